"""Multi-GPU plumbing: one process per GPU, no data-path collective.

Sample points are independent (PointSamples_interpolation.jl:38 loops over them with
@threads), so the path shards without any exchange: every rank either interpolates its
own snapshot (weak scaling, what bench.py measures) or a contiguous slice of one shared
grid against a replicated particle set.  The only collectives are the timing barrier and
a max-over-ranks reduction of the measured times, through torch.distributed (NCCL on
GPUs, gloo on CPU).
"""
import numpy as np


def query_shard(npts, rank, world):
    """Contiguous [lo, hi) slice of npts sample points owned by ``rank`` (sizes differ by <= 1)."""
    if world < 1 or not (0 <= rank < world):
        raise ValueError("bad rank/world")
    base, extra = divmod(int(npts), int(world))
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def max_over_ranks(values, device="cpu"):
    """Element-wise max of a list of floats over all ranks (identity without a process group)."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size() == 1:
        return list(values)
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def gather_shards(local, npts, rank, world, device="cpu"):
    """Assemble per-rank output slices (each rank's query_shard) into the full array on every rank."""
    import torch
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or world == 1:
        return np.asarray(local)
    sizes = [query_shard(npts, r, world) for r in range(world)]
    width = max(hi - lo for lo, hi in sizes)
    buf = torch.zeros(width, dtype=torch.float64, device=device)
    buf[:len(local)] = torch.as_tensor(np.asarray(local), dtype=torch.float64, device=device)
    parts = [torch.zeros(width, dtype=torch.float64, device=device) for _ in range(world)]
    dist.all_gather(parts, buf)
    return np.concatenate([parts[r][:hi - lo].cpu().numpy() for r, (lo, hi) in enumerate(sizes)])
