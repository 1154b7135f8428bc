#!/usr/bin/env python
"""Benchmark of the LBVH build + SPH grid interpolation path on B200.

Default workload (the configuration the headline metric is quoted on): a seeded
2^21-particle warped gas disc (M4 kernel) interpolated onto a cylindrical grid of 256
log-spaced radii x 256 phi x 64 z (4,194,304 points) with the catalog rho, vx, vy, vz
(scalars), grad rho, div v and curl v (L = 11 outputs), strategy itpSymmetric, kernel sums
in FP32 with compensated accumulation (FP64 distance tests and pair offsets).

One step = one pass of the hot path over the snapshot with inputs resident in HBM:
LinearBVH! (quantise, encode, radix sort, dedupe, gather, topology, refit) followed by the
interpolation of every grid point: nearest-h search, symmetric walk emitting accepted runs,
kernel sums over the runs (FP32 compensated; FP64 for queries with <= 4096 neighbours).
--config c5 runs the clumped 16M-particle disc (C4 Wendland, rho + curl v, 256^3 grid);
"schedules" compares the plain, tuned and learned query schedules (identical outputs).
  value     grid points / s of the interpolation stage (build excluded; CUDA events on
            the launching stream), summed over ranks (weak scaling: one snapshot per GPU)
  build_ms  LBVH build time per step (CUDA events)
  e2e       the same metric through the public API (PointSamples_interpolation) with
            pinned host buffers: H2D of the particles and sample points, build,
            interpolation, D2H of the outputs and of the in-place-permuted particle columns
  roofline  algorithmic bytes of the reference algorithm's traversal events (per query:
            24 B point + 8 B x L outputs; nearest pass 32 B per internal visit + 24 B per
            leaf test; main pass 36 B per internal visit + 28 B per leaf test + (2+k) x 4 B
            per accepted neighbour, k = quantity columns read) / traversal kernel time,
            against the measured HBM copy bandwidth
  fp64      the same workload in FP64 mode (the reference's arithmetic) on the same GPU
  c5        (one GPU, default run) the clumped 16M-particle disc: build ms, plain / tuned /
            learned interpolation with identical-output hashes, pair roofline, FP32C error
  cpu_baseline  the CPU oracle port on all host threads over a fixed seeded sample of 65,536
            grid points (the sample's and the full grid's mean accepted neighbours beside it)
--impl reference runs the CPU oracle port (the restated reference algorithm, all host
threads) on the same fixed sample, dealt over the timed steps.
"""
import argparse
import datetime
import json
import os
import subprocess
import sys
import time

import numpy as np

REPO = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, REPO)

METRIC = "interp grid pts/s (LBVH build ms reported beside it)"
UNIT = "grid pts/s"
L2_FLUSH_BYTES = 256 << 20
# thread instructions per pair of k_pairs32w<itpSymmetric, M4, grad+div+curl> measured by ncu
# (smsp__inst_executed.sum x 32 / pairs; profiles/k_pairs32w_c2disc_96x96x24.md)
PAIRS32_THREAD_INST_PER_PAIR = 113.7


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--precision", default="fp32c", choices=["fp32c", "fp64"])
    ap.add_argument("--c4-discs", type=int, default=16, help="discs of the C4 batch (the full workload has 64)")
    ap.add_argument("--c4-nmax", type=int, default=4_000_000, help="largest disc of the C4 batch (particles)")
    ap.add_argument("--c4-edges", default="32,64,128,256", help="grid edges the C4 discs draw from")
    ap.add_argument("--config", default="c2", choices=["c2", "c3", "c4", "c5"],
                    help="c2: warped disc, cylindrical grid, L=11 (the headline); c3: two-species 8M disc, "
                         "face-on column density + column-averaged vz image (line integrals, itpScatter); "
                         "c5: clumped 16M disc, C4 Wendland, rho + curl v on a 256^3 Cartesian grid")
    ap.add_argument("--schedule", default="learned", choices=["plain", "tuned", "learned"],
                    help="query schedule of the FP32C path (outputs are identical)")
    ap.add_argument("--no-schedules", action="store_true", help="skip the plain/tuned/learned comparison")
    ap.add_argument("--particles", type=int, default=None)
    ap.add_argument("--grid", default=None)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true", help="skip the FP64-mode timing of the same workload")
    ap.add_argument("--no-c5", action="store_true", help="skip the clumped 16M-particle (C5) block of the default run")
    ap.add_argument("--c5-grid", type=int, default=256, help="grid edge of the C5 block")
    ap.add_argument("--c5-particles", type=int, default=1 << 24, help="particles of the C5 block")
    ap.add_argument("--no-accuracy", action="store_true")
    ap.add_argument("--no-roofline", action="store_true", help="skip the event-count pass (profiling runs)")
    ap.add_argument("--json-out", default=None)
    return ap.parse_args()


def workload(args, rank):
    from distorteddustydiscanalysistoolkits_b200 import synthetic
    import distorteddustydiscanalysistoolkits_b200 as pb
    if args.config == "c5":
        n = args.particles or (1 << 24)
        g = int(args.grid or 256)
        p = synthetic.clumped_disc(n, seed=5 + rank)
        flat = pb.flatten(pb.Cartesian, synthetic.cartesian_box_grid(p, n=g))
        cols = synthetic.C2_COLUMNS
        cat = pb.InterpolationCatalog(cols, scalars=("rho",), curls=("v",))
        config = {"workload": "clumped disc (two log spirals + 2000 clumps), %d particles (C4 Wendland), "
                              "Cartesian %d^3 grid, itpSymmetric, L=%d (rho; curl v)" % (n, g, cat.L),
                  "particles": n, "grid_points": len(flat), "outputs": cat.L, "kernel": "C4_Wendland",
                  "strategy": "itpSymmetric", "precision": args.precision}
        return p, flat, cols, cat, config, pb.C4_Wendland
    n = args.particles or (1 << 21)
    ns, nphi, nz = (int(v) for v in (args.grid or "256,256,64").split(","))
    p = synthetic.disc(n, seed=2 + rank)
    grid = synthetic.log_cylindrical_grid(ns, nphi, nz)
    flat = pb.flatten(pb.Cylindrical, grid)
    cols = synthetic.C2_COLUMNS
    cat = pb.InterpolationCatalog(cols, **synthetic.C2_CATALOG)
    config = {"workload": "warped gas disc, %d particles (M4), cylindrical %dx%dx%d log-r grid, itpSymmetric, "
                          "L=%d (rho,vx,vy,vz; grad rho; div v; curl v)" % (n, ns, nphi, nz, cat.L),
              "particles": n, "grid_points": len(flat), "outputs": cat.L, "kernel": "M4_spline",
              "strategy": "itpSymmetric", "precision": args.precision}
    return p, flat, cols, cat, config, pb.M4_spline


def _max_over_ranks(vals, world):
    if world == 1:
        return vals
    import torch
    import torch.distributed as dist
    t = torch.tensor(vals, dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


class ClockSampler:
    """nvidia-smi clock/throttle samples while the timed region runs."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu = gpu
        self.proc = None
        self.path = os.path.join("/tmp", "pb_clocks_%d_%d.csv" % (os.getpid(), gpu))

    def start(self):
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "100"], stdout=self.f,
                                         stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            parts = [s.strip() for s in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def algorithmic_bytes(stats, L, k_cols, s):
    """Reference-algorithm bytes of the two kernel phases over all queries (see module doc):
    the traversal (nearest search + walk: query points and tree visits) and the pair sums
    (per accepted neighbour m, rho and k quantity columns at s bytes, per query L outputs)."""
    nv, nl, mv, ml, acc = (stats[:, i].astype(np.float64).sum() for i in range(5))
    nq = stats.shape[0]
    return {"walk": nq * 24 + 32 * nv + 24 * nl + 36 * mv + 28 * ml, "pairs": nq * 8 * L + acc * (2 + k_cols) * s}


CPU_SAMPLE_POINTS = 65536
CPU_SAMPLE_SEED = 2024


def cpu_sample(n, m=CPU_SAMPLE_POINTS, seed=CPU_SAMPLE_SEED):
    """The fixed seeded uniform sample of grid points the CPU oracle is timed on (sorted), the
    same in the cpu_baseline leg and in the --impl reference arm: the per-point work is
    heavy-tailed and varies with position, so a large random sample represents the grid."""
    g = np.random.default_rng(seed)
    return np.sort(g.choice(n, size=min(m, n), replace=False))


def cpu_baseline(p, flat, cols, cat):
    """Oracle port on all host cores: full LBVH build, then the fixed sample of grid points."""
    import oracle
    threads = oracle.max_threads()
    t0 = time.perf_counter()
    o = oracle.OracleLBVH(p["x"], p["y"], p["z"], p["h"]).attach(p["m"], p["rho"], [p[c] for c in cols])
    build_s = time.perf_counter() - t0
    idx = cpu_sample(len(flat))
    t0 = time.perf_counter()
    _, st = o.interp_points(cat.oracle_dict(), *(c[idx] for c in flat.coor), strategy="itpSymmetric", stats=True)
    dt = time.perf_counter() - t0
    return {"value": len(idx) / dt, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": "oracle (C, OpenMP, FP64) on a fixed seeded uniform sample of %d of %d grid points (seed %d), "
                      "after a full %d-particle LBVH build (%.0f ms)" % (len(idx), len(flat), CPU_SAMPLE_SEED,
                                                                         len(p["x"]), build_s * 1e3),
            "build_ms": build_s * 1e3, "sample_mean_accepted": float(st[:, 4].mean())}


def run_reference(args, rank, world):
    if rank != 0:
        return 0
    import oracle
    import distorteddustydiscanalysistoolkits_b200 as pb  # noqa: F401  (catalog/grid host types only)
    p, flat, cols, cat, config, _ = workload(args, 0)
    threads = oracle.max_threads()
    t0 = time.perf_counter()
    o = oracle.OracleLBVH(p["x"], p["y"], p["z"], p["h"]).attach(p["m"], p["rho"], [p[c] for c in cols])
    build_ms = (time.perf_counter() - t0) * 1e3
    idx = cpu_sample(len(flat))
    # the fixed sample is dealt round-robin over the timed steps (each step a representative
    # part of it), so all timed steps together evaluate exactly the cpu_baseline sample;
    # warm-up steps take small slices of it
    steps = max(1, args.steps)
    for w in range(args.warmup):
        o.interp_points(cat.oracle_dict(), *(c[idx[w::steps * 8][:256]] for c in flat.coor), strategy="itpSymmetric")
    times, acc = [], []
    for k in range(steps):
        part = idx[k::steps]
        t0 = time.perf_counter()
        _, st = o.interp_points(cat.oracle_dict(), *(c[part] for c in flat.coor), strategy="itpSymmetric", stats=True)
        times.append(time.perf_counter() - t0)
        acc.append(st[:, 4])
    total = float(np.sum(times))
    value = len(idx) / total
    ms = 1e3 * total / steps
    sample = ("fixed seeded uniform sample of %d of %d grid points (seed %d), dealt round-robin over the %d timed "
              "steps; LBVH build of all %d particles once (%.0f ms)" % (len(idx), len(flat), CPU_SAMPLE_SEED, steps,
                                                                         len(p["x"]), build_ms))
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded disc)",
            "config": dict(config, precision="fp64"), "build_ms": build_ms,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port", "sample": sample,
                             "sample_mean_accepted": float(np.concatenate(acc).mean())},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
            "note": "reference Julia code cannot run on this box (no Julia toolchain); this arm is the C "
                    "restatement of the reference algorithm (oracle/), OpenMP over all host threads"}
    print(json.dumps(line), flush=True)
    return 0


def run_lines(args, rank, world):
    """C3: line-integrated column density and column-averaged v_z of a 6M gas + 2M dust disc
    (tilt 30 deg) on a face-on npix^2 image, both species per step; device-resident inputs."""
    import ctypes
    import torch
    import distorteddustydiscanalysistoolkits_b200 as pb
    from distorteddustydiscanalysistoolkits_b200 import _lib, synthetic
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    ng, nd = (args.particles or 6291456), (args.particles or 6291456) // 3
    npix = int(args.grid or 2048)
    gas, dust = synthetic.dusty_disc(ng, nd, seed=3 + rank, tilt_deg=30.0)
    prec = _lib.PB_FP32C if args.precision == "fp32c" else _lib.PB_FP64
    be = pb.CUDAComputeBackend(int(os.environ.get("LOCAL_RANK", "0")))
    H = be.handle
    # the face-on image's lines are generated on the device (pb_line_image): origins on z = 0
    # over the gas disc's x/y extent, direction (0, 0, 1)
    xs = pb.grids.linrange(float(np.min(gas["x"])), float(np.max(gas["x"])), npix)
    ys = pb.grids.linrange(float(np.min(gas["y"])), float(np.max(gas["y"])), npix)
    lines = pb.LineSamples_image(be, xs, ys)
    nl = len(lines)
    H.set_option("timing", 1)
    H.set_stream(torch.cuda.current_stream().cuda_stream)
    cat = pb.InterpolationCatalog(("rho", "vz"), scalars=("rho", "vz"))
    o, d = lines.origin, lines.direction
    species = []
    for sp in (gas, dust):
        dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in sp.items()}
        inp = pb.InterpolationInput(dev["x"], dev["y"], dev["z"], dev["m"], dev["h"], dev["rho"],
                                    (dev["rho"], dev["vz"]), smoothed_kernel=pb.M4_spline)
        outs = [torch.empty(nl, dtype=torch.float64, device="cuda") for _ in range(cat.L)]
        species.append((dev, inp, inp._c_struct(), outs, (ctypes.c_void_p * cat.L)(*[x.data_ptr() for x in outs])))
    ccat = cat._c_struct()

    def step():
        b = i = 0.0
        for dev, inp, cin, outs, optrs in species:
            rc = H.lib.pb_line_samples_interpolation(H.h, ctypes.byref(cin), ctypes.byref(ccat), nl, o[0].data_ptr(),
                                                     o[1].data_ptr(), o[2].data_ptr(), d[0].data_ptr(),
                                                     d[1].data_ptr(), d[2].data_ptr(), pb.itpScatter.code, prec,
                                                     optrs, 0)
            H.check(rc, "pb_line_samples_interpolation")
            tb, ti, _ = H.timings()
            b += tb
            i += ti
        return b, i

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    res = [step() for _ in range(args.steps)]
    build_ms = float(np.mean([r[0] for r in res]))
    interp_ms = float(np.mean([r[1] for r in res]))
    line = {"metric": "line samples/s (both species)", "value": 2 * nl / (interp_ms / 1e3), "unit": "lines/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": build_ms + interp_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded two-species disc)",
            "config": {"workload": "dusty disc %d gas + %d dust (M4, tilt 30 deg), face-on %d^2 image, itpScatter, "
                                   "column rho + column-averaged vz per species" % (ng, nd, npix),
                       "precision": args.precision,
                       "note": "line integrals use the FP64 kernel in both precision modes"},
            "build_ms": build_ms, "interp_ms": interp_ms}
    if rank == 0:
        print(json.dumps(line), flush=True)
        if args.json_out:
            with open(args.json_out, "w") as f:
                f.write(json.dumps(line) + "\n")
    return 0


def c5_block(local, model, sched_modes, args):
    """The clumped-disc target measured inside the default run (one GPU): 2^24 particles (two
    log spirals + 2000 clumps, C4 Wendland), rho + curl v on a 256^3 Cartesian grid, itpSymmetric,
    FP32C.  Reports the LBVH build time (CUDA events, 10 builds), the interpolation time of the
    plain, tuned and learned schedules (one timed run each after one warm-up run) with a hash
    of each one's outputs (they must be identical), the pair kernels' roofline from the pair
    phase time and the sample's accepted counts, and the FP32C error against the FP64 mode
    (bit-exact with the oracle) on a seeded sample of 2^20 grid points."""
    import ctypes
    import hashlib
    import torch
    import distorteddustydiscanalysistoolkits_b200 as pb
    from distorteddustydiscanalysistoolkits_b200 import _lib, accuracy, scheduler, synthetic
    n = args.c5_particles
    p = synthetic.clumped_disc(n, seed=5)
    flat = pb.flatten(pb.Cartesian, synthetic.cartesian_box_grid(p, n=args.c5_grid))
    npts = len(flat)
    cols = synthetic.C2_COLUMNS
    cat = pb.InterpolationCatalog(cols, scalars=("rho",), curls=("v",))
    backend = pb.CUDAComputeBackend(local)
    H = backend.handle
    H.set_option("timing", 1)
    if model is not None:
        scheduler.set_model(H, model)
    H.set_stream(torch.cuda.current_stream().cuda_stream)
    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in p.items()}
    q = [torch.from_numpy(np.ascontiguousarray(c)).cuda() for c in flat.coor]
    outs = [torch.empty(npts, dtype=torch.float64, device="cuda") for _ in range(cat.L)]
    inp = pb.InterpolationInput(dev["x"], dev["y"], dev["z"], dev["m"], dev["h"], dev["rho"],
                                tuple(dev[c] for c in cols), smoothed_kernel=pb.C4_Wendland)
    cin, ccat = inp._c_struct(), cat._c_struct()
    optrs = (ctypes.c_void_p * cat.L)(*[o.data_ptr() for o in outs])
    qp = [c.data_ptr() for c in q]
    builds = []
    for k in range(12):
        H.check(H.lib.pb_linear_bvh(H.h, ctypes.byref(cin), 0), "pb_linear_bvh")
        if k >= 2:
            builds.append(H.timings()[0])

    def interp(prec=_lib.PB_FP32C):
        H.check(H.lib.pb_interpolate_points(H.h, ctypes.byref(ccat), npts, qp[0], qp[1], qp[2], pb.itpSymmetric.code,
                                            prec, optrs), "pb_interpolate_points")
        return H.timings()[1]

    runs = {}
    H.set_option("schedule", scheduler.TUNED)
    interp()   # warm-up: grows the run pool to its working size
    for name in ("learned", "tuned", "plain"):
        if name == "learned" and model is None:
            continue
        H.set_option("schedule", sched_modes[name])
        ms = interp()
        hs = hashlib.sha256()
        for o in outs:
            hs.update(o.cpu().numpy().tobytes())
        ph = H.phase_times()
        runs[name] = {"interp_ms": ms, "pts_per_s": npts / (ms / 1e3), "nearest_ms": ph[0], "walk_ms": ph[1],
                      "pairs_ms": ph[2], "walk_rounds": H.schedule()[0], "deferred_queries": H.schedule()[1],
                      "pair_split": dict(zip(("heavy_queries", "light_queries", "heavy_pairs", "light_pairs"),
                                             H.pair_split())),
                      "outputs_sha256": hs.hexdigest()}
    H.set_option("schedule", scheduler.TUNED)
    hashes = {r["outputs_sha256"] for r in runs.values()}
    out = {"workload": "clumped disc, %d particles (2 log spirals + 2000 clumps, C4 Wendland), Cartesian %d^3 grid, "
                       "itpSymmetric, rho + curl v (L=%d), FP32C" % (n, args.c5_grid, cat.L),
           "build_ms": float(np.mean(builds)), "build_ms_min": float(np.min(builds)), "build_reps": len(builds),
           "schedules": runs, "outputs_identical": len(hashes) == 1}
    if "plain" in runs:
        for name in runs:
            out["%s_vs_plain" % name] = runs["plain"]["interp_ms"] / runs[name]["interp_ms"]
    if "learned" in runs and "tuned" in runs:
        out["learned_vs_tuned"] = runs["tuned"]["interp_ms"] / runs["learned"]["interp_ms"]
    # accuracy and accepted counts on a seeded sample of grid points
    g = np.random.default_rng(55)
    idx = np.sort(g.choice(npts, size=min(npts, 1 << 20), replace=False))
    qs = [torch.from_numpy(np.ascontiguousarray(c[idx])).cuda() for c in flat.coor]
    lb = pb.LinearBVH(backend, n)
    ref = pb.interpolate_points(lb, cat, qs, pb.itpSymmetric, pb.FP64)
    got = pb.interpolate_points(lb, cat, qs, pb.itpSymmetric, pb.FP32C)
    out["accuracy_fp32c_vs_fp64"] = accuracy.field_errors([a.cpu().numpy() for a in got],
                                                          [r.cpu().numpy() for r in ref], cat.ordered_names)
    out["accuracy_fp32c_vs_fp64"]["sample_points"] = len(idx)
    st = pb.traversal_stats(lb, [c.cpu().numpy() for c in qs], pb.itpSymmetric)
    mean_acc = float(st[:, 4].mean())
    best = min(runs.values(), key=lambda r: r["interp_ms"]) if runs else None
    if best is not None and best["pairs_ms"] > 0:
        pair_bytes = npts * 8 * cat.L + mean_acc * npts * (2 + len(cols)) * 4
        peak = _peak_gbs()
        ach = pair_bytes / (best["pairs_ms"] / 1e3) / 1e9
        out["roofline_pairs"] = {"achieved": ach, "peak": peak[0], "frac": ach / peak[0], "unit": "GB/s",
                                 "peak_source": peak[1], "algorithmic_bytes": pair_bytes,
                                 "mean_accepted_per_query_sample": mean_acc,
                                 "note": "pair-phase bytes from the sample's mean accepted count x all grid points"}
    backend.close()
    return out


def _peak_gbs():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        return float(json.load(open(path))["hbm_gbs"]), "MEASURED_PEAKS.json hbm_gbs (of measured)"
    return 6650.0, "fallback 6.65 TB/s"


def run_c4(args, rank, world):
    """C4: seeded discs of log-uniform particle counts (50k .. --c4-nmax), each with its own
    Cartesian grid (edge drawn from --c4-edges) and tilt, rho + grad rho, M4, itpSymmetric,
    FP32C.  Times the per-call loop (one PointSamples_interpolation per disc) against one step of
    the device batch (every disc's build + one batched launch) replayed from a CUDA graph with
    the autotuned schedule, and checks that both give the same bits."""
    import torch
    import distorteddustydiscanalysistoolkits_b200 as pb
    from distorteddustydiscanalysistoolkits_b200 import batch
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    edges = tuple(int(e) for e in args.c4_edges.split(","))
    descs = batch.c4_discs(args.c4_discs, seed=100 + 1000 * rank, n_max=args.c4_nmax, edges=edges)
    prec = pb.FP32C if args.precision == "fp32c" else pb.FP64
    jobs = [batch.make_job(d) for d in descs]
    npts = sum(len(j["points"]) for j in jobs)
    npart = sum(j["input"].Npart for j in jobs)
    # per-call loop, one handle, inputs on the host as a caller of the reference API holds them
    be = pb.CUDAComputeBackend(local)
    loop_out = None
    loop_ms = []
    for step in range(args.warmup + args.steps):
        fresh = [batch.make_job(d) for d in descs] if step == 0 else None
        if fresh is None:
            fresh = [dict(j, input=pb.InterpolationInput(*(np.array(c) for c in j["input"].coord), np.array(j["input"].m),
                                                         np.array(j["input"].h), np.array(j["input"].rho),
                                                         tuple(np.array(q) for q in j["input"].quant),
                                                         smoothed_kernel=j["input"].smoothed_kernel)) for j in jobs]
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        outs, _ = batch.batch_point_interpolation(be, fresh, None, precision=prec)
        dt = (time.perf_counter() - t0) * 1e3
        if step >= args.warmup:
            loop_ms.append(dt)
        if loop_out is None:
            loop_out = [np.stack([g.grid for g in o.grids]) for o in outs]
    be.close()
    db = batch.DeviceBatch(jobs, device=local, precision=prec)
    # the per-call loop on the same device-resident inputs (build + two-phase interpolation per
    # disc, CUDA events of the library), the like-for-like reference for the batched launch
    import ctypes
    from distorteddustydiscanalysistoolkits_b200 import _lib
    res_ms = []
    hd = db.backends[0].handle
    hd.set_option("timing", 1)
    for step in range(args.warmup + args.steps):
        tot = 0.0
        for k in range(db.K):
            outs_k = (ctypes.c_void_p * db.L)(*[o.data_ptr() for o in db.outs[k]])
            q = db.queries[k]
            rc = hd.lib.pb_point_samples_interpolation(hd.h, ctypes.byref(db.cin[k]), ctypes.byref(db.ccat),
                                                       len(q[0]), q[0].data_ptr(), q[1].data_ptr(), q[2].data_ptr(),
                                                       pb.itpSymmetric.code, db.precision, outs_k, 0)
            hd.check(rc, "pb_point_samples_interpolation")
            b, i, _ = hd.timings()
            tot += b + i
        if step >= args.warmup:
            res_ms.append(tot)
    hd.set_option("timing", 0)
    tuner = batch.BatchAutotuner(leaf_size=(1, 8), order=(0, 1), blocks_per_sm=(0,), walk_split=(16, 32, 64),
                                 repeats=1)
    best = tuner.tune(db)
    db.timed(args.warmup)
    ms = db.timed(args.steps)
    same = all(np.array_equal(a.view(np.uint64), b.view(np.uint64)) for a, b in zip(db.outputs(), loop_out))
    db.close()
    line = {"metric": "batched interp grid pts/s (all discs built + interpolated per step)", "value": npts / (ms / 1e3),
            "unit": "grid pts/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32" if prec == pb.FP32C else "f64", "data": "synthetic (seeded discs)",
            "config": {"workload": "%d seeded discs, %d..%d particles (log-uniform), Cartesian grids with edges from %s, "
                                   "tilt 0-30 deg, rho + grad rho, M4, itpSymmetric" % (len(descs), 50_000, args.c4_nmax,
                                                                                         edges),
                       "discs": len(descs), "particles": npart, "grid_points": npts},
            "batch": {"ms_per_step": ms, "graph": True, "options": best,
                      "autotune": [{"options": o, "ms": t} for o, t in tuner.timings]},
            "per_call_loop": {"ms_per_step": float(np.mean(loop_ms)), "pts_per_s": npts / (float(np.mean(loop_ms)) / 1e3),
                              "note": "one PointSamples_interpolation per disc, host arrays (H2D and D2H inside)"},
            "per_call_loop_resident": {"ms_per_step": float(np.mean(res_ms)),
                                       "pts_per_s": npts / (float(np.mean(res_ms)) / 1e3),
                                       "note": "one pb_point_samples_interpolation per disc on the batch's device "
                                               "arrays: build + two-phase interpolation (library CUDA events)"},
            "batch_vs_loop": float(np.mean(loop_ms)) / ms, "batch_vs_loop_resident": float(np.mean(res_ms)) / ms,
            "outputs_identical": bool(same)}
    if rank == 0:
        print(json.dumps(line), flush=True)
        if args.json_out:
            with open(args.json_out, "w") as f:
                f.write(json.dumps(line) + "\n")
    return 0


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank, world)
    if args.config == "c3":
        return run_lines(args, rank, world)
    if args.config == "c4":
        return run_c4(args, rank, world)

    import torch
    import distorteddustydiscanalysistoolkits_b200 as pb
    from distorteddustydiscanalysistoolkits_b200 import _lib

    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    p, flat, cols, cat, config, skern = workload(args, rank)
    nparticles = len(p["x"])
    prec = pb.FP32C if args.precision == "fp32c" else pb.FP64
    npts = len(flat)
    backend = pb.CUDAComputeBackend(local)
    H = backend.handle
    H.set_option("timing", 1)
    from distorteddustydiscanalysistoolkits_b200 import scheduler
    sched_modes = {"plain": scheduler.PLAIN, "tuned": scheduler.TUNED, "learned": scheduler.LEARNED}
    model = scheduler.Model.load() if os.path.exists(scheduler.MODEL_PATH) else None
    if model is not None:
        scheduler.set_model(H, model)
    if args.schedule == "learned" and model is None:
        args.schedule = "tuned"
    H.set_option("schedule", sched_modes[args.schedule])
    stream = torch.cuda.current_stream()
    H.set_stream(stream.cuda_stream)

    dev = {k: torch.from_numpy(np.ascontiguousarray(v)).cuda() for k, v in p.items()}
    q = [torch.from_numpy(np.ascontiguousarray(c)).cuda() for c in flat.coor]
    outs = [torch.empty(npts, dtype=torch.float64, device="cuda") for _ in range(cat.L)]
    inp = pb.InterpolationInput(dev["x"], dev["y"], dev["z"], dev["m"], dev["h"], dev["rho"],
                                tuple(dev[c] for c in cols), smoothed_kernel=skern)
    import ctypes
    cin, ccat = inp._c_struct(), cat._c_struct()
    optrs = (ctypes.c_void_p * cat.L)(*[o.data_ptr() for o in outs])
    qp = [c.data_ptr() for c in q]
    pcode = _lib.PB_FP32C if prec == pb.FP32C else _lib.PB_FP64

    def step():
        rc = H.lib.pb_point_samples_interpolation(H.h, ctypes.byref(cin), ctypes.byref(ccat), npts, qp[0], qp[1],
                                                  qp[2], pb.itpSymmetric.code, pcode, optrs, 0)
        H.check(rc, "pb_point_samples_interpolation")
        b, i, nl = H.timings()
        phases.append(H.phase_times())
        return b, i

    phases = []

    flush = torch.empty(L2_FLUSH_BYTES // 8, dtype=torch.float64, device="cuda")
    for _ in range(args.warmup):
        step()
    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    launches0 = H.launch_count()
    builds, interps = [], []
    phases.clear()
    for _ in range(args.steps):
        flush.zero_()            # L2 flush between timed steps, outside the per-step events
        b, i = step()
        builds.append(b)
        interps.append(i)
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    launches = H.launch_count() - launches0
    sched = H.schedule()
    main_phases = list(phases)
    clocks = sampler.stop()
    build_ms, interp_ms = float(np.mean(builds)), float(np.mean(interps))
    build_ms, interp_ms, step_ms = _max_over_ranks([build_ms, interp_ms, build_ms + interp_ms], world)
    value = world * npts / (interp_ms / 1e3)

    # the same step under each query schedule (identical outputs): plain = input order, one walk
    # per query, no ordering; tuned = Morton order, split walks, heaviest-first pairs; learned =
    # tuned + walk order binned by the MLP's predicted work
    schedules = None
    if prec == pb.FP32C and not args.no_schedules:
        schedules = {}
        for name, mode in sched_modes.items():
            if mode == scheduler.LEARNED and model is None:
                continue
            H.set_option("schedule", mode)
            for _ in range(2):
                step()
            phases.clear()
            ts = []
            for _ in range(max(2, min(args.steps, 3))):
                flush.zero_()
                ts.append(step()[1])
            ph = np.mean(np.array(phases), axis=0)
            schedules[name] = {"interp_ms": float(np.mean(ts)), "pts_per_s": npts / (float(np.mean(ts)) / 1e3),
                               "nearest_ms": float(ph[0]), "walk_ms": float(ph[1]), "pairs_ms": float(ph[2])}
        H.set_option("schedule", sched_modes[args.schedule])
        if "plain" in schedules:
            for name in schedules:
                schedules[name]["speedup_vs_plain"] = schedules["plain"]["interp_ms"] / schedules[name]["interp_ms"]
        phases.clear()

    # roofline of the dominant kernel phase (walk kernels vs pair kernels, per-phase CUDA events
    # of the library)
    lb = pb.LinearBVH(backend, nparticles)
    roofline = None
    if not args.no_roofline:
        stats = pb.traversal_stats(lb, [c.cpu().numpy() for c in q], pb.itpSymmetric)
        s = 4 if prec == pb.FP32C else 8
        alg = algorithmic_bytes(stats, cat.L, len(cols), s)
        peak, peak_source = _peak_gbs()
        ph = np.mean(np.array(main_phases), axis=0) if main_phases else np.zeros(3)
        kname = {"M4_spline": "M4", "C4_Wendland": "C4"}.get(config["kernel"], config["kernel"])
        pk = "k_pairs32w<itpSymmetric,%s> (+ k_pairs64w for light queries)" % kname if prec == pb.FP32C \
            else "k_pairs64w<itpSymmetric>"
        kern = {"walk": ("k_nearest_list + k_item_filter + k_walk_list<itpSymmetric>", ph[0] + ph[1]), "pairs": (pk, ph[2])}
        per = {}
        for key, (name, ms) in kern.items():
            a = alg[key] / (ms / 1e3) / 1e9 if ms > 0 else None
            per[key] = {"kernel": name, "ms": float(ms), "algorithmic_bytes": alg[key], "achieved_gbs": a}
        dom = max(per, key=lambda k: per[k]["ms"])
        traffic = None
        prof = os.path.join(REPO, "profiles", {"pairs": "k_pairs32w", "walk": "k_walk_items"}[dom] + "_c2_traffic.json")
        if os.path.exists(prof) and args.precision == "fp32c" and args.config == "c2" and \
                args.particles in (None, 1 << 21) and args.grid in (None, "256,256,64"):
            traffic = json.load(open(prof)).get("dram_bytes_per_launch")
        achieved = per[dom]["achieved_gbs"]
        # The pair kernel is bound by instruction issue, not by DRAM (its DRAM traffic is 3 % of
        # peak; the records are re-read from L2): pairs/s against the issue ceiling, SMs x 4
        # schedulers x SM clock / warp instructions per pair, with the instructions per pair of
        # the committed ncu capture of k_pairs32w (profiles/k_pairs32w_c2disc_96x96x24.md)
        issue = None
        acc_pairs = float(stats[:, 4].astype(np.float64).sum())
        if prec == pb.FP32C and ph[2] > 0:
            props = torch.cuda.get_device_properties(local)
            sm_mhz = (clocks or {}).get("sm_mhz") or 1965.0
            warp_inst_per_pair = PAIRS32_THREAD_INST_PER_PAIR / 32.0
            ceiling = props.multi_processor_count * 4 * sm_mhz * 1e6 / warp_inst_per_pair
            got = acc_pairs / (ph[2] / 1e3)
            issue = {"pairs_per_s": got, "issue_ceiling_pairs_per_s": ceiling, "frac": got / ceiling,
                     "thread_inst_per_pair": PAIRS32_THREAD_INST_PER_PAIR, "sm_mhz": sm_mhz,
                     "note": "issue ceiling = SMs x 4 schedulers x SM clock / (thread instructions per pair / 32)"}
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak if achieved else None, "traffic": traffic,
                    "kernel": per[dom]["kernel"], "algorithmic_bytes_per_launch": alg[dom],
                    "peak_source": peak_source,
                    "phases": per, "pair_issue": issue,
                    "events_per_query": {k: float(stats[:, i].mean()) for i, k in enumerate(
                        ("nearest_internal", "nearest_leaf", "main_internal", "main_leaf", "accepted"))}}

    # accuracy of the FP32-compensated fields against the FP64 path (bit-exact to the oracle)
    accuracy = None
    if prec == pb.FP32C and not args.no_accuracy:
        from distorteddustydiscanalysistoolkits_b200 import accuracy as acc_mod
        ref = pb.interpolate_points(lb, cat, q, pb.itpSymmetric, pb.FP64)
        got = pb.interpolate_points(lb, cat, q, pb.itpSymmetric, pb.FP32C)
        split = H.pair_split()
        accuracy = acc_mod.field_errors([a.cpu().numpy() for a in got], [r.cpu().numpy() for r in ref],
                                        cat.ordered_names)
        accuracy["pair_split"] = dict(zip(("heavy_queries", "light_queries", "heavy_pairs", "light_pairs"), split))

    # end to end through the public API with pinned host buffers
    e2e = None
    if not args.no_e2e:
        def pinned(a):
            t = torch.empty(len(a), dtype=torch.float64, pin_memory=True)
            t.numpy()[:] = a
            return t.numpy()

        hp = {k: pinned(v) for k, v in p.items()}
        pristine = {k: v.copy() for k, v in hp.items()}
        hq = [pinned(c) for c in flat.coor]
        hout = [pinned(np.zeros(npts)) for _ in range(cat.L)]
        grid = pb.PointSamples(np.zeros(npts), hq)
        H.set_stream(None)
        times = []
        for k in range(args.warmup + args.steps):
            for key in hp:
                hp[key][:] = pristine[key]
            inp_h = pb.InterpolationInput(hp["x"], hp["y"], hp["z"], hp["m"], hp["h"], hp["rho"],
                                          tuple(hp[c] for c in cols), smoothed_kernel=skern)
            t0 = time.perf_counter()
            pb.PointSamples_interpolation(backend, grid, inp_h, cat, pb.itpSymmetric, precision=prec, out=hout)
            dt = time.perf_counter() - t0
            if k >= args.warmup:
                times.append(dt)
        e2e_s = _max_over_ranks([float(np.mean(times))], world)[0]
        ncols_in = 6 + len(cols)
        e2e = {"value": world * npts / e2e_s, "unit": UNIT, "ms_per_step": e2e_s * 1e3,
               "h2d_bytes_per_step": ncols_in * 8 * nparticles + 24 * npts,
               "d2h_bytes_per_step": cat.L * 8 * npts + ncols_in * 8 * nparticles,
               "path": "PointSamples_interpolation(CUDAComputeBackend) with pinned host arrays: H2D, build, "
                       "interpolation, D2H of outputs and of the permuted particle columns"}

    # the same workload in FP64 mode (the reference's arithmetic, bit-exact with the oracle):
    # the like-for-like GPU figure beside the FP64 CPU arm
    fp64 = None
    if prec == pb.FP32C and world == 1 and not args.no_fp64:
        H.set_stream(stream.cuda_stream)
        ts = []
        for k in range(3):
            flush.zero_()
            rc = H.lib.pb_interpolate_points(H.h, ctypes.byref(ccat), npts, qp[0], qp[1], qp[2], pb.itpSymmetric.code,
                                             _lib.PB_FP64, optrs)
            H.check(rc, "pb_interpolate_points(FP64)")
            if k > 0:
                ts.append(H.timings()[1])
        fp64 = {"interp_ms": float(np.mean(ts)), "pts_per_s": npts / (float(np.mean(ts)) / 1e3), "steps": len(ts),
                "note": "FP64 mode on the same resident LBVH (every pair in the reference's FP64 arithmetic)"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(p, flat, cols, cat)
        if roofline is not None:
            cpu["full_grid_mean_accepted"] = roofline["events_per_query"]["accepted"]

    c5 = None
    if rank == 0 and world == 1 and args.config == "c2" and not args.no_c5:
        backend.close()
        c5 = c5_block(local, model, sched_modes, args)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f32" if prec == pb.FP32C else "f64",
                "data": "synthetic (seeded Philox disc, no dataset exists for this path)",
                "config": dict(config, parallelism="replicas x%d (one snapshot per GPU)" % world,
                               l2_flush="256 MiB write between timed steps, outside the step events"),
                "build_ms": build_ms, "interp_ms": interp_ms,
                "pts_per_s_with_build": world * npts / (step_ms / 1e3),
                "gpu_launches": int(launches), "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "fp64": fp64,
                "c5": c5,
                "schedule": dict(zip(("walk_rounds", "deferred_queries", "pool_chunks"), sched), mode=args.schedule),
                "schedules": schedules,
                "clocks": clocks, "accuracy_fp32c_vs_fp64": accuracy}
        txt = json.dumps(line)
        print(txt, flush=True)
        if args.json_out:
            with open(args.json_out, "w") as f:
                f.write(txt + "\n")
    if c5 is None:
        backend.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
