"""Schedule invariance of the FP32-compensated point path.

The per-query arithmetic depends only on the query and the tree: the accepted leaves are
summed in DFS order with the k-th leaf on lane k mod 32, whatever the query order, the
number of subtrees a walk is split into, the size of the run pool (queries that find it full
are walked again in later rounds, or finished by the fused walk-and-sum kernel), or which of
the two kernels ran.  Every configuration must therefore give the same bits.
"""
import os

import numpy as np
import pytest

import distorteddustydiscanalysistoolkits_b200 as pb
from distorteddustydiscanalysistoolkits_b200 import synthetic

pytestmark = pytest.mark.gpu

COLS = ("rho", "vx", "vy", "vz")


def _run(p, flat, strategy, options=(), env=None, precision=pb.FP32C):
    old = {k: os.environ.get(k) for k in ("PB_RUN_POOL_CHUNKS", "PB_RUN_POOL_MB")}
    for k in old:
        os.environ.pop(k, None)
    os.environ.update(env or {})
    be = pb.CUDAComputeBackend(0)
    try:
        for k, v in options:
            be.handle.set_option(k, v)
        inp = pb.InterpolationInput(p["x"].copy(), p["y"].copy(), p["z"].copy(), p["m"].copy(), p["h"].copy(),
                                    p["rho"].copy(), tuple(p[c].copy() for c in COLS))
        cat = pb.InterpolationCatalog(COLS, **synthetic.C2_CATALOG)
        out = pb.PointSamples_interpolation(be, flat, inp, cat, strategy, precision=precision)
        return np.stack([g.grid for g in out.grids]), be.handle.schedule()
    finally:
        be.close()
        for k, v in old.items():
            os.environ.pop(k, None)
            if v is not None:
                os.environ[k] = v


def _same_bits(a, b):
    assert a.shape == b.shape
    assert np.array_equal(a.view(np.uint64), b.view(np.uint64))


@pytest.fixture(scope="module")
def case():
    p = synthetic.disc(30000, seed=21)
    flat = pb.flatten(pb.Cylindrical, synthetic.log_cylindrical_grid(20, 16, 8))
    return p, flat


@pytest.mark.parametrize("strategy", [pb.itpGather, pb.itpScatter, pb.itpSymmetric])
def test_fp32c_identical_across_schedules(case, strategy):
    p, flat = case
    ref, (rounds, deferred, _) = _run(p, flat, strategy, env={"PB_RUN_POOL_MB": "512"})
    assert rounds == 1 and deferred == 0
    got, _ = _run(p, flat, strategy)   # default pool size
    _same_bits(got, ref)
    for opts in ((("walk_split", 1),), (("walk_split", 7),), (("walk_split", 300),), (("sort_queries", 0),)):
        got, _ = _run(p, flat, strategy, options=opts)
        _same_bits(got, ref)
    # small pools: queries are deferred to later walk rounds (or to the fused kernel)
    for chunks in ("8000", "3000"):
        got, (rounds, deferred, cap) = _run(p, flat, strategy, env={"PB_RUN_POOL_CHUNKS": chunks})
        assert cap == int(chunks) and deferred > 0
        _same_bits(got, ref)
    # a pool of one chunk: the fused kernel finishes the deferred queries
    got, (rounds, deferred, _) = _run(p, flat, strategy, env={"PB_RUN_POOL_CHUNKS": "1"})
    assert deferred > 0
    _same_bits(got, ref)


@pytest.mark.parametrize("strategy", [pb.itpGather, pb.itpSymmetric])
def test_light_queries_are_summed_exactly_in_fp64(case, strategy):
    """FP32C mode sums queries with at most 4096 accepted neighbours (option fp64_light_max) with
    the FP64 kernels: their values are the FP64 mode's, bit for bit."""
    p, flat = case
    got, _ = _run(p, flat, strategy)
    exact, _ = _run(p, flat, strategy, precision=pb.FP64)
    be = pb.CUDAComputeBackend(0)
    try:
        inp = pb.InterpolationInput(p["x"], p["y"], p["z"], p["m"], p["h"], p["rho"], ())
        lb = pb.LinearBVH_build(inp, be)
        acc = pb.traversal_stats(lb, flat.coor, strategy)[:, 4]
    finally:
        be.close()
    light = acc <= 4096
    assert light.any() and (~light).any()
    assert np.array_equal(got[:, light].view(np.uint64), exact[:, light].view(np.uint64))
    alt, _ = _run(p, flat, strategy, options=(("fp64_light_max", 0),))
    nonempty = light & (acc > 0)
    assert not np.array_equal(alt[:, nonempty].view(np.uint64), exact[:, nonempty].view(np.uint64))
