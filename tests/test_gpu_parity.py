"""GPU parity: the CUDA library against the CPU oracle on the same seeded inputs.

Bit-exact: Morton codes, sort order, tree topology, FP64 boxes/hmax, nearest leaves,
neighbour lists (DFS order), and every FP64-mode interpolated value (the FP64 kernels run
the reference's expressions in the reference's order, so equality is exact, NaN included).
FP32-compensated mode: |gpu - oracle| <= 1e-5 * max|field| per field (the FP32 tolerance,
scaled per field because several fields -- div v of a Keplerian flow, grad rho at the
midplane -- pass through zero).  With the default routing (queries of at most 4096 accepted
neighbours summed in FP64) the density, a field that does not change sign, also meets
|gpu - oracle| / |oracle| <= 1e-5 at every point.  The FP32 pair kernel itself is pinned by
runs that send every query to it (option fp64_light_max = 0); there only the field-scaled
bound is asserted: a query with a handful of neighbours near the edge of their support gets
its value from kernel terms f(q) = (2 - q)^3 / 4 whose condition number 3q / (2 - q) grows
without bound, so an FP32 evaluation of such a point can be off by far more than 1e-5 of its
own (tiny) value -- the reason those queries are routed to FP64 by default.  The pointwise
relative error of every field is computed (accuracy.field_errors) and printed.
"""
import numpy as np
import pytest

import distorteddustydiscanalysistoolkits_b200 as pb
from distorteddustydiscanalysistoolkits_b200 import accuracy, synthetic
import oracle

pytestmark = pytest.mark.gpu

COLS = ("rho", "vx", "vy", "vz")
FP32_TOL = 1e-5


def _prime_coords(n, off, dim=3):
    primes = (37, 61, 97, 131, 197, 263)
    return [np.array([((primes[d] * i + primes[d + dim] * off) % 1021) / 1021 for i in range(1, n + 1)])
            for d in range(dim)]


def _input(p, cols=COLS, kernel=pb.M4_spline):
    return pb.InterpolationInput(p["x"].copy(), p["y"].copy(), p["z"].copy(), p["m"].copy(), p["h"].copy(),
                                 p["rho"].copy(), tuple(p[c].copy() for c in cols), smoothed_kernel=kernel)


def _oracle(p, cols=COLS, kernel="M4_spline"):
    return oracle.OracleLBVH(p["x"], p["y"], p["z"], p["h"]).attach(p["m"], p["rho"], [p[c] for c in cols], kernel)


def _assert_same(a, b):
    a, b = np.asarray(a), np.asarray(b)
    assert a.shape == b.shape
    na, nb = np.isnan(a), np.isnan(b)
    assert np.array_equal(na, nb), "NaN positions differ (%d vs %d)" % (na.sum(), nb.sum())
    diff = a[~na] != b[~nb]
    assert not diff.any(), "%d values differ, max |diff| %g" % (diff.sum(), np.max(np.abs(a[~na] - b[~nb])))


def _check_build(backend, x, y, z, h):
    n = len(x)
    one = np.ones(n)
    inp = pb.InterpolationInput(x.copy(), y.copy(), z.copy(), one.copy(), h.copy(), one.copy(), ())
    lb = pb.LinearBVH_build(inp, backend)
    codes, order = lb.encoding()
    t = lb.tree()
    o = oracle.OracleLBVH(x, y, z, h)
    assert np.array_equal(codes, o.codes)
    assert np.array_equal(order, o.order)
    assert t["root"] == o.root
    for k in ("left", "right", "escape", "parent"):
        assert np.array_equal(t[k], getattr(o, k)), k
    if n > 1:
        for k in ("bmin", "bmax", "hmax"):
            assert np.array_equal(t[k], getattr(o, k)), k
    # the reference permutes the caller's arrays in place
    assert np.array_equal(inp.coord[0], x[order]) and np.array_equal(inp.h, h[order])
    return lb, o


@pytest.mark.parametrize("n", [1, 2, 3, 5, 17, 257, 4096, 100003])
def test_build_bitexact_random(backend, n):
    g = np.random.default_rng(n)
    x, y, z = g.random((3, n)) * 10 - 5
    _check_build(backend, x, y, z, g.random(n) * 0.3 + 0.01)


@pytest.mark.parametrize("off", range(5))
def test_build_prime_hash_coords(backend, off):
    # deterministic coordinates of Partia.jl/test/neighbor_search_tests.jl:49-61
    for n in range(1, 21):
        x, y, z = _prime_coords(n, off)
        _check_build(backend, x, y, z, np.full(n, 0.1))


@pytest.mark.parametrize("n", [2, 8, 16, 1000])
def test_build_identical_and_duplicate_codes(backend, n):
    # identical coordinates: every code equal, the bump makes them consecutive
    _check_build(backend, np.full(n, 0.5), np.full(n, 0.5), np.full(n, 0.5), np.full(n, 0.5))
    # heavy duplicates on a coarse lattice (bump collisions with neighbouring codes)
    g = np.random.default_rng(n)
    x, y, z = (g.integers(0, 3, (3, n)) / 2.0)
    _check_build(backend, x, y, z, np.full(n, 0.2))


def test_build_disc_full_size(backend):
    p = synthetic.disc(1 << 21, seed=2)
    _check_build(backend, p["x"], p["y"], p["z"], p["h"])


def test_nearest_and_query_bitexact(backend):
    p = synthetic.disc(20000, seed=7)
    lb, o = _check_build(backend, p["x"], p["y"], p["z"], p["h"])
    g = np.random.default_rng(1)
    q = [g.uniform(-100, 100, 3000), g.uniform(-100, 100, 3000), g.normal(0, 5, 3000)]
    idx = pb.LBVH_find_nearest(lb, q)
    hh = pb.LBVH_find_nearest_h(lb, q)
    for i in range(0, 3000, 7):
        hv, b = o.find_nearest_h((q[0][i], q[1][i], q[2][i]))
        assert idx[i] == b and hh[i] == hv
    radius = g.uniform(0.5, 6.0, 3000)
    sel = pb.LBVH_query(lb, q, radius)
    for i in range(0, 3000, 11):
        pool, near = o.query((q[0][i], q[1][i], q[2][i]), radius[i])
        assert np.array_equal(sel[i].valid_indices(), pool)
        assert sel[i].nearest == near


def _full_catalog():
    # 2 scalars (rho: no Shepard), column gradient, density gradient (slot 0), div, curl:
    # more than one launch's register budget, so the host splits it
    return pb.InterpolationCatalog.from_slots(
        scalar_names=("rho", "vx"), scalar_slots=(1, 2), grad_names=("rho", "ρ"), grad_slots=(1, 0),
        div_names=("v",), div_slots=((2, 3, 4),), curl_names=("v",), curl_slots=((2, 3, 4),))


@pytest.mark.parametrize("kernel", ["M4_spline", "M5_spline", "M6_spline", "C2_Wendland", "C4_Wendland",
                                    "C6_Wendland"])
@pytest.mark.parametrize("strategy", ["itpGather", "itpScatter", "itpSymmetric"])
def test_points_fp64_bitexact(backend, kernel, strategy):
    p = synthetic.disc(6000, seed=5)
    grid = synthetic.cartesian_box_grid(p, n=14, pad=2.0)
    flat = pb.flatten(pb.Cartesian, grid)
    K = getattr(pb, kernel)
    cat = _full_catalog()
    inp = _input(p, kernel=K)
    out = pb.PointSamples_interpolation(backend, flat, inp, cat, getattr(pb, strategy), precision=pb.FP64)
    got = np.stack([g.grid for g in out.grids])
    exp = _oracle(p, kernel=kernel).interp_points(cat.oracle_dict(), *flat.coor, strategy=strategy)
    assert out.names == cat.ordered_names
    assert np.isfinite(exp).any()
    _assert_same(got, exp)


def _fp32c_run(backend, flat, inp, cat, strategy, light_max):
    """FP32C interpolation with queries of more than `light_max` neighbours on the FP32 pair
    kernel (0: every query); returns the outputs and the handle's pair split."""
    H = backend.handle
    H.set_option("fp64_light_max", light_max)
    try:
        out = pb.PointSamples_interpolation(backend, flat, inp, cat, strategy, precision=pb.FP32C)
        split = H.pair_split()
    finally:
        H.set_option("fp64_light_max", 4096)
    return np.stack([g.grid for g in out.grids]), split


def _check_fp32c(got, exp, names, positive=()):
    assert np.array_equal(np.isnan(got), np.isnan(exp))
    st = accuracy.field_errors(got, exp, names)
    print({k: {m: "%.2e" % v[m] for m in ("max_field_scaled", "max_rel", "rms_rel") if m in v} for k, v in st.items()})
    bad = {k: v["max_field_scaled"] for k, v in st.items() if not v["max_field_scaled"] <= FP32_TOL}
    assert not bad, bad
    for k in positive:
        if k in st:
            assert st[k]["max_rel"] <= FP32_TOL, (k, st[k])
    return st


@pytest.mark.parametrize("light_max", [4096, 0])
@pytest.mark.parametrize("strategy", ["itpGather", "itpScatter", "itpSymmetric"])
def test_points_fp32c_tolerance(backend, strategy, light_max):
    p = synthetic.disc(20000, seed=9)
    grid = synthetic.log_cylindrical_grid(24, 24, 8)
    flat = pb.flatten(pb.Cylindrical, grid)
    cat = pb.InterpolationCatalog(COLS, **synthetic.C2_CATALOG)
    got, (hq, lq, hp, lp) = _fp32c_run(backend, flat, _input(p), cat, getattr(pb, strategy), light_max)
    exp, st = _oracle(p).interp_points(cat.oracle_dict(), *flat.coor, strategy=strategy, stats=True)
    # every accepted pair went through one of the two pair kernels
    assert hp + lp == int(st[:, 4].sum()) and hq + lq == len(flat)
    if light_max == 0:
        # the FP32 pair kernel summed every query that has a neighbour
        assert lp == 0 and hp > 0 and hq == int((st[:, 4] > 0).sum())
    _check_fp32c(got, exp, cat.ordered_names, positive=("rho",) if light_max else ())


@pytest.mark.parametrize("light_max", [4096, 0])
def test_points_density_gradient_fp32c(backend, light_max):
    p = synthetic.disc(20000, seed=13)
    grid = synthetic.cartesian_box_grid(p, n=10)
    flat = pb.flatten(pb.Cartesian, grid)
    cat = _full_catalog()
    got, (hq, lq, hp, lp) = _fp32c_run(backend, flat, _input(p), cat, pb.itpSymmetric, light_max)
    if light_max == 0:
        assert lp == 0 and hp > 0
    exp = _oracle(p).interp_points(cat.oracle_dict(), *flat.coor, strategy="itpSymmetric")
    _check_fp32c(got, exp, cat.ordered_names, positive=("rho",) if light_max else ())


@pytest.mark.parametrize("kernel", ["M5_spline", "M6_spline", "C2_Wendland", "C4_Wendland", "C6_Wendland"])
def test_points_fp32_pair_kernel_every_kernel(backend, kernel):
    """The FP32 pair kernel's shapes of every kernel family against the oracle (every query on it)."""
    p = synthetic.disc(12000, seed=23)
    grid = synthetic.cartesian_box_grid(p, n=10, pad=1.0)
    flat = pb.flatten(pb.Cartesian, grid)
    cat = pb.InterpolationCatalog(COLS, scalars=("rho",), curls=("v",))
    got, (hq, lq, hp, lp) = _fp32c_run(backend, flat, _input(p, kernel=getattr(pb, kernel)), cat, pb.itpSymmetric, 0)
    assert lp == 0 and hp > 0
    exp = _oracle(p, kernel=kernel).interp_points(cat.oracle_dict(), *flat.coor, strategy="itpSymmetric")
    _check_fp32c(got, exp, cat.ordered_names)


@pytest.mark.parametrize("kernel", ["M4_spline", "C4_Wendland"])
def test_lines_fp64_bitexact_and_fp32c(backend, kernel):
    gas, dust = synthetic.dusty_disc(30000, 10000, seed=3)
    for p in (gas, dust):
        lines = synthetic.face_on_lines(p, npix=48)
        cat = pb.InterpolationCatalog(("rho", "vz"), scalars=("rho", "vz"))
        exp = _oracle(p, cols=("rho", "vz"), kernel=kernel).interp_lines(cat.oracle_dict(), lines.origin,
                                                                        lines.direction)
        out = pb.LineSamples_interpolation(backend, lines, _input(p, cols=("rho", "vz"), kernel=getattr(pb, kernel)),
                                           cat, pb.itpScatter, precision=pb.FP64)
        _assert_same(np.stack([g.grid for g in out.grids]), exp)
        out = pb.LineSamples_interpolation(backend, lines, _input(p, cols=("rho", "vz"), kernel=getattr(pb, kernel)),
                                           cat, pb.itpScatter, precision=pb.FP32C)
        got = np.stack([g.grid for g in out.grids])
        assert np.array_equal(np.isnan(got), np.isnan(exp))
        scale = np.nanmax(np.abs(exp), axis=1, keepdims=True)
        assert np.nanmax(np.abs(got - exp) / scale) <= FP32_TOL


def test_oblique_lines_fp64(backend):
    p = synthetic.disc(20000, seed=21)
    g = np.random.default_rng(2)
    n = 500
    d = g.normal(size=(3, n))
    d /= np.linalg.norm(d, axis=0)
    o = [g.uniform(-60, 60, n), g.uniform(-60, 60, n), g.uniform(-5, 5, n)]
    lines = pb.LineSamples(np.zeros(n), o, tuple(d))
    cat = pb.InterpolationCatalog(("rho", "vz"), scalars=("rho", "vz"))
    exp = _oracle(p, cols=("rho", "vz")).interp_lines(cat.oracle_dict(), lines.origin, lines.direction)
    out = pb.LineSamples_interpolation(backend, lines, _input(p, cols=("rho", "vz")), cat, pb.itpScatter)
    _assert_same(np.stack([g.grid for g in out.grids]), exp)


def test_reference_fixture_points_and_lines(backend):
    # the 4-particle fixtures of Partia.jl/test/grid_interpolation_test_common.jl:17-121
    from golden import load
    fx = load("grid_interpolation_fixture")
    p = {k: np.array(v) for k, v in fx["particles"].items()}
    cols = ("temp", "vx", "vy", "vz")
    cat = pb.InterpolationCatalog(cols, scalars=("temp",), divergences=("v",))
    q = [np.array(a) for a in fx["point_samples"]]
    for strategy in ("itpGather", "itpScatter", "itpSymmetric"):
        out = pb.PointSamples_interpolation(backend, pb.PointSamples(np.zeros(len(q[0])), q), _input(p, cols), cat,
                                            getattr(pb, strategy))
        exp = _oracle(p, cols).interp_points(cat.oracle_dict(), *q, strategy=strategy)
        _assert_same(np.stack([g.grid for g in out.grids]), exp)
    lcols = ("temp", "vx")
    lcat = pb.InterpolationCatalog(lcols, scalars=lcols)
    lines = pb.LineSamples(np.zeros(3), [np.array(a) for a in fx["line_origin"]],
                           [np.array(a) for a in fx["line_direction"]])
    out = pb.LineSamples_interpolation(backend, lines, _input(p, lcols), lcat, pb.itpScatter)
    exp = _oracle(p, lcols).interp_lines(lcat.oracle_dict(), lines.origin, lines.direction)
    _assert_same(np.stack([g.grid for g in out.grids]), exp)


def test_structured_grid_interpolation_roundtrip(backend):
    p = synthetic.disc(5000, seed=4)
    grid = pb.StructuredGrid.cylindrical((5.0, 60.0, 6), (0.0, 2 * np.pi, 5), (-3.0, 3.0, 4))
    cat = pb.InterpolationCatalog(COLS, scalars=("rho", "vx"))
    out = pb.StructuredGrid_interpolation(backend, pb.Cylindrical, grid, _input(p), cat, pb.itpSymmetric)
    flat = pb.flatten(pb.Cylindrical, grid)
    exp = _oracle(p).interp_points(cat.oracle_dict(), *flat.coor, strategy="itpSymmetric")
    for l, g in enumerate(out.grids):
        assert g.grid.shape == (6, 5, 4)
        _assert_same(g.grid.reshape(-1, order="F"), exp[l])


def test_probe_neighbors_bitexact(backend):
    """LBVH_probe_neighbors (LinearBVHQueries.jl:22-42): count, closest leaf and its d2."""
    p = synthetic.disc(20000, seed=19)
    lb, o = _check_build(backend, p["x"], p["y"], p["z"], p["h"])
    g = np.random.default_rng(5)
    q = [g.uniform(-100, 100, 2000), g.uniform(-100, 100, 2000), g.normal(0, 5, 2000)]
    radius = g.uniform(0.1, 8.0, 2000)
    radius[:50] = 1e-9   # mostly empty
    cnt, idx, d2 = pb.LBVH_probe_neighbors(lb, q, radius)
    for i in range(0, 2000, 3):
        c, ci, cd = o.probe_neighbors((q[0][i], q[1][i], q[2][i]), radius[i])
        assert cnt[i] == c and idx[i] == ci and d2[i] == cd, i
    assert (idx[cnt == 0] == -1).all() and np.isinf(d2[cnt == 0]).all()


def test_errors(backend):
    p = synthetic.disc(1000, seed=1)
    lines = synthetic.face_on_lines(p, npix=4)
    cat = pb.InterpolationCatalog(("rho",), scalars=("rho",))
    for s in (pb.itpGather, pb.itpSymmetric):
        with pytest.raises(pb.ArgumentError):
            pb.LineSamples_interpolation(backend, lines, _input(p, ("rho",)), cat, s)
    bad = dict(p)
    bad["x"] = p["x"].copy()
    bad["x"][17] = np.nan
    flat = pb.PointSamples(np.zeros(3), (np.zeros(3), np.zeros(3), np.zeros(3)))
    with pytest.raises(pb.ArgumentError):
        pb.PointSamples_interpolation(backend, flat, _input(bad, ("rho",)), cat)
    with pytest.raises(pb.DimensionMismatch):
        pb.InterpolationInput(np.zeros(3), np.zeros(3), np.zeros(2), np.zeros(3), np.zeros(3), np.zeros(3))
    with pytest.raises(KeyError):
        pb.InterpolationCatalog(("rho",), scalars=("temp",))
    # the C ABI's own classes: a catalog column beyond the input's columns is KeyError
    import ctypes
    from distorteddustydiscanalysistoolkits_b200 import _lib
    lb = pb.LinearBVH_build(_input(p, ("rho",)), backend)
    H = lb.handle
    cols = (ctypes.c_int32 * 1)(5)
    shep = (ctypes.c_int32 * 1)(1)
    ccat = _lib.PBCatalog(1, cols, shep, 0, None, 0, None, 0, None)
    o = np.zeros(3)
    optr = (ctypes.c_void_p * 1)(o.ctypes.data)
    z3 = np.zeros(3)
    rc = H.lib.pb_interpolate_points(H.h, ctypes.byref(ccat), 3, z3.ctypes.data, z3.ctypes.data, z3.ctypes.data,
                                     pb.itpSymmetric.code, _lib.PB_FP64, optr)
    assert rc == _lib.PB_ERR_KEY
    # a neighbour pool shorter than the counts is DimensionMismatch
    off = np.array([0, 0, 0, 0], np.int64)
    pool = np.zeros(1, np.int64)
    rr = np.full(3, 1e3)
    rc = H.lib.pb_query_neighbors(H.h, 3, z3.ctypes.data, z3.ctypes.data, z3.ctypes.data, rr.ctypes.data,
                                  off.ctypes.data, pool.ctypes.data, None)
    assert rc == _lib.PB_ERR_DIMENSION
    empty = {k: np.zeros(0) for k in ("x", "y", "z", "m", "h", "rho")}
    with pytest.raises(pb.ArgumentError):
        pb.PointSamples_interpolation(backend, flat, _input(empty, ()), pb.InterpolationCatalog((), scalars=()))
    # the handle stays usable after the errors
    out = pb.PointSamples_interpolation(backend, flat, _input(p, ("rho",)), cat)
    assert len(out.grids) == 1


def test_device_resident_inputs(backend):
    torch = pytest.importorskip("torch")
    p = synthetic.disc(8000, seed=31)
    grid = synthetic.cartesian_box_grid(p, n=8)
    flat = pb.flatten(pb.Cartesian, grid)
    cat = pb.InterpolationCatalog(COLS, **synthetic.C2_CATALOG)
    dev = {k: torch.from_numpy(v.copy()).cuda() for k, v in p.items()}
    inp = pb.InterpolationInput(dev["x"], dev["y"], dev["z"], dev["m"], dev["h"], dev["rho"],
                                tuple(dev[c] for c in COLS), smoothed_kernel=pb.M4_spline)
    lb = pb.LinearBVH_build(inp, backend)
    q = [torch.from_numpy(c.copy()).cuda() for c in flat.coor]
    outs = pb.interpolate_points(lb, cat, q, pb.itpSymmetric, pb.FP64)
    got = np.stack([o.cpu().numpy() for o in outs])
    exp = _oracle(p).interp_points(cat.oracle_dict(), *flat.coor, strategy="itpSymmetric")
    _assert_same(got, exp)
    _, order = lb.encoding()
    assert np.array_equal(dev["x"].cpu().numpy(), p["x"][order])


@pytest.mark.parametrize("strategy", ["itpGather", "itpScatter", "itpSymmetric"])
def test_traversal_stats_match_oracle(backend, strategy):
    p = synthetic.disc(20000, seed=17)
    inp = _input(p)
    lb = pb.LinearBVH_build(inp, backend)
    grid = synthetic.cartesian_box_grid(p, n=12, pad=1.0)
    flat = pb.flatten(pb.Cartesian, grid)
    st = pb.traversal_stats(lb, flat.coor, getattr(pb, strategy))
    cat = pb.InterpolationCatalog(COLS, scalars=("rho",))
    _, exp = _oracle(p).interp_points(cat.oracle_dict(), *flat.coor, strategy=strategy, stats=True)
    assert np.array_equal(st, exp)


def test_c1_full_size_fp64_bitexact(backend):
    """The CPU-runnable configuration at full size: 131,072-particle disc (seed 1), M4, scalar rho
    (no Shepard normalisation for :rho) on a 64^3 Cartesian grid over the disc, FP64,
    itpSymmetric -- every one of the 262,144 values equals the oracle's bit for bit."""
    p = synthetic.disc(131072, seed=1)
    flat = pb.flatten(pb.Cartesian, synthetic.cartesian_box_grid(p, n=64))
    cat = pb.InterpolationCatalog(("rho",), scalars=("rho",))
    assert cat.scalar_snormalization == (False,)
    out = pb.PointSamples_interpolation(backend, flat, _input(p, cols=("rho",)), cat, pb.itpSymmetric,
                                        precision=pb.FP64)
    exp = _oracle(p, cols=("rho",)).interp_points(cat.oracle_dict(), *flat.coor, strategy="itpSymmetric")
    got = np.stack([g.grid for g in out.grids])
    assert np.isfinite(exp).sum() > 0.5 * exp.size
    _assert_same(got, exp)
