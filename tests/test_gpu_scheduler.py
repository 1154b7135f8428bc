"""Learned work prediction: the device MLP against the CPU oracle, training on the device, and
the learned schedule's outputs against the plain schedule's (bit-identical).

Gradients: the device kernels round weights and layer inputs to bfloat16 and sum in float32;
the oracle does the same in numpy, so gradients agree to float32 summation-order effects
(relative 2e-3 of the largest component).  The gain of the trained network is measured as the
SIMT efficiency of the walk order: sum over queries of the work / (32 x sum over warps of the
largest work in the warp), with work = exact accepted-neighbour counts.
"""
import numpy as np
import pytest

import distorteddustydiscanalysistoolkits_b200 as pb
from distorteddustydiscanalysistoolkits_b200 import scheduler, synthetic
from oracle import mlp_oracle as mo

pytestmark = pytest.mark.gpu


def _model(seed=7):
    g = np.random.default_rng(seed)
    norm = np.concatenate([g.normal(0, 1, mo.F), np.exp(g.normal(0, 0.3, mo.F))]).astype(np.float32)
    return scheduler.Model(scheduler.init_params(seed), norm)


def test_predict_and_gradients_match_oracle(backend):
    m = _model()
    g = np.random.default_rng(11)
    X = g.normal(0, 1.5, (300, mo.F)).astype(np.float32) + m.norm[:mo.F]
    T = g.normal(2, 1, 300).astype(np.float32)
    got = scheduler.predict(backend.handle, m, X)
    exp, _ = mo.forward(m.params, m.norm, X)
    np.testing.assert_allclose(got, exp, rtol=1e-4, atol=1e-4)
    grads, loss = scheduler.gradients(backend.handle, m, X, T)
    eloss, egrads = mo.loss_and_grad(m.params, m.norm, X, T)
    assert abs(loss - eloss) <= 1e-4 * max(1.0, abs(eloss))
    scale = np.abs(egrads).max()
    assert np.abs(grads - egrads).max() <= 2e-3 * scale


def test_training_on_device_reduces_loss(backend):
    p = synthetic.clumped_disc(60000, seed=1003)
    inp = pb.InterpolationInput(p["x"], p["y"], p["z"], p["m"], p["h"], p["rho"], (), smoothed_kernel=pb.C4_Wendland)
    lb = pb.LinearBVH_build(inp, backend)
    flat = pb.flatten(pb.Cartesian, synthetic.cartesian_box_grid(p, n=24))
    X = scheduler.features(lb, flat.coor)
    y = scheduler.labels(lb, flat.coor, pb.itpSymmetric)
    assert np.isfinite(X).all() and np.isfinite(y).all()
    model, losses = scheduler.train(backend.handle, X, y, steps=600, batch=2048, lr=3e-3, seed=2)
    assert losses[-50:].mean() < 0.25 * losses[:10].mean()
    pred = scheduler.predict(backend.handle, model, X)
    assert np.mean((pred - y) ** 2) < 0.25 * np.var(y)


def _interp(p, flat, mode, model=None, strategy=pb.itpSymmetric, slice_queries=None, walk_split=None):
    be = pb.CUDAComputeBackend(0)
    try:
        if model is not None:
            scheduler.set_model(be.handle, model)
        be.handle.set_option("schedule", mode)
        if slice_queries:
            be.handle.set_option("slice_queries", slice_queries)
        if walk_split:
            be.handle.set_option("walk_split", walk_split)
        cols = ("rho", "vx", "vy", "vz")
        inp = pb.InterpolationInput(p["x"].copy(), p["y"].copy(), p["z"].copy(), p["m"].copy(), p["h"].copy(),
                                    p["rho"].copy(), tuple(p[c].copy() for c in cols), smoothed_kernel=pb.C4_Wendland)
        cat = pb.InterpolationCatalog(cols, scalars=("rho",), curls=("v",))
        out = pb.PointSamples_interpolation(be, flat, inp, cat, strategy, precision=pb.FP32C)
        return np.stack([g.grid for g in out.grids])
    finally:
        be.close()


@pytest.mark.parametrize("strategy", [pb.itpSymmetric, pb.itpGather, pb.itpScatter])
def test_learned_schedule_outputs_identical(strategy):
    p = synthetic.clumped_disc(40000, seed=17, n_clumps=50)
    flat = pb.flatten(pb.Cartesian, synthetic.cartesian_box_grid(p, n=20))
    model = _model(3)
    model.bin_width = 0.5
    ref = _interp(p, flat, scheduler.PLAIN, strategy=strategy)
    for mode, kw in ((scheduler.TUNED, {}), (scheduler.LEARNED, {"model": model}),
                     (scheduler.LEARNED, {"model": model, "slice_queries": 1500}),
                     (scheduler.PLAIN, {"slice_queries": 1024})):
        got = _interp(p, flat, mode, strategy=strategy, **kw)
        assert np.array_equal(got.view(np.uint64), ref.view(np.uint64)), (mode, kw)


def _simt_efficiency(work, order):
    w = work[order]
    pad = (-len(w)) % 32
    w = np.concatenate([w, np.zeros(pad)]).reshape(-1, 32)
    return w.sum() / (32.0 * w.max(1).sum())


def test_trained_network_improves_warp_work_balance(backend):
    model = scheduler.Model.load()
    p = synthetic.clumped_disc(1 << 19, seed=4242)
    inp = pb.InterpolationInput(p["x"], p["y"], p["z"], p["m"], p["h"], p["rho"], (), smoothed_kernel=pb.C4_Wendland)
    lb = pb.LinearBVH_build(inp, backend)
    flat = pb.flatten(pb.Cartesian, synthetic.cartesian_box_grid(p, n=48))
    work = pb.traversal_stats(lb, flat.coor, pb.itpSymmetric)[:, 4].astype(np.float64)
    # Morton order of the points on the particle box (10 bits per axis), as the library sorts them
    lo = np.array([p[k].min() for k in "xyz"])
    ext = np.array([p[k].max() for k in "xyz"]) - lo
    q = np.clip(np.stack(flat.coor, 1) - lo, 0, None) / np.where(ext > 0, ext, 1)
    c = np.minimum((np.clip(q, 0, 1) * 1023).astype(np.uint64), 1023)

    def spread(v):
        out = np.zeros_like(v)
        for b in range(10):
            out |= ((v >> np.uint64(b)) & np.uint64(1)) << np.uint64(3 * b)
        return out

    code = (spread(c[:, 0]) << np.uint64(2)) | (spread(c[:, 1]) << np.uint64(1)) | spread(c[:, 2])
    morton = np.argsort(code, kind="stable")
    pred = scheduler.predict(backend.handle, model, scheduler.features(lb, flat.coor))
    cls = np.clip(np.floor(pred[morton] / model.bin_width), 0, model.nclass - 1)
    learned = morton[np.argsort(model.nclass - 1 - cls, kind="stable")]
    e_m = _simt_efficiency(work, morton)
    e_l = _simt_efficiency(work, learned)
    assert e_l > 1.2 * e_m, (e_m, e_l)
