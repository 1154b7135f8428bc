"""Host side of the learned schedule (no GPU): the shipped model file, its save/load round trip,
parameter layout and normalisation."""
import numpy as np

from distorteddustydiscanalysistoolkits_b200 import scheduler
from oracle import mlp_oracle as mo


def test_shipped_model_loads_with_the_documented_layout():
    m = scheduler.Model.load()
    assert m.params.shape == (scheduler.NPARAM,) == (mo.NPARAM,)
    assert m.norm.shape == (2 * scheduler.NF,)
    assert np.isfinite(m.params).all() and np.isfinite(m.norm).all() and (m.norm[scheduler.NF:] > 0).all()
    assert m.bin_width > 0 and m.nclass >= 1
    assert len(scheduler.FEATURES) == scheduler.NF == mo.F


def test_model_round_trip(tmp_path):
    g = np.random.default_rng(5)
    X = g.normal(3, 2, (500, scheduler.NF)).astype(np.float32)
    norm = scheduler.normalisation(X)
    np.testing.assert_allclose(norm[:scheduler.NF], X.mean(0), rtol=1e-5)
    m = scheduler.Model(scheduler.init_params(3), norm, bin_width=0.5, nclass=12)
    path = str(tmp_path / "m.npz")
    m.save(path)
    r = scheduler.Model.load(path)
    assert np.array_equal(r.params, m.params) and np.array_equal(r.norm, m.norm)
    assert r.bin_width == 0.5 and r.nclass == 12
    y, _ = mo.forward(r.params, r.norm, X)
    assert np.isfinite(y).all()
