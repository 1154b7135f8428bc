"""The CPU oracle of the work-prediction MLP against finite differences (float64, no rounding),
and its bfloat16 rounding against the definition (nearest, ties to even)."""
import numpy as np

from oracle import mlp_oracle as mo


def test_bf16_rounding():
    x = np.array([1.0, 1.00390625, 1.005859375, 1.0078125, -3.14159, 0.0, 1e-40], np.float32)
    r = mo.bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0            # halfway between 1 and 1+2^-7 rounds to even (1)
    assert r[2] == np.float32(1.0078125)          # above halfway rounds up
    assert r[3] == np.float32(1.0078125)
    assert abs(r[4] + 3.140625) < 1e-6
    bits = r.view(np.uint32)
    assert (bits & 0xFFFF).max() == 0


def test_backward_matches_finite_differences():
    g = np.random.default_rng(3)
    p = g.normal(0, 0.3, mo.NPARAM)
    norm = np.concatenate([g.normal(0, 1, mo.F), np.exp(g.normal(0, 0.3, mo.F))])
    X = g.normal(0, 1, (40, mo.F))
    T = g.normal(0, 1, 40)
    loss, grad = mo.loss_and_grad(p, norm, X, T, bf=False, dtype=np.float64)
    idx = g.choice(mo.NPARAM, 60, replace=False)
    eps = 1e-6
    for i in idx:
        q = p.copy()
        q[i] += eps
        lp, _ = mo.loss_and_grad(q, norm, X, T, bf=False, dtype=np.float64)
        q[i] -= 2 * eps
        lm, _ = mo.loss_and_grad(q, norm, X, T, bf=False, dtype=np.float64)
        fd = (lp - lm) / (2 * eps)
        assert abs(fd - grad[i]) <= 1e-6 + 1e-5 * abs(fd), (i, fd, grad[i])
