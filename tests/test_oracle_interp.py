"""Interpolation semantics of the oracle against independent brute-force evaluators.

The brute-force evaluators restate Partia.jl/test/interpolation_test_common.jl:15-335 (an
O(N) loop over all particles with the acceptance predicate d2 <= (K*h_sel)^2, h_sel = ha
(gather), hb (scatter) or max(ha, hb) (symmetric), ha = smoothing length of the nearest
particle) in vectorised numpy.  Tolerances are the reference's (atol 1e-12, rtol 1e-10,
Partia.jl/test/point_samples_interpolation_tests.jl:30-31).  Also covered: the
no-neighbour behaviour (all outputs NaN, general_interpolation.jl:128-131), vanishing
divergence and curl of a uniform field (interpolation_tests.jl:302-333), and the analytic
linear-field regression on a uniform lattice (point_samples_interpolation_tests.jl:84-112).
"""
import math

import numpy as np
import pytest

import oracle
from golden import load

SIG = 1.0 / math.pi
STRATS = ["itpGather", "itpScatter", "itpSymmetric"]


def f_m4(q):
    a = np.clip(2 - q, 0, None)
    b = np.clip(1 - q, 0, None)
    return 0.25 * a ** 3 - b ** 3


def df_m4(q):
    a = np.clip(2 - q, 0, None)
    b = np.clip(1 - q, 0, None)
    return -0.75 * a ** 2 + 3 * b ** 2


def W(r, h):
    return SIG / h ** 3 * f_m4(r / h)


def gW(d, r, h):
    with np.errstate(invalid="ignore", divide="ignore"):
        c = np.where(r > 0, SIG / h ** 4 * df_m4(r / h) / np.where(r > 0, r, 1), 0.0)
    return d * c


def brute(p, P, cols, cat, strategy):
    """General interpolation at point p by brute force; returns the L outputs."""
    x, y, z, m, h, rho = (P[k] for k in ("x", "y", "z", "m", "h", "rho"))
    d = np.stack([p[0] - x, p[1] - y, p[2] - z])
    d2 = (d ** 2).sum(0)
    ha = h[np.argmin(d2)]
    hs = {"itpGather": np.full_like(h, ha), "itpScatter": h, "itpSymmetric": np.maximum(ha, h)}[strategy]
    sel = d2 <= (2.0 * hs) ** 2
    r = np.sqrt(d2)
    if strategy == "itpSymmetric":
        w = 0.5 * (W(r, ha) + W(r, h))
        g = 0.5 * (gW(d, r, ha) + gW(d, r, h))
    else:
        hh = ha if strategy == "itpGather" else h
        w, g = W(r, hh), gW(d, r, hh)
    w, g = np.where(sel, w, 0.0), np.where(sel, g, 0.0)
    wt = m * w / rho
    S1 = wt.sum()
    L = len(cat["scalar_cols"]) + 3 * len(cat.get("grad_cols", [])) + len(cat.get("div_cols", [])) + \
        3 * len(cat.get("curl_cols", []))
    if S1 == 0:
        return np.full(L, np.nan)
    out = []
    for c, sh in zip(cat["scalar_cols"], cat["scalar_shepard"]):
        s = (cols[c] * wt).sum()
        out.append(s / S1 if sh else s)
    gq = m / rho * g
    B = gq.sum(1)
    for c in cat.get("grad_cols", []):
        if c < 0:
            F, Bd, A = (m * g).sum(1), (m / rho * g).sum(1), (m * w).sum() / S1
            out += list(F - A * Bd)
        else:
            A = (cols[c] * wt).sum() / S1
            out += list((gq * cols[c]).sum(1) - A * B)
    for cx, cy, cz in cat.get("div_cols", []):
        V = np.stack([cols[cx], cols[cy], cols[cz]])
        Abar = (V * wt).sum(1) / S1
        out.append((gq * V).sum() - Abar @ B)
    for cx, cy, cz in cat.get("curl_cols", []):
        V = np.stack([cols[cx], cols[cy], cols[cz]])
        Abar = (V * wt).sum(1) / S1
        C = np.cross(V.T, gq.T).sum(0)
        out += list(-(C - np.cross(Abar, B)))
    return np.array(out)


def _oracle(P, cols):
    return oracle.OracleLBVH(P["x"], P["y"], P["z"], P["h"]).attach(P["m"], P["rho"], cols, "M4_spline")


def _check(P, cols, cat, q, strategy, atol=1e-12, rtol=1e-10):
    o = _oracle(P, cols)
    got = o.interp_points(cat, *q, strategy=strategy)
    for i in range(q.shape[1]):
        exp = brute(q[:, i], P, cols, cat, strategy)
        np.testing.assert_allclose(got[:, i], exp, atol=atol, rtol=rtol, equal_nan=True)


FULL = {"scalar_cols": [0, 1], "scalar_shepard": [1, 1], "grad_cols": [0, -1], "div_cols": [[1, 2, 3]],
        "curl_cols": [[1, 2, 3]]}


@pytest.mark.parametrize("strategy", STRATS)
def test_reference_fixture(strategy):
    fx = load("grid_interpolation_fixture")
    P = {k: np.array(v) for k, v in fx["particles"].items()}
    cols = [P["temp"], P["vx"], P["vy"], P["vz"]]
    q = np.array(fx["point_samples"])
    _check(P, cols, FULL, q, strategy)


@pytest.mark.parametrize("strategy", STRATS)
def test_random_set(strategy):
    g = np.random.default_rng(0xBADA55)
    n = 300
    P = {"x": g.random(n), "y": g.random(n), "z": g.random(n), "m": g.random(n) * 0.1 + 0.01,
         "h": g.random(n) * 0.1 + 0.05, "rho": g.random(n) + 0.5}
    cols = [g.normal(size=n) for _ in range(4)]
    q = g.random((3, 25))
    _check(P, cols, FULL, q, strategy)


def test_no_neighbour_gives_nan():
    g = np.random.default_rng(0xDEAD)
    n = 20
    P = {"x": g.random(n), "y": g.random(n), "z": g.random(n), "m": np.ones(n), "h": np.full(n, 1e-3),
         "rho": np.ones(n)}
    cols = [np.ones(n)] * 4
    o = _oracle(P, cols)
    for s in ("itpScatter",):
        out = o.interp_points(FULL, [2.0], [2.0], [2.0], strategy=s)
        assert np.isnan(out).all()


def test_uniform_field_has_zero_div_and_curl():
    x = np.array([0.0, 0.05, 0.11, -0.08])
    y = np.array([0.02, -0.03, 0.04, 0.01])
    z = np.array([0.0, 0.01, -0.02, 0.03])
    n = 4
    P = {"x": x, "y": y, "z": z, "m": np.ones(n), "h": np.full(n, 0.12), "rho": np.ones(n)}
    cols = [np.full(n, 1.0), np.full(n, -2.0), np.full(n, 0.5)]
    cat = {"scalar_cols": [], "scalar_shepard": [], "div_cols": [[0, 1, 2]], "curl_cols": [[0, 1, 2]]}
    o = _oracle(P, cols)
    for s in STRATS:
        out = o.interp_points(cat, [x[0]], [y[0]], [z[0]], strategy=s)
        assert np.abs(out).max() <= 1e-12


def uniform_cloud(nx, eta=1.2, variable_h=True):
    dx = 1.0 / nx
    c = np.arange(dx / 2, 1.0, dx)[:nx]
    X, Y, Z = np.meshgrid(c, c, c, indexing="ij")
    x, y, z = X.ravel(), Y.ravel(), Z.ravel()
    n = len(x)
    h = eta * dx * (1.0 + 0.18 * (x - 0.5) - 0.10 * (y - 0.5) + 0.08 * (z - 0.5)) if variable_h else np.full(n, eta * dx)
    P = {"x": x, "y": y, "z": z, "m": np.full(n, dx ** 3), "h": h, "rho": np.ones(n)}
    cols = [x + y + z, x.copy(), y.copy(), z.copy()]
    return P, cols


@pytest.mark.parametrize("strategy", STRATS)
def test_analytic_linear_field(strategy):
    P, cols = uniform_cloud(12)
    cat = {"scalar_cols": [0], "scalar_shepard": [1], "grad_cols": [0], "div_cols": [[1, 2, 3]],
           "curl_cols": [[1, 2, 3]]}
    q = np.array([[0.35, 0.45, 0.55], [0.40, 0.50, 0.45], [0.45, 0.35, 0.50]])
    out = _oracle(P, cols).interp_points(cat, *q, strategy=strategy)
    for i in range(3):
        p = q[:, i]
        assert out[0, i] == pytest.approx(p.sum(), abs=2e-2, rel=1e-2)
        for d in range(3):
            assert out[1 + d, i] == pytest.approx(1.0, abs=6e-2, rel=1e-2)
        assert out[4, i] == pytest.approx(3.0, abs=1e-1, rel=2e-2)
        for d in range(3):
            assert out[5 + d, i] == pytest.approx(0.0, abs=5e-2)
