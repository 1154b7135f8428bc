"""Seeded synthetic dusty discs and sample grids (the stand-in for real Phantom dumps).

The reference's only data file is missing and it names no public dataset, so workloads
are generated here: Philox-seeded (numpy ``Philox``) gas/dust discs with r ~ U[1, 100]
(Sigma ~ 1/r), z ~ N(0, H) with H = 0.05 r^1.25, smoothing lengths from the analytic
density h = 1.2 (m/rho)^(1/3), a warp (rotation about the x axis by an angle ramping
linearly in r), Keplerian velocities with 1 % Gaussian noise, plus the sample geometries
of the benchmark configurations (Cartesian box, log-radius cylindrical grid, face-on
image lines).
"""
import math

import numpy as np

from .grids import LineSamples, PointSamples, StructuredGrid, Cylindrical, Cartesian, flatten, linrange, steprange


def _rng(seed):
    return np.random.Generator(np.random.Philox(key=int(seed)))


def disc(n, seed=1, mass=1e-6, tilt_deg=15.0, h_scale=1.0, rmin=1.0, rmax=100.0, sigma_total=None):
    """One species.  Returns dict with x, y, z, m, h, rho, vx, vy, vz (float64 arrays)."""
    g = _rng(seed)
    r = g.uniform(rmin, rmax, n)
    phi = g.uniform(0.0, 2.0 * np.pi, n)
    H = 0.05 * r ** 1.25 * h_scale
    zp = g.normal(0.0, 1.0, n) * H
    total = n * mass if sigma_total is None else sigma_total
    sigma = total / (2.0 * np.pi * (rmax - rmin) * r)
    rho = sigma / (math.sqrt(2.0 * np.pi) * H) * np.exp(-zp * zp / (2.0 * H * H))
    h = 1.2 * (mass / rho) ** (1.0 / 3.0)
    beta = np.deg2rad(tilt_deg) * (r - rmin) / (rmax - rmin)
    cb, sb = np.cos(beta), np.sin(beta)
    x0, y0 = r * np.cos(phi), r * np.sin(phi)
    vk = r ** -0.5
    vx0, vy0 = -vk * np.sin(phi), vk * np.cos(phi)
    x = x0
    y = y0 * cb - zp * sb
    z = y0 * sb + zp * cb
    vx = vx0
    vy = vy0 * cb
    vz = vy0 * sb
    noise = g.normal(0.0, 1.0, (3, n)) * (0.01 * vk)
    return {"x": x, "y": y, "z": z, "m": np.full(n, mass), "h": h, "rho": rho,
            "vx": vx + noise[0], "vy": vy + noise[1], "vz": vz + noise[2]}


def dusty_disc(n_gas, n_dust, seed=3, tilt_deg=30.0, dust_to_gas=0.01):
    """Two species: gas, and dust with 0.1 H scale height and the given mass ratio."""
    m_gas = 1e-6
    m_dust = dust_to_gas * m_gas * n_gas / n_dust
    gas = disc(n_gas, seed=seed, mass=m_gas, tilt_deg=tilt_deg)
    dust = disc(n_dust, seed=seed + 7919, mass=m_dust, tilt_deg=tilt_deg, h_scale=0.1)
    return gas, dust


def cartesian_box_grid(p, n=64, pad=0.0):
    """Cartesian n^3 grid spanning the particle bounding box."""
    lo = [float(np.min(p[k])) - pad for k in "xyz"]
    hi = [float(np.max(p[k])) + pad for k in "xyz"]
    return StructuredGrid.cartesian(*[(lo[d], hi[d], n) for d in range(3)])


def log_cylindrical_grid(ns=256, nphi=256, nz=64, rmin=1.0, rmax=100.0):
    """Cylindrical grid with log-spaced radius, half-open phi in [0, 2pi) and z in +-3 H(rmax)."""
    hz = 3.0 * 0.05 * rmax ** 1.25
    s = np.exp(linrange(math.log(rmin), math.log(rmax), ns))
    phi = steprange(0.0, 2.0 * np.pi / nphi, nphi)
    z = linrange(-hz, hz, nz)
    return StructuredGrid(None, (s, phi, z))


def face_on_lines(p, npix=2048):
    """Face-on image: one line per pixel through z = 0 with direction (0, 0, 1)."""
    x = linrange(float(np.min(p["x"])), float(np.max(p["x"])), npix)
    y = linrange(float(np.min(p["y"])), float(np.max(p["y"])), npix)
    X, Y = np.meshgrid(x, y, indexing="ij")
    n = npix * npix
    xo = np.ascontiguousarray(X.reshape(-1, order="F"))
    yo = np.ascontiguousarray(Y.reshape(-1, order="F"))
    return LineSamples(np.zeros(n), (xo, yo, np.zeros(n)), (np.zeros(n), np.zeros(n), np.ones(n)))


def c2_workload(n=1 << 21, seed=2, ns=256, nphi=256, nz=64):
    """Disc of n particles, catalog rho/vx/vy/vz scalars, grad rho, div v, curl v (L = 11),
    on the log-radius cylindrical grid."""
    p = disc(n, seed=seed)
    grid = log_cylindrical_grid(ns, nphi, nz)
    return p, grid, flatten(Cylindrical, grid)


C2_COLUMNS = ("rho", "vx", "vy", "vz")
C2_CATALOG = dict(scalars=("rho", "vx", "vy", "vz"), gradients=("rho",), divergences=("v",), curls=("v",))
