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


def clumped_disc(n, seed=5, mass=None, tilt_deg=30.0, n_clumps=2000, clump_fraction=0.1, pitch_deg=12.0,
                 arm_contrast=5.0, arm_width=0.1, rmin=1.0, rmax=100.0):
    """Disc with two logarithmic spiral arms and Gaussian clumps (about 100x spread in h).

    The base disc is ``disc``'s (Sigma ~ 1/r, H = 0.05 r^1.25, warp ramping to ``tilt_deg``);
    its azimuths follow two log spirals phi_arm = phi0 + ln(r) / tan(pitch) (+ pi) with a
    Gaussian profile of width ``arm_width`` rad and an arm/inter-arm density contrast
    ``arm_contrast``.  ``n_clumps`` Gaussian clumps (centres drawn from the disc, sigma
    log-uniform in [0.05, 0.5] H(r)) share ``clump_fraction`` of the particles equally.  Every
    particle has the same mass (total 1 unless given); h = 1.2 (m/rho)^(1/3) from the analytic
    density of its own component."""
    g = _rng(seed)
    m = (1.0 / n) if mass is None else mass
    n_cl_each = int(n * clump_fraction) // n_clumps
    n_cl = n_cl_each * n_clumps
    nd = n - n_cl
    r = g.uniform(rmin, rmax, nd)
    # azimuths by rejection against the arm profile w(phi) = 1 + (c - 1) exp(-dphi^2 / 2 w^2)
    k = 1.0 / math.tan(math.radians(pitch_deg))
    phi0 = g.uniform(0.0, 2.0 * np.pi)
    phi = np.empty(nd)
    todo = np.arange(nd)
    while len(todo):
        cand = g.uniform(0.0, 2.0 * np.pi, len(todo))
        d = np.mod(cand - (phi0 + k * np.log(r[todo])), np.pi)
        d = np.minimum(d, np.pi - d)
        w = 1.0 + (arm_contrast - 1.0) * np.exp(-d * d / (2.0 * arm_width ** 2))
        ok = g.uniform(0.0, arm_contrast, len(todo)) < w
        phi[todo[ok]] = cand[ok]
        todo = todo[~ok]
    d = np.mod(phi - (phi0 + k * np.log(r)), np.pi)
    d = np.minimum(d, np.pi - d)
    w = 1.0 + (arm_contrast - 1.0) * np.exp(-d * d / (2.0 * arm_width ** 2))
    wmean = 1.0 + (arm_contrast - 1.0) * arm_width * math.sqrt(2.0 * math.pi) / np.pi
    H = 0.05 * r ** 1.25
    zp = g.normal(0.0, 1.0, nd) * H
    sigma = nd * m / (2.0 * np.pi * (rmax - rmin) * r)
    rho = sigma / (math.sqrt(2.0 * np.pi) * H) * np.exp(-zp * zp / (2.0 * H * H)) * w / wmean
    # clumps: centres drawn from the disc particles, isotropic Gaussians
    ci = g.integers(0, nd, n_clumps)
    cr, cphi, cz = r[ci], phi[ci], zp[ci]
    csig = np.exp(g.uniform(math.log(0.05), math.log(0.5), n_clumps)) * (0.05 * cr ** 1.25)
    off = g.normal(0.0, 1.0, (3, n_cl)) * np.repeat(csig, n_cl_each)
    cx0 = np.repeat(cr * np.cos(cphi), n_cl_each) + off[0]
    cy0 = np.repeat(cr * np.sin(cphi), n_cl_each) + off[1]
    cz0 = np.repeat(cz, n_cl_each) + off[2]
    q2 = (off ** 2).sum(0) / np.repeat(csig, n_cl_each) ** 2
    rho_c = n_cl_each * m / ((2.0 * np.pi) ** 1.5 * np.repeat(csig, n_cl_each) ** 3) * np.exp(-0.5 * q2)
    x0 = np.concatenate([r * np.cos(phi), cx0])
    y0 = np.concatenate([r * np.sin(phi), cy0])
    z0 = np.concatenate([zp, cz0])
    rho = np.concatenate([rho, rho_c])
    rr = np.sqrt(x0 * x0 + y0 * y0)
    h = 1.2 * (m / rho) ** (1.0 / 3.0)
    beta = np.deg2rad(tilt_deg) * (np.clip(rr, rmin, rmax) - rmin) / (rmax - rmin)
    cb, sb = np.cos(beta), np.sin(beta)
    vk = np.maximum(rr, rmin) ** -0.5
    ph = np.arctan2(y0, x0)
    vx0, vy0 = -vk * np.sin(ph), vk * np.cos(ph)
    noise = g.normal(0.0, 1.0, (3, n)) * (0.01 * vk)
    return {"x": x0, "y": y0 * cb - z0 * sb, "z": y0 * sb + z0 * cb, "m": np.full(n, m), "h": h, "rho": rho,
            "vx": vx0 + noise[0], "vy": vy0 * cb + noise[1], "vz": vy0 * sb + noise[2]}


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
