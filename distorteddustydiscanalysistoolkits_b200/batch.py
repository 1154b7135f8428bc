"""Batches of snapshots and grids of uneven size, with an autotuned schedule.

``c4_discs`` generates the batched workload: seeded discs (seeds 100 + k) with log-uniform
particle counts, each with its own Cartesian grid (edge drawn from a set of sizes) and a random
tilt.  ``batch_point_interpolation`` runs every job on one handle and one stream: buffers stay
resident and only grow, and each job runs with the schedule options ``Autotuner`` picked for
its size class.  The options change only the schedule, so a batch gives the same bits as
separate calls (tests/test_gpu_batch.py).

The autotuner times the interpolation of a representative job of each size class (particles
and points rounded to powers of 4) under every candidate setting of the walk split, the slice
size and the scheduler bin width, and keeps the fastest.
"""
import itertools
import math
import time

import numpy as np

from . import scheduler, synthetic
from .grids import Cartesian, flatten
from .interpolation import (C4_Wendland, InterpolationCatalog, InterpolationInput, M4_spline,
                            PointSamples_interpolation, FP32C, itpSymmetric)


def c4_discs(n_discs=64, seed=100, n_min=50_000, n_max=4_000_000, edges=(32, 64, 128, 256)):
    """Descriptors (seed, particles, grid edge, tilt) of the batched workload."""
    out = []
    for k in range(n_discs):
        g = np.random.default_rng(seed + k)
        n = int(round(math.exp(g.uniform(math.log(n_min), math.log(n_max)))))
        out.append({"seed": seed + k, "particles": n, "edge": int(g.choice(edges)), "tilt": float(g.uniform(0.0, 30.0))})
    return out


def make_job(desc, columns=("rho",), kernel=M4_spline):
    """Particles, flattened grid points and catalog (scalar + gradient of rho) of one disc."""
    p = synthetic.disc(desc["particles"], seed=desc["seed"], tilt_deg=desc["tilt"])
    flat = flatten(Cartesian, synthetic.cartesian_box_grid(p, n=desc["edge"]))
    inp = InterpolationInput(p["x"], p["y"], p["z"], p["m"], p["h"], p["rho"], tuple(p[c] for c in columns),
                             smoothed_kernel=kernel)
    cat = InterpolationCatalog(columns, scalars=("rho",), gradients=("rho",))
    return {"desc": desc, "input": inp, "points": flat, "catalog": cat}


def size_class(n_particles, n_points):
    return (int(round(math.log(max(n_particles, 1), 4))), int(round(math.log(max(n_points, 1), 4))))


class Autotuner:
    """Per size class, the fastest of the candidate schedule options (results are unaffected)."""

    def __init__(self, walk_split=(16, 32, 64, 128), slice_queries=(1 << 20, 1 << 22), bin_width=(0.5, 1.0, 2.0),
                 repeats=2):
        self.grid = {"walk_split": walk_split, "slice_queries": slice_queries, "bin_width": bin_width}
        self.repeats = repeats
        self.table = {}
        self.timings = {}

    def options(self, job):
        return self.table.get(size_class(job["input"].Npart, len(job["points"])))

    def tune(self, backend, job, strategy=itpSymmetric, precision=FP32C):
        key = size_class(job["input"].Npart, len(job["points"]))
        if key in self.table:
            return self.table[key]
        H = backend.handle
        H.set_option("timing", 1)
        model = scheduler.Model.load() if self._have_model() else None
        best, best_ms, tried = None, math.inf, []
        for ws, sq, bw in itertools.product(*self.grid.values()):
            opts = {"walk_split": ws, "slice_queries": sq, "bin_width": bw}
            apply_options(backend, opts, model)
            ms = []
            for _ in range(self.repeats + 1):
                PointSamples_interpolation(backend, job["points"], job["input"], job["catalog"], strategy,
                                           precision=precision)
                ms.append(H.timings()[1])
            t = float(np.min(ms[1:]))
            tried.append((opts, t))
            if t < best_ms:
                best, best_ms = opts, t
        self.table[key] = best
        self.timings[key] = tried
        return best

    @staticmethod
    def _have_model():
        import os
        return os.path.exists(scheduler.MODEL_PATH)


def apply_options(backend, opts, model=None):
    H = backend.handle
    H.set_option("walk_split", int(opts["walk_split"]))
    H.set_option("slice_queries", int(opts["slice_queries"]))
    if model is not None:
        m = scheduler.Model(model.params, model.norm, opts.get("bin_width", model.bin_width), model.nclass)
        scheduler.set_model(H, m)
        H.set_option("schedule", scheduler.LEARNED)
    else:
        H.set_option("schedule", scheduler.TUNED)


def batch_point_interpolation(backend, jobs, tuner=None, strategy=itpSymmetric, precision=FP32C):
    """Interpolate every job on one handle; returns (list of GridBundle, list of per-job ms)."""
    model = scheduler.Model.load() if Autotuner._have_model() else None
    H = backend.handle
    H.set_option("timing", 1)
    out, ms = [], []
    for job in jobs:
        if tuner is not None:
            opts = tuner.options(job) or tuner.tune(backend, job, strategy, precision)
            apply_options(backend, opts, model)
        t0 = time.perf_counter()
        out.append(PointSamples_interpolation(backend, job["points"], job["input"], job["catalog"], strategy,
                                              precision=precision))
        b, i, _ = H.timings()
        ms.append({"build_ms": b, "interp_ms": i, "wall_ms": (time.perf_counter() - t0) * 1e3})
    return out, ms
