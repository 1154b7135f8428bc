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

``DeviceBatch`` is the one-launch form: every disc's particles, sample points and outputs stay
on the device, each disc has its own handle (its tree), all handles share one stream, and a
step enqueues every disc's LBVH build (PB_BUILD_ASYNC) and one pb_batch_points launch that
interpolates the sample points of all discs.  The step can be captured in a CUDA graph and
replayed.  ``BatchAutotuner`` picks its schedule options -- the walk's leaf size (subtrees of at
most that many leaves scanned linearly), the disc order (given or most work first) and the
blocks per SM -- by timing graph replays; outputs do not depend on them.
"""
import ctypes
import itertools
import math
import time

import numpy as np

from . import _lib, scheduler, synthetic
from .grids import Cartesian, flatten
from .interpolation import (C4_Wendland, CUDAComputeBackend, FP32C, FP64, InterpolationCatalog, InterpolationInput,
                            M4_spline, PointSamples_interpolation, _precision, itpSymmetric)


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


class DeviceBatch:
    """Every job resident on one device, interpolated by one batched launch per step."""

    def __init__(self, jobs, device=0, precision=FP32C, strategy=itpSymmetric):
        import torch
        if not jobs:
            raise ValueError("no jobs")
        self.torch = torch
        self.device = device
        self.precision = _precision(precision)
        self.strategy = strategy
        cat = jobs[0]["catalog"]
        self.catalog = cat
        self.L = cat.L
        dev = "cuda:%d" % device
        self.stream = torch.cuda.Stream(device=dev)
        self.backends = [CUDAComputeBackend(device) for _ in jobs]
        for b in self.backends:
            b.handle.set_stream(self.stream.cuda_stream)
        self.inputs, self.queries, self.outs, self.cin = [], [], [], []
        for job in jobs:
            inp = job["input"]
            t = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.float64)).to(dev)   # noqa: E731
            d = InterpolationInput(t(inp.coord[0]), t(inp.coord[1]), t(inp.coord[2]), t(inp.m), t(inp.h), t(inp.rho),
                                   tuple(t(q) for q in inp.quant), smoothed_kernel=inp.smoothed_kernel)
            self.inputs.append(d)
            self.cin.append(d._c_struct())
            q = [t(c) for c in job["points"].coor]
            self.queries.append(q)
            self.outs.append([torch.empty(len(q[0]), dtype=torch.float64, device=dev) for _ in range(self.L)])
        K = len(jobs)
        self.K = K
        self.ccat = cat._c_struct()
        self.handles = (ctypes.c_void_p * K)(*[b.handle.h.value for b in self.backends])
        self.npts = (ctypes.c_int64 * K)(*[len(q[0]) for q in self.queries])
        self.qptr = [(ctypes.c_void_p * K)(*[q[d].data_ptr() for q in self.queries]) for d in range(3)]
        self.optr = (ctypes.c_void_p * (K * self.L))(*[o.data_ptr() for outs in self.outs for o in outs])
        self.lib = self.backends[0].handle.lib
        self.graph = None

    @property
    def npoints(self):
        return int(sum(self.npts))

    def set_options(self, leaf_size=1, order=0, blocks_per_sm=0, walk_split=16):
        H = self.backends[0].handle
        H.set_option("leaf_size", int(leaf_size))
        H.set_option("batch_walk_split", int(walk_split))
        H.set_option("batch_order", int(order))
        H.set_option("batch_blocks_per_sm", int(blocks_per_sm))

    def _enqueue(self, flags):
        for b, cin in zip(self.backends, self.cin):
            b.handle.check(self.lib.pb_linear_bvh(b.handle.h, ctypes.byref(cin), _lib.PB_BUILD_ASYNC), "LinearBVH!")
        rc = self.lib.pb_batch_points(self.handles, self.K, ctypes.byref(self.ccat), self.npts, self.qptr[0],
                                      self.qptr[1], self.qptr[2], self.optr, self.strategy.code, self.precision,
                                      flags)
        self.backends[0].handle.check(rc, "pb_batch_points")

    def run(self):
        """One step, eagerly: build every disc, interpolate all of them, wait and check."""
        with self.torch.cuda.stream(self.stream):
            self._enqueue(0)

    def capture(self):
        """Record one step (after an eager one has sized every buffer) in a CUDA graph."""
        self.run()
        g = self.torch.cuda.CUDAGraph()
        with self.torch.cuda.graph(g, stream=self.stream):
            self._enqueue(_lib.PB_BATCH_ASYNC)
        self.graph = g
        return g

    def replay(self, check=True):
        with self.torch.cuda.stream(self.stream):   # a graph replays on the current stream
            self.graph.replay()
        if check:
            self.backends[0].handle.check(self.lib.pb_batch_check(self.handles, self.K), "pb_batch_check")

    def timed(self, steps=3, graph=True):
        """Mean ms per step (CUDA events on the batch's stream) over `steps` steps."""
        torch = self.torch
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        self.stream.synchronize()
        with torch.cuda.stream(self.stream):   # the graph replays on the current stream
            e0.record(self.stream)
            for _ in range(steps):
                if graph:
                    self.graph.replay()
                else:
                    self._enqueue(_lib.PB_BATCH_ASYNC)
            e1.record(self.stream)
        e1.synchronize()
        self.backends[0].handle.check(self.lib.pb_batch_check(self.handles, self.K), "pb_batch_check")
        return e0.elapsed_time(e1) / steps

    def outputs(self):
        return [np.stack([o.cpu().numpy() for o in outs]) for outs in self.outs]

    def close(self):
        self.graph = None
        for b in self.backends:
            b.close()


class BatchAutotuner:
    """Schedule options of a DeviceBatch (outputs do not depend on them): every combination of
    the candidates is captured and timed over `repeats` graph replays; the fastest is kept."""

    def __init__(self, leaf_size=(1, 4, 8, 16), order=(0, 1), blocks_per_sm=(0, 2), walk_split=(8, 16, 32),
                 repeats=2):
        self.grid = {"leaf_size": leaf_size, "order": order, "blocks_per_sm": blocks_per_sm, "walk_split": walk_split}
        self.repeats = repeats
        self.best = None
        self.timings = []

    def tune(self, batch):
        best, best_ms = None, math.inf
        for ls, od, bp, ws in itertools.product(*self.grid.values()):
            opts = {"leaf_size": ls, "order": od, "blocks_per_sm": bp, "walk_split": ws}
            batch.set_options(**opts)
            batch.capture()
            ms = batch.timed(self.repeats)
            self.timings.append((opts, ms))
            if ms < best_ms:
                best, best_ms = opts, ms
        batch.set_options(**best)
        batch.capture()
        self.best = best
        return best
