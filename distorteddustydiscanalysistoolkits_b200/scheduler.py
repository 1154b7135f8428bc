"""Learned work prediction for the point-interpolation schedule.

A 3-layer BF16 MLP of width 64 predicts, for each sample point, log2(1 + accepted
neighbours) from 16 features the library computes on the device before the walk
(``FEATURES``).  It is trained on the GPU by the library's own forward/backward/Adam kernels
(``pb_scheduler_train``) on exact neighbour counts that the plain traversal itself produces
(``pb_traversal_stats``), on held-out seeded discs.  With option ``schedule = LEARNED`` the
walk takes the queries binned by predicted work, heaviest class first (Morton order inside a
class), so the 32 queries of a walk warp carry similar work.  Only the order changes; the
outputs are bit-identical to the plain schedule (``PLAIN``), which stays the fallback.
"""
import ctypes
import os

import numpy as np

from . import _lib
from .neighbor import traversal_stats

PLAIN, TUNED, LEARNED = 0, 1, 2
FEATURES = ("log2 h_nearest", "log2 d_nearest/extent", "x/extent", "y/extent", "z/extent", "log2 |p|/extent") + \
    tuple("%s (subtree >= 2^%d)" % (k, l) for l in (4, 8, 12, 16, 20) for k in ("log2 hmax", "log2 half-diagonal"))
NF, NPARAM = _lib.SCHED_FEATURES, _lib.SCHED_PARAMS
MODEL_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "sched_mlp.npz")


class Model:
    """Weights (PB_SCHED_PARAMS floats), input normalisation (mean, 1/std) and bin width."""

    def __init__(self, params, norm, bin_width=1.0, nclass=24, meta=None):
        self.params = np.ascontiguousarray(params, np.float32)
        self.norm = np.ascontiguousarray(norm, np.float32)
        self.bin_width = float(bin_width)
        self.nclass = int(nclass)
        self.meta = dict(meta or {})
        assert self.params.shape == (NPARAM,) and self.norm.shape == (2 * NF,)

    def save(self, path=MODEL_PATH):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez(path, params=self.params, norm=self.norm, bin_width=self.bin_width, nclass=self.nclass,
                 meta=np.array(repr(self.meta)))

    @classmethod
    def load(cls, path=MODEL_PATH):
        z = np.load(path)
        return cls(z["params"], z["norm"], float(z["bin_width"]), int(z["nclass"]), {"file": os.path.basename(path)})


def init_params(seed=0):
    """He-normal weights, zero biases."""
    g = np.random.default_rng(seed)
    H = 64
    parts = [g.normal(0, np.sqrt(2.0 / NF), H * NF), np.zeros(H), g.normal(0, np.sqrt(2.0 / H), H * H), np.zeros(H),
             g.normal(0, np.sqrt(1.0 / H), H), np.zeros(1)]
    return np.concatenate(parts).astype(np.float32)


def normalisation(X):
    mu = X.mean(0)
    sd = X.std(0)
    return np.concatenate([mu, 1.0 / np.where(sd > 1e-6, sd, 1.0)]).astype(np.float32)


def features(lbvh, points):
    """(N, 16) float32 features of sample points on the last build of ``lbvh``'s handle."""
    qx, qy, qz = (np.ascontiguousarray(c, np.float64) for c in points)
    n = len(qx)
    out = np.empty((n, NF), np.float32)
    H = lbvh.handle
    H.check(H.lib.pb_scheduler_features(H.h, n, qx.ctypes.data, qy.ctypes.data, qz.ctypes.data, out.ctypes.data),
            "scheduler_features")
    return out


def labels(lbvh, points, strategy):
    """log2(1 + exact accepted-neighbour count) of each point, from the reference traversal."""
    st = traversal_stats(lbvh, points, strategy)
    return np.log2(1.0 + st[:, 4].astype(np.float64)).astype(np.float32)


def set_model(handle, model):
    handle.check(handle.lib.pb_scheduler_set(handle.h, model.params.ctypes.data, model.norm.ctypes.data,
                                             ctypes.c_float(model.bin_width), model.nclass), "scheduler_set")


def predict(handle, model, X):
    set_model(handle, model)
    X = np.ascontiguousarray(X, np.float32)
    out = np.empty(len(X), np.float32)
    handle.check(handle.lib.pb_scheduler_predict(handle.h, X.ctypes.data, len(X), out.ctypes.data), "predict")
    return out


def gradients(handle, model, X, y):
    """Gradient of the batch MSE (PB_SCHED_PARAMS floats) and the loss, computed on the device."""
    set_model(handle, model)
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    g = np.empty(NPARAM, np.float32)
    loss = ctypes.c_float()
    handle.check(handle.lib.pb_scheduler_gradients(handle.h, X.ctypes.data, y.ctypes.data, len(y), g.ctypes.data,
                                                   ctypes.byref(loss)), "gradients")
    return g, loss.value


def train(handle, X, y, steps=3000, batch=4096, lr=2e-3, seed=0, init=None, bin_width=1.0, nclass=24):
    """Train on the device from ``init`` (He-normal by default); returns (Model, per-step losses)."""
    X = np.ascontiguousarray(X, np.float32)
    y = np.ascontiguousarray(y, np.float32)
    model = Model(init_params(seed) if init is None else init, normalisation(X), bin_width, nclass)
    set_model(handle, model)
    losses = np.empty(steps, np.float32)
    handle.check(handle.lib.pb_scheduler_train(handle.h, X.ctypes.data, y.ctypes.data, len(y), steps, batch,
                                               ctypes.c_float(lr), ctypes.c_uint64(seed), losses.ctypes.data),
                 "scheduler_train")
    p = np.empty(NPARAM, np.float32)
    handle.check(handle.lib.pb_scheduler_get(handle.h, p.ctypes.data), "scheduler_get")
    model.params = p
    return model, losses


def use(backend, model=None, mode=LEARNED):
    """Load ``model`` (the shipped one by default) into the backend and select the schedule."""
    H = backend.handle
    if mode == LEARNED:
        set_model(H, model or Model.load())
    H.set_option("schedule", mode)
