"""Train the work-prediction MLP on held-out seeded discs (run on a CUDA device).

    python -m distorteddustydiscanalysistoolkits_b200.train_scheduler [--particles N] [--grid G] [--out PATH]

For each of the 8 held-out clumped discs (seeds 1001..1008, never used by the benchmarks or
tests) it builds the LBVH, computes the 16 features of every point of a G^3 Cartesian grid
over the disc and of as many uniformly random points, and labels them with the exact
accepted-neighbour counts of the plain reference traversal (itpSymmetric, C4 Wendland
support).  The network is trained on the device by the library's own kernels; the held-out
loss of disc 1008 is reported and the model is written to ``--out``.
"""
import argparse
import json
import sys
import time

import numpy as np

from . import scheduler, synthetic
from .grids import Cartesian, flatten
from .interpolation import CUDAComputeBackend, InterpolationInput, C4_Wendland, itpSymmetric
from .neighbor import LinearBVH_build


def dataset(backend, seed, n, grid):
    p = synthetic.clumped_disc(n, seed=seed)
    inp = InterpolationInput(p["x"], p["y"], p["z"], p["m"], p["h"], p["rho"], (), smoothed_kernel=C4_Wendland)
    lb = LinearBVH_build(inp, backend)
    flat = flatten(Cartesian, synthetic.cartesian_box_grid(p, n=grid))
    g = np.random.default_rng(seed)
    lo = np.array([p[k].min() for k in "xyz"])
    hi = np.array([p[k].max() for k in "xyz"])
    rnd = lo + (hi - lo) * g.random((len(flat), 3))
    pts = [np.concatenate([flat.coor[d], rnd[:, d]]) for d in range(3)]
    return scheduler.features(lb, pts), scheduler.labels(lb, pts, itpSymmetric)


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--particles", type=int, default=1 << 20)
    ap.add_argument("--grid", type=int, default=48)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--out", default=scheduler.MODEL_PATH)
    args = ap.parse_args(argv)
    be = CUDAComputeBackend(0)
    t0 = time.time()
    Xs, ys = [], []
    for seed in range(1001, 1009):
        X, y = dataset(be, seed, args.particles, args.grid)
        Xs.append(X)
        ys.append(y)
    t_data = time.time() - t0
    Xtr, ytr = np.concatenate(Xs[:-1]), np.concatenate(ys[:-1])
    Xte, yte = Xs[-1], ys[-1]
    t0 = time.time()
    model, losses = scheduler.train(be.handle, Xtr, ytr, steps=args.steps, batch=args.batch, lr=args.lr, seed=1)
    t_train = time.time() - t0
    pred = scheduler.predict(be.handle, model, Xte)
    test_mse = float(np.mean((pred - yte) ** 2))
    base_mse = float(np.mean((ytr.mean() - yte) ** 2))
    model.meta = {"discs": "clumped_disc seeds 1001-1007 (train), 1008 (held out)", "particles": args.particles,
                  "points_per_disc": len(ys[0]), "steps": args.steps, "batch": args.batch, "lr": args.lr,
                  "train_mse_last100": float(losses[-100:].mean()), "heldout_mse": test_mse,
                  "heldout_mse_of_mean_predictor": base_mse, "data_s": t_data, "train_s": t_train}
    model.save(args.out)
    print(json.dumps(model.meta), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
