"""Trains the learned warm start on seeded synthetic box piles and writes the
weights (with their normalisation and an evaluation summary) to
avbd_b200/warm_start_pile.npz.

Data: piles of nx*nz*ny boxes (half extents U[0.2, 0.4], random orientation,
density 1000, friction 0.4, mu_s = 1.25 mu, one box in 500 corner-pinned),
the distribution of the 100k-box pile benchmark at a smaller footprint,
seeds 0..49 by default.  At a few frames of each pile's fall and settle the
plain solver runs one substep of 50 iterations with the contact cache
emptied; every box-box contact then gives one sample: its 20 features
(logged at emission) labelled with the lambda (normal and both friction
rows) and normal penalty it converged to in those 50 iterations.  Three
rows per contact: 50 seeds x 4 snapshots give about 2 M rows.  Training:
the package's FP32 forward/backward kernels and Adam, 20 epochs.

Evaluation on held-out seeds (1000..1009 by default; disjoint from
training): for each snapshot, one substep of up to 256 iterations from
three starts -- the plain zero start and the learned start, both with the cache
emptied so every contact is new, and the full contact cache (the start the
learned one stands in for).  Score: iterations until the max violation over
all rows is <= 1e-4 m (up to 256; 257 = not reached); the same over the
box-box contact rows alone is reported beside it.

    python -m avbd_b200.train_warm_start
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import scenes
from .learned import SHIPPED, WarmStartMLP, cold_start_violation, collect_converged, iterations_to
from .solver import Solver6DOF

PARAMS = dict(dt=1.0 / 60.0, iterations=10, substeps=4, friction_static_mult=1.25, coloring_mode="jones_plassmann")
ARMS = (("plain", False, True), ("learned", True, True), ("cached", False, False))


def make_pile(seed: int, nx: int, nz: int, ny: int, model=None) -> Solver6DOF:
    s = Solver6DOF(mlp_warm_start=model, **PARAMS)
    scenes.pile(s, nx=nx, nz=nz, ny=ny, seed=seed)
    return s


def snapshots(s: Solver6DOF, frames):
    """Steps the pile and yields at each frame in `frames`."""
    last = 0
    for f in sorted(frames):
        for _ in range(f - last):
            s.step()
        last = f
        yield f


def collect(seeds, size, frames, label_iterations=50):
    feats, targs = [], []
    for seed in seeds:
        s = make_pile(seed, *size)
        for _ in snapshots(s, frames):
            f, t = collect_converged(s, label_iterations)
            feats.append(f)
            targs.append(t)
    return np.concatenate(feats), np.concatenate(targs)


def score_snapshot(s, iterations=256, tol=1e-4) -> dict:
    """Iterations to `tol` max violation (all rows, and box-box contacts
    alone) from each of the three starts, at the solver's current state."""
    row = {}
    for arm, learned, clear in ARMS:
        h, st = cold_start_violation(s, iterations, learned=learned, clear_cache=clear)
        row[arm + "_max_iters"] = iterations_to(h, tol)
        row[arm + "_box_iters"] = iterations_to(st["contact_violation"], tol)
        if learned:
            row.update(new=int(st["n_new_logged"]), applied=int(st["n_mlp_applied"]),
                       fallback=int(st["n_mlp_fallback"]), reverted=int(st["n_mlp_reverted"]))
    return row


def evaluate(model, seeds, size, frames, iterations=256, tol=1e-4):
    rows = []
    for seed in seeds:
        s = make_pile(seed, *size, model=model)
        for f in snapshots(s, frames):
            rows.append(dict(seed=seed, frame=f, **score_snapshot(s, iterations, tol)))
    return rows


def summarize(ev) -> dict:
    d = {}
    for arm, _, _ in ARMS:
        for k in ("max", "box"):
            d[f"{arm}_{k}_iters"] = float(np.mean([r[f"{arm}_{k}_iters"] for r in ev]))
    for k in ("max", "box"):
        d[f"learned_{k}_reduction"] = 1.0 - d[f"learned_{k}_iters"] / d[f"plain_{k}_iters"]
        d[f"cached_{k}_reduction"] = 1.0 - d[f"cached_{k}_iters"] / d[f"plain_{k}_iters"]
    d["applied_fraction"] = float(sum(r["applied"] for r in ev) / max(1, sum(r["new"] for r in ev)))
    return d


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train-seeds", type=int, default=50)
    ap.add_argument("--eval-seeds", type=int, default=10)
    ap.add_argument("--size", type=int, nargs=3, default=[16, 16, 8])
    ap.add_argument("--frames", type=int, nargs="+", default=[60, 120, 240, 400])
    ap.add_argument("--eval-frames", type=int, nargs="+", default=[240, 400])
    ap.add_argument("--label-iterations", type=int, default=50)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--out", default=SHIPPED)
    args = ap.parse_args(argv)
    t0 = time.time()
    size = tuple(args.size)
    X, Y = collect(range(args.train_seeds), size, args.frames, args.label_iterations)
    keep = X[:, 3] > 0  # separated contacts always keep the zero start
    t1 = time.time()
    model = WarmStartMLP(seed=0)
    hist = model.fit(X[keep], Y[keep], epochs=args.epochs, batch=2048, lr=2e-3)
    t2 = time.time()
    ev = evaluate(model, range(1000, 1000 + args.eval_seeds), size, args.eval_frames)
    t3 = time.time()
    summary = dict(contacts=int(X.shape[0]), rows=int(3 * X.shape[0]), trained_on=int(keep.sum()), size=list(size),
                   frames=args.frames, eval_frames=args.eval_frames, train_seeds=args.train_seeds,
                   eval_seeds=args.eval_seeds, label_iterations=args.label_iterations, epochs=args.epochs,
                   loss_first=hist[0], loss_last=hist[-1], scores=summarize(ev), collect_s=t1 - t0,
                   train_s=t2 - t1, eval_s=t3 - t2)
    model.save(args.out, summary=json.dumps(summary), eval=json.dumps(ev))
    print(json.dumps(summary))
    return summary


if __name__ == "__main__":
    main()
