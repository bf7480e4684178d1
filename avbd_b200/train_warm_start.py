"""Trains the learned warm start on seeded synthetic box piles and writes the
weights (with their normalisation and an evaluation summary) to
avbd_b200/warm_start_pile.npz.

Data: piles of nx*nz*ny boxes (half extents U[0.2, 0.4], random orientation,
density 1000, friction 0.4, mu_s = 1.25 mu, pins every 500th box), the
distribution of the 100k-box pile benchmark at a smaller footprint.  At a
few frames of each pile's fall and settle, every box-box contact gives one
sample: its 20 features (logged by a substep run with the contact cache
emptied, so every contact is new) labelled with the state the cache held for
it -- the warm start the learned start stands in for.  Training seeds and
held-out evaluation seeds are disjoint.

Evaluation: for each held-out snapshot, one substep of up to 64 iterations
from three starts: the plain zero start and the learned start, both with the
cache emptied, and the full cache for reference.  Two scores per start:
iterations until the max violation over all rows is <= 1e-4 m, and until the
mean violation of the box-box contacts (the rows the warm start sets) is
<= 1e-5 m.  The max over all rows is dominated by floor rows and deep
interpenetrations that no contact warm start touches (the full cache barely
moves it), so the contact mean is the score that measures the warm start.

    python -m avbd_b200.train_warm_start --train-seeds 24 --eval-seeds 6
"""

from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import scenes
from .learned import SHIPPED, WarmStartMLP, collect_cold_start, cold_start_violation, iterations_to
from .solver import Solver6DOF

PARAMS = dict(dt=1.0 / 60.0, iterations=10, substeps=4, friction_static_mult=1.25, coloring_mode="jones_plassmann")


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


def collect(seeds, size, frames):
    feats, targs = [], []
    for seed in seeds:
        s = make_pile(seed, *size)
        s.log_new_contacts = True
        for _ in snapshots(s, frames):
            f, t = collect_cold_start(s)
            feats.append(f)
            targs.append(t)
    return np.concatenate(feats), np.concatenate(targs)


def evaluate(model, seeds, size, frames, iterations=64, tol_max=1e-4, tol_contact=1e-5):
    rows = []
    for seed in seeds:
        s = make_pile(seed, *size, model=model)
        for f in snapshots(s, frames):
            row = dict(seed=seed, frame=f)
            for arm, learned, clear in (("plain", False, True), ("learned", True, True), ("cached", False, False)):
                h, st = cold_start_violation(s, iterations, learned=learned, clear_cache=clear)
                hc = st["contact_violation"]
                row[arm + "_max_iters"] = iterations_to(h, tol_max)
                row[arm + "_contact_iters"] = iterations_to(hc, tol_contact)
                row[arm + "_viol"] = h.tolist()
                row[arm + "_contact_viol"] = hc.tolist()
                if learned:
                    row.update(new=int(st["n_new_logged"]), applied=int(st["n_mlp_applied"]),
                               fallback=int(st["n_mlp_fallback"]))
            rows.append(row)
    return rows


def summarize(ev, frames):
    out = {}
    for f in ["all"] + list(frames):
        rs = [r for r in ev if f == "all" or r["frame"] == f]
        d = {}
        for arm in ("plain", "learned", "cached"):
            for k in ("max", "contact"):
                d[f"{arm}_{k}_iters"] = float(np.mean([r[f"{arm}_{k}_iters"] for r in rs]))
        d["contact_reduction"] = 1.0 - d["learned_contact_iters"] / d["plain_contact_iters"]
        d["max_reduction"] = 1.0 - d["learned_max_iters"] / d["plain_max_iters"]
        out[str(f)] = d
    return out


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--train-seeds", type=int, default=24)
    ap.add_argument("--eval-seeds", type=int, default=6)
    ap.add_argument("--size", type=int, nargs=3, default=[16, 16, 8])
    ap.add_argument("--frames", type=int, nargs="+", default=[60, 120, 240, 400])
    ap.add_argument("--epochs", type=int, default=150)
    ap.add_argument("--out", default=SHIPPED)
    args = ap.parse_args(argv)
    t0 = time.time()
    size = tuple(args.size)
    X, Y = collect(range(args.train_seeds), size, args.frames)
    keep = X[:, 3] > 0  # separated contacts always keep the zero start
    t1 = time.time()
    model = WarmStartMLP(seed=0)
    hist = model.fit(X[keep], Y[keep], epochs=args.epochs, batch=2048, lr=2e-3)
    t2 = time.time()
    ev = evaluate(model, range(1000, 1000 + args.eval_seeds), size, args.frames)
    t3 = time.time()
    summary = dict(samples=int(keep.sum()), size=list(size), frames=args.frames, train_seeds=args.train_seeds,
                   eval_seeds=args.eval_seeds, loss_first=hist[0], loss_last=hist[-1],
                   scores=summarize(ev, args.frames), collect_s=t1 - t0, train_s=t2 - t1, eval_s=t3 - t2)
    model.save(args.out, summary=json.dumps(summary), eval=json.dumps(ev))
    print(json.dumps(summary))
    return summary


if __name__ == "__main__":
    main()
