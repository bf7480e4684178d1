"""Writes tests/golden/reference_*.npz: substeps of the reference's OWN
Solver6DOF (src/avbd3d/solver_6dof.py + kernels_6dof.py, unmodified, run on
the CPU through the pure-Python warp stand-in in oracle/warp_shim).

Each fixture holds, for K consecutive substeps of one scene, the reference's
persistent state before the substep (bodies, static-row lambda / penalty /
active / static-friction flags, contact hash as (a, b, ordinal) keys with
their state, colors), the coloring the substep used, and what the substep
produced: broadphase pairs with SAT axis and contact count, the emitted
contact keys in row order, and the poses and velocities after it.

The reference checkout is needed to run this (python
tests/golden/make_reference_golden.py, from the repository root, where
/root/reference or $AVBD_REFERENCE_ROOT holds it); the fixtures are committed
so the checks run anywhere.  Scenes are built by avbd_b200.scenes, seeded.
"""

from __future__ import annotations

import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from avbd_b200 import scenes  # noqa: E402

# name: (solver keywords, scene builder, frames run before the recorded substeps, substeps recorded)
SCENES = {
    "pyramid20_jacobi": (dict(dt=1 / 60, iterations=10, substeps=4, friction_static_mult=1.2,
                              coloring_mode="jacobi"), lambda s: scenes.pyramid20(s), 0, 8),
    "pyramid20_jacobi_f20": (dict(dt=1 / 60, iterations=10, substeps=4, friction_static_mult=1.2,
                                  coloring_mode="jacobi"), lambda s: scenes.pyramid20(s), 20, 6),
    "towers_jp": (dict(dt=1 / 60, iterations=12, substeps=4, coloring_mode="jones_plassmann"),
                  lambda s: scenes.tower_grid(s, grid=2, height=3), 2, 8),
    "heap27_walls_jacobi_f20": (dict(dt=1 / 60, iterations=10, substeps=4, friction_static_mult=1.25),
                                lambda s: scenes.heap(s, n_side=3, spacing=1.0), 20, 8),
    "pile27_pins_jp_f10": (dict(dt=1 / 60, iterations=10, substeps=4, friction_static_mult=1.25,
                                coloring_mode="jones_plassmann"),
                           lambda s: scenes.pile(s, nx=3, nz=3, ny=3, spacing=0.8, pin_every=4), 10, 8),
}

STATE_KEYS = ("x", "q", "v", "w", "pv", "pw", "row_lam", "row_pen", "row_active", "row_was", "cache_abc",
              "cache_state")


def record(name: str) -> dict:
    from oracle.warp_shim import reference
    S = reference.load()
    params, build, frames, k_sub = SCENES[name]
    s = S.Solver6DOF(device="cpu", **params)
    build(s)
    s._flush()
    for _ in range(frames):
        s.step()
    out: dict = {}
    for k in range(k_sub):
        sd = reference.state_dict(s)
        reference.substep(s)
        for key in STATE_KEYS:
            out[f"s{k}_in_{key}"] = sd[key]
        out[f"s{k}_colors"] = s.body_color.numpy()[:len(s._x)].astype(np.int32).copy()
        out[f"s{k}_n_colors"] = np.int32(s._n_active_colors)
        p = reference.pairs(s)
        for key in ("a", "b", "overlap", "sat_idx", "count"):
            out[f"s{k}_pairs_{key}"] = p[key]
        out[f"s{k}_contacts"] = reference.contacts(s)
        out[f"s{k}_out_x"] = s.x.numpy()[:len(s._x)].copy()
        out[f"s{k}_out_q"] = s.q.numpy()[:len(s._x)].copy()
        out[f"s{k}_out_v"] = s.v.numpy()[:len(s._x)].copy()
        out[f"s{k}_out_w"] = s.omega.numpy()[:len(s._x)].copy()
        out[f"s{k}_out_row_lam"] = s.c_lambda.numpy()[:s._gpu_pool_n_static].copy()
    out["n_substeps"] = np.int32(k_sub)
    out["frames_before"] = np.int32(frames)
    return out


def main(names=None):
    for name in names or SCENES:
        t = time.time()
        data = record(name)
        path = os.path.join(HERE, f"reference_{name}.npz")
        np.savez_compressed(path, **data)
        print(f"{path}: {os.path.getsize(path)} bytes, {time.time() - t:.0f} s")


if __name__ == "__main__":
    main(sys.argv[1:] or None)
