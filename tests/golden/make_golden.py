"""Writes the golden fixtures of the substep parity tests.

For each seeded scene the FP64 oracle (oracle/, the C++ restatement of the
reference substep) is run to a few snapshot frames; at each snapshot the
fixture holds the complete persistent state (bodies, static-row lambda /
penalty / active / was_static, contact cache, colors) and the outcome of one
substep from it: poses and velocities, the broad-phase pair list with SAT
axes and contact counts, the emitted contact keys and the colors.

    python tests/golden/make_golden.py        # rewrites tests/golden/*.npz

tests/test_golden.py checks that the oracle still reproduces these files
(CPU) and that the GPU substep matches them from the same state (gpu).
"""

from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from avbd_b200 import scenes  # noqa: E402  (scene builders only; no device code)
from oracle.oracle import OracleSolver6DOF  # noqa: E402

CASES = {
    "pyramid20_jacobi": (lambda s: scenes.pyramid20(s), dict(dt=1 / 60, iterations=10, substeps=4,
                                                             friction_static_mult=1.2, coloring_mode="jacobi")),
    "heap64_jacobi": (lambda s: scenes.heap(s, n_side=4, spacing=1.2), dict(dt=1 / 60, iterations=10, substeps=4,
                                                                             friction_static_mult=1.25)),
    "pile_pins_jp": (lambda s: scenes.pile(s, nx=6, nz=6, ny=4, spacing=0.95, pin_every=7),
                     dict(dt=1 / 60, iterations=10, substeps=4, friction_static_mult=1.25,
                          coloring_mode="jones_plassmann")),
    "towers_jp": (lambda s: scenes.tower_grid(s, grid=3, height=4), dict(dt=1 / 60, iterations=12, substeps=4,
                                                                        coloring_mode="jones_plassmann")),
}
SNAPSHOTS = (0, 25)


def oracle_state(so: OracleSolver6DOF, fresh: bool) -> dict:
    """The persistent state; `fresh`: no coloring exists yet (the first
    substep colors from scratch)."""
    x, q, v, w, pv, pw = so.get_bodies()
    ns = so.counts()["n_static"]
    r = so.rows()
    abc, st = so.cache()
    order = np.lexsort((abc[:, 2], abc[:, 1], abc[:, 0])) if len(abc) else np.zeros(0, np.int64)
    colors, nc = so.colors()
    return dict(x=x, q=q, v=v, w=w, pv=pv, pw=pw, row_lam=r["lam"][:ns], row_pen=r["pen"][:ns],
                row_active=r["active"][:ns], row_was=r["was"][:ns], cache_abc=abc[order], cache_state=st[order],
                colors=colors, n_colors=np.int32(nc), color_dirty=np.int32(1 if fresh else 0))


def inject(so: OracleSolver6DOF, sd: dict) -> None:
    so.set_bodies(sd["x"], sd["q"], sd["v"], sd["w"], sd["pv"], sd["pw"])
    so.set_static_rows(sd["row_lam"], sd["row_pen"], sd["row_active"], sd["row_was"])
    so.set_cache(sd["cache_abc"], sd["cache_state"])
    so.set_colors(sd["colors"], int(sd["n_colors"]), bool(sd["color_dirty"]))


def make_oracle(name: str) -> OracleSolver6DOF:
    build, params = CASES[name]
    so = OracleSolver6DOF(precision="float64", threads=1, **params)
    build(so)
    so._flush()
    return so


def outcome(so: OracleSolver6DOF) -> dict:
    x, q, v, w, _, _ = so.get_bodies()
    p = so.pairs()
    colors, nc = so.colors()
    return dict(next_x=x, next_q=q, next_v=v, next_w=w, pair_a=p["a"], pair_b=p["b"], pair_overlap=p["overlap"],
                pair_sat=p["sat_idx"], pair_count=p["count"], contacts=so.contacts(), next_colors=colors,
                next_n_colors=np.int32(nc))


def main() -> None:
    for name in CASES:
        so = make_oracle(name)
        done = 0
        for k in SNAPSHOTS:
            for _ in range(k - done):
                so.step()
            done = k
            sd = oracle_state(so, fresh=(k == 0))
            so.substep()
            out = outcome(so)
            inject(so, sd)  # back to the snapshot, so stepping continues from it
            np.savez_compressed(os.path.join(HERE, f"{name}_f{k}.npz"), **sd, **out)
            print(name, k, len(sd["x"]), "bodies", len(out["pair_a"]), "pairs", len(out["contacts"]), "contacts")


if __name__ == "__main__":
    main()
