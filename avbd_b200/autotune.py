"""Launch-shape autotuner for the substep solve.

Three knobs decide how the persistent solve kernel maps onto the 148 SMs:

* lanes per body in the primal sweep -- the reference's `primal_group_size`
  (src/avbd3d/solver_6dof.py:627-637; 1..32 lanes gather one body's
  constraint groups and reduce its 6x6 system by shuffles);
* CTAs per SM of the cooperative grid (2 or 3; each count has its own
  register budget, 128 or 80 registers per thread);
* how the color passes are ordered: a grid barrier per color, or per-body
  completion flags (each body waits only for its neighbours, so passes of
  small colors overlap);
* with barriers, whether colors too small to fill the resident warps get
  more lanes per body (`adaptive_lanes`).

The best pair depends on the scene: bodies per color, groups per body and
whether the group records fit in L2.  `autotune` times every candidate on the
solver's live scene with CUDA events on the solver's stream and keeps the
fastest; the simulation state is saved before and restored after, so tuning
does not advance the scene.
"""

from __future__ import annotations

import itertools

import torch


def _time_frames(solver, frames: int, warm: int) -> float:
    """Device milliseconds per frame over `frames` frames after `warm`."""
    for _ in range(warm):
        solver.step()
    st = solver._cuda_stream
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ms = 0.0
    for _ in range(frames):
        with torch.cuda.stream(st):
            t0.record(st)
        solver._enqueue_step()
        with torch.cuda.stream(st):
            t1.record(st)
        solver._after_frame()
        ms += t0.elapsed_time(t1)
    return ms / frames


def autotune(solver, group_sizes=(4, 8, 16), blocks_per_sm=(2, 3), flag_sweep=(False, True),
             adaptive_lanes=(False, True), frames: int = 2, warm: int = 2, apply: bool = True) -> dict:
    """Times each (group size, CTAs per SM, sweep ordering, adaptive lanes)
    candidate for `frames` frames (after `warm` untimed frames: a frame is
    one CUDA graph per LBVH rebuild pattern, and consecutive frames can
    differ in pattern, so two warm frames capture both before timing) and
    returns {"best": {...}, "table":
    [...]}; sets the best candidate on the solver when `apply`.  Adaptive
    lanes only apply to the barrier sweep, so flag-sweep candidates are timed
    without them.  The scene state is restored afterwards."""
    solver._flush()
    sd = solver.state_dict()
    knobs = ("primal_group_size", "blocks_per_sm", "flag_sweep", "adaptive_lanes")
    keep = [getattr(solver, k) for k in knobs]
    table = []
    for g, b, f, a in itertools.product(group_sizes, blocks_per_sm, flag_sweep, adaptive_lanes):
        if f and a:
            continue
        solver.load_state_dict(sd)
        for k, v in zip(knobs, (g, b, f, a)):
            setattr(solver, k, v)
        table.append({"group_size": g, "blocks_per_sm": b, "flag_sweep": f, "adaptive_lanes": a,
                      "ms_per_frame": _time_frames(solver, frames, warm)})
    best = min(table, key=lambda r: r["ms_per_frame"])
    solver.load_state_dict(sd)
    chosen = ([best["group_size"], best["blocks_per_sm"], best["flag_sweep"], best["adaptive_lanes"]]
              if apply else keep)
    for k, v in zip(knobs, chosen):
        setattr(solver, k, v)
    return {"best": best, "table": table}
