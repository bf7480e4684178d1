"""Launch-shape autotuner for the substep solve.

Two knobs decide how the persistent solve kernel maps onto the 148 SMs:

* lanes per body in the primal sweep -- the reference's `primal_group_size`
  (src/avbd3d/solver_6dof.py:627-637; 1..32 lanes gather one body's
  constraint groups and reduce its 6x6 system by shuffles);
* CTAs per SM of the cooperative grid (2 or 3; each count has its own
  register budget, 128 or 80 registers per thread).

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


def autotune(solver, group_sizes=(4, 8, 16, 32), blocks_per_sm=(2, 3), frames: int = 2, warm: int = 1,
             apply: bool = True) -> dict:
    """Times each (group size, CTAs per SM) pair for `frames` frames and
    returns {"best": {...}, "table": [...]}; sets the best pair on the solver
    when `apply`.  The scene state is restored afterwards."""
    solver._flush()
    sd = solver.state_dict()
    g0, b0 = solver.primal_group_size, solver.blocks_per_sm
    table = []
    for g, b in itertools.product(group_sizes, blocks_per_sm):
        solver.load_state_dict(sd)
        solver.primal_group_size = g
        solver.blocks_per_sm = b
        table.append({"group_size": g, "blocks_per_sm": b, "ms_per_frame": _time_frames(solver, frames, warm)})
    best = min(table, key=lambda r: r["ms_per_frame"])
    solver.load_state_dict(sd)
    if apply:
        solver.primal_group_size = best["group_size"]
        solver.blocks_per_sm = best["blocks_per_sm"]
    else:
        solver.primal_group_size, solver.blocks_per_sm = g0, b0
    return {"best": best, "table": table}
