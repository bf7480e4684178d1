"""Loads the reference's own Solver6DOF (src/avbd3d/solver_6dof.py and
kernels_6dof.py, unmodified, read from the reference checkout) on top of the
pure-Python warp stand-in in this folder -- TEST INFRASTRUCTURE ONLY.

The reference checkout is needed at run time, so this runs only where it is
mounted (the build container), never on a GPU box; the fixtures it produces
are committed under tests/golden/.
"""

from __future__ import annotations

import importlib
import os
import sys
import types

HERE = os.path.dirname(os.path.abspath(__file__))
DEFAULT_ROOT = "/root/reference"


def reference_root() -> str:
    return os.environ.get("AVBD_REFERENCE_ROOT", DEFAULT_ROOT)


def available() -> bool:
    return os.path.isfile(os.path.join(reference_root(), "src", "avbd3d", "solver_6dof.py"))


def load():
    """Import avbd3d.solver_6dof from the reference checkout with `warp`
    bound to the shim.  The package's __init__ is not executed (it also
    imports the 3-DOF deformable module, whose trimesh dependency is absent);
    a bare package object points Python at the reference's source folder."""
    src = os.path.join(reference_root(), "src", "avbd3d")
    if not os.path.isdir(src):
        raise FileNotFoundError(f"reference source not found: {src}")
    w = sys.modules.get("warp")
    if w is not None and not getattr(w, "__version__", "").endswith("avbd-shim"):
        raise RuntimeError("a real warp module is already imported; the shim must be the one bound")
    if HERE not in sys.path:
        sys.path.insert(0, HERE)
    import warp  # noqa: F401  (the shim)
    if "avbd3d" not in sys.modules:
        pkg = types.ModuleType("avbd3d")
        pkg.__path__ = [src]
        pkg.__file__ = os.path.join(src, "__init__.py")
        sys.modules["avbd3d"] = pkg
    return importlib.import_module("avbd3d.solver_6dof")


# ---------------------------------------------------------------------------
# Read-outs of a reference Solver6DOF in the layout of
# avbd_b200.Solver6DOF.state_dict / pairs / contacts, so the oracle and the
# GPU solver can be loaded from, and compared with, the reference's own run.
# ---------------------------------------------------------------------------
def substep(solver, dt=None) -> None:
    """One substep of dt / substeps, as step() runs it (solver_6dof.py:1178-1197)."""
    import numpy as np  # noqa: F401
    full = solver.dt
    solver.dt = full / solver.substeps if dt is None else dt
    try:
        solver._step_one()
    finally:
        solver.dt = full


def state_dict(solver) -> dict:
    """Persistent state between substeps: bodies, static rows (the first
    _gpu_pool_n_static rows of the c_* pool), the contact hash decoded into
    (a, b, manifold ordinal) keys (kernels_6dof.py:2588-2594) with its 8
    state floats, and the body colors."""
    import numpy as np
    n = len(solver._x)
    ns = solver._gpu_pool_n_static
    f = lambda a: np.asarray(a.numpy()[:n], np.float64).reshape(n, -1)
    if solver.hash_keys is not None:
        keys = solver.hash_keys.numpy()
        live = keys >= 0
        k = keys[live].astype(np.int64)
        st = solver.hash_state.numpy().reshape(-1, 8)[live].astype(np.float64)
    else:
        k, st = np.zeros(0, np.int64), np.zeros((0, 8))
    abc = np.stack([k // (16384 * 4), (k // 4) % 16384, k % 4], 1).astype(np.int32)
    o = np.lexsort((abc[:, 2], abc[:, 1], abc[:, 0])) if k.size else np.zeros(0, np.int64)
    return dict(x=f(solver.x), q=f(solver.q), v=f(solver.v), w=f(solver.omega), pv=f(solver.prev_v),
                pw=f(solver.prev_omega), row_lam=solver.c_lambda.numpy()[:ns].astype(np.float64),
                row_pen=solver.c_penalty.numpy()[:ns].astype(np.float64),
                row_active=solver.c_active.numpy()[:ns].astype(np.int32),
                row_was=solver.c_was_static.numpy()[:ns].astype(np.int32), cache_abc=abc[o],
                cache_state=st[o], colors=solver.body_color.numpy()[:n].astype(np.int32).copy(),
                n_colors=int(solver._n_active_colors), color_dirty=bool(solver._color_dirty))


def pairs(solver) -> dict:
    """Broadphase pairs of the last substep with SAT axis (-1 when separated)
    and contact count (kernels_6dof.py:1946-2130, 2208-2537)."""
    import numpy as np
    n = int(solver._bp_pair_count.numpy()[0]) if solver._bp_pair_count is not None else 0
    n = min(n, solver._bp_max_pairs)
    ov = solver._bp_pair_overlap.numpy()[:n].astype(np.int32) if n else np.zeros(0, np.int32)
    si = solver._bp_pair_sat_idx.numpy()[:n] if n else np.zeros(0, np.int32)
    cnt = solver._mf_contact_count.numpy()[:n] if n else np.zeros(0, np.int32)
    return dict(a=solver._bp_pair_a.numpy()[:n].astype(np.int32), b=solver._bp_pair_b.numpy()[:n].astype(np.int32),
                overlap=ov, sat_idx=np.where(ov == 1, si, -1).astype(np.int32),
                count=np.where(ov == 1, cnt, 0).astype(np.int32))


def contacts(solver):
    """(reference body, incident body, manifold ordinal) of every emitted
    contact, in row order (kernels_6dof.py:2695-2912)."""
    import numpy as np
    if solver.pool_count is None:
        return np.zeros((0, 3), np.int32)
    m = int(solver.pool_count.numpy()[0])
    rn = solver.pool_idx_n.numpy()[:m]
    c = solver.pool_idx_c.numpy()[:m]
    o = np.argsort(rn, kind="stable")
    return np.stack([solver.c_body_a.numpy()[rn][o], solver.c_body_b.numpy()[rn][o], c[o]], 1).astype(np.int32)
