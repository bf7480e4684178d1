"""Drop-in `Solver6DOF` running the substep on a B200 through libavbd6.so.

Mirrors the public API of the reference solver (src/avbd3d/solver_6dof.py:
177-2052): constructor keywords, scene building (`add_box`,
`add_floor_contact_box`, `add_pin_corner`, `enable_self_collision`), `step`,
getters / setters, `read_state_batched`, `count_color_conflicts` and the
runtime properties.  All device state lives in ONE PyTorch-owned arena whose
layout the C library defines (`avbd_layout`); this module fills the scene
arrays, then calls the C ABI with raw pointers and the current CUDA stream.

There is no CPU path: constructing a solver without a CUDA device, or with the
extension missing, raises.
"""

from __future__ import annotations

import ctypes as C
import itertools
import math
import warnings
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib

# Constraint type codes (solver_6dof.py:31-34).
FLOOR_CONTACT_6DOF = 0
CONTACT_TANGENT_6DOF = 1
PIN_6DOF = 2
BOX_BOX_CONTACT_6DOF = 3

KIND_FLOOR, KIND_PIN, KIND_BOX = 0, 1, 2
META_IMPLICIT = 512  # implicit floor corner (corner index in meta bits 6-8; csrc/common.cuh)
MAX_COLORS = 32
_INF = math.inf


def _obb_sat(c_A, R_A, e_A, c_B, R_B, e_B, margin: float = 0.005):
    """Host 15-axis SAT (solver_6dof.py:37-102): (axis_idx, n_hat B->A,
    overlap) or None when separated by more than `margin` (face axes) or at
    all (edge axes)."""
    t = np.asarray(c_B, np.float64) - np.asarray(c_A, np.float64)
    R_A = np.asarray(R_A, np.float64)
    R_B = np.asarray(R_B, np.float64)
    e_A = np.asarray(e_A, np.float64)
    e_B = np.asarray(e_B, np.float64)
    best_idx, best_ov, best_axis = -1, np.inf, None
    axes = [(k, R_A[:, k], None) for k in range(3)] + [(3 + k, R_B[:, k], None) for k in range(3)]
    for idx, L, _ in axes:
        rA = e_A[idx] if idx < 3 else float(np.sum(e_A * np.abs(L @ R_A)))
        rB = e_B[idx - 3] if idx >= 3 else float(np.sum(e_B * np.abs(L @ R_B)))
        ov = rA + rB - abs(float(t @ L))
        if ov < -margin:
            return None
        if ov < best_ov:
            best_idx, best_ov, best_axis = idx, ov, (-L if float(t @ L) > 0 else L)
    for i in range(3):
        for j in range(3):
            L = np.cross(R_A[:, i], R_B[:, j])
            n = float(np.linalg.norm(L))
            if n < 1e-6:
                continue
            L = L / n
            ov = float(np.sum(e_A * np.abs(L @ R_A)) + np.sum(e_B * np.abs(L @ R_B))) - abs(float(t @ L))
            if ov < 0:
                return None
            if ov < best_ov:
                best_idx, best_ov, best_axis = 6 + 3 * i + j, ov, (-L if float(t @ L) > 0 else L)
    return best_idx, np.asarray(best_axis, np.float32), float(best_ov)


@dataclass
class RigidBody:
    """Handle returned by add_box (solver_6dof.py:105-110)."""
    index: int
    half_extents: tuple


@dataclass
class _Row:  # solver_6dof.py:113-129
    type: int
    body_a: int
    body_b: int = -1
    world_anchor: tuple = (0.0, 0.0, 0.0)
    off_a: tuple = (0.0, 0.0, 0.0)
    off_b: tuple = (0.0, 0.0, 0.0)
    rest: float = 0.0
    stiffness: float = _INF
    fracture: float = _INF
    fmin: float = -_INF
    fmax: float = _INF
    sibling: int = -1
    friction: float = 0.0
    friction_static: float = 0.0
    partner: int = -1


# Corner order of add_floor_contact_box (solver_6dof.py:474-520): x outer, z inner.
_CORNER_SIGNS = np.array([(sx, sy, sz) for sx in (-1.0, 1.0) for sy in (-1.0, 1.0) for sz in (-1.0, 1.0)])


class _RowTable:
    """The reference's constraint-row list (row numbering of the c_* arrays,
    solver_6dof.py:1067-1129), stored compactly: explicit rows (pins) plus
    one record per add_floor_contact_box call, whose 8 corners x (1 or 3)
    rows are materialised only when a row is looked up.  A 100k-box pile has
    2.4 M floor rows; they exist here as 100 k block records, and the
    static groups are built from them with array operations."""

    def __init__(self):
        self._starts: list[int] = []  # first row of each segment
        self._segs: list = []  # list[_Row] (explicit rows) or a floor-block tuple
        self._n = 0
        # the floor blocks again, column by column, for array construction
        self._fb_cols: tuple = ([], [], [], [], [], [], [], [], [], [])  # body, hx, hy, hz, fy, mu, mus, stiff, start, per

    def __len__(self) -> int:
        return self._n

    def append(self, row: _Row) -> None:
        if not self._segs or not isinstance(self._segs[-1], list):
            self._starts.append(self._n)
            self._segs.append([])
        self._segs[-1].append(row)
        self._n += 1

    def add_floor_block(self, body: int, he: tuple, floor_y: float, mu: float, mus: float,
                        stiffness: float) -> int:
        start = self._n
        per = 3 if mu > 0.0 else 1
        self._starts.append(start)
        self._segs.append((body, he, floor_y, mu, mus, stiffness, start, per))
        for col, v in zip(self._fb_cols, (body, he[0], he[1], he[2], floor_y, mu, mus, stiffness, start, per)):
            col.append(v)
        self._n += 8 * per
        return start

    @staticmethod
    def _block_row(blk, k: int) -> _Row:
        body, he, floor_y, mu, mus, stiff, start, per = blk
        c, s = divmod(k, per)
        off = tuple(float(v) for v in _CORNER_SIGNS[c] * np.asarray(he))
        n = start + c * per
        if s == 0:
            return _Row(FLOOR_CONTACT_6DOF, body, world_anchor=(0.0, float(floor_y), 0.0), off_a=off,
                        stiffness=stiff, fmin=-_INF, fmax=0.0)
        t = n + 1
        return _Row(CONTACT_TANGENT_6DOF, body, world_anchor=(1.0, 0.0, 0.0) if s == 1 else (0.0, 0.0, 1.0),
                    off_a=off, stiffness=stiff, sibling=n, friction=mu, friction_static=mus,
                    partner=t + 1 if s == 1 else t)

    def __getitem__(self, i):
        if isinstance(i, slice):
            return [self[k] for k in range(*i.indices(self._n))]
        if i < 0:
            i += self._n
        if not 0 <= i < self._n:
            raise IndexError(i)
        j = int(np.searchsorted(self._starts, i, side="right")) - 1
        seg = self._segs[j]
        k = i - self._starts[j]
        return seg[k] if isinstance(seg, list) else self._block_row(seg, k)

    def __iter__(self):
        for j, seg in enumerate(self._segs):
            if isinstance(seg, list):
                yield from seg
            else:
                for k in range(8 * seg[7]):
                    yield self._block_row(seg, k)

    def floor_blocks(self) -> list:
        return [seg for seg in self._segs if not isinstance(seg, list)]

    def n_floor_blocks(self) -> int:
        return len(self._fb_cols[0])

    def floor_columns(self) -> dict:
        """The floor blocks as arrays: body, he [n, 3], floor_y, mu, mus,
        stiffness, first row, rows per corner."""
        c = self._fb_cols
        return dict(body=np.asarray(c[0], np.int64), he=np.stack([np.asarray(c[k], np.float64) for k in (1, 2, 3)], 1)
                    if c[0] else np.zeros((0, 3)), fy=np.asarray(c[4], np.float32), mu=np.asarray(c[5], np.float32),
                    mus=np.asarray(c[6], np.float32), stiff=np.asarray(c[7], np.float32),
                    start=np.asarray(c[8], np.int64), per=np.asarray(c[9], np.int64))


def box_inertia_local(mass: float, hx: float, hy: float, hz: float) -> np.ndarray:
    """Solid-box body inertia (solver_6dof.py:132-142); zero for static bodies."""
    if mass <= 0.0:
        return np.zeros((3, 3), dtype=np.float32)
    return np.diag([mass / 3.0 * (hy * hy + hz * hz), mass / 3.0 * (hx * hx + hz * hz),
                    mass / 3.0 * (hx * hx + hy * hy)]).astype(np.float32)


def _box_inertia_diag_batch(mass: np.ndarray, he: np.ndarray) -> np.ndarray:
    """box_inertia_local's diagonal for arrays of bodies (same float64
    arithmetic, then float32)."""
    hx, hy, hz = he[:, 0], he[:, 1], he[:, 2]
    d = np.stack([mass / 3.0 * (hy * hy + hz * hz), mass / 3.0 * (hx * hx + hz * hz),
                  mass / 3.0 * (hx * hx + hy * hy)], 1)
    d[mass <= 0.0] = 0.0
    return d.astype(np.float32)


def box_inv_inertia_local(mass: float, hx: float, hy: float, hz: float) -> np.ndarray:
    """Inverse of box_inertia_local (solver_6dof.py:145-152)."""
    if mass <= 0.0:
        return np.zeros((3, 3), dtype=np.float32)
    return np.linalg.inv(box_inertia_local(mass, hx, hy, hz)).astype(np.float32)


def _snap_group_size(g: int) -> int:
    """Largest power of two <= g in [1, 32] (solver_6dof.py:165-174)."""
    g = max(1, min(32, int(g)))
    p = 1
    while p * 2 <= g:
        p *= 2
    return p


def _on_stream(fn):
    """Run a method with the solver's CUDA stream current, so torch copies and
    the library's launches are ordered on one non-default stream (required
    for CUDA-graph capture)."""

    def wrapped(self, *a, **k):
        with torch.cuda.device(self.device), torch.cuda.stream(self._cuda_stream):
            return fn(self, *a, **k)

    wrapped.__name__ = fn.__name__
    wrapped.__doc__ = fn.__doc__
    return wrapped


def _next_pow2(n: int) -> int:
    p = 1
    while p < n:
        p <<= 1
    return p


class _Arena:
    """One device allocation holding every array of the C layout."""

    def __init__(self, dims: _lib.AvbdDims, device: torch.device):
        L = _lib.load()
        n = L.avbd_num_arrays()
        offs = (C.c_size_t * n)()
        total = C.c_size_t(0)
        _lib.check(L.avbd_layout(C.byref(dims), offs, C.byref(total)), "layout")
        self.names = [L.avbd_array_name(i).decode() for i in range(n)]
        self.off = {nm: int(offs[i]) for i, nm in enumerate(self.names)}
        self.total = int(total.value)
        self.buf = torch.zeros(self.total, dtype=torch.uint8, device=device)
        self.dims = dims

    def ptr(self) -> int:
        return self.buf.data_ptr()

    def view(self, name: str, dtype: torch.dtype, shape) -> torch.Tensor:
        o = self.off[name]
        n = int(np.prod(shape)) * torch.tensor([], dtype=dtype).element_size()
        return self.buf[o:o + n].view(dtype).view(*shape)


_COLOR_ALIASES = {"jp": "jones_plassmann", "jones-plassmann": "jones_plassmann",
                  "jones plassmann": "jones_plassmann", "speculative": "jacobi",
                  "speculative_greedy": "jacobi", "greedy": "jacobi"}


class Solver6DOF:
    """6-DOF AVBD rigid-body solver; the substep runs in libavbd6.so on the GPU."""

    _COLORING_MODES = ("jones_plassmann", "jacobi")

    def __init__(self, dt: float = 1.0 / 60.0, iterations: int = 10, gravity=(0.0, -9.81, 0.0), alpha: float = 0.99,
                 beta: float = 1.0e5, gamma: float = 0.99, post_stabilize: bool = True, device: str = "cpu",
                 max_linear_speed: float = 30.0, max_angular_speed: float = 50.0, substeps: int = 1,
                 friction_static_mult: float = 1.5, coloring_mode: str = "jacobi",
                 unsafe_fixed_capacity: bool = False, primal_group_size: int = 8, primal_shuffle: bool = True,
                 primal_fused: bool = True, gpu_resident: bool = True, recolor_every_substep: bool = False,
                 persistent: bool = True, use_graph: bool = True, mlp_warm_start=None):
        if not torch.cuda.is_available():
            raise RuntimeError("avbd_b200.Solver6DOF needs a CUDA device (there is no CPU path)")
        _lib.load()
        # `device` names the CUDA device; "cpu" (the reference default) maps to
        # the current CUDA device so reference code runs unchanged.
        dev = str(device)
        self.device = torch.device(dev if dev.startswith("cuda") else f"cuda:{torch.cuda.current_device()}")
        self._cuda_stream = torch.cuda.Stream(self.device)
        self._ctx = None
        self._arena = None
        self._primal_group_size = _snap_group_size(primal_group_size)
        self._primal_shuffle = bool(primal_shuffle)
        self._primal_fused = bool(primal_fused)
        self._gpu_resident = bool(gpu_resident)
        self._recolor_every_substep = bool(recolor_every_substep)
        self._unsafe_fixed_capacity = bool(unsafe_fixed_capacity)
        self._coloring_mode = None
        self._color_dirty = True
        self.coloring_mode = coloring_mode
        self.dt = float(dt)
        self.iterations = int(iterations)
        self.gravity = tuple(float(g) for g in gravity)
        self.alpha, self.beta, self.gamma = float(alpha), float(beta), float(gamma)
        self.post_stabilize = bool(post_stabilize)
        self.max_linear_speed = float(max_linear_speed)
        self.max_angular_speed = float(max_angular_speed)
        self.substeps = max(1, int(substeps))
        self.friction_static_mult = max(1.0, float(friction_static_mult))
        self.persistent = bool(persistent)
        self.use_graph = bool(use_graph)
        self.record_violation = False
        self.blocks_per_sm = 0
        self.timing = False  # stamp the solve kernel's phases (phase_profile())
        # persistent solve: order the color passes by per-body completion
        # flags instead of one grid barrier per color (same results).  With
        # 8 lanes per body (the primal_group_size default; the reference's
        # default is 16, and any value passed is used as given) and 2 CTAs per
        # SM this is the fastest shape the autotuner measured on the 100k
        # pile, so a plain Solver6DOF(...) runs it without autotune().
        self.flag_sweep = True
        self.adaptive_lanes = False  # more lanes per body for small colors (barrier sweep)
        # barrier sweep: floor corners resting above the floor in their start
        # state are evaluated from the body's pose alone (same poses; fewer
        # group reads); the flag sweep always reads them
        self.resting_floor = True
        # LBVH rebuilt every this many substeps, refit in between (same pairs)
        self.bvh_rebuild_every = 8
        # initial dynamic-row pool (None: the reference's 192 rows per body)
        self.dyn_row_capacity = None
        self._anchor_keys = False  # cache_key_mode "anchor_5mm"
        self._debug_skip_arrive = False
        self._mlp = mlp_warm_start
        self._log_new = False
        # batched scenes (avbd_b200.batch.SceneBatch): scene of each body and
        # per scene (substeps per frame, iterations); empty for one scene
        self._scene_of: list[int] = []
        self._scene_tab: list[tuple[int, int]] = []
        self._cur_scene = -1

        self._x, self._q, self._v, self._omega = [], [], [], []
        self._mass, self._half_extents, self._friction = [], [], []
        self._rows = _RowTable()
        # explicit static groups (pins): (kind, body, row0, three, off, extra3, mu, mus, stiffness, fracture);
        # floor-contact groups live in the row table's floor blocks (8 each)
        self._groups: list[tuple] = []
        self._layout = None
        self._row_map_cache = None
        self._dirty = True
        self._self_collide = False
        self._self_friction = 0.0

        self._arena = None
        self._ctx = None
        self._stats = _lib.AvbdStats()
        self.num_colors = MAX_COLORS
        self._max_colors = MAX_COLORS
        self.num_active_colors = MAX_COLORS
        self._n_active_colors = MAX_COLORS
        self.broadphase_ms = 0.0
        self.solve_ms = 0.0
        self._graph_signature = None
        self._gpu_pool_n_static = 0
        self._gpu_pool_n_capacity = 0
        self._gpu_pool_n_dyn_capacity = 0
        self._gpu_pool_max_pairs = 0
        self._bp_max_pairs = 0
        self._gpu_pool_hash_cap = 0
        self._fixed_cap_overflow_warned = False
        self._pair_overflow_warned = False
        self.host_syncs = 0  # host<->device synchronisations issued by step()

    def __del__(self):
        try:
            if self._ctx is not None:
                _lib.load().avbd_destroy(self._ctx)
                self._ctx = None
        except Exception:
            pass

    # ---- scene building (solver_6dof.py:446-578) -----------------------------
    def add_box(self, position, half_extents, mass, orientation=(0.0, 0.0, 0.0, 1.0), velocity=(0.0, 0.0, 0.0),
                angular_velocity=(0.0, 0.0, 0.0), friction=0.0) -> RigidBody:
        idx = len(self._x)
        px, py, pz = position
        qx, qy, qz, qw = orientation
        vx, vy, vz = velocity
        wx, wy, wz = angular_velocity
        hx, hy, hz = half_extents
        hx, hy, hz = float(hx), float(hy), float(hz)
        self._x.append((float(px), float(py), float(pz)))
        self._q.append((float(qx), float(qy), float(qz), float(qw)))
        self._v.append((float(vx), float(vy), float(vz)))
        self._omega.append((float(wx), float(wy), float(wz)))
        self._mass.append(float(mass))
        self._half_extents.append((hx, hy, hz))
        self._friction.append(max(0.0, float(friction)))
        if self._scene_tab:
            if self._cur_scene < 0:
                raise RuntimeError("a batched solver needs a current scene (SceneBatch.add_scene) for add_box")
            self._scene_of.append(self._cur_scene)
        self._dirty = True
        return RigidBody(index=idx, half_extents=(hx, hy, hz))

    def add_floor_contact_box(self, body: RigidBody, floor_y: float = 0.0, friction=None,
                              stiffness: float = _INF) -> list[int]:
        mu = float(friction) if friction is not None else self._friction[body.index]
        mus = mu * self.friction_static_mult if mu > 0.0 else 0.0
        hx, hy, hz = body.half_extents
        start = self._rows.add_floor_block(body.index, (float(hx), float(hy), float(hz)), float(floor_y),
                                           mu, mus, float(stiffness))
        per = 3 if mu > 0.0 else 1
        out = list(range(start, start + 8 * per, per))
        self._dirty = True
        return out

    def add_pin_corner(self, body: RigidBody, body_local, world_point, stiffness: float = _INF,
                       fracture: float = _INF) -> list[int]:
        start = len(self._rows)
        out = []
        for axis in (0, 1, 2):
            out.append(len(self._rows))
            self._rows.append(_Row(PIN_6DOF, body.index, body_b=axis,
                                   world_anchor=tuple(float(p) for p in world_point),
                                   off_a=tuple(float(v) for v in body_local), stiffness=stiffness,
                                   fracture=fracture))
        self._groups.append((KIND_PIN, body.index, start, True, tuple(float(v) for v in body_local),
                             tuple(float(p) for p in world_point), 0.0, 0.0, float(stiffness), float(fracture)))
        self._dirty = True
        return out

    def enable_self_collision(self, enabled: bool = True, default_friction: float = 0.0) -> None:
        self._self_collide = bool(enabled)
        self._self_friction = max(0.0, float(default_friction))
        self._dirty = True

    # ---- runtime properties (solver_6dof.py:597-661) -------------------------
    @property
    def coloring_mode(self) -> str:
        return self._coloring_mode

    @coloring_mode.setter
    def coloring_mode(self, mode: str) -> None:
        m = str(mode).strip().lower()
        m = _COLOR_ALIASES.get(m, m)
        if m not in self._COLORING_MODES:
            raise ValueError(f"coloring_mode must be one of {self._COLORING_MODES}, got {mode!r}")
        if m != self._coloring_mode:
            self._coloring_mode = m
            self._color_dirty = True
            if self._ctx is not None:
                _lib.load().avbd_mark_color_dirty(self._ctx, self._stream())

    @property
    def primal_group_size(self) -> int:
        return self._primal_group_size

    @primal_group_size.setter
    def primal_group_size(self, g: int) -> None:
        self._primal_group_size = _snap_group_size(g)

    @property
    def gpu_resident(self) -> bool:
        return self._gpu_resident

    @gpu_resident.setter
    def gpu_resident(self, on: bool) -> None:
        self._gpu_resident = bool(on)

    @property
    def recolor_every_substep(self) -> bool:
        return self._recolor_every_substep

    @recolor_every_substep.setter
    def recolor_every_substep(self, on: bool) -> None:
        self._recolor_every_substep = bool(on)

    # ---- device upload (solver_6dof.py:904-1174) -------------------------------
    def _stream(self):
        return C.c_void_p(self._cuda_stream.cuda_stream)

    def _dims(self, pair_cap=None, dyn_rows=None) -> _lib.AvbdDims:
        n = len(self._x)
        if self._self_collide:
            max_pairs = max(64, 16 * max(1, n))
            pc = max(256, 16 * n) if pair_cap is None else pair_cap
            # the reference's pool size (16 pairs x 12 rows per body) unless a
            # caller sized it (dyn_row_capacity); overflow grows it either way
            dr = (self.dyn_row_capacity or max_pairs * 12) if dyn_rows is None else dyn_rows
            hc = _next_pow2(max(1024, 8 * max_pairs))
        else:
            pc, dr, hc = 0, 0, 1024
        d = _lib.AvbdDims()
        d.n_bodies = n
        d.n_static_groups = self._n_static_groups
        d.n_static_rows = len(self._rows)
        d.pair_cap = pc
        d.dyn_row_cap = dr
        d.dyn_group_cap = dr
        d.hash_cap = hc
        d.mlp_floats = 0 if self._mlp is None else int(self._mlp.n_floats)
        # new-contact queue: allocated only when a warm-start model or the
        # training log can use it
        d.new_cap = max(1024, 8 * n) if self._self_collide and (self._mlp is not None or self._log_new) else 0
        d.n_scenes = len(self._scene_tab)
        d.anchor_keys = int(self._anchor_keys)
        return d

    def _views(self):
        A = self._arena
        n = max(1, len(self._x))
        f4 = lambda nm: A.view(nm, torch.float32, (n, 4))
        self.x4, self.q, self.v4, self.w4 = f4("BX"), f4("BQ"), f4("BV"), f4("BW")
        self.pv4, self.pw4 = f4("BPV"), f4("BPW")
        self.x = self.x4[:, :3]
        self.v = self.v4[:, :3]
        self.omega = self.w4[:, :3]
        self.prev_v, self.prev_omega = self.pv4[:, :3], self.pw4[:, :3]
        self._he4, self._iloc4 = f4("BHE"), f4("BILOC")
        self._prio = A.view("BPRIO", torch.float32, (n,))
        self._color = A.view("COLOR", torch.int32, (n,))
        self._color_starts = A.view("COLOR_STARTS", torch.int32, (64,))
        self._color_bodies = A.view("COLOR_BODIES", torch.int32, (n,))
        self._sg_start = A.view("SG_START", torch.int32, (n + 1,))
        g = max(1, A.dims.n_static_groups + A.dims.dyn_group_cap)
        self._g_body = A.view("G_BODY", torch.int32, (g, 2))
        self._g_meta = A.view("G_META", torch.int32, (g,))
        self._g_row0 = A.view("G_ROW0", torch.int32, (g,))
        self._g_flags = A.view("G_FLAGS", torch.int32, (g,))
        for nm in ("G_OFFA", "G_OFFB", "G_N", "G_MAT", "G_LAM", "G_PEN", "G_AC0"):
            setattr(self, "_" + nm.lower(), A.view(nm, torch.float32, (g, 4)))
        p = max(1, A.dims.pair_cap)
        self._pair_ab = A.view("PAIR_AB", torch.int32, (p, 2))
        self._pair_info = A.view("PAIR_INFO", torch.int32, (p,))
        self._pair_nrm = A.view("PAIR_NRM", torch.float32, (p, 4))
        self._pair_kept = A.view("PAIR_KEPT", torch.int32, (p,))
        h = A.dims.hash_cap
        self._h_key = A.view("H_KEY", torch.int64, (h,))
        self._h_s0 = A.view("H_S0", torch.float32, (h, 4))
        self._h_s1 = A.view("H_S1", torch.float32, (h, 4))

    @property
    def _n_static_groups(self) -> int:
        return 8 * self._rows.n_floor_blocks() + len(self._groups)

    def _static_group_arrays(self):
        """Host construction of the static groups, sorted by body (stable: by
        first row within a body), so each body's groups are one contiguous
        range; returns numpy arrays and the static row -> (group, slot) map.
        The solver builds the same records on the device
        (_upload_static_groups); this host form is what the tests compare
        the device build with."""
        n = len(self._x)
        nblk = self._rows.n_floor_blocks()
        nf = 8 * nblk
        ng = nf + len(self._groups)
        G = max(ng, 1)
        body = np.full((G, 2), -1, np.int32)
        meta = np.zeros(G, np.int32)
        row0 = np.zeros(G, np.int64)
        offa = np.zeros((G, 4), np.float32)
        gn = np.zeros((G, 4), np.float32)
        mat = np.zeros((G, 4), np.float32)
        three = np.zeros(G, bool)
        if nblk:
            fc = self._rows.floor_columns()
            bb, he, fy, mu, mus, st, r0, per = (fc[k] for k in ("body", "he", "fy", "mu", "mus", "stiff", "start",
                                                                "per"))
            body[:nf, 0] = np.repeat(bb, 8)
            row0[:nf] = (r0[:, None] + np.arange(8)[None, :] * per[:, None]).reshape(-1)
            three[:nf] = np.repeat(per == 3, 8)
            hard = np.repeat(~(st < _INF), 8)
            meta[:nf] = KIND_FLOOR | np.where(three[:nf], 4, 0) | np.where(hard, 8, 0)
            mat[:nf] = np.repeat(np.stack([mu, mus, st, np.full_like(st, _INF)], 1), 8, axis=0)
            # Implicit corners: a block whose half extents are its body's
            # stores no offsets; the kernels rebuild them from the body's half
            # extents and the corner index (meta bits 6-8), and the floor
            # height sits in mat.w.  Other blocks keep explicit offsets.
            body_he = np.asarray(self._half_extents, np.float32).reshape(-1, 3)[bb]
            imp = np.all(he.astype(np.float32) == body_he, axis=1)
            imp8 = np.repeat(imp, 8)
            corner = np.tile(np.arange(8), nblk)
            meta[:nf] |= np.where(imp8, META_IMPLICIT | (corner << 6), 0).astype(np.int32)
            explicit = (he[:, None, :] * _CORNER_SIGNS[None, :, :]).reshape(-1, 3).astype(np.float32)
            offa[:nf, :3] = np.where(imp8[:, None], 0.0, explicit)
            offa[:nf, 3] = np.where(imp8, 0.0, np.repeat(fy, 8))
            mat[:nf, 3] = np.where(imp8, np.repeat(fy, 8), mat[:nf, 3])
        for j, (kind, b, r0_, th, off, extra, mu_, mus_, stiff, frac) in enumerate(self._groups):
            k = nf + j
            body[k, 0] = b
            hard = not (stiff < _INF)
            meta[k] = kind | (4 if th else 0) | (8 if hard else 0)
            row0[k] = r0_
            three[k] = th
            offa[k, :3] = off
            if kind == KIND_FLOOR:
                offa[k, 3] = extra[1]
            else:
                gn[k, :3] = extra
            mat[k] = (mu_, mus_, stiff, frac)
        order = np.lexsort((row0[:ng], body[:ng, 0])) if ng else np.zeros(0, np.int64)
        out = dict(body=body[order] if ng else body, meta=meta[order] if ng else meta,
                   row0=(row0[order] if ng else row0).astype(np.int32), offa=offa[order] if ng else offa,
                   n=gn[order] if ng else gn, mat=mat[order] if ng else mat)
        th = three[order] if ng else three
        out["flags"] = np.where(th, 7, 1).astype(np.int32)
        row_map = np.zeros((len(self._rows), 2), np.int64)
        if ng:
            g_idx = np.arange(ng, dtype=np.int64)
            r0s = out["row0"][:ng].astype(np.int64)
            row_map[r0s, 0] = g_idx
            row_map[r0s, 1] = 0
            t = th[:ng]
            for s_ in (1, 2):
                row_map[r0s[t] + s_, 0] = g_idx[t]
                row_map[r0s[t] + s_, 1] = s_
        counts = np.bincount(body[:ng, 0].astype(np.int64), minlength=n) if ng else np.zeros(n, np.int64)
        sg_start = np.zeros(n + 1, np.int32)
        sg_start[1:] = np.cumsum(counts[:n])
        return out, sg_start, row_map

    def _static_layout(self):
        """Where each static group goes: floor blocks (8 corner groups each)
        and explicit groups (pins) in one order, by body and then first row,
        so a body's groups form one range.  Returns (floor-block columns,
        first group of each block, group of each explicit group,
        sg_start [n+1])."""
        n = len(self._x)
        fc = self._rows.floor_columns()
        nblk = len(fc["body"])
        ne = len(self._groups)
        eb = np.fromiter((g[1] for g in self._groups), np.int64, ne)
        er = np.fromiter((g[2] for g in self._groups), np.int64, ne)
        body = np.concatenate([fc["body"], eb])
        size = np.concatenate([np.full(nblk, 8, np.int64), np.ones(ne, np.int64)])
        order = np.lexsort((np.concatenate([fc["start"], er]), body))
        first = np.zeros(len(order), np.int64)
        if len(order):
            first[order] = np.concatenate([[0], np.cumsum(size[order])[:-1]])
        counts = np.bincount(body, weights=size, minlength=n)[:n].astype(np.int64) if len(body) else np.zeros(n, np.int64)
        sg_start = np.zeros(n + 1, np.int32)
        sg_start[1:] = np.cumsum(counts)
        return fc, first[:nblk], first[nblk:], sg_start

    def _build_row_map(self) -> np.ndarray:
        """Static row -> (group, row within the group) in the reference's row
        numbering, from the static layout (computed when first needed)."""
        fc, bfirst, efirst, _ = self._layout
        rm = np.zeros((len(self._rows), 2), np.int64)
        per = fc["per"]
        if len(per):
            nr = 8 * per
            rel = np.arange(int(nr.sum())) - np.repeat(np.cumsum(nr) - nr, nr)
            pr = np.repeat(per, nr)
            rows = np.repeat(fc["start"], nr) + rel
            rm[rows, 0] = np.repeat(bfirst, nr) + rel // pr
            rm[rows, 1] = rel % pr
        for j, g in enumerate(self._groups):
            for s_ in range(3 if g[3] else 1):
                rm[g[2] + s_] = (efirst[j], s_)
        return rm

    @property
    def _row_map(self) -> np.ndarray:
        if self._row_map_cache is None:
            self._row_map_cache = self._build_row_map()
        return self._row_map_cache

    def _explicit_group_arrays(self, efirst):
        """Records of the explicit static groups (pins) at their groups."""
        ne = len(self._groups)
        body = np.full((ne, 2), -1, np.int32)
        meta = np.zeros(ne, np.int32)
        row0 = np.zeros(ne, np.int32)
        offa = np.zeros((ne, 4), np.float32)
        gn = np.zeros((ne, 4), np.float32)
        mat = np.zeros((ne, 4), np.float32)
        flags = np.zeros(ne, np.int32)
        for j, (kind, b, r0_, th, off, extra, mu_, mus_, stiff, frac) in enumerate(self._groups):
            body[j, 0] = b
            meta[j] = kind | (4 if th else 0) | (8 if not (stiff < _INF) else 0)
            row0[j] = r0_
            offa[j, :3] = off
            if kind == KIND_FLOOR:
                offa[j, 3] = extra[1]
            else:
                gn[j, :3] = extra
            mat[j] = (mu_, mus_, stiff, frac)
            flags[j] = 7 if th else 1
        return dict(body=body, meta=meta, row0=row0, offa=offa, n=gn, mat=mat, flags=flags)

    def _upload_static_groups(self) -> None:
        """Static groups on the device: floor blocks expanded by
        avbd_build_floor_groups (8 corner groups per block), explicit groups
        (pins) written from host records, the per-body ranges (SG_START)."""
        self._layout = fc, bfirst, efirst, sg_start = self._static_layout()
        self._row_map_cache = None
        dev = self.device
        nblk = len(fc["body"])
        if nblk:
            i32 = lambda a: torch.from_numpy(np.ascontiguousarray(a, np.int32)).to(dev)
            he_fy = np.zeros((nblk, 4), np.float32)
            he_fy[:, :3] = fc["he"]
            he_fy[:, 3] = fc["fy"]
            mat = np.zeros((nblk, 4), np.float32)
            mat[:, 0], mat[:, 1], mat[:, 2] = fc["mu"], fc["mus"], fc["stiff"]
            t = [i32(fc["body"]), torch.from_numpy(he_fy).to(dev), torch.from_numpy(mat).to(dev), i32(fc["start"]),
                 i32(fc["per"]), i32(bfirst)]
            _lib.check(_lib.load().avbd_build_floor_groups(self._ctx, nblk, *[C.c_void_p(x.data_ptr()) for x in t],
                                                           self._stream()), "build floor groups")
        if len(self._groups):
            eg = self._explicit_group_arrays(efirst)
            idx = torch.from_numpy(efirst).to(dev)
            for name, arr in (("_g_body", eg["body"]), ("_g_meta", eg["meta"]), ("_g_row0", eg["row0"]),
                              ("_g_offa", eg["offa"]), ("_g_n", eg["n"]), ("_g_mat", eg["mat"]),
                              ("_g_flags", eg["flags"])):
                getattr(self, name).index_copy_(0, idx, torch.from_numpy(arr).to(dev))
            self._g_lam.index_fill_(0, idx, 0.0)
            self._g_pen.index_fill_(0, idx, 1.0)  # solver_6dof.py:1121 (penalty seeded to 1)
        self._sg_start.copy_(torch.from_numpy(sg_start))

    @_on_stream
    def _flush(self) -> None:
        if not self._dirty:
            return
        n = len(self._x)
        prev = None
        if self._arena is not None:
            k = min(n, self._arena.dims.n_bodies)
            prev = (k, self.x4[:k].clone(), self.q[:k].clone(), self.v4[:k].clone(), self.w4[:k].clone(),
                    self.pv4[:k].clone(), self.pw4[:k].clone())
        if self._ctx is not None:
            _lib.load().avbd_destroy(self._ctx)
            self._ctx = None
        dims = self._dims()
        self._arena = _Arena(dims, self.device)
        self._views()
        dev = self.device
        if n:
            m = np.fromiter(self._mass, np.float32, n)
            rows = lambda lst, k: np.fromiter(itertools.chain.from_iterable(lst), np.float32, k * n).reshape(n, k)
            x4 = np.zeros((n, 4), np.float32)
            x4[:, :3] = rows(self._x, 3)
            x4[:, 3] = m
            self.x4.copy_(torch.from_numpy(x4))
            self.q.copy_(torch.from_numpy(rows(self._q, 4)))
            self.v4[:, :3].copy_(torch.from_numpy(rows(self._v, 3)))
            self.w4[:, :3].copy_(torch.from_numpy(rows(self._omega, 3)))
            he = rows(self._half_extents, 3)
            he4 = np.zeros((n, 4), np.float32)
            he4[:, :3] = he
            he4[:, 3] = np.fromiter(self._friction, np.float32, n)
            self._he4.copy_(torch.from_numpy(he4))
            il = np.zeros((n, 4), np.float32)
            il[:, :3] = _box_inertia_diag_batch(np.fromiter(self._mass, np.float64, n),
                                                np.fromiter(itertools.chain.from_iterable(self._half_extents),
                                                            np.float64, 3 * n).reshape(n, 3))
            self._iloc4.copy_(torch.from_numpy(il))
            prio = np.random.default_rng(seed=0xA5BD).uniform(0.0, 1.0, size=n).astype(np.float32)
            self._prio.copy_(torch.from_numpy(prio))
        if prev is not None:
            k = prev[0]
            for dst, src in zip((self.x4, self.q, self.v4, self.w4, self.pv4, self.pw4), prev[1:]):
                dst[:k].copy_(src)
        if self._mlp is not None:
            self._arena.view("MLP_W", torch.float32, (self._mlp.n_floats,)).copy_(self._mlp.packed(dev))
        if self._scene_tab:
            if len(self._scene_of) != n:
                raise RuntimeError("every body of a batched solver must belong to a scene")
            self._arena.view("SCENE_OF", torch.int32, (n,)).copy_(torch.tensor(self._scene_of, dtype=torch.int32))
        L = _lib.load()
        ctx = C.c_void_p()
        _lib.check(L.avbd_create(C.byref(dims), C.c_void_p(self._arena.ptr()), self._arena.total, C.byref(ctx)),
                   "create")
        self._ctx = ctx
        st = self._stream()
        self._upload_static_groups()
        _lib.check(L.avbd_reset_state(self._ctx, st), "reset")
        self._pushed = None  # a new context starts without parameters
        self._push_params()
        self._gpu_pool_n_static = len(self._rows)
        self._gpu_pool_n_dyn_capacity = dims.dyn_row_cap
        self._gpu_pool_n_capacity = len(self._rows) + dims.dyn_row_cap
        self._gpu_pool_max_pairs = dims.dyn_row_cap // 12
        self._bp_max_pairs = dims.pair_cap
        self._gpu_pool_hash_cap = dims.hash_cap if self._self_collide else 0
        self.num_colors = MAX_COLORS
        self.num_active_colors = MAX_COLORS
        self._n_active_colors = MAX_COLORS
        self._color_dirty = True
        self._dirty = False

    def _params(self) -> _lib.AvbdParams:
        p = _lib.AvbdParams()
        p.dt = self.dt
        p.iterations = self.iterations
        p.gravity[:] = self.gravity
        p.alpha, p.beta, p.gamma = self.alpha, self.beta, self.gamma
        p.post_stabilize = int(self.post_stabilize)
        p.max_linear_speed = self.max_linear_speed
        p.max_angular_speed = self.max_angular_speed
        p.substeps = self.substeps
        p.friction_static_mult = self.friction_static_mult
        p.coloring_mode = 0 if self._coloring_mode == "jacobi" else 1
        p.recolor_every_substep = int(self._recolor_every_substep)
        p.self_collide = int(self._self_collide)
        p.self_friction = self._self_friction
        p.group_size = self._primal_group_size
        p.use_graph = int(self.use_graph)
        p.persistent = int(self.persistent)
        p.record_violation = int(self.record_violation)
        p.mlp_warm_start = int(self._mlp is not None and getattr(self._mlp, "enabled", True))
        p.debug_skip_arrive = int(self._debug_skip_arrive)
        p.blocks_per_sm = int(self.blocks_per_sm)
        p.timing = int(self.timing)
        p.log_new_contacts = int(self._log_new)
        p.flag_sweep = int(bool(self.flag_sweep))
        p.adaptive_lanes = int(bool(self.adaptive_lanes))
        p.resting_floor = int(bool(self.resting_floor))
        p.bvh_rebuild_every = max(1, int(self.bvh_rebuild_every))
        if self._scene_tab:  # the device loops cover the largest scene settings
            p.substeps = max(sc for sc, _ in self._scene_tab)
            p.iterations = max(it for _, it in self._scene_tab)
        return p

    def _push_params(self):
        p = self._params()
        key = bytes(p) + repr(self._scene_tab).encode()
        if getattr(self, "_pushed", None) != key:
            _lib.check(_lib.load().avbd_set_params(self._ctx, C.byref(p), self._stream()), "set_params")
            if self._scene_tab:  # per scene: (substep dt, iterations, substeps, 0)
                tab = torch.tensor([(self.dt / sc, float(it), float(sc), 0.0) for sc, it in self._scene_tab],
                                   dtype=torch.float32)
                with torch.cuda.stream(self._cuda_stream):
                    self._arena.view("SCENE_TAB", torch.float32, (len(self._scene_tab), 4)).copy_(tab)
            self._pushed = key

    def _current_graph_signature(self) -> tuple:
        """Scalars of the solve (solver_6dof.py:1466-1491).  They live in a
        device parameter block, so changing one never requires a recapture;
        the tuple is kept for API compatibility."""
        return (int(self.iterations), int(self.post_stabilize), int(self._max_colors), int(self._n_active_colors),
                int(self._primal_group_size), int(self._primal_shuffle), int(self._primal_fused),
                int(self._gpu_resident), int(self._recolor_every_substep), float(self.dt), float(self.alpha),
                float(self.beta), float(self.gamma), float(self.max_linear_speed), float(self.max_angular_speed))

    # ---- stepping (solver_6dof.py:1178-1230) ----------------------------------
    @_on_stream
    def step(self) -> None:
        self._enqueue_step()
        self._after_frame()

    def _enqueue_step(self) -> None:
        """Launch one frame without reading anything back."""
        if self._dirty:
            self._flush()
        self._graph_signature = self._current_graph_signature()
        if len(self._x) == 0:
            return
        self._push_params()
        _lib.check(_lib.load().avbd_step(self._ctx, self._stream()), "step")

    @_on_stream
    def substep(self, dt=None) -> None:
        """One substep of `dt` (default dt / substeps) -- the unit the parity
        tests compare against the oracle."""
        if self._dirty:
            self._flush()
        if len(self._x) == 0:
            return
        self._push_params()
        d = self.dt / self.substeps if dt is None else float(dt)
        _lib.check(_lib.load().avbd_substep(self._ctx, C.c_float(d), self._stream()), "substep")
        self._after_frame()

    def _after_frame(self) -> None:
        if len(self._x) == 0 or self._ctx is None:
            return
        L = _lib.load()
        code = L.avbd_read_stats(self._ctx, C.byref(self._stats), self._stream())
        self.host_syncs += 1
        s = self._stats
        if code < 0 or (s.err & _lib.AVBD_ERR_BARRIER_TIMEOUT):
            raise RuntimeError(f"libavbd6 step failed: {L.avbd_last_error().decode()} (err bits {s.err})")
        cc, sc = C.c_float(0.0), C.c_float(0.0)
        L.avbd_step_ms(self._ctx, C.byref(cc), C.byref(sc))
        self.broadphase_ms = float(cc.value)
        self.solve_ms = float(sc.value)
        self._n_active_colors = max(1, min(int(s.n_colors), MAX_COLORS))
        self.num_active_colors = self._n_active_colors
        self._color_dirty = False
        self._check_overflow()

    def _check_overflow(self) -> None:
        """Once per frame (solver_6dof.py:1199-1230): warn when contacts were
        dropped and grow the pools so the next frame has room."""
        s = self._stats
        dims = self._arena.dims
        pair_over = s.n_pairs_found > dims.pair_cap
        row_over = s.n_dyn_rows_req > dims.dyn_row_cap
        if not (pair_over or row_over):
            return
        msg = (f"avbd_b200: row pool overflow ({s.n_dyn_rows_req} rows requested > {dims.dyn_row_cap} dynamic "
               f"capacity; {s.n_pairs_found} broadphase pairs, pair capacity {dims.pair_cap}) -- contacts were "
               "dropped this frame; growing the pools for the next frame.")
        warnings.warn(msg, RuntimeWarning, stacklevel=3)
        new_pairs = max(dims.pair_cap, 2 * s.n_pairs_found) if pair_over else dims.pair_cap
        est_rows = s.n_dyn_rows_req
        if pair_over and s.n_pairs > 0:
            est_rows = int(est_rows * s.n_pairs_found / max(1, s.n_pairs))
        new_rows = max(dims.dyn_row_cap, 2 * est_rows) if (row_over or pair_over) else dims.dyn_row_cap
        self._grow(new_pairs, new_rows)

    @_on_stream
    def _grow(self, pair_cap: int, dyn_rows: int) -> None:
        old, old_ctx = self._arena, self._ctx
        dims = self._dims(pair_cap=pair_cap, dyn_rows=dyn_rows)
        dims.hash_cap = old.dims.hash_cap
        new = _Arena(dims, self.device)
        keep = ["BX", "BQ", "BV", "BW", "BPV", "BPW", "BILOC", "BHE", "BPRIO", "COLOR", "COLOR_STARTS",
                "COLOR_BODIES", "SG_START", "H_KEY", "H_S0", "H_S1", "MLP_W", "PARAMS", "COUNTERS"]
        ng = old.dims.n_static_groups
        nxt = {nm: old.off[old.names[i + 1]] for i, nm in enumerate(old.names[:-1])}
        for nm in keep:
            nbytes = nxt.get(nm, old.total) - old.off[nm]
            nbytes = min(nbytes, (new.off[new.names[new.names.index(nm) + 1]] if nm != new.names[-1] else new.total)
                         - new.off[nm])
            new.buf[new.off[nm]:new.off[nm] + nbytes].copy_(old.buf[old.off[nm]:old.off[nm] + nbytes])
        for nm, w in (("G_BODY", 8), ("G_META", 4), ("G_ROW0", 4), ("G_FLAGS", 4), ("G_OFFA", 16), ("G_OFFB", 16),
                      ("G_N", 16), ("G_MAT", 16), ("G_LAM", 16), ("G_PEN", 16), ("G_AC0", 16)):
            nbytes = w * ng
            new.buf[new.off[nm]:new.off[nm] + nbytes].copy_(old.buf[old.off[nm]:old.off[nm] + nbytes])
        L = _lib.load()
        ctx = C.c_void_p()
        _lib.check(L.avbd_create(C.byref(dims), C.c_void_p(new.ptr()), new.total, C.byref(ctx)), "create")
        self._cuda_stream.synchronize()
        L.avbd_destroy(old_ctx)
        self._arena, self._ctx = new, ctx
        self._views()
        self._pushed = None
        self._push_params()
        self._gpu_pool_n_dyn_capacity = dims.dyn_row_cap
        self._gpu_pool_n_capacity = len(self._rows) + dims.dyn_row_cap
        self._bp_max_pairs = dims.pair_cap

    # ---- diagnostics -------------------------------------------------------------
    @_on_stream
    def count_color_conflicts(self) -> int:
        """Active two-body contacts whose bodies share a color (solver_6dof.py:846-862)."""
        if self._ctx is None:
            return 0
        return int(_lib.load().avbd_count_color_conflicts(self._ctx, self._stream()))

    def phase_profile(self) -> dict:
        """Device time (ms) per phase of the last substep's persistent solve
        kernel and the number of grid barriers of each (needs timing=True)."""
        cap = 256
        t = (C.c_longlong * cap)()
        ph = (C.c_int * cap)()
        n = _lib.check(_lib.load().avbd_read_phase_marks(self._ctx, t, ph, cap, self._stream()), "phase marks")
        out = {}
        for k in range(1, n):
            name = _lib.PHASES[ph[k]] if 0 <= ph[k] < len(_lib.PHASES) else str(ph[k])
            ms, cnt = out.get(name, (0.0, 0))
            out[name] = (ms + (t[k] - t[k - 1]) * 1e-6, cnt + 1)
        return out

    @_on_stream
    def collision_profile(self) -> dict:
        """Runs one substep whose collision pipeline replays as a one-off
        graph with an event after each stage, and returns {stage: device ms} (a scan
        stage covers its three launches).  The substep is a real one: the
        scene advances."""
        self._flush()
        L = _lib.load()
        _lib.check(L.avbd_profile_next_substep(self._ctx), "profile")
        self.substep()
        cap = 48
        ms = (C.c_float * cap)()
        n = _lib.check(L.avbd_collision_profile(self._ctx, ms, cap), "collision profile")
        return {L.avbd_collision_stage(self._ctx, k).decode(): float(ms[k]) for k in range(n)}

    def clear_errors(self) -> None:
        """Clear the sticky device error bits (after handling a reported error)."""
        if self._ctx is not None:
            _lib.check(_lib.load().avbd_clear_errors(self._ctx, self._stream()), "clear_errors")
            self._stats.err = 0

    # ---- learned warm start (no reference counterpart) ----------------------
    @property
    def log_new_contacts(self) -> bool:
        """Queue the 20 features (and group id) of every new contact each
        substep; new_contact_log() reads the queue of the last substep."""
        return self._log_new

    @log_new_contacts.setter
    def log_new_contacts(self, on: bool) -> None:
        self._log_new = bool(on)
        if self._arena is not None and self._log_new and self._arena.dims.new_cap == 0:
            self._dirty = True  # re-flush with a queue (keeps bodies, empties the contact cache)

    @property
    def warm_start(self):
        """The learned warm-start model (avbd_b200.learned.WarmStartMLP) or None."""
        return self._mlp

    @warm_start.setter
    def warm_start(self, model) -> None:
        had = self._mlp is not None
        self._mlp = model
        if self._arena is None:
            return
        if (model is not None) != had or (model is not None and self._arena.dims.new_cap == 0):
            self._dirty = True
        elif model is not None:
            with torch.cuda.stream(self._cuda_stream):
                self._arena.view("MLP_W", torch.float32, (model.n_floats,)).copy_(model.packed(self.device))

    @_on_stream
    def new_contact_log(self):
        """(features [n, 20] float32, group ids [n] int32) of the new contacts
        queued by the last substep (queue order is not deterministic)."""
        if self._arena is None or self._arena.dims.new_cap == 0:
            return np.zeros((0, _lib.MLP_IN), np.float32), np.zeros(0, np.int32)
        n = min(int(self._stats.n_new_logged), self._arena.dims.new_cap)
        cap = self._arena.dims.new_cap
        feat = self._arena.view("MLP_FEAT", torch.float32, (cap, _lib.MLP_IN))[:n].cpu().numpy()
        gid = self._arena.view("NEW_LIST", torch.int32, (cap,))[:n].cpu().numpy()
        return feat, gid

    @_on_stream
    def group_state(self, gid):
        """(lambda [n, 4], penalty [n, 4]) of contact groups `gid` (the state
        the contact cache stores for them after this substep)."""
        idx = torch.as_tensor(np.asarray(gid, np.int64), device=self.device)
        return self._g_lam[idx].cpu().numpy(), self._g_pen[idx].cpu().numpy()

    @property
    def cache_key_mode(self) -> str:
        """How the contact cache identifies a contact across substeps:
        "ordinal" -- (a, b, place in the pair's manifold), the key of the
        reference's live cache (kernels_6dof.py:2588-2594); "anchor_5mm" --
        (a, b, contact point in body a's frame rounded to 5 mm), the key of
        its documented cache (PERFORMANCE_PROGRESS.md:122-125), which
        survives reordering of the manifold.  Changing it empties the cache."""
        return "anchor_5mm" if self._anchor_keys else "ordinal"

    @cache_key_mode.setter
    def cache_key_mode(self, mode: str) -> None:
        if mode not in ("ordinal", "anchor_5mm"):
            raise ValueError(f"cache_key_mode must be 'ordinal' or 'anchor_5mm', got {mode!r}")
        on = mode == "anchor_5mm"
        if on != self._anchor_keys:
            self._anchor_keys = on
            self._dirty = True  # re-flush: the arena gains / drops the per-group key array

    @property
    def _contact_cache(self) -> dict:
        """The warm-start contact cache as {key: state}: key (a, b, ordinal)
        with a < b the bodies and ordinal the contact's place in the pair's
        manifold (the raw 50-bit anchor fingerprint in "anchor_5mm" mode),
        state 8 floats (lambda n/t1/t2, penalty n/t1/t2, was_static t1/t2).
        A host copy of the device hash (kernels_6dof.py:2915-2995 keep the
        same contents in hash_keys / hash_state)."""
        sd = self.state_dict()
        if self._anchor_keys:
            return {int(k): st for k, st in zip(sd["cache_keys"], sd["cache_state"])}
        return {tuple(int(v) for v in k): st for k, st in zip(sd["cache_abc"], sd["cache_state"])}

    @_on_stream
    def clear_contact_cache(self) -> None:
        """Empties the contact cache: every contact of the next substep is new."""
        self._flush()
        if self._ctx is not None:
            _lib.check(_lib.load().avbd_cache_load(self._ctx, 0, None, None, self._stream()), "cache clear")

    def stats(self) -> dict:
        s = self._stats
        return {k: getattr(s, k) for k, _ in _lib.AvbdStats._fields_ if k not in ("viol", "viol_contact")}

    def violation_history(self) -> np.ndarray:
        """Max constraint violation after each iteration of the last substep
        (record_violation): max(0, -C) of contact normals, |C| of pins, C
        relative to alpha*C0 for hard rows."""
        s = self._stats
        return np.array(s.viol[: s.n_viol], np.float64)

    def contact_violation_history(self) -> np.ndarray:
        """Max violation over the box-box contacts (the rows a contact warm
        start sets) after each iteration of the last substep
        (record_violation)."""
        s = self._stats
        return np.array(s.viol_contact[: s.n_viol], np.float64)

    @property
    def n_active_rows(self) -> torch.Tensor:
        """Live row count, [n_static + dynamic rows] (host tensor with .numpy())."""
        return torch.tensor([len(self._rows) + int(self._stats.n_dyn_rows)], dtype=torch.int32)

    @property
    def _bp_pair_count(self) -> torch.Tensor:
        return torch.tensor([int(self._stats.n_pairs_found)], dtype=torch.int32)

    @property
    @_on_stream
    def body_color(self) -> torch.Tensor:
        """Per-body color (host tensor with .numpy())."""
        if self._arena is None:
            return torch.full((max(1, len(self._x)),), -1, dtype=torch.int32)
        return self._color[: len(self._x)].cpu()

    # ---- read-back (solver_6dof.py:1920-2052) -----------------------------------
    @_on_stream
    def positions(self) -> np.ndarray:
        if self._arena is None:
            return np.array(self._x, dtype=np.float32).reshape(-1, 3)
        return self.x[: len(self._x)].cpu().numpy().copy()

    @_on_stream
    def orientations(self) -> np.ndarray:
        if self._arena is None:
            return np.array(self._q, dtype=np.float32).reshape(-1, 4)
        return self.q[: len(self._x)].cpu().numpy().copy()

    @_on_stream
    def velocities(self) -> np.ndarray:
        if self._arena is None:
            return np.array(self._v, dtype=np.float32).reshape(-1, 3)
        return self.v[: len(self._x)].cpu().numpy().copy()

    @_on_stream
    def angular_velocities(self) -> np.ndarray:
        if self._arena is None:
            return np.array(self._omega, dtype=np.float32).reshape(-1, 3)
        return self.omega[: len(self._x)].cpu().numpy().copy()

    @_on_stream
    def _row_state(self):
        """Per-row (lambda, penalty, alpha*C0, active, was_static, type) over the
        row capacity, in the reference's row numbering."""
        cap = self._gpu_pool_n_capacity if self._arena is not None else len(self._rows)
        lam = np.zeros(cap, np.float32)
        pen = np.ones(cap, np.float32)
        ac0 = np.zeros(cap, np.float32)
        act = np.zeros(cap, np.int32)
        was = np.zeros(cap, np.int32)
        typ = np.zeros(cap, np.int32)
        if self._arena is None:
            act[: len(self._rows)] = 1
            return lam, pen, ac0, act, was, typ
        ng = self._n_static_groups + int(self._stats.n_dyn_groups)
        ng = min(ng, self._g_meta.shape[0])
        meta = self._g_meta[:ng].cpu().numpy()
        row0 = self._g_row0[:ng].cpu().numpy()
        fl = self._g_flags[:ng].cpu().numpy()
        L = self._g_lam[:ng].cpu().numpy()
        P = self._g_pen[:ng].cpu().numpy()
        A = self._g_ac0[:ng].cpu().numpy()
        three = (meta & 4) != 0
        kind = meta & 3
        for s in range(3):
            sel = np.ones(ng, bool) if s == 0 else three
            r = row0[sel] + s
            ok = r < cap
            r = r[ok]
            lam[r] = L[sel, s][ok]
            pen[r] = P[sel, s][ok]
            ac0[r] = A[sel, s][ok]
            act[r] = ((fl[sel] >> s) & 1)[ok]
            k = kind[sel][ok]
            if s == 0:
                typ[r] = np.where(k == KIND_FLOOR, FLOOR_CONTACT_6DOF, np.where(k == KIND_PIN, PIN_6DOF,
                                                                               BOX_BOX_CONTACT_6DOF))
                was[r] = np.where(k == KIND_PIN, 0, (fl[sel][ok] >> 3) & 1)
            else:
                typ[r] = np.where(k == KIND_PIN, PIN_6DOF, CONTACT_TANGENT_6DOF)
                was[r] = np.where(k == KIND_PIN, 0, (fl[sel][ok] >> (3 + s)) & 1)
        return lam, pen, ac0, act, was, typ

    def lambdas(self) -> np.ndarray:
        return self._row_state()[0]

    def active(self) -> np.ndarray:
        return self._row_state()[3]

    @property
    def stream(self) -> torch.cuda.Stream:
        """The CUDA stream every launch of this solver is enqueued on."""
        return self._cuda_stream

    def state_views(self) -> dict:
        """Zero-copy device views of the body state (torch tensors on the
        solver's device, valid until the scene is rebuilt): positions [N, 3],
        orientations [N, 4] (xyzw), velocities [N, 3], angular_velocities
        [N, 3].  The host-copy getters and read_state_batched
        (solver_6dof.py:1920-2052) stay available; consumers on another
        stream wait on `stream` before reading.  Writes through the views
        change the simulation."""
        self._flush()
        n = len(self._x)
        return {"positions": self.x[:n], "orientations": self.q[:n], "velocities": self.v[:n],
                "angular_velocities": self.omega[:n]}

    def read_state_batched(self, include_rows: bool = True) -> dict:
        """Positions, orientations, angular velocities and per-row diagnostics
        (solver_6dof.py:1952-2052)."""
        n_c = int(self.n_active_rows[0]) if (include_rows and self._arena is not None) else (
            len(self._rows) if include_rows else 0)
        out = {"positions": self.positions(), "orientations": self.orientations(),
               "angular_velocities": self.angular_velocities()}
        if include_rows:
            lam, _, _, act, was, typ = self._row_state()
            out.update(lambdas=lam[:n_c].copy(), active=act[:n_c].copy(), was_static=was[:n_c].copy(),
                       c_type=typ[:n_c].copy())
        else:
            out.update(lambdas=np.zeros(0, np.float32), active=np.zeros(0, np.int32),
                       was_static=np.zeros(0, np.int32), c_type=np.zeros(0, np.int32))
        out["n_rows"] = n_c
        return out

    # ---- in-place setters (solver_6dof.py:878-900) -------------------------------
    # They write into the existing device buffers (never rebind them), so
    # captured CUDA graphs keep operating on the live state.
    @_on_stream
    def _set_row(self, name: str, idx: int, vals) -> None:
        self._flush()
        t = getattr(self, name)
        t[idx, : len(vals)] = torch.tensor([float(v) for v in vals], dtype=torch.float32, device=self.device)

    def set_position(self, body, p) -> None:
        self._set_row("x4", body.index, p)

    def set_orientation(self, body, q_xyzw) -> None:
        self._set_row("q", body.index, q_xyzw)

    def set_velocity(self, body, v) -> None:
        self._set_row("v4", body.index, v)

    def set_angular_velocity(self, body, w) -> None:
        self._set_row("w4", body.index, w)

    @_on_stream
    def upload_body_state(self, x4, q, v4=None, w4=None) -> None:
        """Bulk in-place overwrite of the body state from host (pinned) (N,4)
        float32 tensors: x (w = mass), q (xyzw), v, w.  Asynchronous."""
        self._flush()
        n = len(self._x)
        for dst, src in ((self.x4, x4), (self.q, q), (self.v4, v4), (self.w4, w4)):
            if src is not None:
                dst[:n].copy_(src, non_blocking=True)

    @_on_stream
    def download_poses(self, x_out, q_out) -> None:
        """Copy positions (x, mass) and orientations into host (pinned) (N,4)
        float32 tensors and wait for them."""
        n = len(self._x)
        x_out.copy_(self.x4[:n], non_blocking=True)
        q_out.copy_(self.q[:n], non_blocking=True)
        self._cuda_stream.synchronize()

    # ---- state transfer (parity tests, checkpoints) ------------------------------
    @_on_stream
    def state_dict(self) -> dict:
        """Every piece of state that persists across substeps, as numpy."""
        self._flush()
        n = len(self._x)
        lam, pen, _, act, was, _ = self._row_state()
        ns = len(self._rows)
        tag = 1 + (int(self._stats.epoch) % 16000)
        keys = self._h_key.cpu().numpy().view(np.uint64)
        live = (keys >> np.uint64(50)) == np.uint64(tag)
        k = keys[live]
        abc = np.stack([((k >> np.uint64(26)) & np.uint64(0xFFFFFF)).astype(np.int64),
                        ((k >> np.uint64(2)) & np.uint64(0xFFFFFF)).astype(
            np.int64), (k & np.uint64(3)).astype(np.int64)], axis=1).astype(np.int32) if k.size else np.zeros(
            (0, 3), np.int32)
        st = np.concatenate([self._h_s0.cpu().numpy()[live], self._h_s1.cpu().numpy()[live]], axis=1)
        raw = k & np.uint64((1 << 50) - 1)
        if self._anchor_keys:  # fingerprints: no (a, b, ordinal) to decode
            order = np.argsort(raw, kind="stable")
            abc = np.zeros((0, 3), np.int32)
        else:
            order = np.lexsort((abc[:, 2], abc[:, 1], abc[:, 0])) if k.size else np.zeros(0, np.int64)
            abc = abc[order]
        return dict(x=self.x[:n].cpu().numpy().astype(np.float64), q=self.q[:n].cpu().numpy().astype(np.float64),
                    v=self.v[:n].cpu().numpy().astype(np.float64), w=self.omega[:n].cpu().numpy().astype(np.float64),
                    pv=self.prev_v[:n].cpu().numpy().astype(np.float64),
                    pw=self.prev_omega[:n].cpu().numpy().astype(np.float64),
                    row_lam=lam[:ns].astype(np.float64), row_pen=pen[:ns].astype(np.float64),
                    row_active=act[:ns].copy(), row_was=was[:ns].copy(),
                    cache_abc=abc, cache_keys=raw[order], cache_state=st[order].astype(np.float64),
                    colors=self._color[:n].cpu().numpy().copy(), n_colors=int(self._stats.n_colors),
                    color_dirty=bool(self._color_dirty))

    @_on_stream
    def load_state_dict(self, sd: dict) -> None:
        """Inverse of state_dict (bodies, static rows, contact cache, colors)."""
        self._flush()
        n = len(self._x)
        dev = self.device
        f = lambda a: torch.as_tensor(np.asarray(a, np.float32), device=dev)
        self.x4[:n, :3] = f(sd["x"])
        self.q[:n] = f(sd["q"])
        self.v4[:n, :3] = f(sd["v"])
        self.w4[:n, :3] = f(sd["w"])
        self.pv4[:n, :3] = f(sd["pv"])
        self.pw4[:n, :3] = f(sd["pw"])
        ns = len(self._rows)
        if ns:
            rm = self._row_map
            ng = self._n_static_groups
            lam = self._g_lam[:ng].cpu().numpy()
            pen = self._g_pen[:ng].cpu().numpy()
            fl = self._g_flags[:ng].cpu().numpy()
            meta = self._g_meta[:ng].cpu().numpy()
            g_of, s_of = rm[:ns, 0], rm[:ns, 1]
            lam[g_of, s_of] = np.asarray(sd["row_lam"], np.float32)[:ns]
            pen[g_of, s_of] = np.asarray(sd["row_pen"], np.float32)[:ns]
            act = np.asarray(sd["row_active"], np.int32)[:ns]
            was = np.asarray(sd["row_was"], np.int32)[:ns]
            for s in range(3):  # one row per group in each pass
                m = s_of == s
                g = g_of[m]
                fl[g] = (fl[g] & ~(1 << s)) | (act[m] << s)
                if s == 0:
                    nonpin = (meta[g] & 3) != KIND_PIN
                    g2 = g[nonpin]
                    fl[g2] = (fl[g2] & ~8) | (was[m][nonpin] << 3)
            self._g_lam[:ng] = torch.from_numpy(lam).to(dev)
            self._g_pen[:ng] = torch.from_numpy(pen).to(dev)
            self._g_flags[:ng] = torch.from_numpy(fl).to(dev)
        stt = np.ascontiguousarray(sd["cache_state"], np.float32)
        ts = torch.from_numpy(stt).to(dev) if stt.size else torch.zeros((1, 8), dtype=torch.float32, device=dev)
        if self._anchor_keys:
            ks = np.ascontiguousarray(sd["cache_keys"], np.uint64).view(np.int64)
            tk = torch.from_numpy(ks.copy()).to(dev) if ks.size else torch.zeros(1, dtype=torch.int64, device=dev)
            _lib.check(_lib.load().avbd_cache_load_keys(self._ctx, int(ks.shape[0]), C.c_void_p(tk.data_ptr()),
                                                        C.c_void_p(ts.data_ptr()), self._stream()), "cache_load")
        else:
            abc = np.ascontiguousarray(sd["cache_abc"], np.int32)
            ta = torch.from_numpy(abc).to(dev) if abc.size else torch.zeros((1, 3), dtype=torch.int32, device=dev)
            _lib.check(_lib.load().avbd_cache_load(self._ctx, int(abc.shape[0]), C.c_void_p(ta.data_ptr()),
                                                   C.c_void_p(ts.data_ptr()), self._stream()), "cache_load")
        colors = np.asarray(sd["colors"], np.int32)
        self._color[:n] = torch.from_numpy(colors).to(dev)
        cs = np.zeros(64, np.int32)
        cnt = np.bincount(np.clip(colors, 0, MAX_COLORS - 1), minlength=MAX_COLORS)
        cs[1:MAX_COLORS + 1] = np.cumsum(cnt)
        self._color_starts.copy_(torch.from_numpy(cs))
        self._color_bodies[:n] = torch.from_numpy(np.argsort(colors, kind="stable").astype(np.int32)).to(dev)
        ctr = self._arena.view("COUNTERS", torch.int32, (8,))
        ctr[7] = int(sd["n_colors"])  # DevCounters.n_colors
        dirty = self._arena.view("COUNTERS", torch.int32, (12,))
        dirty[11] = int(bool(sd["color_dirty"]))  # DevCounters.color_dirty
        self._color_dirty = bool(sd["color_dirty"])
        self._cuda_stream.synchronize()
        ta, ts = None, None

    # ---- debug views of the last substep ---------------------------------------
    @_on_stream
    def pairs(self) -> dict:
        """Broadphase pairs (i<j, sorted) with SAT / manifold outcome."""
        np_ = min(int(self._stats.n_pairs), self._pair_ab.shape[0])
        ab = self._pair_ab[:np_].cpu().numpy()
        info = self._pair_info[:np_].cpu().numpy()
        ov = info & 1
        return dict(a=ab[:, 0].copy(), b=ab[:, 1].copy(), overlap=ov, sat_idx=np.where(ov == 1, (info >> 1) & 31, -1),
                    count=(info >> 6) & 7, n_hat=self._pair_nrm[:np_, :3].cpu().numpy())

    @_on_stream
    def contacts(self) -> np.ndarray:
        """(ref body, inc body, ordinal) of every emitted dynamic contact, row order."""
        ns = self._n_static_groups
        nd = int(self._stats.n_dyn_groups)
        b = self._g_body[ns:ns + nd].cpu().numpy()
        meta = self._g_meta[ns:ns + nd].cpu().numpy()
        row0 = self._g_row0[ns:ns + nd].cpu().numpy()
        o = np.argsort(row0, kind="stable")
        return np.stack([b[o, 0], b[o, 1], (meta[o] >> 4) & 3], axis=1).astype(np.int32)
