"""Python front end of the CPU oracle -- TEST INFRASTRUCTURE ONLY.

`OracleSolver6DOF` restates the scene-building API of the reference
`Solver6DOF` (src/avbd3d/solver_6dof.py:446-578) and runs the substep through
`oracle/_build/liboracle.so` (the C++ restatement in `avbd_oracle.cpp`).

Only the test-suite, `__graft_entry__.smoke()` and the `cpu_baseline` leg of
`bench.py` import this module.  The product package `avbd_b200` never does.
"""

from __future__ import annotations

import ctypes as C
import math
import os
import subprocess
from dataclasses import dataclass

import numpy as np

FLOOR_CONTACT_6DOF = 0
CONTACT_TANGENT_6DOF = 1
PIN_6DOF = 2
BOX_BOX_CONTACT_6DOF = 3

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build() -> str:
    """Compile the oracle with its Makefile (g++, -ffp-contract=off)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        vp, i, d = C.c_void_p, C.c_int, C.c_double
        L.orc_create.restype = vp
        L.orc_create.argtypes = [i]
        L.orc_destroy.argtypes = [vp]
        L.orc_set_params.argtypes = [vp, d, i, d, d, d, d, d, d, i, d, d, i, d, i, i, i, d, i]
        L.orc_load_scene.argtypes = [vp, i] + [vp] * 9 + [i] + [vp] * 14 + [i, i]
        for name in ("orc_step", "orc_substep", "orc_count_conflicts"):
            getattr(L, name).argtypes = [vp]
        L.orc_set_dt.argtypes = [vp, d]
        L.orc_set_caps.argtypes = [vp, i, i]
        L.orc_set_record_violation.argtypes = [vp, i]
        L.orc_get_violation.argtypes = [vp, vp, i]
        L.orc_get_bodies.argtypes = [vp] * 7
        L.orc_set_bodies.argtypes = [vp] * 7
        L.orc_get_counts.argtypes = [vp, vp]
        L.orc_get_rows.argtypes = [vp, i] + [vp] * 8
        L.orc_set_static_rows.argtypes = [vp] * 5
        L.orc_get_cache.argtypes = [vp, i, vp, vp]
        L.orc_set_cache.argtypes = [vp, i, vp, vp]
        L.orc_set_key_mode.argtypes = [vp, i]
        L.orc_get_cache_keys.argtypes = [vp, i, vp, vp]
        L.orc_set_cache_keys.argtypes = [vp, i, vp, vp]
        L.orc_get_colors.argtypes = [vp, vp]
        L.orc_set_colors.argtypes = [vp, vp, i, i]
        L.orc_get_pairs.argtypes = [vp, i] + [vp] * 6
        L.orc_get_contacts.argtypes = [vp, i, vp]
        L.orc_sat.argtypes = [vp] * 9
        L.orc_sat.restype = i
        L.orc_geom_stiffness_diag.argtypes = [vp, vp, vp]
        _lib = L
    return _lib


def _p(a: np.ndarray):
    return a.ctypes.data_as(C.c_void_p)


def obb_sat(c_A, R_A, e_A, c_B, R_B, e_B, q_A=None, q_B=None):
    """15-axis SAT known-answer probe (kernels_6dof.py:1991-2130).  Poses are
    given as quaternions (xyzw); identity when `q_*` is None.  Returns
    (axis_idx, n_hat, overlap) or None, like solver_6dof.py:_obb_sat."""
    qa = np.array(q_A if q_A is not None else (0, 0, 0, 1), np.float32)
    qb = np.array(q_B if q_B is not None else (0, 0, 0, 1), np.float32)
    ca, cb = np.asarray(c_A, np.float32), np.asarray(c_B, np.float32)
    ea, eb = np.asarray(e_A, np.float32), np.asarray(e_B, np.float32)
    idx = np.zeros(1, np.int32)
    n = np.zeros(3, np.float32)
    dep = np.zeros(1, np.float32)
    ok = lib().orc_sat(_p(ca), _p(qa), _p(ea), _p(cb), _p(qb), _p(eb), _p(idx), _p(n), _p(dep))
    if not ok:
        return None
    return int(idx[0]), n, float(dep[0])


def geom_stiffness_diag(n, r) -> np.ndarray:
    """kernels_6dof.py:280-316 in FP64."""
    nn, rr = np.asarray(n, np.float64), np.asarray(r, np.float64)
    out = np.zeros(3, np.float64)
    lib().orc_geom_stiffness_diag(_p(nn), _p(rr), _p(out))
    return out


@dataclass
class RigidBody:
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
    stiffness: float = math.inf
    fracture: float = math.inf
    fmin: float = -math.inf
    fmax: float = math.inf
    sibling: int = -1
    friction: float = 0.0
    friction_static: float = 0.0
    partner: int = -1


def box_inertia_diag(mass: float, hx: float, hy: float, hz: float) -> np.ndarray:
    """Diagonal of solver_6dof.py:132-142 (zero for static bodies), float32."""
    if mass <= 0.0:
        return np.zeros(3, np.float32)
    return np.array([mass / 3.0 * (hy * hy + hz * hz), mass / 3.0 * (hx * hx + hz * hz),
                     mass / 3.0 * (hx * hx + hy * hy)], np.float32)


def body_priorities(n_b: int) -> np.ndarray:
    """Seeded coloring priorities of solver_6dof.py:1004-1009."""
    if n_b <= 0:
        return np.zeros(0, np.float32)
    return np.random.default_rng(seed=0xA5BD).uniform(0.0, 1.0, size=n_b).astype(np.float32)


_MODES = {"jacobi": 0, "speculative": 0, "speculative_greedy": 0, "greedy": 0,
          "jones_plassmann": 1, "jp": 1, "jones-plassmann": 1, "jones plassmann": 1}


class OracleSolver6DOF:
    """CPU restatement of the reference Solver6DOF (scene API + substep)."""

    def __init__(self, dt=1.0 / 60.0, iterations=10, gravity=(0.0, -9.81, 0.0), alpha=0.99, beta=1.0e5,
                 gamma=0.99, post_stabilize=True, max_linear_speed=30.0, max_angular_speed=50.0, substeps=1,
                 friction_static_mult=1.5, coloring_mode="jacobi", precision="float32", threads=1, **_ignored):
        self.dt = float(dt)
        self.iterations = int(iterations)
        self.gravity = tuple(float(g) for g in gravity)
        self.alpha, self.beta, self.gamma = float(alpha), float(beta), float(gamma)
        self.post_stabilize = bool(post_stabilize)
        self.max_linear_speed = float(max_linear_speed)
        self.max_angular_speed = float(max_angular_speed)
        self.substeps = max(1, int(substeps))
        self.friction_static_mult = max(1.0, float(friction_static_mult))
        m = str(coloring_mode).strip().lower()
        if m not in _MODES:
            raise ValueError(f"coloring_mode must be one of ('jones_plassmann', 'jacobi'), got {coloring_mode!r}")
        self.coloring_mode = "jacobi" if _MODES[m] == 0 else "jones_plassmann"
        self.recolor_every_substep = False
        self.precision = 0 if precision in ("float32", "f32", 32) else 1
        self.threads = max(1, int(threads))
        self._x, self._q, self._v, self._w = [], [], [], []
        self._mass, self._he, self._fric = [], [], []
        self._rows: list[_Row] = []
        self._self_collide = False
        self._self_friction = 0.0
        # coloring priorities: the reference's seeded draw over this solver's
        # bodies, unless a checker sets them (a scene cut out of a batch keeps
        # the batch's priorities)
        self.priorities = None
        self._h = lib().orc_create(self.precision)
        self._dirty = True
        self.pair_cap = 0
        self.dyn_cap = 0

    def __del__(self):
        if getattr(self, "_h", None) and _lib is not None:
            _lib.orc_destroy(self._h)
            self._h = None

    # ---- scene building (solver_6dof.py:446-578) ---------------------------
    def add_box(self, position, half_extents, mass, orientation=(0.0, 0.0, 0.0, 1.0), velocity=(0.0, 0.0, 0.0),
                angular_velocity=(0.0, 0.0, 0.0), friction=0.0):
        idx = len(self._x)
        self._x.append(tuple(float(v) for v in position))
        self._q.append(tuple(float(v) for v in orientation))
        self._v.append(tuple(float(v) for v in velocity))
        self._w.append(tuple(float(v) for v in angular_velocity))
        self._mass.append(float(mass))
        he = tuple(float(h) for h in half_extents)
        self._he.append(he)
        self._fric.append(max(0.0, float(friction)))
        self._dirty = True
        return RigidBody(index=idx, half_extents=he)

    def add_floor_contact_box(self, body, floor_y=0.0, friction=None, stiffness=math.inf):
        mu = float(friction) if friction is not None else self._fric[body.index]
        hx, hy, hz = body.half_extents
        out = []
        for sx in (-1.0, 1.0):
            for sy in (-1.0, 1.0):
                for sz in (-1.0, 1.0):
                    off = (sx * hx, sy * hy, sz * hz)
                    n = len(self._rows)
                    self._rows.append(_Row(FLOOR_CONTACT_6DOF, body.index, world_anchor=(0.0, float(floor_y), 0.0),
                                           off_a=off, stiffness=stiffness, fmin=-math.inf, fmax=0.0))
                    out.append(n)
                    if mu > 0.0:
                        mus = mu * self.friction_static_mult
                        t = len(self._rows)
                        self._rows.append(_Row(CONTACT_TANGENT_6DOF, body.index, world_anchor=(1.0, 0.0, 0.0),
                                               off_a=off, stiffness=stiffness, sibling=n, friction=mu,
                                               friction_static=mus, partner=t + 1))
                        self._rows.append(_Row(CONTACT_TANGENT_6DOF, body.index, world_anchor=(0.0, 0.0, 1.0),
                                               off_a=off, stiffness=stiffness, sibling=n, friction=mu,
                                               friction_static=mus, partner=t))
        self._dirty = True
        return out

    def add_pin_corner(self, body, body_local, world_point, stiffness=math.inf, fracture=math.inf):
        out = []
        for axis in (0, 1, 2):
            out.append(len(self._rows))
            self._rows.append(_Row(PIN_6DOF, body.index, body_b=axis,
                                   world_anchor=tuple(float(p) for p in world_point),
                                   off_a=tuple(float(v) for v in body_local), stiffness=stiffness,
                                   fracture=fracture))
        self._dirty = True
        return out

    def enable_self_collision(self, enabled=True, default_friction=0.0):
        self._self_collide = bool(enabled)
        self._self_friction = max(0.0, float(default_friction))
        self._dirty = True

    # ---- upload ----------------------------------------------------------
    def _params(self):
        L = lib()
        L.orc_set_params(self._h, self.dt, self.iterations, *self.gravity, self.alpha, self.beta, self.gamma,
                         int(self.post_stabilize), self.max_linear_speed, self.max_angular_speed, self.substeps,
                         self.friction_static_mult, 0 if self.coloring_mode == "jacobi" else 1,
                         int(self.recolor_every_substep), int(self._self_collide), self._self_friction, self.threads)

    def _flush(self):
        if not self._dirty:
            return
        n = len(self._x)
        prev = None
        if getattr(self, "_nb_loaded", 0) > 0:
            prev = self.get_bodies()
        x = np.array(self._x, np.float32).reshape(-1, 3)
        q = np.array(self._q, np.float32).reshape(-1, 4)
        v = np.array(self._v, np.float32).reshape(-1, 3)
        w = np.array(self._w, np.float32).reshape(-1, 3)
        mass = np.array(self._mass, np.float32)
        he = np.array(self._he, np.float32).reshape(-1, 3)
        fric = np.array(self._fric, np.float32)
        iloc = np.stack([box_inertia_diag(m, *h) for m, h in zip(self._mass, self._he)]) if n else np.zeros((0, 3),
                                                                                                         np.float32)
        iloc = np.ascontiguousarray(iloc, np.float32)
        prio = body_priorities(n) if self.priorities is None else np.ascontiguousarray(self.priorities, np.float32)
        rows = self._rows
        nr = len(rows)
        ia = lambda f: np.array([f(r) for r in rows], np.int32) if nr else np.zeros(0, np.int32)
        fa = lambda f: np.array([f(r) for r in rows], np.float32) if nr else np.zeros(0, np.float32)
        va = lambda f: np.array([f(r) for r in rows], np.float32).reshape(-1, 3) if nr else np.zeros((0, 3), np.float32)
        arrs = [ia(lambda r: r.type), ia(lambda r: r.body_a), ia(lambda r: r.body_b), va(lambda r: r.world_anchor),
                va(lambda r: r.off_a), va(lambda r: r.off_b), fa(lambda r: r.stiffness), fa(lambda r: r.fracture),
                fa(lambda r: r.fmin), fa(lambda r: r.fmax), ia(lambda r: r.sibling), ia(lambda r: r.partner),
                fa(lambda r: r.friction), fa(lambda r: r.friction_static)]
        arrs = [np.ascontiguousarray(a) for a in arrs]
        if self._self_collide:
            self.pair_cap = max(256, 16 * max(1, n))
            self.dyn_cap = max(64, 16 * max(1, n)) * 12
        else:
            self.pair_cap, self.dyn_cap = 0, 0
        self._params()
        keep = [x, q, v, w, mass, he, fric, iloc, prio]
        lib().orc_load_scene(self._h, n, *[_p(a) for a in keep], nr, *[_p(a) for a in arrs], self.pair_cap,
                             self.dyn_cap)
        self._keep = keep + arrs
        if prev is not None:
            k = min(prev[0].shape[0], n)
            cur = self.get_bodies()
            for a, b in zip(cur, prev):
                a[:k] = b[:k]
            self.set_bodies(*cur)
        self._nb_loaded = n
        self._dirty = False

    # ---- stepping ---------------------------------------------------------
    def step(self):
        self._flush()
        self._params()
        lib().orc_step(self._h)
        self._grow_if_needed()

    def substep(self, dt=None):
        """One substep at `dt` (default: dt / substeps)."""
        self._flush()
        self._params()
        lib().orc_set_dt(self._h, self.dt / self.substeps if dt is None else dt)
        lib().orc_substep(self._h)
        lib().orc_set_dt(self._h, self.dt)
        self._grow_if_needed()

    def _grow_if_needed(self):
        c = self.counts()
        grow = False
        if c["pairs_found"] > self.pair_cap:
            self.pair_cap = max(2 * self.pair_cap, 2 * c["pairs_found"])
            grow = True
        if c["rows_reserved"] > c["capacity"]:
            self.dyn_cap = max(2 * self.dyn_cap, 2 * (c["rows_reserved"] - c["n_static"]))
            grow = True
        if grow:
            lib().orc_set_caps(self._h, self.pair_cap, self.dyn_cap)
        self.overflowed = grow

    # ---- readback ---------------------------------------------------------
    def counts(self) -> dict:
        out = np.zeros(9, np.int64)
        lib().orc_get_counts(self._h, _p(out))
        keys = ["n_static", "n_rows", "capacity", "rows_reserved", "pairs_found", "n_pairs", "n_colors",
                "recolored", "color_dirty"]
        return {k: int(v) for k, v in zip(keys, out)}

    def get_bodies(self):
        n = len(self._x)
        arrs = [np.zeros((n, 3)), np.zeros((n, 4)), np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3)),
                np.zeros((n, 3))]
        lib().orc_get_bodies(self._h, *[_p(a) for a in arrs])
        return arrs

    def set_bodies(self, x=None, q=None, v=None, w=None, pv=None, pw=None):
        arrs = [None if a is None else np.ascontiguousarray(a, np.float64) for a in (x, q, v, w, pv, pw)]
        lib().orc_set_bodies(self._h, *[None if a is None else _p(a) for a in arrs])

    def positions(self):
        self._flush()
        return self.get_bodies()[0]

    def orientations(self):
        self._flush()
        return self.get_bodies()[1]

    def velocities(self):
        self._flush()
        return self.get_bodies()[2]

    def angular_velocities(self):
        self._flush()
        return self.get_bodies()[3]

    def rows(self, n=None):
        c = self.counts()
        n = c["n_rows"] if n is None else n
        lam, pen, ac0 = np.zeros(n), np.zeros(n), np.zeros(n)
        act, was, ty, a, b = (np.zeros(n, np.int32) for _ in range(5))
        lib().orc_get_rows(self._h, n, *[_p(z) for z in (lam, pen, ac0, act, was, ty, a, b)])
        return dict(lam=lam, pen=pen, ac0=ac0, active=act, was=was, type=ty, body_a=a, body_b=b)

    def lambdas(self):
        return self.rows()["lam"]

    def active(self):
        return self.rows()["active"]

    def set_static_rows(self, lam, pen, active, was):
        arrs = [np.ascontiguousarray(lam, np.float64), np.ascontiguousarray(pen, np.float64),
                np.ascontiguousarray(active, np.int32), np.ascontiguousarray(was, np.int32)]
        lib().orc_set_static_rows(self._h, *[_p(a) for a in arrs])

    def _set_one(self, idx, k, val):
        arrs = self.get_bodies()
        arrs[k][idx] = val
        self.set_bodies(*arrs)

    def set_position(self, body, p):
        self._flush()
        self._set_one(body.index, 0, p)

    def set_orientation(self, body, q):
        self._flush()
        self._set_one(body.index, 1, q)

    def set_velocity(self, body, v):
        self._flush()
        self._set_one(body.index, 2, v)

    def set_angular_velocity(self, body, w):
        self._flush()
        self._set_one(body.index, 3, w)

    def cache(self):
        cap = 1 << 22
        abc = np.zeros((cap, 3), np.int32)
        st = np.zeros((cap, 8))
        n = lib().orc_get_cache(self._h, cap, _p(abc), _p(st))
        return abc[:n].copy(), st[:n].copy()

    def set_key_mode(self, mode: str) -> None:
        """'ordinal' (a, b, manifold ordinal) or 'anchor_5mm' cache keys;
        empties the cache."""
        lib().orc_set_key_mode(self._h, 1 if mode == "anchor_5mm" else 0)

    def cache_keys(self):
        cap = 1 << 22
        keys = np.zeros(cap, np.uint64)
        st = np.zeros((cap, 8))
        n = lib().orc_get_cache_keys(self._h, cap, _p(keys), _p(st))
        return keys[:n].copy(), st[:n].copy()

    def set_cache_keys(self, keys, st):
        keys = np.ascontiguousarray(keys, np.uint64)
        st = np.ascontiguousarray(st, np.float64)
        lib().orc_set_cache_keys(self._h, keys.shape[0], _p(keys), _p(st))

    def set_cache(self, abc, st):
        abc = np.ascontiguousarray(abc, np.int32)
        st = np.ascontiguousarray(st, np.float64)
        lib().orc_set_cache(self._h, abc.shape[0], _p(abc), _p(st))

    def colors(self):
        out = np.zeros(len(self._x), np.int32)
        nc = lib().orc_get_colors(self._h, _p(out))
        return out, nc

    def set_colors(self, colors, n_colors, dirty=False):
        c = np.ascontiguousarray(colors, np.int32)
        lib().orc_set_colors(self._h, _p(c), int(n_colors), int(dirty))

    def count_color_conflicts(self):
        return lib().orc_count_conflicts(self._h)

    def pairs(self):
        n = self.counts()["n_pairs"]
        pa, pb, ov, si, cnt = (np.zeros(n, np.int32) for _ in range(5))
        nrm = np.zeros((n, 3), np.float32)
        lib().orc_get_pairs(self._h, n, *[_p(a) for a in (pa, pb, ov, si, cnt, nrm)])
        return dict(a=pa, b=pb, overlap=ov, sat_idx=si, count=cnt, n_hat=nrm)

    def contacts(self):
        cap = 1 << 22
        abc = np.zeros((cap, 3), np.int32)
        n = lib().orc_get_contacts(self._h, cap, _p(abc))
        return abc[:n].copy()

    def record_violation(self, on=True):
        lib().orc_set_record_violation(self._h, int(on))

    def violation_history(self):
        out = np.zeros(256)
        n = lib().orc_get_violation(self._h, _p(out), 256)
        return out[:n].copy()

    @property
    def num_active_colors(self):
        return self.counts()["n_colors"]
