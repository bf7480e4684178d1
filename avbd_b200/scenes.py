"""Seeded synthetic scenes for tests and benchmarks.

Each builder takes any object with the Solver6DOF scene API (the GPU solver
or the CPU oracle) and fills it, so the same scene is built bit-identically on
both.  No public dataset is involved: the scene distributions follow the
workload descriptions of the benchmark configurations (box counts, extents,
densities, friction, grids).
"""

from __future__ import annotations

import math

import numpy as np


def _rand_quat(rng) -> tuple:
    """Uniform random unit quaternion (Shoemake), xyzw."""
    u1, u2, u3 = rng.uniform(0.0, 1.0, 3)
    a, b = math.sqrt(1.0 - u1), math.sqrt(u1)
    return (a * math.sin(2 * math.pi * u2), a * math.cos(2 * math.pi * u2), b * math.sin(2 * math.pi * u3),
            b * math.cos(2 * math.pi * u3))


def _yaw_quat(deg: float) -> tuple:
    h = math.radians(deg) * 0.5
    return (0.0, math.sin(h), 0.0, math.cos(h))


def pyramid20(s, seed: int = 0, friction: float = 0.5):
    """20 one-metre cubes (density 1000) in 4 tiers of 8/6/4/2, +-1 mm xz and
    +-0.5 deg yaw jitter, floor rows on every box, self collision on."""
    rng = np.random.default_rng(seed)
    s.enable_self_collision(True, default_friction=friction)
    boxes = []
    h = 0.5
    for tier, count in enumerate((8, 6, 4, 2)):
        x0 = -(count - 1) * 0.5 * 1.0
        for k in range(count):
            j = rng.uniform(-1e-3, 1e-3, 2)
            yaw = rng.uniform(-0.5, 0.5)
            b = s.add_box((x0 + k * 1.0 + float(j[0]), h + 2 * h * tier, float(j[1])), (h, h, h), mass=1000.0,
                          orientation=_yaw_quat(yaw), friction=friction)
            s.add_floor_contact_box(b, friction=friction)
            boxes.append(b)
    return boxes


def heap(s, n_side: int = 20, spacing: float = 1.2, seed: int = 0, friction: float = 0.4, walls: bool = True,
         he_range=(0.1, 0.5)):
    """n_side^3 OBBs (half extents uniform in he_range, uniform random
    orientation, density 1000) on a jittered grid above the floor, inside a
    square container of 4 static walls (mass 0), floor rows on every box."""
    rng = np.random.default_rng(seed)
    s.enable_self_collision(True, default_friction=friction)
    boxes = []
    off = -(n_side - 1) * spacing * 0.5
    for iy in range(n_side):
        for ix in range(n_side):
            for iz in range(n_side):
                he = rng.uniform(he_range[0], he_range[1], 3)
                m = 8.0 * float(he[0] * he[1] * he[2]) * 1000.0
                j = rng.uniform(-0.05, 0.05, 3)
                p = (off + ix * spacing + float(j[0]), 1.0 + iy * spacing + float(j[1]),
                     off + iz * spacing + float(j[2]))
                b = s.add_box(p, tuple(float(v) for v in he), mass=m, orientation=_rand_quat(rng),
                              friction=friction)
                s.add_floor_contact_box(b, friction=friction)
                boxes.append(b)
    if walls:
        half = max(20.0, -off + 2.0)
        t = 0.5
        for (cx, cz, hx, hz) in ((half + t, 0.0, t, half + 2 * t), (-half - t, 0.0, t, half + 2 * t),
                                 (0.0, half + t, half + 2 * t, t), (0.0, -half - t, half + 2 * t, t)):
            boxes.append(s.add_box((cx, 2.0, cz), (hx, 2.0, hz), mass=0.0, friction=friction))
    return boxes


def pile(s, nx: int = 100, nz: int = 100, ny: int = 10, spacing: float = 1.4, seed: int = 0, friction: float = 0.4,
         pin_every: int = 500, pin_fracture: float = 5.0e4):
    """nx*nz*ny OBBs (half extents uniform in [0.2, 0.4], random orientation,
    density 1000) on a jittered grid; every `pin_every`-th box is pinned by a
    corner to its initial world position with a breakable pin."""
    rng = np.random.default_rng(seed)
    s.enable_self_collision(True, default_friction=friction)
    boxes = []
    ox, oz = -(nx - 1) * spacing * 0.5, -(nz - 1) * spacing * 0.5
    k = 0
    for iy in range(ny):
        for ix in range(nx):
            for iz in range(nz):
                he = rng.uniform(0.2, 0.4, 3)
                m = 8.0 * float(he[0] * he[1] * he[2]) * 1000.0
                j = rng.uniform(-0.05, 0.05, 3)
                q = _rand_quat(rng)
                p = (ox + ix * spacing + float(j[0]), 0.8 + iy * spacing + float(j[1]),
                     oz + iz * spacing + float(j[2]))
                b = s.add_box(p, tuple(float(v) for v in he), mass=m, orientation=q, friction=friction)
                s.add_floor_contact_box(b, friction=friction)
                if pin_every and k % pin_every == 0:
                    corner = tuple(float(v) for v in he)
                    R = _quat_matrix(q)
                    w = np.asarray(p) + R @ np.asarray(corner)
                    s.add_pin_corner(b, body_local=corner, world_point=tuple(float(v) for v in w),
                                     fracture=pin_fracture)
                boxes.append(b)
                k += 1
    return boxes


def _quat_matrix(q) -> np.ndarray:
    x, y, z, w = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def tower_grid(s, grid: int = 3, height: int = 3, h: float = 0.12, spacing: float = 0.55, seed: int = 0,
               friction: float = 0.5):
    """Grid of cube towers (the reference viewer's default scene layout)."""
    rng = np.random.default_rng(seed)
    s.enable_self_collision(True, default_friction=friction)
    boxes = []
    o = -(grid - 1) * spacing * 0.5
    for ix in range(grid):
        for iz in range(grid):
            for k in range(height):
                j = rng.uniform(-1e-3, 1e-3, 2)
                b = s.add_box((o + ix * spacing + float(j[0]), h + 2 * h * k, o + iz * spacing + float(j[1])),
                              (h, h, h), mass=1.0, friction=friction)
                s.add_floor_contact_box(b, friction=friction)
                boxes.append(b)
    return boxes
