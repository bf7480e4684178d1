"""Batched scenes: many independent Solver6DOF scenes in one solver.

Every scene keeps its own bodies, floor rows, pins, contacts, substeps per
frame and iterations per substep; all scenes advance together in the same
launches -- one collision graph and one persistent solve kernel per substep
slot -- instead of one launch sequence per scene.  How it maps onto the
device:

* bodies of all scenes share one arena; `SCENE_OF` tags each body with its
  scene and `SCENE_TAB` holds per scene (substep dt, iterations, substeps);
* the broad phase never pairs bodies of different scenes, and the scenes are
  laid out on a grid `spacing` metres apart so the BVH keeps them apart too;
* a frame is `max substeps` slots; a scene with S substeps takes part in the
  first S slots, each at dt / S, and sits the rest out untouched;
* the color passes run to the largest iteration count; each body follows its
  own scene's count (its post-stabilization pass, or its last dual update
  and finalize, at its own iteration index); colors are shared, since no
  contact joins two scenes.

No counterpart in the reference, which runs one scene per Solver6DOF.
"""

from __future__ import annotations

import math

import numpy as np

from .solver import RigidBody, Solver6DOF


class Scene:
    """One scene of a batch.  Positions passed to and returned by it are in
    the scene's own frame (the batch offsets them by `origin`)."""

    def __init__(self, batch: "SceneBatch", index: int, origin: tuple, substeps: int, iterations: int):
        self.batch = batch
        self.index = index
        self.origin = np.asarray(origin, np.float64)
        self.substeps = substeps
        self.iterations = iterations
        self.bodies: list[RigidBody] = []

    def _enter(self) -> Solver6DOF:
        s = self.batch.solver
        s._cur_scene = self.index
        return s

    def add_box(self, position, half_extents, mass, orientation=(0.0, 0.0, 0.0, 1.0), velocity=(0.0, 0.0, 0.0),
                angular_velocity=(0.0, 0.0, 0.0), friction=0.0) -> RigidBody:
        p = tuple(float(v) for v in np.asarray(position, np.float64) + self.origin)
        b = self._enter().add_box(p, half_extents, mass, orientation, velocity, angular_velocity, friction)
        self.bodies.append(b)
        return b

    def add_floor_contact_box(self, body: RigidBody, floor_y: float = 0.0, friction=None, **kw):
        return self._enter().add_floor_contact_box(body, floor_y=floor_y, friction=friction, **kw)

    def add_pin_corner(self, body: RigidBody, body_local, world_point, **kw):
        w = tuple(float(v) for v in np.asarray(world_point, np.float64) + self.origin)
        return self._enter().add_pin_corner(body, body_local, w, **kw)

    def positions(self) -> np.ndarray:
        idx = [b.index for b in self.bodies]
        return self.batch.solver.positions()[idx] - self.origin

    def orientations(self) -> np.ndarray:
        idx = [b.index for b in self.bodies]
        return self.batch.solver.orientations()[idx]

    def velocities(self) -> np.ndarray:
        idx = [b.index for b in self.bodies]
        return self.batch.solver.velocities()[idx]


class SceneBatch:
    """Independent scenes stepped together.  `solver_kw` are Solver6DOF
    keywords shared by all scenes (dt is the frame time of every scene;
    substeps and iterations are per scene)."""

    def __init__(self, dt: float = 1.0 / 60.0, spacing: float = 100.0, self_collide: bool = True,
                 default_friction: float = 0.0, **solver_kw):
        solver_kw.pop("substeps", None)
        solver_kw.pop("iterations", None)
        self.solver = Solver6DOF(dt=dt, substeps=1, iterations=1, **solver_kw)
        if self_collide:
            self.solver.enable_self_collision(True, default_friction=default_friction)
        self.spacing = float(spacing)
        self.scenes: list[Scene] = []

    def add_scene(self, substeps: int = 4, iterations: int = 10) -> Scene:
        if not (1 <= iterations <= 63) or substeps < 1:
            raise ValueError("a scene needs 1..63 iterations and >= 1 substeps")
        k = len(self.scenes)
        # scenes on a square grid in x/z, filled row by row
        side = 32
        origin = ((k % side) * self.spacing, 0.0, (k // side) * self.spacing)
        sc = Scene(self, k, origin, int(substeps), int(iterations))
        self.solver._scene_tab.append((sc.substeps, sc.iterations))
        self.scenes.append(sc)
        self.solver._dirty = True
        return sc

    def step(self) -> None:
        """One frame of every scene (each scene's own substeps)."""
        self.solver.step()

    def stats(self) -> dict:
        return self.solver.stats()

    def body_substeps_per_frame(self) -> int:
        """Dynamic body-substeps one frame advances (the throughput unit)."""
        m = np.asarray(self.solver._mass)
        tab = np.asarray([sc.substeps for sc in self.scenes])
        of = np.asarray(self.solver._scene_of)
        return int(np.sum(tab[of][m > 0]))


def c4_scene(sc: Scene, n_bodies: int, rng: np.random.Generator) -> None:
    """One scene of the batched benchmark: `n_bodies` OBBs with half extents
    U[0.1, 0.5] m, uniform random orientations, density 1000, on a jittered
    grid at 1.2 m over the floor inside 4 static walls; mu_s U[0.3, 0.8] and
    mu_d = 0.8 mu_s (mu_s = 1.25 mu_d is the solver's friction_static_mult)."""
    mu_d = 0.8 * float(rng.uniform(0.3, 0.8))
    side = int(math.ceil(math.sqrt(n_bodies / 4.0)))  # 4 layers at most per column
    layers = int(math.ceil(n_bodies / float(side * side)))
    half = 0.5 * side * 1.2 + 1.0
    for (cx, cz, hx, hz) in ((half + 0.5, 0.0, 0.5, half + 1.0), (-half - 0.5, 0.0, 0.5, half + 1.0),
                             (0.0, half + 0.5, half + 1.0, 0.5), (0.0, -half - 0.5, half + 1.0, 0.5)):
        sc.add_box((cx, 2.0, cz), (hx, 2.0, hz), mass=0.0, friction=mu_d)
    k = 0
    for iy in range(layers):
        for ix in range(side):
            for iz in range(side):
                if k >= n_bodies:
                    break
                he = rng.uniform(0.1, 0.5, 3)
                m = 8.0 * float(he[0] * he[1] * he[2]) * 1000.0
                u1, u2, u3 = rng.uniform(0.0, 1.0, 3)
                q = (math.sqrt(1 - u1) * math.sin(2 * math.pi * u2), math.sqrt(1 - u1) * math.cos(2 * math.pi * u2),
                     math.sqrt(u1) * math.sin(2 * math.pi * u3), math.sqrt(u1) * math.cos(2 * math.pi * u3))
                j = rng.uniform(-0.05, 0.05, 3)
                p = ((ix - (side - 1) * 0.5) * 1.2 + j[0], 0.6 + iy * 1.2 + j[1], (iz - (side - 1) * 0.5) * 1.2 + j[2])
                b = sc.add_box(p, tuple(float(v) for v in he), mass=m, orientation=q, friction=mu_d)
                sc.add_floor_contact_box(b, friction=mu_d)
                k += 1


def c4_specs(n_scenes: int = 512, seed: int = 0, min_bodies: int = 16, max_bodies: int = 2048,
             substep_choices=(2, 4, 8), iteration_choices=(5, 10, 20)) -> list:
    """Per scene (bodies, substeps, iterations, scene seed) of the batched
    benchmark: body counts log-uniform in [min_bodies, max_bodies]."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n_scenes):
        n = int(round(math.exp(rng.uniform(math.log(min_bodies), math.log(max_bodies)))))
        out.append((n, int(rng.choice(substep_choices)), int(rng.choice(iteration_choices)), seed * 100003 + k))
    return out


def c4_batch(specs, **solver_kw) -> SceneBatch:
    """A SceneBatch holding the scenes of `specs` (see c4_specs)."""
    kw = dict(friction_static_mult=1.25, coloring_mode="jones_plassmann", spacing=40.0)
    kw.update(solver_kw)
    batch = SceneBatch(**kw)
    for n, sub, its, sseed in specs:
        c4_scene(batch.add_scene(substeps=sub, iterations=its), n, np.random.default_rng(sseed))
    return batch


def c4_single(spec, **solver_kw) -> Solver6DOF:
    """One scene of `specs` as its own Solver6DOF (the one-at-a-time baseline)."""
    n, sub, its, sseed = spec
    kw = dict(friction_static_mult=1.25, coloring_mode="jones_plassmann")
    kw.update(solver_kw)
    s = Solver6DOF(dt=1.0 / 60.0, substeps=sub, iterations=its, **kw)
    s.enable_self_collision(True, default_friction=0.0)
    c4_scene(s, n, np.random.default_rng(sseed))
    return s
