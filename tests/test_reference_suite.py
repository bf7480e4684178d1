"""The reference's 6-DOF acceptance tests, run on both backends.

Restated from tests/test_solver_6dof.py and tests/test_kernel_face_clip.py of
the reference (nanli9/AVBD): the same scenes, step counts and tolerances.
`oracle` runs the CPU restatement (pins the oracle to the reference's known
answers); `gpu` runs the sm_100a library through the drop-in Solver6DOF.
"""

import math

import numpy as np
import pytest

from backends import BACKENDS, factory, quat_matrix


@pytest.fixture(params=BACKENDS)
def S(request):
    return factory(request.param)


def test_free_fall_constant_acceleration(S):  # test_solver_6dof.py:20-28
    s = S(dt=1 / 60, iterations=5)
    s.add_box((0., 5., 0.), (0.5, 0.5, 0.5), mass=1.0)
    for _ in range(60):
        s.step()
    assert s.velocities()[0][1] == pytest.approx(-9.81, rel=1e-3)


def test_free_spin_preserves_angular_velocity(S):  # :31-47
    s = S(dt=1 / 60, iterations=5, gravity=(0., 0., 0.))
    s.add_box((0., 0., 0.), (0.5, 0.5, 0.5), mass=1.0, angular_velocity=(0., 0., 2.0))
    for _ in range(60):
        s.step()
    w = s.angular_velocities()[0]
    assert np.linalg.norm(w - np.array([0., 0., 2.0])) < 1e-3
    q = s.orientations()[0]
    expected = np.array([0., 0., math.sin(1.0), math.cos(1.0)])
    assert min(np.linalg.norm(q - expected), np.linalg.norm(q + expected)) < 5e-3


def test_box_drops_on_floor_settles_at_half_extent(S):  # :50-60
    h = 0.3
    s = S(dt=1 / 60, iterations=20)
    b = s.add_box((0., 2.0, 0.), (h, h, h), mass=1.0, friction=0.5)
    s.add_floor_contact_box(b, floor_y=0.0, friction=0.5)
    for _ in range(300):
        s.step()
    assert abs(s.positions()[0][1] - h) < 0.01
    assert abs(s.velocities()[0][1]) < 0.1


def test_spinning_box_on_floor_friction_brakes_omega(S):  # :63-77
    s = S(dt=1 / 60, iterations=25)
    h = 0.3
    b = s.add_box((0., h + 0.15, 0.), (h, h, h), mass=1.0, friction=0.8, angular_velocity=(0., 5.0, 0.))
    s.add_floor_contact_box(b, friction=0.8)
    for _ in range(300):
        s.step()
    assert np.linalg.norm(s.angular_velocities()[0]) < 0.1
    assert abs(s.positions()[0][1] - h) < 0.02


def test_tilted_box_drops_and_settles(S):  # :80-100
    s = S(dt=1 / 60, iterations=15, substeps=8)
    h = 0.3
    ang = math.radians(30)
    b = s.add_box((0., 1.5, 0.), (h, h, h), mass=1.0, friction=0.5,
                  orientation=(math.sin(ang / 2), 0., 0., math.cos(ang / 2)))
    s.add_floor_contact_box(b, friction=0.5)
    for _ in range(300):
        s.step()
    assert np.linalg.norm(s.angular_velocities()[0]) < 0.05
    assert np.linalg.norm(s.velocities()[0]) < 0.05
    assert h - 0.02 < s.positions()[0][1] < h + 0.02


def test_box_corner_pin_holds_against_gravity(S):  # :103-130
    s = S(dt=1 / 60, iterations=30)
    h = 0.3
    world_pin = (h, 2.0, h)
    b = s.add_box((0., 2.0 - h, 0.), (h, h, h), mass=1.0)
    s.add_pin_corner(b, body_local=(h, h, h), world_point=world_pin)
    for _ in range(180):
        s.step()
    corner = s.positions()[0] + quat_matrix(s.orientations()[0]) @ np.array([h, h, h])
    assert np.linalg.norm(corner - np.array(world_pin)) < 0.02


def test_two_cubes_stack_axis_aligned(S):  # :133-152
    h = 0.20
    s = S(dt=1 / 60, iterations=15, substeps=8)
    bot = s.add_box((0., 0.20, 0.), (h, h, h), mass=1.0, friction=0.5)
    top = s.add_box((0., 0.55, 0.), (h, h, h), mass=1.0, friction=0.5)
    for b in (bot, top):
        s.add_floor_contact_box(b, friction=0.5)
    s.enable_self_collision(True, default_friction=0.5)
    for _ in range(300):
        s.step()
    ys = s.positions()[:, 1]
    assert abs(ys[0] - h) < 0.01
    assert abs(ys[1] - 3 * h) < 0.02
    assert abs(ys[1] - ys[0] - 2 * h) < 0.01
    assert np.abs(s.velocities()[:, 1]).max() < 0.05


def test_three_cubes_stack(S):  # :155-170
    h = 0.20
    s = S(dt=1 / 60, iterations=15, substeps=8)
    bs = [s.add_box((0., y, 0.), (h, h, h), mass=1.0, friction=0.5) for y in (0.20, 0.62, 1.04)]
    for b in bs:
        s.add_floor_contact_box(b, friction=0.5)
    s.enable_self_collision(True, default_friction=0.5)
    for _ in range(360):
        s.step()
    ys = s.positions()[:, 1]
    for i, e in enumerate([h, 3 * h, 5 * h]):
        assert abs(ys[i] - e) < 0.03


def test_cube_on_floor_friction_brakes_translation(S):  # :173-189
    h, v0, mu = 0.20, 2.0, 0.4
    s = S(dt=1 / 60, iterations=15, substeps=8)
    b = s.add_box((0., h, 0.), (h, h, h), mass=1.0, friction=mu, velocity=(v0, 0., 0.))
    s.add_floor_contact_box(b, friction=mu)
    x0 = s.positions()[0][0]
    for _ in range(240):
        s.step()
    expected = v0 * v0 / (2 * mu * 9.81)
    assert abs((s.positions()[0][0] - x0) - expected) / expected < 0.10


def test_static_body_does_not_move(S):  # :220-229
    s = S(dt=1 / 60, iterations=5)
    s.add_box((0.5, 1.0, 0.5), (0.3, 0.3, 0.3), mass=0.0)
    x0 = s.positions()[0].copy()
    q0 = s.orientations()[0].copy()
    for _ in range(60):
        s.step()
    assert np.allclose(s.positions()[0], x0)
    assert np.allclose(s.orientations()[0], q0)


def test_pinned_box_with_spin_stays_bounded(S):  # :266-283
    s = S(dt=1 / 60, iterations=20, max_angular_speed=50.0)
    h = 0.2
    b = s.add_box((0., 2.0 - h, 0.), (h, h, h), mass=1.0, angular_velocity=(0., 6.0, 0.))
    s.add_pin_corner(b, body_local=(h, h, h), world_point=(h, 2.0, h))
    max_w = 0.0
    for _ in range(180):
        s.step()
        max_w = max(max_w, float(np.linalg.norm(s.angular_velocities()[0])))
    assert max_w < 12.0


def _pushed_box(S, force):
    s = S(dt=1 / 60, iterations=20, substeps=4, friction_static_mult=1.5)
    h = 0.2
    b = s.add_box((0., h, 0.), (h, h, h), mass=1.0, friction=0.4)
    s.add_floor_contact_box(b, friction=0.4)
    for _ in range(60):
        s.step()
    x0 = float(s.positions()[0][0])
    for _ in range(60):
        v = s.velocities()[0]
        s.set_velocity(b, (float(v[0] + force * s.dt), float(v[1]), float(v[2])))
        s.step()
    return float(s.positions()[0][0]) - x0


def test_static_friction_holds_under_small_push(S):  # :286-307
    assert abs(_pushed_box(S, 3.0)) < 0.05


def test_kinetic_friction_slips_under_large_push(S):  # :310-330
    assert _pushed_box(S, 10.0) > 1.0


def test_bvh_broadphase_settles_column(S):  # :333-355 (asserts heights; the pair count is not pinned there)
    h = 0.15
    s = S(dt=1 / 60, iterations=10, substeps=4)
    s.enable_self_collision(True, default_friction=0.3)
    for k in range(3):
        b = s.add_box((0., h + 2 * h * k + 0.02 * k, 0.), (h, h, h), mass=1.0, friction=0.3)
        s.add_floor_contact_box(b, friction=0.3)
    s.step()
    if hasattr(s, "broadphase_ms"):
        assert s.broadphase_ms > 0.0
    for _ in range(120):
        s.step()
    ys = s.positions()[:, 1]
    for i in range(3):
        assert abs(ys[i] - (h + 2 * h * i)) < 0.03


def test_bvh_broadphase_scales_to_27_bodies(S):  # :358-385
    h, spacing = 0.12, 0.6
    s = S(dt=1 / 60, iterations=15, substeps=6)
    s.enable_self_collision(True, default_friction=0.5)
    for ix in range(3):
        for iz in range(3):
            for k in range(3):
                b = s.add_box(((ix - 1) * spacing, h + 2 * h * k, (iz - 1) * spacing), (h, h, h), mass=1.0,
                              friction=0.5)
                s.add_floor_contact_box(b, friction=0.5)
    for _ in range(120):
        s.step()
    p = s.positions()
    for tower in range(9):
        assert 4.5 * h < p[tower * 3 + 2][1] < 5.5 * h


def test_edge_edge_contact_two_rotated_boxes_separate(S):  # :388-422
    s = S(dt=1.0 / 240.0, iterations=20, substeps=2, gravity=(0., 0., 0.))
    s.enable_self_collision(True, default_friction=0.0)
    h = 0.25
    qz45 = (0., 0., math.sin(math.pi / 8), math.cos(math.pi / 8))
    s.add_box((0., 0., 0.), (h, h, h), mass=1.0, orientation=qz45, friction=0.0)
    qx45 = (math.sin(math.pi / 8), 0., 0., math.cos(math.pi / 8))
    s.add_box((0.0, 0.6, 0.0), (h, h, h), mass=1.0, orientation=qx45, friction=0.0, velocity=(0., -2.0, 0.))
    for _ in range(120):
        s.step()
    p = s.positions()
    assert abs(p[1][1] - p[0][1]) > 2 * h - 0.05
    assert np.all(np.isfinite(p)) and np.all(np.isfinite(s.velocities()))


def test_eq14_hessian_rescaling_settles_box_on_floor(S):  # :425-456
    h = 0.3
    s = S(dt=1.0 / 60.0, iterations=15, gravity=(0., -9.81, 0.))
    b = s.add_box((0., 1.5, 0.), (h, h, h), mass=1.0, friction=0.5)
    s.add_floor_contact_box(b, friction=0.5)
    for _ in range(180):
        s.step()
    y_settled = s.positions()[0][1]
    ys = []
    for _ in range(120):
        s.step()
        ys.append(s.positions()[0][1])
    assert max(ys) - min(ys) < 2.0e-3
    assert abs(y_settled - h) < 2.0e-3


def test_kernel_face_clip_settles_3_cube_stack(S):  # test_kernel_face_clip.py:20-42
    h = 0.20
    s = S(dt=1.0 / 60.0, iterations=15, substeps=8)
    s.enable_self_collision(True, default_friction=0.5)
    bs = [s.add_box((0., y, 0.), (h, h, h), mass=1.0, friction=0.5) for y in (0.20, 0.62, 1.04)]
    for b in bs:
        s.add_floor_contact_box(b, friction=0.5)
    for _ in range(360):
        s.step()
    ys, vs = s.positions()[:, 1], s.velocities()[:, 1]
    for i, e in enumerate((0.20, 0.60, 1.00)):
        assert abs(float(ys[i]) - e) < 0.03
    assert float(np.abs(vs).max()) < 0.05
