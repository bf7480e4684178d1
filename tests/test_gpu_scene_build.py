"""Scene build on the device (avbd_build_floor_groups): the static groups
the kernel writes from the floor-block records, with the pins placed beside
them, equal the host construction of the same groups (solver_6dof.py:
474-541 floor corners, :543-578 pins, row numbering :1067-1129) field for
field -- implicit and explicit corners, with and without friction, hard and
soft rows -- and the per-body ranges and the row -> group map agree."""

import numpy as np
import pytest
import torch

from backends import make_gpu

pytestmark = pytest.mark.gpu


def _mixed_scene(s):
    s.enable_self_collision(True, default_friction=0.4)
    rng = np.random.default_rng(3)
    for k in range(60):
        he = tuple(float(v) for v in rng.uniform(0.1, 0.5, 3))
        b = s.add_box((float(k) * 1.2, 1.0, 0.0), he, mass=1.0 + k, friction=0.3 if k % 3 else 0.0)
        if k % 5 == 1:  # a pin before the floor block
            s.add_pin_corner(b, body_local=he, world_point=(float(k) * 1.2 + he[0], 1.0 + he[1], he[2]),
                             fracture=5e4)
        if k % 4 == 2:  # a block with other half extents: explicit corners
            s.add_floor_contact_box(type(b)(index=b.index, half_extents=(he[0] * 0.5, he[1], he[2])),
                                    floor_y=-0.25, friction=0.5)
        else:
            s.add_floor_contact_box(b, stiffness=1e7 if k % 7 == 0 else float("inf"))
        if k % 6 == 0:
            s.add_pin_corner(b, body_local=(0.0, he[1], 0.0), world_point=(float(k) * 1.2, 1.0 + he[1], 0.0))
    s.add_box((0.0, -3.0, 0.0), (5.0, 0.5, 5.0), mass=0.0)  # a static body without rows


def test_device_groups_equal_host_construction():
    s = make_gpu(dt=1 / 60, iterations=4, substeps=1)
    _mixed_scene(s)
    s._flush()
    want, sg_start, row_map = s._static_group_arrays()
    ng = s._n_static_groups
    got = {"body": s._g_body[:ng], "meta": s._g_meta[:ng], "row0": s._g_row0[:ng], "offa": s._g_offa[:ng],
           "n": s._g_n[:ng], "mat": s._g_mat[:ng], "flags": s._g_flags[:ng]}
    for k, t in got.items():
        np.testing.assert_array_equal(t.cpu().numpy(), want[k][:ng], err_msg=k)
    np.testing.assert_array_equal(s._sg_start.cpu().numpy(), sg_start)
    np.testing.assert_array_equal(s._row_map, row_map)
    np.testing.assert_array_equal(s._g_pen[:ng].cpu().numpy(), np.ones((ng, 4), np.float32))
    np.testing.assert_array_equal(s._g_lam[:ng].cpu().numpy(), np.zeros((ng, 4), np.float32))
    s.step()  # and it runs
    assert s.stats()["err"] == 0


def test_state_round_trip_uses_the_device_row_map():
    s = make_gpu(dt=1 / 60, iterations=4, substeps=2)
    _mixed_scene(s)
    for _ in range(5):
        s.step()
    sd = s.state_dict()
    s.load_state_dict(sd)
    sd2 = s.state_dict()
    for k in ("row_lam", "row_pen", "row_active", "row_was"):
        np.testing.assert_array_equal(sd[k], sd2[k], err_msg=k)


def test_pile_scene_build_time():
    """The library's share of building the 100k-box pile (arena, body
    arrays, static groups on the device, upload): well under a second."""
    import time
    from avbd_b200 import scenes
    s = make_gpu(dt=1 / 60, iterations=10, substeps=4, coloring_mode="jones_plassmann")
    scenes.pile(s, nx=100, nz=100, ny=10)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    s._flush()
    s.stream.synchronize()
    dt = time.perf_counter() - t0
    assert s._n_static_groups == 800_200
    assert dt < 1.0, dt
