"""GPU robustness, residency and API tests (restating tests/test_robustness.py
and the CUDA-graph buffer-ownership tests of tests/test_solver_6dof.py of the
reference), plus device failure detection without faulting the GPU."""

import numpy as np
import pytest

from avbd_b200 import Solver6DOF, scenes

pytestmark = pytest.mark.gpu


def _stack(mode="jacobi", n=6, gap=0.85, **kw):
    s = Solver6DOF(gravity=(0, -9.8, 0), iterations=4, coloring_mode=mode, **kw)
    for i in range(n):
        s.add_box((0.0, 0.5 + i * gap, 0.0), (0.5, 0.5, 0.5), mass=1.0, friction=0.3)
    s.enable_self_collision(True)
    return s


def test_dense_cluster_no_crash():  # test_robustness.py:26-46
    s = Solver6DOF(gravity=(0, -9.8, 0), iterations=4)
    for i in range(60):
        s.add_box((0.01 * i, 2.0, 0.0), (0.5, 0.5, 0.5), mass=1.0, friction=0.3)
    s.enable_self_collision(True)
    s._flush()
    with pytest.warns(RuntimeWarning, match="row pool overflow"):
        s.step()
    for _ in range(4):
        s.step()
    assert int(s.n_active_rows.numpy()[0]) <= s._gpu_pool_n_capacity
    assert np.all(np.isfinite(s.positions()))


def test_coloring_safety_for_touching_bodies():  # :49-63
    s = Solver6DOF(gravity=(0, -9.8, 0), iterations=4)
    s.add_box((0.0, 2.0, 0.0), (0.5, 0.5, 0.5), mass=1.0, friction=0.3)
    s.add_box((0.6, 2.0, 0.0), (0.5, 0.5, 0.5), mass=1.0, friction=0.3)
    s.enable_self_collision(True)
    s.step()
    c = s.body_color.numpy()
    assert c[0] != c[1]


def test_coloring_safety_for_stack():  # :66-78
    s = _stack(n=5, gap=1.0)
    s.step()
    c = s.body_color.numpy()
    for i in range(4):
        assert c[i] != c[i + 1]


@pytest.mark.parametrize("mode", ["jones_plassmann", "jacobi"])
def test_coloring_mode_conflict_free(mode):  # :81-96
    s = _stack(mode)
    s.step()
    assert s.coloring_mode == mode
    assert s.count_color_conflicts() == 0
    assert 1 <= s.num_active_colors <= s._max_colors


def test_coloring_mode_switch_takes_effect_at_runtime():  # :99-140
    s = _stack("jones_plassmann")
    s.step()
    jp = s.num_active_colors
    assert s._color_dirty is False
    s.coloring_mode = "jacobi"
    assert s._color_dirty is True
    s.step()
    assert s.coloring_mode == "jacobi"
    assert s.count_color_conflicts() == 0
    assert s.num_active_colors <= jp
    assert s.stats()["recolored"] == 1
    s.step()
    assert s._color_dirty is False
    s.coloring_mode = "jacobi"
    assert s._color_dirty is False


def test_jacobi_packs_no_worse_than_jp():  # :143-154
    def colors(mode):
        s = _stack(mode)
        s.step()
        return s.num_active_colors
    assert colors("jacobi") <= colors("jones_plassmann")


def test_coloring_after_dynamic_contact():  # :157-185
    s = Solver6DOF(gravity=(0, -9.8, 0), iterations=4, dt=1 / 240)
    s.enable_self_collision(True)
    a = s.add_box((0.0, 2.0, 0.0), (0.2, 0.2, 0.2), mass=1.0, friction=0.3)
    b = s.add_box((5.0, 2.0, 0.0), (0.2, 0.2, 0.2), mass=1.0, friction=0.3)
    s.set_velocity(b, (-40.0, 0.0, 0.0))
    for _ in range(80):
        s.step()
        if int(s._bp_pair_count.numpy()[0]) > 0 and s.stats()["n_dyn_groups"] > 0:
            break
    assert int(s._bp_pair_count.numpy()[0]) > 0
    c = s.body_color.numpy()
    assert c[a.index] != c[b.index]


def test_graph_signature_tracks_iterations():  # :188-209
    s = _stack(n=2, gap=0.6)
    s.step()
    sig = s._graph_signature
    assert sig[0] == 4
    s.iterations = 9
    s.step()
    assert s._graph_signature[0] == 9 and s._graph_signature != sig


def test_primal_group_size_in_signature():  # :212-227
    s = _stack(n=2, gap=0.6)
    s.step()
    sig = s._graph_signature
    s.primal_group_size = 8
    assert s.primal_group_size == 8
    s.step()
    assert s._graph_signature != sig


def _tower(s):
    s.enable_self_collision(True, default_friction=0.5)
    for k in range(4):
        b = s.add_box((0.0, 0.13 + 0.24 * k, 0.0), (0.12, 0.12, 0.12), mass=1.0, friction=0.5)
        s.add_floor_contact_box(b, friction=0.5)
    return s


@pytest.mark.parametrize("group", [8, 16, 32])
def test_warp_per_body_matches_serial(group):  # :230-260 (the reference compares group 8 with serial)
    a = _tower(Solver6DOF(gravity=(0, -9.81, 0), iterations=20, substeps=4, dt=1 / 60, primal_group_size=1))
    b = _tower(Solver6DOF(gravity=(0, -9.81, 0), iterations=20, substeps=4, dt=1 / 60, primal_group_size=group))
    for _ in range(40):
        a.step()
        b.step()
    assert float(np.abs(a.positions() - b.positions()).max()) < 1.0e-3


@pytest.mark.parametrize("group", [1, 2, 4, 8, 16, 32])
def test_every_group_size_matches_fp64_oracle_per_substep(group):
    """Per substep (state injected), every lane count agrees with the FP64
    oracle to 1e-5 m.  Over 40 frames the symmetric tower is sensitive to the
    summation order, so trajectory comparisons between lane counts drift;
    the per-substep check is the exact criterion."""
    from backends import sync_oracle_from_gpu
    from oracle.oracle import OracleSolver6DOF
    kw = dict(gravity=(0, -9.81, 0), iterations=20, substeps=4, dt=1 / 60)
    sg = _tower(Solver6DOF(primal_group_size=group, **kw))
    so = _tower(OracleSolver6DOF(precision="float64", **kw))
    sg._flush()
    so._flush()
    worst = 0.0
    for _ in range(80):
        sync_oracle_from_gpu(sg, so)
        sg.substep()
        so.substep()
        worst = max(worst, float(np.abs(sg.state_dict()["x"] - so.get_bodies()[0]).max()))
    assert worst < 1e-5


def test_one_host_sync_per_frame():  # :335-395 (the hot loop is readback-free)
    s = _stack(n=4, gap=0.9)
    s.substeps = 4
    for _ in range(8):
        s.step()
    before = s.host_syncs
    s.step()
    assert s.host_syncs - before == 1


def test_recolor_every_substep_stays_conflict_free():
    s = _stack("jacobi", recolor_every_substep=True)
    for _ in range(5):
        s.step()
        assert s.stats()["recolored"] == 1
    assert s.count_color_conflicts() == 0


def test_set_velocity_writes_live_buffer():  # test_solver_6dof.py:467-526
    h = 0.15
    s = Solver6DOF(dt=1 / 60, iterations=15, substeps=4, post_stabilize=True)
    s.enable_self_collision(True, default_friction=0.5)
    for k in range(2):
        b = s.add_box((0., h + 2 * h * k + 0.02 * k, 0.), (h, h, h), mass=1.0, friction=0.5)
        s.add_floor_contact_box(b, friction=0.5)
    for _ in range(60):
        s.step()
    nb = s.add_box((0.3, 2.0, 0.3), (h, h, h), mass=1.0, friction=0.5)
    s.add_floor_contact_box(nb, friction=0.5)
    s._flush()
    for _ in range(60):
        s.step()
    target = (1.7, 2.3, -1.1)
    s.set_velocity(type("B", (), {"index": 0})(), target)
    s.step()
    v = s.velocities()[0]
    assert not np.allclose(v, target, atol=1e-4)
    assert np.all(np.isfinite(s.positions())) and np.all(np.isfinite(s.velocities()))


def test_kick_all_after_midsim_add_box_settles_under_gravity():  # test_solver_6dof.py:529-580
    h = 0.12
    s = Solver6DOF(dt=1 / 60, iterations=20, substeps=6, post_stabilize=True)
    s.enable_self_collision(True, default_friction=0.5)
    for ix in range(2):
        for iz in range(2):
            for k in range(3):
                b = s.add_box((0.5 * ix, h + 2 * h * k, 0.5 * iz), (h, h, h), mass=1.0, friction=0.5)
                s.add_floor_contact_box(b, friction=0.5)
    for _ in range(80):
        s.step()
    nb = s.add_box((0.25, 2.0, 0.25), (h, h, h), mass=1.0, friction=0.5)
    s.add_floor_contact_box(nb, friction=0.5)
    s._flush()
    for _ in range(80):
        s.step()
    rng = np.random.default_rng(0)
    for i in range(s.positions().shape[0]):
        body = type("B", (), {"index": i})()
        v = s.velocities()[i]
        w = s.angular_velocities()[i]
        s.set_velocity(body, tuple(float(v[j] + rng.uniform(-2.5, 2.5)) for j in range(3)))
        s.set_angular_velocity(body, tuple(float(w[j] + rng.uniform(-3., 3.)) for j in range(3)))
    for _ in range(120):
        s.step()
    pos, vel = s.positions(), s.velocities()
    assert np.all(np.isfinite(pos)) and np.all(np.isfinite(vel))
    assert float(pos[:, 1].max()) < 1.2
    assert float(np.linalg.norm(vel, axis=1).mean()) < 0.6


def test_barrier_timeout_is_reported_not_hung():
    """A test-only flag makes block 0 skip its first barrier arrival: every
    other block's bounded wait runs out (~0.2 s), the kernel returns, and the
    host gets an error status; the context stays usable."""
    s = _stack(n=3, gap=0.9)
    s.step()
    s._debug_skip_arrive = True
    with pytest.raises(RuntimeError, match="barrier"):
        s.step()
    assert s.stats()["err"] & 1
    s._debug_skip_arrive = False
    s.clear_errors()
    s.step()
    assert s.stats()["err"] == 0
    assert np.all(np.isfinite(s.positions()))


def test_nonfinite_state_is_flagged():
    s = _stack(n=2, gap=1.0)
    s.step()
    s.set_position(type("B", (), {"index": 1})(), (float("nan"), 1.0, 0.0))
    s.step()
    assert s.stats()["err"] & 16


def test_pile_properties_at_scale():
    """Size-independent properties on a 20x20x10 pile (4,000 boxes with pins):
    canonical pair list sorted and unique, every emitted contact has a key,
    the coloring is conflict-free after a recolor, state stays finite."""
    s = Solver6DOF(dt=1 / 60, iterations=10, substeps=4, coloring_mode="jones_plassmann",
                   friction_static_mult=1.25)
    scenes.pile(s, nx=20, nz=20, ny=10, pin_every=50)
    for _ in range(60):
        s.step()
    p = s.pairs()
    key = p["a"].astype(np.int64) * (1 << 32) + p["b"]
    assert np.all(p["a"] < p["b"]) and np.all(np.diff(key) > 0)
    c = s.contacts()
    keys = np.unique(np.minimum(c[:, 0], c[:, 1]).astype(np.int64) * (1 << 34)
                     + np.maximum(c[:, 0], c[:, 1]).astype(np.int64) * 4 + c[:, 2])
    assert keys.size == c.shape[0]
    s.recolor_every_substep = True
    s.step()
    assert s.count_color_conflicts() == 0
    assert np.all(np.isfinite(s.positions())) and s.stats()["err"] == 0
