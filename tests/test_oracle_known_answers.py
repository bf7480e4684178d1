"""Known-answer tests that pin the CPU oracle (CPU only).

SAT and the geometric-stiffness diagonal against the closed forms asserted in
the reference's tests/test_solver_6dof.py:192-263, and the reference's
coloring tests (tests/test_robustness.py:49-185) on the oracle.
"""

import math

import numpy as np
import pytest

from oracle.oracle import OracleSolver6DOF, geom_stiffness_diag, obb_sat


def test_obb_sat_detects_axis_aligned_overlap():  # test_solver_6dof.py:192-207
    e = [0.2, 0.2, 0.2]
    res = obb_sat([0., 0., 0.], None, e, [0., 0.30, 0.], None, e)
    assert res is not None
    idx, n, ov = res
    assert idx == 1
    assert abs(ov - 0.1) < 1e-4
    assert abs(n[1] + 1.0) < 1e-4


def test_obb_sat_separated_returns_none():  # test_solver_6dof.py:209-217
    e = [0.2, 0.2, 0.2]
    assert obb_sat([0., 0., 0.], None, e, [0., 0.50, 0.], None, e) is None


def test_obb_sat_margin_applies_to_face_axes_only():
    # Face axes reject below -margin, edge axes below 0 (kernels_6dof.py:2056,
    # 2116).  For aligned boxes the edge cross products coincide with face
    # normals, so a 3 mm gap is rejected by an edge axis ...
    e = [0.2, 0.2, 0.2]
    assert obb_sat([0., 0., 0.], None, e, [0., 0.403, 0.], None, e) is None
    # ... and a touching pair (gap 0) is kept, depth 0 on the first face axis.
    res = obb_sat([0., 0., 0.], None, e, [0., 0.4, 0.], None, e)
    assert res is not None and res[0] == 1 and abs(res[2]) < 1e-6


def test_geom_stiffness_diag_matches_closed_form():  # test_solver_6dof.py:237-263
    g = geom_stiffness_diag([1.0, 0.0, 0.0], [0.3, 0.4, 0.5])
    exp = [0.5 * math.sqrt(0.4 ** 2 + 0.5 ** 2), math.sqrt(0.4 ** 2 / 4.0 + 0.3 ** 2),
           math.sqrt(0.5 ** 2 / 4.0 + 0.3 ** 2)]
    assert np.allclose(g, exp, atol=1e-6)


def _stack(mode, n=6, gap=0.85):
    s = OracleSolver6DOF(gravity=(0, -9.8, 0), iterations=4, coloring_mode=mode)
    for i in range(n):
        s.add_box((0.0, 0.5 + i * gap, 0.0), (0.5, 0.5, 0.5), mass=1.0, friction=0.3)
    s.enable_self_collision(True)
    s.step()
    return s


def test_coloring_touching_bodies_differ():  # test_robustness.py:49-63
    s = OracleSolver6DOF(gravity=(0, -9.8, 0), iterations=4)
    s.add_box((0.0, 2.0, 0.0), (0.5, 0.5, 0.5), mass=1.0, friction=0.3)
    s.add_box((0.6, 2.0, 0.0), (0.5, 0.5, 0.5), mass=1.0, friction=0.3)
    s.enable_self_collision(True)
    s.step()
    c, _ = s.colors()
    assert c[0] != c[1]


def test_coloring_stack_adjacent_differ():  # test_robustness.py:66-78
    s = _stack("jacobi", n=5, gap=1.0)
    c, _ = s.colors()
    for i in range(4):
        assert c[i] != c[i + 1]


@pytest.mark.parametrize("mode", ["jones_plassmann", "jacobi"])
def test_coloring_mode_conflict_free(mode):  # test_robustness.py:81-96
    s = _stack(mode)
    assert s.count_color_conflicts() == 0
    assert 1 <= s.num_active_colors <= 32


def test_jacobi_packs_no_worse_than_jp():  # test_robustness.py:143-154
    assert _stack("jacobi").num_active_colors <= _stack("jones_plassmann").num_active_colors


def test_dense_cluster_overflow_grows():  # test_robustness.py:26-46
    s = OracleSolver6DOF(gravity=(0, -9.8, 0), iterations=4)
    for i in range(60):
        s.add_box((0.01 * i, 2.0, 0.0), (0.5, 0.5, 0.5), mass=1.0, friction=0.3)
    s.enable_self_collision(True)
    s.step()
    assert s.overflowed
    for _ in range(2):
        s.step()
    c = s.counts()
    assert c["rows_reserved"] <= c["capacity"]
    assert np.all(np.isfinite(s.positions()))


def test_fp32_and_fp64_oracles_agree_per_substep():
    """The algorithm is well conditioned on the pyramid: the FP32 restatement
    stays within 1e-6 m of an FP64 replay of each substep."""
    from avbd_b200 import scenes
    P = dict(dt=1 / 60, iterations=10, substeps=4, friction_static_mult=1.2)
    a = OracleSolver6DOF(precision="float32", **P)
    b = OracleSolver6DOF(precision="float64", **P)
    scenes.pyramid20(a)
    scenes.pyramid20(b)
    a._flush()
    b._flush()
    worst = 0.0
    for _ in range(16):
        b.set_bodies(*a.get_bodies())
        r = a.rows(len(a._rows))
        b.set_static_rows(r["lam"], r["pen"], r["active"], r["was"])
        b.set_cache(*a.cache())
        c, nc = a.colors()
        b.set_colors(c, nc, a.counts()["color_dirty"])
        a.substep()
        b.substep()
        worst = max(worst, float(np.abs(a.get_bodies()[0] - b.get_bodies()[0]).max()))
    assert worst < 1e-6
