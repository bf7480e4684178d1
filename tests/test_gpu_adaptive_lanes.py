"""Adaptive lanes per body (barrier sweep): colors too small to fill the
resident warps run with more lanes per body.  Only the order of each body's
sums changes, so a substep matches the fixed-lane sweep to float rounding and
the FP64 oracle to the parity tolerance, and runs stay bit-reproducible."""

import numpy as np
import pytest

from backends import make_gpu

pytestmark = pytest.mark.gpu


def _pile(adaptive, seed=0, nx=12, nz=12, ny=5, group_size=4):
    from avbd_b200 import scenes
    s = make_gpu(dt=1 / 60, iterations=10, substeps=4, friction_static_mult=1.25,
                 coloring_mode="jones_plassmann")
    s.adaptive_lanes = adaptive
    s.primal_group_size = group_size
    scenes.pile(s, nx=nx, nz=nz, ny=ny, seed=seed, pin_every=97)
    return s


@pytest.mark.parametrize("group_size", [1, 4, 8])
def test_adaptive_substep_matches_fixed_lanes(group_size):
    a, b = _pile(False, group_size=group_size), _pile(True, group_size=group_size)
    for _ in range(30):
        a.step()
    sd = a.state_dict()
    for _ in range(4):
        a.load_state_dict(sd)
        b.load_state_dict(sd)
        a.substep()
        b.substep()
        sa, sb = a.state_dict(), b.state_dict()
        np.testing.assert_allclose(sb["x"], sa["x"], atol=2e-6)
        np.testing.assert_allclose(np.abs(sb["q"]), np.abs(sa["q"]), atol=2e-6)
        np.testing.assert_array_equal(sb["colors"], sa["colors"])
        assert b.stats()["err"] == 0
        sd = sa


def test_adaptive_parity_with_oracle():
    from oracle.oracle import OracleSolver6DOF
    from avbd_b200 import scenes
    from backends import sync_oracle_from_gpu
    s = _pile(True, seed=3)
    so = OracleSolver6DOF(precision="float64", dt=1 / 60, iterations=10, substeps=4, friction_static_mult=1.25,
                          coloring_mode="jones_plassmann")
    scenes.pile(so, nx=12, nz=12, ny=5, seed=3, pin_every=97)
    for _ in range(40):
        s.step()
    s._flush()
    so._flush()
    worst = 0.0
    for _ in range(6):
        sync_oracle_from_gpu(s, so)
        s.substep()
        so.substep()
        worst = max(worst, float(np.abs(s.state_dict()["x"] - so.get_bodies()[0]).max()))
    assert worst <= 1e-5, worst


def test_adaptive_is_bit_reproducible():
    runs = []
    for _ in range(2):
        s = _pile(True, seed=5)
        for _ in range(15):
            s.step()
        runs.append((s.positions(), s.orientations()))
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    np.testing.assert_array_equal(runs[0][1], runs[1][1])
