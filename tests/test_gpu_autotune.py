"""The launch-shape autotuner: it times every candidate on the live scene,
applies the fastest, and leaves the simulation state as it found it."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_autotune_restores_state_and_applies_best():
    from avbd_b200 import Solver6DOF, scenes
    from avbd_b200.autotune import autotune
    s = Solver6DOF(dt=1 / 60, iterations=10, substeps=4, friction_static_mult=1.25, coloring_mode="jones_plassmann")
    scenes.pile(s, nx=10, nz=10, ny=4, seed=3, pin_every=0)
    for _ in range(30):
        s.step()
    before = s.state_dict()
    res = autotune(s, group_sizes=(4, 8, 16), blocks_per_sm=(2, 3), frames=1, warm=1)
    after = s.state_dict()
    for k in ("x", "q", "v", "w"):
        np.testing.assert_array_equal(before[k], after[k])
    # 3 group sizes x 2 CTA counts x (barrier, barrier + adaptive lanes, flags)
    assert len(res["table"]) == 18 and all(r["ms_per_frame"] > 0 for r in res["table"])
    best = res["best"]
    assert (s.primal_group_size, s.blocks_per_sm, s.flag_sweep, s.adaptive_lanes) == (
        best["group_size"], best["blocks_per_sm"], best["flag_sweep"], best["adaptive_lanes"])
    assert best["ms_per_frame"] == min(r["ms_per_frame"] for r in res["table"])
    # the tuned solver still steps: same trajectory as an untuned twin loaded with the same state
    s.step()
    t = Solver6DOF(dt=1 / 60, iterations=10, substeps=4, friction_static_mult=1.25, coloring_mode="jones_plassmann")
    scenes.pile(t, nx=10, nz=10, ny=4, seed=3, pin_every=0)
    t.primal_group_size = best["group_size"]
    t.blocks_per_sm = best["blocks_per_sm"]
    t.flag_sweep = best["flag_sweep"]
    t.adaptive_lanes = best["adaptive_lanes"]
    t.load_state_dict(before)
    t.step()
    np.testing.assert_allclose(s.state_dict()["x"], t.state_dict()["x"], atol=1e-6)
