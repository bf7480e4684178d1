"""Resting floor corners (resting_floor, barrier sweep): a floor corner above
the floor in its resting start state is evaluated from the body's pose
alone.  Its contribution and its (unchanged) dual state are the ones a read
of the group gives, so whole trajectories match the all-reads run bit for
bit."""

import numpy as np
import pytest

from backends import make_gpu

pytestmark = pytest.mark.gpu


def _pile(rest, seed=0, nx=12, nz=12, ny=5):
    from avbd_b200 import scenes
    s = make_gpu(dt=1 / 60, iterations=10, substeps=4, friction_static_mult=1.25,
                 coloring_mode="jones_plassmann")
    s.flag_sweep = False
    s.resting_floor = rest
    scenes.pile(s, nx=nx, nz=nz, ny=ny, seed=seed, pin_every=97)
    return s


def _resting_bodies(s) -> int:
    import torch
    fs = s._arena.view("FSEP", torch.float32, (len(s.positions()),)).cpu().numpy()
    return int(np.isfinite(fs).sum())


def _same(a, b):
    for k in ("x", "q", "v", "w", "pv", "pw"):
        xa, xb = np.ascontiguousarray(a[k], np.float64), np.ascontiguousarray(b[k], np.float64)
        np.testing.assert_array_equal(xa.view(np.uint64), xb.view(np.uint64), err_msg=k)
    # stored multipliers compare as numbers: a skipped write keeps a +0 where
    # the clamp of a read group may store -0
    for k in ("row_lam", "row_pen", "row_active", "row_was", "cache_state"):
        np.testing.assert_array_equal(np.asarray(a[k]), np.asarray(b[k]), err_msg=k)
    np.testing.assert_array_equal(np.asarray(a["colors"]), np.asarray(b["colors"]))


def test_resting_floor_same_trajectory():
    """The pile falls onto the floor (corners go from resting to touching
    within a substep, which clears the body's resting state) and settles;
    both runs agree bit for bit at every frame."""
    a, b = _pile(False), _pile(True)
    for f in range(60):
        a.step()
        b.step()
        if f % 10 == 9:
            _same(a.state_dict(), b.state_dict())
    assert a.stats()["err"] == 0 and b.stats()["err"] == 0
    # most boxes stand on other boxes: their corners rest
    assert _resting_bodies(b) > 0.5 * 12 * 12 * 5


def test_resting_floor_batched_scenes():
    from avbd_b200.batch import SceneBatch, c4_scene
    out = []
    for rest in (False, True):
        b = SceneBatch(dt=1 / 60, spacing=40.0, friction_static_mult=1.25, coloring_mode="jones_plassmann")
        for sub, its, n, seed in [(2, 5, 40, 1), (4, 10, 60, 2), (1, 3, 30, 3)]:
            c4_scene(b.add_scene(substeps=sub, iterations=its), n, np.random.default_rng(seed))
        b.solver.flag_sweep = False
        b.solver.resting_floor = rest
        out.append(b)
    for _ in range(30):
        for b in out:
            b.step()
    _same(out[0].solver.state_dict(), out[1].solver.state_dict())
