"""read_state_batched (solver_6dof.py:1952-2052): the viewer's packed
read-out equals the per-array getters, with the reference's keys, dtypes and
row count (the live static + dynamic rows), and include_rows=False returns
the bodies with empty row arrays."""

import numpy as np
import pytest

from avbd_b200 import scenes
from backends import make_gpu

pytestmark = pytest.mark.gpu


def _pile():
    s = make_gpu(dt=1 / 60, iterations=10, substeps=4, friction_static_mult=1.25, coloring_mode="jones_plassmann")
    scenes.pile(s, nx=6, nz=6, ny=4, spacing=0.95, pin_every=7)
    for _ in range(30):
        s.step()
    return s


def test_read_state_batched_matches_getters():
    s = _pile()
    out = s.read_state_batched()
    n_c = int(s.n_active_rows[0])
    assert out["n_rows"] == n_c > len(s._rows)  # static prefix plus live contact rows
    for key, want in (("positions", s.positions()), ("orientations", s.orientations()),
                      ("angular_velocities", s.angular_velocities())):
        assert out[key].dtype == np.float32 and out[key].shape == want.shape
        np.testing.assert_array_equal(out[key], want)
    np.testing.assert_array_equal(out["lambdas"], s.lambdas()[:n_c])
    np.testing.assert_array_equal(out["active"], s.active()[:n_c])
    for key in ("lambdas", "active", "was_static", "c_type"):
        assert out[key].shape == (n_c,)
    assert out["lambdas"].dtype == np.float32
    for key in ("active", "was_static", "c_type"):
        assert out[key].dtype == np.int32
    # row types: 24 floor-corner rows per box (normal + 2 tangents), 3 per pin,
    # then 3 rows per box-box contact (normal BOX_BOX + 2 tangents)
    ct = out["c_type"]
    assert set(np.unique(ct)) <= {0, 1, 2, 3}
    assert (ct == 3).sum() > 0 and (ct == 2).sum() == 3 * sum(1 for g in s._groups if g[0] == 1)
    assert np.all(np.isin(out["was_static"], (0, 1)))


def test_read_state_batched_without_rows():
    s = _pile()
    out = s.read_state_batched(include_rows=False)
    assert out["n_rows"] == 0
    for key in ("lambdas", "active", "was_static", "c_type"):
        assert out[key].shape == (0,)
    np.testing.assert_array_equal(out["positions"], s.positions())
