"""Between LBVH rebuilds the collision pipeline only refits the tree to the
bodies' new boxes.  The pair list is sorted by body, not by tree, so a refit
tree must give exactly the pairs of a rebuilt one, and the whole trajectory
stays bit-identical (kernels_6dof.py:1946-1978 rebuilds every substep)."""

import numpy as np
import pytest

from backends import make_gpu

pytestmark = pytest.mark.gpu


def _pile(every, seed=2):
    from avbd_b200 import scenes
    s = make_gpu(dt=1 / 60, iterations=8, substeps=4, friction_static_mult=1.25, coloring_mode="jones_plassmann")
    s.bvh_rebuild_every = every
    scenes.pile(s, nx=12, nz=12, ny=6, seed=seed, pin_every=0)
    return s


@pytest.mark.parametrize("every", [2, 8, 1000])
def test_refit_tree_gives_the_rebuilt_trajectory(every):
    a, b = _pile(1), _pile(every)
    for frame in range(25):  # the pile falls and collapses: boxes move a lot
        a.step()
        b.step()
        pa, pb = a.pairs(), b.pairs()
        for k in ("a", "b", "overlap", "sat_idx", "count"):
            np.testing.assert_array_equal(pa[k], pb[k], err_msg=f"frame {frame} {k}")
    np.testing.assert_array_equal(a.positions(), b.positions())
    np.testing.assert_array_equal(a.orientations(), b.orientations())
    st = b.stats()
    assert st["err"] == 0 and st["graph_state"] == 7  # each frame one whole-frame graph


def test_refit_after_teleport():
    """Moving bodies far away between substeps (a user setter) only makes the
    refit tree loose; the pairs stay exact."""
    a, b = _pile(1, seed=5), _pile(1000, seed=5)
    for _ in range(6):
        a.step()
        b.step()
    from avbd_b200.solver import RigidBody
    for s in (a, b):
        x = s.positions()
        for i in range(0, len(x), 7):
            s.set_position(RigidBody(index=i, half_extents=(0.0, 0.0, 0.0)),
                           (float(x[i, 0]) + 30.0, float(x[i, 1]), float(x[i, 2])))
    for _ in range(3):
        a.substep()
        b.substep()
        np.testing.assert_array_equal(a.pairs()["a"], b.pairs()["a"])
        np.testing.assert_array_equal(a.pairs()["b"], b.pairs()["b"])
    np.testing.assert_array_equal(a.positions(), b.positions())
