"""The 5 mm anchor-keyed contact cache (the reference's documented cache key:
bodies plus the contact point in the lower body's frame at 5 mm) against the
oracle keyed the same way, and its behaviour where the ordinal key loses
contacts."""

import numpy as np
import pytest

from backends import make_gpu, sync_oracle_from_gpu

pytestmark = pytest.mark.gpu


def _pair(seed=0):
    from oracle.oracle import OracleSolver6DOF
    from avbd_b200 import scenes
    params = dict(dt=1 / 60, iterations=10, substeps=4, friction_static_mult=1.25, coloring_mode="jones_plassmann")
    sg = make_gpu(**params)
    sg.cache_key_mode = "anchor_5mm"
    so = OracleSolver6DOF(precision="float64", **params)
    so.set_key_mode("anchor_5mm")
    for s in (sg, so):
        scenes.pile(s, nx=7, nz=7, ny=4, spacing=0.95, seed=seed, pin_every=11)
    return sg, so


def test_anchor_keyed_substeps_match_oracle():
    sg, so = _pair()
    for _ in range(30):
        sg.step()
    sg._flush()
    so._flush()
    worst = 0.0
    for _ in range(6):
        sync_oracle_from_gpu(sg, so)
        sg.substep()
        so.substep()
        kg = sg.state_dict()["cache_keys"]
        ko, _ = so.cache_keys()
        np.testing.assert_array_equal(np.sort(kg), ko)
        np.testing.assert_array_equal(sg.contacts(), so.contacts())
        worst = max(worst, float(np.abs(sg.state_dict()["x"] - so.get_bodies()[0]).max()))
    assert worst <= 1e-5, worst
    assert sg.stats()["n_cache_hits"] > 0


def test_cache_view_and_mode_switch():
    s = make_gpu(dt=1 / 60, iterations=8, substeps=2, friction_static_mult=1.25, coloring_mode="jones_plassmann")
    from avbd_b200 import scenes
    scenes.pile(s, nx=5, nz=5, ny=3, spacing=0.95, seed=1, pin_every=0)
    for _ in range(20):
        s.step()
    view = s._contact_cache
    keys = {(int(a), int(b), int(c)) for a, b, c in s.contacts()}
    assert set(view) == {(min(a, b), max(a, b), c) for a, b, c in keys}
    assert all(len(v) == 8 for v in view.values())
    s.cache_key_mode = "anchor_5mm"  # re-keys: the cache starts empty, then fills
    s.step()
    v2 = s._contact_cache
    assert len(v2) == len(s.contacts()) and all(isinstance(k, int) and k < (1 << 50) for k in v2)
    with pytest.raises(ValueError):
        s.cache_key_mode = "5mm"
