"""Golden fixtures (tests/golden/*.npz, written by make_golden.py from the
FP64 oracle): the complete state at a snapshot of a seeded scene and the
outcome of one substep from it.

* CPU: the oracle still reproduces every fixture (pins the checker itself).
* GPU: the B200 substep from the fixture state matches the fixture: the
  discrete outputs exactly (pairs, SAT axes, contact counts, contact keys,
  colors), poses within 1e-5 m / 1e-5 of the FP64 result.
"""

import glob
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
FILES = sorted(f for f in glob.glob(os.path.join(HERE, "golden", "*.npz"))
               if not os.path.basename(f).startswith("reference_"))  # those: test_reference_pin.py
POS_TOL = 1e-5
QUAT_TOL = 1e-5


def _case(path):
    name = os.path.basename(path).rsplit("_f", 1)[0]
    return name, dict(np.load(path))


def _state(z):
    keys = ("x", "q", "v", "w", "pv", "pw", "row_lam", "row_pen", "row_active", "row_was", "cache_abc",
            "cache_state", "colors")
    sd = {k: z[k] for k in keys}
    sd["n_colors"] = int(z["n_colors"])
    sd["color_dirty"] = bool(z["color_dirty"])
    return sd


def test_fixtures_present():
    assert len(FILES) >= 8


@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f)[:-4] for f in FILES])
def test_oracle_reproduces_fixture(path):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden as G
    name, z = _case(path)
    so = G.make_oracle(name)
    G.inject(so, _state(z))
    so.substep()
    out = G.outcome(so)
    for k in ("pair_a", "pair_b", "pair_overlap", "pair_sat", "pair_count", "contacts", "next_colors"):
        np.testing.assert_array_equal(out[k], z[k], err_msg=k)
    np.testing.assert_allclose(out["next_x"], z["next_x"], atol=1e-9)
    np.testing.assert_allclose(out["next_q"], z["next_q"], atol=1e-9)


@pytest.mark.gpu
@pytest.mark.parametrize("path", FILES, ids=[os.path.basename(f)[:-4] for f in FILES])
def test_gpu_substep_matches_fixture(path):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden as G
    from backends import make_gpu
    name, z = _case(path)
    build, params = G.CASES[name]
    s = make_gpu(**params)
    build(s)
    s.load_state_dict(_state(z))
    s.substep()
    p = s.pairs()
    np.testing.assert_array_equal(p["a"], z["pair_a"])
    np.testing.assert_array_equal(p["b"], z["pair_b"])
    np.testing.assert_array_equal(p["overlap"], z["pair_overlap"])
    np.testing.assert_array_equal(p["sat_idx"], z["pair_sat"])
    np.testing.assert_array_equal(p["count"], z["pair_count"])
    np.testing.assert_array_equal(s.contacts(), z["contacts"])
    sd = s.state_dict()
    np.testing.assert_array_equal(sd["colors"], z["next_colors"])
    assert np.abs(sd["x"] - z["next_x"]).max() <= POS_TOL
    dq = np.minimum(np.abs(sd["q"] - z["next_q"]).max(axis=1), np.abs(sd["q"] + z["next_q"]).max(axis=1))
    assert dq.max() <= QUAT_TOL
