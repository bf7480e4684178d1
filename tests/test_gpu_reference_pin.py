"""The B200 substep against the reference's OWN substeps.

tests/golden/reference_*.npz were recorded from the reference's unmodified
Solver6DOF (src/avbd3d/solver_6dof.py:1178-1679, kernels_6dof.py:122-3336)
run on the CPU through oracle/warp_shim.  For every recorded substep the
reference's state before it (bodies, static rows, contact hash, and the
coloring the reference used) is loaded into the GPU solver through the C ABI
and one substep runs.  Broadphase pairs, SAT overlap and axis, contact counts
and the emitted contact keys must equal the reference's exactly; poses must
be within 1e-5 m / 1e-5 of the reference's float32 results (the GPU's fused
multiply-adds and lane reductions round differently from the CPU).
"""

import os

import numpy as np
import pytest

from backends import make_gpu, pose_diff
from test_reference_pin import FIXTURES, NAMES, _scene, _state

pytestmark = pytest.mark.gpu

POS_TOL = 1e-5
QUAT_TOL = 1e-5
HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.mark.parametrize("name", NAMES)
def test_gpu_substep_matches_reference(name):
    assert FIXTURES
    fx = np.load(os.path.join(HERE, "golden", f"reference_{name}.npz"))
    params, build, _, _ = _scene(name)
    sg = make_gpu(**params)
    build(sg)
    sg._flush()
    worst_x = worst_q = 0.0
    for k in range(int(fx["n_substeps"])):
        sg.load_state_dict(_state(fx, k))
        sg.substep()
        p = sg.pairs()
        for key in ("a", "b", "overlap", "sat_idx", "count"):
            np.testing.assert_array_equal(p[key], fx[f"s{k}_pairs_{key}"], err_msg=f"{name} substep {k} {key}")
        np.testing.assert_array_equal(sg.contacts(), fx[f"s{k}_contacts"], err_msg=f"{name} substep {k}")
        np.testing.assert_array_equal(sg.state_dict()["colors"], fx[f"s{k}_colors"])
        sd = sg.state_dict()
        dx, dq = pose_diff(sd["x"], sd["q"], fx[f"s{k}_out_x"].astype(np.float64),
                           fx[f"s{k}_out_q"].astype(np.float64))
        worst_x, worst_q = max(worst_x, float(dx.max())), max(worst_q, float(dq.max()))
    assert sg.stats()["err"] == 0
    assert worst_x <= POS_TOL and worst_q <= QUAT_TOL, (worst_x, worst_q)
