"""The oracle pinned to the reference's own code.

tests/golden/reference_*.npz hold substeps of the reference's unmodified
Solver6DOF (src/avbd3d/solver_6dof.py:1178-1679 and the kernels of
kernels_6dof.py:122-3336), executed on the CPU through the pure-Python warp
stand-in (oracle/warp_shim), written by tests/golden/make_reference_golden.py.

For every recorded substep the reference's state before it (bodies, static
rows, contact hash, and the coloring it used) is loaded into the oracle's
float32 build, the oracle runs the substep, and its outputs must equal the
reference's BIT FOR BIT: broadphase pairs, SAT overlap and axis, contact
counts, emitted contact keys in row order, positions, orientations, linear
and angular velocities, and the static rows' lambdas.

The coloring is injected because the reference's coloring kernels read
neighbour colors while they are written in the same launch
(kernels_6dof.py:3121-3148, 3247-3262): on Warp's CPU device that is a
sequential greedy coloring, on CUDA a race.  The oracle and the GPU solver
define the coloring rounds on a snapshot of the previous round instead;
test_reference_coloring_semantics shows both colorings are proper.

When the reference checkout is present, test_shim_reproduces_fixture reruns
the first substeps through the stand-in and checks they reproduce the
fixture, so the fixtures are shown to be the reference's output.
"""

import glob
import os

import numpy as np
import pytest

from backends import load_oracle_state

HERE = os.path.dirname(os.path.abspath(__file__))
FIXTURES = sorted(glob.glob(os.path.join(HERE, "golden", "reference_*.npz")))
NAMES = [os.path.basename(f)[len("reference_"):-len(".npz")] for f in FIXTURES]
STATE_KEYS = ("x", "q", "v", "w", "pv", "pw", "row_lam", "row_pen", "row_active", "row_was", "cache_abc",
              "cache_state")


def _scene(name):
    from golden.make_reference_golden import SCENES
    return SCENES[name]


def _state(fx, k):
    sd = {key: fx[f"s{k}_in_{key}"] for key in STATE_KEYS}
    sd["colors"] = fx[f"s{k}_colors"]
    sd["n_colors"] = int(fx[f"s{k}_n_colors"])
    sd["color_dirty"] = False
    return sd


def _oracle(name):
    from oracle.oracle import OracleSolver6DOF
    params, build, _, _ = _scene(name)
    so = OracleSolver6DOF(precision="float32", **params)
    build(so)
    so._flush()
    return so


def test_fixtures_present():
    assert len(FIXTURES) >= 5


@pytest.mark.parametrize("name", NAMES)
def test_oracle_matches_reference_bit_for_bit(name):
    fx = np.load(os.path.join(HERE, "golden", f"reference_{name}.npz"))
    so = _oracle(name)
    n_contacts = 0
    for k in range(int(fx["n_substeps"])):
        load_oracle_state(so, _state(fx, k))
        so.substep()
        p = so.pairs()
        for key in ("a", "b", "overlap", "sat_idx", "count"):
            np.testing.assert_array_equal(p[key], fx[f"s{k}_pairs_{key}"], err_msg=f"{name} substep {k} {key}")
        c = so.contacts()
        np.testing.assert_array_equal(c, fx[f"s{k}_contacts"], err_msg=f"{name} substep {k} contacts")
        n_contacts += len(c)
        x, q, v, w = (a.astype(np.float32) for a in so.get_bodies()[:4])
        for key, got in (("x", x), ("q", q), ("v", v), ("w", w)):
            np.testing.assert_array_equal(got, fx[f"s{k}_out_{key}"], err_msg=f"{name} substep {k} {key}")
        ns = fx[f"s{k}_out_row_lam"].shape[0]
        np.testing.assert_array_equal(so.rows()["lam"][:ns].astype(np.float32), fx[f"s{k}_out_row_lam"],
                                      err_msg=f"{name} substep {k} static lambdas")
    if name != "pyramid20_jacobi":  # the fresh pyramid has no box contacts before it settles
        assert n_contacts > 0


@pytest.mark.parametrize("name", NAMES)
def test_oracle_follows_reference_trajectory(name):
    """Loaded once, at the first recorded substep, the oracle then runs on
    its own (only the reference's coloring of each substep is given) and
    still ends bit-identical to the reference."""
    fx = np.load(os.path.join(HERE, "golden", f"reference_{name}.npz"))
    so = _oracle(name)
    load_oracle_state(so, _state(fx, 0))
    k_last = int(fx["n_substeps"]) - 1
    for k in range(k_last + 1):
        so.set_colors(fx[f"s{k}_colors"], int(fx[f"s{k}_n_colors"]), False)
        so.substep()
    x, q, v, w = (a.astype(np.float32) for a in so.get_bodies()[:4])
    for key, got in (("x", x), ("q", q), ("v", v), ("w", w)):
        np.testing.assert_array_equal(got, fx[f"s{k_last}_out_{key}"], err_msg=f"{name} {key}")


@pytest.mark.parametrize("name", NAMES)
def test_reference_coloring_semantics(name):
    """The reference's coloring of each recorded contact graph and the
    oracle's snapshot coloring of the same graph (the oracle recolors from
    the same state) are both proper -- no contact joins two bodies of one
    color -- though they may differ, by design."""
    fx = np.load(os.path.join(HERE, "golden", f"reference_{name}.npz"))
    so = _oracle(name)
    for k in range(int(fx["n_substeps"])):
        c = fx[f"s{k}_contacts"]
        if not len(c):
            continue
        col = fx[f"s{k}_colors"]
        assert np.all(col[c[:, 0]] != col[c[:, 1]])
        sd = _state(fx, k)
        sd["color_dirty"] = True
        load_oracle_state(so, sd)
        so.substep()
        np.testing.assert_array_equal(so.contacts(), c)
        own, _ = so.colors()
        assert np.all(own[c[:, 0]] != own[c[:, 1]])
        assert so.count_color_conflicts() == 0


@pytest.mark.slow
@pytest.mark.parametrize("name", ["pyramid20_jacobi", "towers_jp"])
def test_shim_reproduces_fixture(name):
    from oracle.warp_shim import reference
    if not reference.available():
        pytest.skip("the reference checkout is not mounted here")
    S = reference.load()
    params, build, frames, _ = _scene(name)
    fx = np.load(os.path.join(HERE, "golden", f"reference_{name}.npz"))
    s = S.Solver6DOF(device="cpu", **params)
    build(s)
    s._flush()
    for _ in range(frames):
        s.step()
    for k in range(2):
        reference.substep(s)
        np.testing.assert_array_equal(s.x.numpy()[:len(s._x)], fx[f"s{k}_out_x"])
        np.testing.assert_array_equal(s.q.numpy()[:len(s._x)], fx[f"s{k}_out_q"])
        np.testing.assert_array_equal(reference.contacts(s), fx[f"s{k}_contacts"])
