"""Jones-Plassmann coloring in the persistent kernel runs as one dataflow
phase (each body publishes its color once its higher-priority neighbours
have); the split path keeps the reference's round loop.  Both must give the
oracle's colors, including bodies still uncolored after the last round
(JP_ROUNDS = 24), which take color 0."""

import numpy as np
import pytest

from backends import make_gpu, sync_oracle_from_gpu
from oracle.oracle import OracleSolver6DOF

pytestmark = pytest.mark.gpu

KW = dict(dt=1 / 60, iterations=6, substeps=2, friction_static_mult=1.25, coloring_mode="jones_plassmann")
N_CHAIN = 40
HE = 0.25


def _priority_chain(s, n=N_CHAIN):
    """A row of boxes on the floor, each overlapping the next by 1 cm, laid
    out so priority falls along the row: the JP round of the k-th box is k,
    so boxes 24.. are still uncolored after the last round."""
    prio = np.random.default_rng(seed=0xA5BD).uniform(0.0, 1.0, size=n).astype(np.float32)
    order = np.lexsort((np.arange(n), -prio))  # decreasing priority, ties by index
    slot = np.empty(n, np.int64)
    slot[order] = np.arange(n)
    s.enable_self_collision(True, default_friction=0.5)
    for i in range(n):
        b = s.add_box((float(slot[i]) * (2 * HE - 0.01), HE, 0.0), (HE, HE, HE), mass=1.0, friction=0.5)
        s.add_floor_contact_box(b, friction=0.5)
    return slot


def _expected_colors(slot):
    # greedy along the chain alternates 0/1; rounds >= 24 stay uncolored -> 0
    return np.where(slot >= 24, 0, slot % 2).astype(np.int32)


@pytest.mark.parametrize("persistent", [True, False])
def test_chain_colors_match_oracle_with_stragglers(persistent):
    sg = make_gpu(persistent=persistent, **KW)
    so = OracleSolver6DOF(precision="float64", **KW)
    slot = _priority_chain(sg)
    _priority_chain(so)
    sg._flush()
    so._flush()
    sync_oracle_from_gpu(sg, so)
    sg.substep()
    so.substep()
    assert sg.stats()["n_pairs"] == N_CHAIN - 1
    cg = sg.state_dict()["colors"]
    co, nco = so.colors()
    np.testing.assert_array_equal(cg, co)
    np.testing.assert_array_equal(cg, _expected_colors(slot))
    assert sg.stats()["n_colors"] == nco == 2
    assert sg.stats()["err"] == 0


def test_dataflow_and_round_loop_agree_on_a_pile():
    """Same state, one substep on each path: identical colors and color
    counts (the contact graph comes from the same collision kernels)."""
    from avbd_b200 import scenes
    a = make_gpu(persistent=True, recolor_every_substep=True, **KW)
    b = make_gpu(persistent=False, recolor_every_substep=True, **KW)
    for s in (a, b):
        scenes.pile(s, nx=14, nz=14, ny=5, seed=4, pin_every=0)
    for _ in range(25):
        a.step()
    sd = a.state_dict()
    for _ in range(3):
        a.load_state_dict(sd)
        b.load_state_dict(sd)
        a.substep()
        b.substep()
        np.testing.assert_array_equal(a.state_dict()["colors"], b.state_dict()["colors"])
        assert a.stats()["n_colors"] == b.stats()["n_colors"]
        assert a.stats()["recolored"] == 1
        sd = a.state_dict()
