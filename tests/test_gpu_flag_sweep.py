"""The flag-ordered color sweep (no grid barrier between colors; each body
waits only for its own previous pass and its neighbours) against the oracle
and against the barrier sweep it replaces."""

import numpy as np
import pytest

from backends import make_gpu

pytestmark = pytest.mark.gpu


def _pile(flag, seed=0, nx=12, nz=12, ny=5, **kw):
    from avbd_b200 import scenes
    s = make_gpu(dt=1 / 60, iterations=10, substeps=4, friction_static_mult=1.25,
                 coloring_mode="jones_plassmann", **kw)
    s.flag_sweep = flag
    scenes.pile(s, nx=nx, nz=nz, ny=ny, seed=seed, pin_every=97)
    return s


@pytest.mark.parametrize("group_size", [4, 8, 16])
def test_flag_sweep_substep_matches_barrier_sweep(group_size):
    """Same state in, one substep each way: the per-body arithmetic is the
    same, only the ordering mechanism differs."""
    a, b = _pile(False), _pile(True)
    a.primal_group_size = b.primal_group_size = group_size
    for _ in range(30):
        a.step()
    sd = a.state_dict()
    for _ in range(4):
        b.load_state_dict(sd)
        a.load_state_dict(sd)
        a.substep()
        b.substep()
        sa, sb = a.state_dict(), b.state_dict()
        np.testing.assert_allclose(sb["x"], sa["x"], atol=2e-6)
        np.testing.assert_allclose(np.abs(sb["q"]), np.abs(sa["q"]), atol=2e-6)
        np.testing.assert_array_equal(sb["colors"], sa["colors"])
        assert b.stats()["err"] == 0
        sd = sa


def test_flag_sweep_parity_with_oracle():
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


def test_flag_sweep_is_bit_reproducible():
    runs = []
    for _ in range(2):
        s = _pile(True, seed=5)
        for _ in range(15):
            s.step()
        runs.append((s.positions(), s.orientations()))
    np.testing.assert_array_equal(runs[0][0], runs[1][0])
    np.testing.assert_array_equal(runs[0][1], runs[1][1])


def test_flag_sweep_in_batched_scenes():
    """Batched scenes with their own iteration counts under the flag sweep
    give the barrier sweep's substep."""
    from avbd_b200.batch import SceneBatch, c4_scene
    out = []
    for flag in (False, True):
        b = SceneBatch(dt=1 / 60, spacing=40.0, friction_static_mult=1.25, coloring_mode="jones_plassmann")
        for sub, its, n, seed in [(2, 5, 40, 1), (4, 10, 60, 2), (1, 3, 30, 3)]:
            c4_scene(b.add_scene(substeps=sub, iterations=its), n, np.random.default_rng(seed))
        b.solver.flag_sweep = flag
        out.append(b)
    for _ in range(20):
        out[0].step()
    sd = out[0].solver.state_dict()
    out[1].solver.load_state_dict(sd)
    for b in out:
        b.solver.load_state_dict(sd)
        b.solver.step()
    np.testing.assert_allclose(out[1].solver.state_dict()["x"], out[0].solver.state_dict()["x"], atol=2e-5)
