"""Batched scenes: one solver stepping independent scenes with their own
substeps and iterations.  Each scene of a batched substep is checked against
the FP64 oracle run on that scene alone (state injected from the batch, the
scene's own dt and iteration count), and the substep slots of a frame are
checked to leave a scene untouched once its own substeps are done."""

import numpy as np
import pytest

from oracle.oracle import OracleSolver6DOF

pytestmark = pytest.mark.gpu

SPECS = [(2, 5, 12, 11), (4, 10, 20, 12), (1, 3, 8, 13)]  # (substeps, iterations, bodies, seed)


class _Offset:
    """Adds a scene origin to the positions given to an oracle solver, so the
    oracle's scene has the batch scene's rows and world anchors."""

    def __init__(self, s, origin):
        self.s, self.origin = s, np.asarray(origin, np.float64)

    def add_box(self, position, *a, **kw):
        return self.s.add_box(tuple(np.asarray(position, np.float64) + self.origin), *a, **kw)

    def add_floor_contact_box(self, *a, **kw):
        return self.s.add_floor_contact_box(*a, **kw)


def _batch():
    from avbd_b200.batch import SceneBatch, c4_scene
    b = SceneBatch(dt=1 / 60, spacing=40.0, friction_static_mult=1.25, coloring_mode="jones_plassmann")
    for sub, its, n, seed in SPECS:
        c4_scene(b.add_scene(substeps=sub, iterations=its), n, np.random.default_rng(seed))
    return b


def _oracle_scene(k, origin, prio):
    from avbd_b200.batch import c4_scene
    sub, its, n, seed = SPECS[k]
    so = OracleSolver6DOF(precision="float64", dt=1 / 60, iterations=its, substeps=sub, friction_static_mult=1.25,
                          coloring_mode="jones_plassmann")
    so.enable_self_collision(True, default_friction=0.0)
    c4_scene(_Offset(so, origin), n, np.random.default_rng(seed))
    so.priorities = prio  # the batch's coloring priorities of these bodies
    so._flush()  # device-side layout now, so injected state is not rebuilt away
    return so


def _ranges(b):
    """Body and static-row ranges of each scene (scenes are built in order)."""
    of = np.asarray(b.solver._scene_of)
    rows_of = np.asarray([of[r.body_a] for r in b.solver._rows])
    out = []
    for k in range(len(b.scenes)):
        bi = np.nonzero(of == k)[0]
        ri = np.nonzero(rows_of == k)[0]
        out.append((int(bi[0]), int(bi[-1]) + 1, int(ri[0]), int(ri[-1]) + 1))
    return out


def _inject(sd, so, b0, b1, r0, r1, recolor):
    so.set_bodies(sd["x"][b0:b1], sd["q"][b0:b1], sd["v"][b0:b1], sd["w"][b0:b1], sd["pv"][b0:b1], sd["pw"][b0:b1])
    so.set_static_rows(sd["row_lam"][r0:r1], sd["row_pen"][r0:r1], sd["row_active"][r0:r1], sd["row_was"][r0:r1])
    abc = sd["cache_abc"]
    sel = (abc[:, 0] >= b0) & (abc[:, 0] < b1)
    loc = abc[sel].copy()
    loc[:, :2] -= b0
    so.set_cache(loc, sd["cache_state"][sel])
    so.set_colors(sd["colors"][b0:b1], sd["n_colors"], recolor)


def test_batched_substep_matches_each_scene_alone():
    b = _batch()
    s = b.solver
    for _ in range(25):
        b.step()
    ranges = _ranges(b)
    prio = s._prio.cpu().numpy()
    oracles = [_oracle_scene(k, b.scenes[k].origin, prio[r[0]:r[1]]) for k, r in enumerate(ranges)]
    recolored = 0
    for _ in range(8):
        sd = s.state_dict()
        s.substep()  # one batched substep: slot 0, every scene at its own dt
        # The batch recolors all scenes when any has a conflict; a scene's
        # part of that coloring is Jones-Plassmann on its own contact graph
        # with the same priorities, which the oracle reproduces when told to
        # recolor.
        rec = bool(s.stats()["recolored"])
        recolored += rec
        for so, (b0, b1, r0, r1) in zip(oracles, ranges):
            _inject(sd, so, b0, b1, r0, r1, rec)
        x = s.state_dict()["x"]
        q = s.state_dict()["q"]
        pairs = s.pairs()
        for k, (so, (b0, b1, r0, r1)) in enumerate(zip(oracles, ranges)):
            sub = SPECS[k][0]
            so.substep(1 / 60 / sub)
            xo, qo = so.get_bodies()[0], so.get_bodies()[1]
            np.testing.assert_allclose(x[b0:b1], xo, atol=1e-5, err_msg=f"scene {k}")
            dq = np.minimum(np.abs(q[b0:b1] - qo).max(axis=1), np.abs(q[b0:b1] + qo).max(axis=1))
            assert dq.max() <= 1e-5, (k, dq.max())
            op = so.pairs()
            mine = (pairs["a"] >= b0) & (pairs["a"] < b1)
            assert not np.any((pairs["b"][mine] < b0) | (pairs["b"][mine] >= b1))  # no cross-scene pair
            np.testing.assert_array_equal(pairs["a"][mine] - b0, op["a"])
            np.testing.assert_array_equal(pairs["b"][mine] - b0, op["b"])
            np.testing.assert_array_equal(pairs["sat_idx"][mine], op["sat_idx"])
            co, _ = so.colors()
            np.testing.assert_array_equal(s.state_dict()["colors"][b0:b1], co)
    assert recolored >= 1  # the recolor path was exercised too


def test_scene_sits_out_slots_beyond_its_substeps():
    """A frame is max-substeps slots; a scene with one substep moves in slot 0
    only, so its state after a whole frame equals one batched substep."""
    b = _batch()
    s = b.solver
    for _ in range(10):
        b.step()
    sd = s.state_dict()
    b0, b1, _, _ = _ranges(b)[2]  # the one-substep scene
    s.step()  # 4 slots
    x_frame = s.state_dict()["x"][b0:b1]
    v_frame = s.state_dict()["v"][b0:b1]
    s.load_state_dict(sd)
    s.substep()  # slot 0 alone
    np.testing.assert_array_equal(s.state_dict()["x"][b0:b1], x_frame)
    np.testing.assert_array_equal(s.state_dict()["v"][b0:b1], v_frame)


def test_batch_runs_and_counts_units():
    b = _batch()
    for _ in range(5):
        b.step()
    n_dyn = [sum(1 for i in range(len(b.solver._mass)) if b.solver._scene_of[i] == k and b.solver._mass[i] > 0)
             for k in range(len(SPECS))]
    assert b.body_substeps_per_frame() == sum(n * sp[0] for n, sp in zip(n_dyn, SPECS))
    assert np.isfinite(b.solver.positions()).all()
    for sc in b.scenes:  # nothing fell through the floor
        assert sc.positions()[:, 1].min() > -0.05
