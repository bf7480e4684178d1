"""The compact row table behind Solver6DOF._rows: floor-contact blocks must
materialise exactly the rows the reference's add_floor_contact_box appends
(solver_6dof.py:474-520), in the same numbering, interleaved with explicit
rows (pins) in call order."""

import math

import numpy as np

from avbd_b200.solver import CONTACT_TANGENT_6DOF, FLOOR_CONTACT_6DOF, PIN_6DOF, _Row, _RowTable

INF = math.inf


def _expected_floor(rows, body, he, floor_y, mu, mus, stiff):
    for sx in (-1.0, 1.0):
        for sy in (-1.0, 1.0):
            for sz in (-1.0, 1.0):
                off = (sx * he[0], sy * he[1], sz * he[2])
                n = len(rows)
                rows.append(_Row(FLOOR_CONTACT_6DOF, body, world_anchor=(0.0, floor_y, 0.0), off_a=off,
                                 stiffness=stiff, fmin=-INF, fmax=0.0))
                if mu > 0.0:
                    t = len(rows)
                    rows.append(_Row(CONTACT_TANGENT_6DOF, body, world_anchor=(1.0, 0.0, 0.0), off_a=off,
                                     stiffness=stiff, sibling=n, friction=mu, friction_static=mus, partner=t + 1))
                    rows.append(_Row(CONTACT_TANGENT_6DOF, body, world_anchor=(0.0, 0.0, 1.0), off_a=off,
                                     stiffness=stiff, sibling=n, friction=mu, friction_static=mus, partner=t))


def test_row_table_matches_explicit_rows():
    tab, ref = _RowTable(), []
    rng = np.random.default_rng(0)
    for k in range(40):
        if k % 7 == 3:  # a pin: three explicit rows
            for axis in range(3):
                r = _Row(PIN_6DOF, k, body_b=axis, world_anchor=(1.0, 2.0, 3.0), off_a=(0.1, 0.2, 0.3))
                tab.append(r)
                ref.append(r)
            continue
        he = tuple(float(v) for v in rng.uniform(0.1, 0.5, 3))
        mu = 0.0 if k % 5 == 0 else 0.4
        start = tab.add_floor_block(k, he, 0.25 * (k % 3), mu, 1.25 * mu, INF if k % 4 else 1e7)
        assert start == len(ref)
        _expected_floor(ref, k, he, 0.25 * (k % 3), mu, 1.25 * mu, INF if k % 4 else 1e7)
    assert len(tab) == len(ref)
    assert list(tab) == ref
    for i in rng.integers(0, len(ref), 50):
        assert tab[int(i)] == ref[int(i)]
    assert tab[-1] == ref[-1] and tab[3:9] == ref[3:9]
    assert len(tab.floor_blocks()) == sum(1 for k in range(40) if k % 7 != 3)


def test_implicit_floor_corners_decode_to_the_reference_offsets():
    """Floor blocks whose half extents are their body's store no offsets: the
    kernels rebuild each corner as +-he by the corner index in meta bits 6-8
    (csrc/common.cuh implicit_corner) and read the floor height from mat.w.
    Decoding that way must give the reference's corner offsets bit for bit;
    a block with other half extents keeps explicit offsets."""
    from avbd_b200.solver import KIND_FLOOR, META_IMPLICIT, Solver6DOF
    s = Solver6DOF.__new__(Solver6DOF)  # host scene state only (no device)
    s._x = [(0.0, 0.0, 0.0)] * 3
    s._half_extents = [(0.3, 0.2, 0.45), (0.1, 0.1, 0.1), (0.25, 0.35, 0.15)]
    s._rows, s._groups = _RowTable(), []
    s._rows.add_floor_block(0, (0.3, 0.2, 0.45), 0.0, 0.5, 0.6, INF)
    s._rows.add_floor_block(1, (0.1, 0.1, 0.1), -1.5, 0.0, 0.0, 1e7)
    s._rows.add_floor_block(2, (0.2, 0.35, 0.15), 0.25, 0.4, 0.5, INF)  # not the body's extents
    out, _, _ = s._static_group_arrays()
    meta, offa, mat, body = out["meta"], out["offa"], out["mat"], out["body"][:, 0]
    assert len(meta) == 24 and np.all(meta & 3 == KIND_FLOOR)
    he = np.asarray(s._half_extents, np.float32)
    for g in range(24):
        blk = s._rows.floor_blocks()[g // 8]
        ref = s._rows._block_row(blk, (g % 8) * blk[7])
        want = np.asarray(ref.off_a, np.float32)
        if meta[g] & META_IMPLICIT:
            c = (meta[g] >> 6) & 7
            h = he[body[g]]
            got = np.array([h[0] if c & 4 else -h[0], h[1] if c & 2 else -h[1], h[2] if c & 1 else -h[2]], np.float32)
            assert np.all(offa[g] == 0.0)
            assert np.float32(mat[g, 3]) == np.float32(ref.world_anchor[1])
        else:
            got = offa[g, :3]
            assert offa[g, 3] == np.float32(ref.world_anchor[1]) and mat[g, 3] == INF
        np.testing.assert_array_equal(got, want)
    assert [bool(m & META_IMPLICIT) for m in meta[::8]] == [True, True, False]
