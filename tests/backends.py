"""Backends for the reference-suite tests: the CPU oracle and the GPU solver."""

import numpy as np
import pytest


def make_oracle(**kw):
    from oracle.oracle import OracleSolver6DOF
    kw.pop("device", None)
    return OracleSolver6DOF(precision="float32", **kw)


def make_gpu(**kw):
    import torch
    if not torch.cuda.is_available():
        raise RuntimeError("GPU test run without a CUDA device")
    from avbd_b200 import Solver6DOF
    kw.pop("device", None)
    return Solver6DOF(**kw)


BACKENDS = [pytest.param("oracle", id="oracle"), pytest.param("gpu", id="gpu", marks=pytest.mark.gpu)]


def factory(name):
    return make_oracle if name == "oracle" else make_gpu


def quat_matrix(q):
    qx, qy, qz, qw = (float(v) for v in q)
    return np.array([[1 - 2 * (qy * qy + qz * qz), 2 * (qx * qy - qw * qz), 2 * (qx * qz + qw * qy)],
                     [2 * (qx * qy + qw * qz), 1 - 2 * (qx * qx + qz * qz), 2 * (qy * qz - qw * qx)],
                     [2 * (qx * qz - qw * qy), 2 * (qy * qz + qw * qx), 1 - 2 * (qx * qx + qy * qy)]])


def sync_oracle_from_gpu(sg, so):
    """Inject the GPU solver's persistent state into the oracle."""
    return load_oracle_state(so, sg.state_dict(), sg.cache_key_mode)


def load_oracle_state(so, sd, cache_key_mode="ordinal"):
    """Load a state_dict (as written by Solver6DOF.state_dict) into the oracle."""
    so.set_bodies(sd["x"], sd["q"], sd["v"], sd["w"], sd["pv"], sd["pw"])
    so.set_static_rows(sd["row_lam"], sd["row_pen"], sd["row_active"], sd["row_was"])
    if cache_key_mode == "anchor_5mm":
        so.set_cache_keys(sd["cache_keys"], sd["cache_state"])
    else:
        so.set_cache(sd["cache_abc"], sd["cache_state"])
    so.set_colors(sd["colors"], sd["n_colors"], sd["color_dirty"])
    return sd


def discrete_equal(sg, so):
    """Broadphase pairs, SAT overlap and axis, contact counts, emitted contact
    keys, colorings and the color count of the last substep: bit-identical."""
    pg, po = sg.pairs(), so.pairs()
    for k in ("a", "b", "overlap", "sat_idx", "count"):
        np.testing.assert_array_equal(pg[k], po[k], err_msg=k)
    np.testing.assert_array_equal(sg.contacts(), so.contacts())
    cg = sg.state_dict()["colors"]
    co, nco = so.colors()
    np.testing.assert_array_equal(cg, co)
    assert sg.stats()["n_colors"] == nco


def pose_error(sg, so):
    """Per body: largest position (m) and quaternion-component difference
    (up to the quaternion's sign) between the GPU state and the oracle's."""
    sd = sg.state_dict()
    xo, qo = so.get_bodies()[0], so.get_bodies()[1]
    return pose_diff(sd["x"], sd["q"], xo, qo)


def pose_diff(xa, qa, xb, qb):
    dx = np.abs(xa - xb).max(axis=1)
    dq = np.minimum(np.abs(qa - qb).max(axis=1), np.abs(qa + qb).max(axis=1))
    return dx, dq
