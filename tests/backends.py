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
    sd = sg.state_dict()
    so.set_bodies(sd["x"], sd["q"], sd["v"], sd["w"], sd["pv"], sd["pw"])
    so.set_static_rows(sd["row_lam"], sd["row_pen"], sd["row_active"], sd["row_was"])
    if sg.cache_key_mode == "anchor_5mm":
        so.set_cache_keys(sd["cache_keys"], sd["cache_state"])
    else:
        so.set_cache(sd["cache_abc"], sd["cache_state"])
    so.set_colors(sd["colors"], sd["n_colors"], sd["color_dirty"])
    return sd
