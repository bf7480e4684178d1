"""The C-ABI library loads and exports every symbol include/avbd6.h declares
(no device calls: this runs without a GPU)."""

import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    src = open(os.path.join(ROOT, "include", "avbd6.h")).read()
    return sorted(set(re.findall(r"^\s*(?:const\s+)?\w+\*?\s+\*?(avbd_\w+)\s*\(", src, flags=re.M)))


def test_header_declares_entry_points():
    names = _declared()
    assert "avbd_step" in names and "avbd_layout" in names and len(names) >= 15


def test_library_exports_every_declared_symbol():
    from avbd_b200 import _lib
    L = _lib.load()
    for name in _declared():
        assert hasattr(L, name), name
        ctypes.cast(getattr(L, name), ctypes.c_void_p)


def test_layout_is_aligned_and_monotone():
    from avbd_b200 import _lib
    L = _lib.load()
    d = _lib.AvbdDims(n_bodies=1000, n_static_groups=8000, n_static_rows=24000, pair_cap=16000,
                      dyn_row_cap=192000, dyn_group_cap=192000, hash_cap=1 << 17, mlp_floats=0)
    n = L.avbd_num_arrays()
    offs = (ctypes.c_size_t * n)()
    tot = ctypes.c_size_t()
    assert L.avbd_layout(ctypes.byref(d), offs, ctypes.byref(tot)) == 0
    o = list(offs)
    assert all(v % 256 == 0 for v in o)
    assert all(b > a for a, b in zip(o, o[1:]))
    assert tot.value > o[-1]
    names = [L.avbd_array_name(i).decode() for i in range(n)]
    assert len(set(names)) == n and "BX" in names and "COUNTERS" in names


def test_layout_rejects_bad_dims():
    from avbd_b200 import _lib
    L = _lib.load()
    d = _lib.AvbdDims(n_bodies=10, hash_cap=1000)  # not a power of two
    n = L.avbd_num_arrays()
    offs = (ctypes.c_size_t * n)()
    tot = ctypes.c_size_t()
    assert L.avbd_layout(ctypes.byref(d), offs, ctypes.byref(tot)) < 0
    assert b"invalid" in L.avbd_last_error()


def test_product_refuses_to_run_without_cuda():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    from avbd_b200 import Solver6DOF
    with pytest.raises(RuntimeError):
        Solver6DOF()
