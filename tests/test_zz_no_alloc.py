"""avbd_exclusive_scan_noalloc: the prefix sum for callers that cannot
allocate device memory (a host application that owns the device-memory
budget, a real-time loop that must not stall on an allocation).

It is checked through the C ABI against the same scan computed by the
regular entry point: avbd_substep scans the per-body upper-neighbour counts
(UP_CNT) into the broadphase pair offsets (PAIR_START) with scratch from the
caller's arena.  Integer results, so the comparison is exact.  This file is
collected last so a failure here never hides the other tests.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _scan_noalloc(lib, src: torch.Tensor, out: torch.Tensor, stream) -> int:
    return lib.avbd_exclusive_scan_noalloc(ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                                           int(src.numel()), ctypes.c_void_p(stream.cuda_stream))


def test_noalloc_scan_matches_substep_scan_twice():
    from avbd_b200 import Solver6DOF, _lib, scenes
    lib = _lib.load()
    s = Solver6DOF(dt=1 / 60, iterations=4, substeps=1, coloring_mode="jones_plassmann")
    scenes.pile(s, nx=12, nz=12, ny=6, spacing=0.9, pin_every=0)
    n = len(s._x)
    for rnd in range(2):
        s.step()  # the regular path: PAIR_START = exclusive scan of UP_CNT (arena scratch)
        up = s._arena.view("UP_CNT", torch.int32, (n,))
        ref = s._arena.view("PAIR_START", torch.int32, (n + 1,)).cpu().numpy()
        assert ref[-1] > 0
        stream = s._cuda_stream
        for call in range(2):  # two calls in a row share the static scratch
            out = torch.full((n + 1,), -7, dtype=torch.int32, device=s.device)
            with torch.cuda.stream(stream):
                assert _scan_noalloc(lib, up, out, stream) == 0, lib.avbd_last_error()
            stream.synchronize()
            np.testing.assert_array_equal(out.cpu().numpy(), ref, err_msg=f"round {rnd} call {call}")


def test_noalloc_scan_rejects_oversized_input():
    from avbd_b200 import _lib
    lib = _lib.load()
    r = lib.avbd_exclusive_scan_noalloc(ctypes.c_void_p(1), ctypes.c_void_p(1), 8388608, None)
    assert r < 0 and b"8388607" in lib.avbd_last_error()


@pytest.mark.parametrize("n", [0, 1, 2048 * 300, 8388607])
def test_noalloc_scan_multi_block_sizes(n):
    """Sizes that reach the scan's carry between batches of 256 block
    partials (2048 x 300 ints: 301 partials) and the largest size the fixed
    scratch holds (8,388,607 ints: 4096 partials, the total in its last
    slot), checked against numpy twice in a row."""
    from avbd_b200 import _lib
    lib = _lib.load()
    rng = np.random.default_rng(n)
    vals = rng.integers(0, 200, size=max(n, 1), dtype=np.int32)[:n]  # total < 2^31
    src = torch.from_numpy(vals.copy()).cuda() if n else torch.zeros(1, dtype=torch.int32, device="cuda")
    want = np.zeros(n + 1, np.int64)
    want[1:] = np.cumsum(vals, dtype=np.int64)
    stream = torch.cuda.current_stream()
    for call in range(2):
        out = torch.full((n + 1,), -7, dtype=torch.int32, device="cuda")
        r = lib.avbd_exclusive_scan_noalloc(ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(out.data_ptr()), n,
                                            ctypes.c_void_p(stream.cuda_stream))
        assert r == 0, lib.avbd_last_error()
        torch.cuda.synchronize()
        np.testing.assert_array_equal(out.cpu().numpy().astype(np.int64), want, err_msg=f"n={n} call {call}")
