"""The allocation-free single-bit-flip entry point (pqi_single_bit_flips_noalloc).

It exists for callers that cannot allocate device memory (their device memory
belongs to another framework's allocator, or their loop must not call
cudaMalloc because it can synchronise the device). It keeps its scratch in a
fixed array inside libpqi instead of a caller workspace, so this test checks,
through the C ABI, that it returns what the allocating pqi_single_bit_flips
returns, on two calls in a row (the array keeps the previous call's contents),
and that it refuses n above its fixed maximum. This file is collected last so
that a failure here leaves every other test already run.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _call_both(dg, words, spin, G, L):
    from pyqrackising_b200 import _lib

    lib = _lib.load()
    out = []
    for name in ("pqi_single_bit_flips", "pqi_single_bit_flips_noalloc"):
        be = torch.empty(1, dtype=torch.float32, device=dg.device)
        bi = torch.empty(1, dtype=torch.int32, device=dg.device)
        args = [ctypes.byref(dg.w), ctypes.c_void_p(words.data_ptr()), spin, G, L,
                ctypes.c_void_p(be.data_ptr()), ctypes.c_void_p(bi.data_ptr())]
        if name == "pqi_single_bit_flips":
            wsp, wsn = dg.wsp(1)
            args += [wsp, wsn]
        args.append(dg.sp())
        assert getattr(lib, name)(*args) == _lib.PQI_OK, lib.pqi_last_error()
        out.append((float(be.item()), int(bi.item())))
    return out


@pytest.mark.parametrize("kind", ["pm1", "normal"])
def test_noalloc_matches_allocating_entry_point_twice(kind):
    from oracle import oracle as O
    from pyqrackising_b200 import workloads as wl
    from pyqrackising_b200.device import DeviceGraph

    n = 700
    W = wl.regular_pm1_fast(n, seed=11) if kind == "pm1" else wl.sherrington_kirkpatrick(n, seed=11)
    dg = DeviceGraph(W)
    rng = np.random.default_rng(3)
    G, L = O.flip_geometry(n, 148)
    for call in range(2):  # two calls in a row: the shared array holds the previous call's data
        th = rng.random(n) < 0.5
        words = dg.pack(th)
        ref, got = _call_both(dg, words, call % 2, G, L)
        assert got[1] == ref[1]
        assert got[0] == pytest.approx(ref[0], rel=1e-6, abs=1e-6)
        # and both agree with the oracle's selection
        oe, oi = O.single_select(W, O.pack32(th), call % 2, G, L)
        assert got[1] == oi


def test_noalloc_rejects_n_above_its_maximum():
    from pyqrackising_b200 import _lib

    lib = _lib.load()
    w = _lib.PqiWeights()
    w.n = _lib.PQI_NOALLOC_MAX_N + 1
    dummy = torch.zeros(16, dtype=torch.int32, device="cuda")
    p = ctypes.c_void_p(dummy.data_ptr())
    rc = lib.pqi_single_bit_flips_noalloc(ctypes.byref(w), p, 0, 32, 32, p, p, None)
    assert rc == _lib.PQI_EINVAL
    assert b"PQI_NOALLOC_MAX_N" in lib.pqi_last_error()
    torch.cuda.synchronize()
