"""The allocation-free exact float sum (rpba_float_sequential_sum_noalloc).

Callers that must not have the library call cudaMalloc/cudaFree -- an
application serving all device memory from its own fixed pool, or a loop
that cannot take cudaFree's device-wide synchronisation -- pass device
buffers they already own; the entry point's scratch is a static device array
of the library.  The test calls it twice in a row through the C ABI (the
shared scratch keeps the first call's contents) and compares each result
with the allocating entry point rpba_float_sequential_sum, bit for bit (the
tolerance the exact-sum tests use).  Device buffers here come from torch,
i.e. from the test, never from the entry point.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NA_MAX_N = 1024 * 4096


def _call(L, dv, n, dout):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    st = L.rpba_float_sequential_sum_noalloc(C.c_void_p(dv.data_ptr()), n, C.c_void_p(dout.data_ptr()),
                                             C.c_void_p(stream))
    torch.cuda.synchronize()
    return st


def test_noalloc_sum_matches_allocating_entry_point_twice():
    import torch
    import rpba_b200 as rb
    L = rb.load()
    rng = np.random.default_rng(123)
    inputs = [
        (rng.normal(0, 0.5, 3_000_001) ** 2 * 2).astype(np.float32),             # ~367 CTAs
        np.where(rng.random(NA_MAX_N) < 0.05, rng.uniform(0, 2500, NA_MAX_N),
                 rng.normal(0, 0.5, NA_MAX_N) ** 2).astype(np.float32),          # the maximum size
    ]
    for v in inputs:
        expect = rb.float_sequential_sum(v)
        dv = torch.from_numpy(v).cuda()
        dout = torch.full((1,), -1.0, dtype=torch.float32, device="cuda")
        assert _call(L, dv, v.size, dout) == 0
        got = np.float32(dout.cpu().numpy()[0])
        assert np.isfinite(got), got  # NaN would mean a failed call
        assert got.tobytes() == expect.tobytes(), (got, expect)


def test_noalloc_small_and_rejects_oversize():
    import torch
    import rpba_b200 as rb
    L = rb.load()
    v = np.arange(1, 5001, dtype=np.float32) * np.float32(0.1)
    dv = torch.from_numpy(v).cuda()
    dout = torch.zeros(1, dtype=torch.float32, device="cuda")
    assert _call(L, dv, v.size, dout) == 0
    assert np.float32(dout.cpu().numpy()[0]).tobytes() == rb.float_sequential_sum(v).tobytes()
    # beyond the fixed scratch: a clear status, nothing launched
    assert _call(L, dv, NA_MAX_N + 1, dout) == 11
    assert L.rpba_status_string(11).startswith(b"input exceeds the fixed scratch")
