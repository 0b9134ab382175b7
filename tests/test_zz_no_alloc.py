"""The numeric entry point that allocates nothing (rvsp_cuda_numeric_noalloc).

It exists for callers that cannot call cudaMalloc when they need C's values
(graph capture, allocators that forbid re-entrant allocation, latency-bound
loops).  Its scratch is a fixed device array inside the library, so this
test checks it through the C-ABI against the regular device-memory
descriptor path on two calls in a row (the second call reuses the array the
first one left behind), with the bit-exact bar of the other parity tests.

This file is named to be collected last, and it sets up everything it needs,
so it passes in a fresh process or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from rvsp import Descriptor, DeviceCSR, gen
from rvsp import _lib as L

pytestmark = pytest.mark.gpu


def _call(lib, A, B, dC, out, b_cols=None):
    import torch
    stream = torch.cuda.current_stream().cuda_stream
    return lib.rvsp_cuda_numeric_noalloc(
        C.c_void_p(stream), A.rows, B.rows, B.cols if b_cols is None else b_cols,
        A.row_ptr.data_ptr(), A.col_idx.data_ptr(), A.values.data_ptr(),
        B.row_ptr.data_ptr(), B.col_idx.data_ptr(), B.values.data_ptr(),
        dC.row_ptr.data_ptr(), dC.col_idx.data_ptr(), out.data_ptr())


def test_noalloc_matches_descriptor_on_two_calls():
    import torch
    lib = L.load()
    hA = gen.random_csr(1500, 1200, 71, mean_len=9.0, heavy_rows=3, heavy_len=900)
    hB = gen.random_csr(1200, 5000, 72, mean_len=12.0, heavy_rows=3, heavy_len=3000)
    A, B = DeviceCSR.from_host(hA), DeviceCSR.from_host(hB)
    with Descriptor(memory=L.MEM_DEVICE) as d:
        ws_bytes, n = d.work_estimation(A, B)
        dC = DeviceCSR.empty(hA.rows, hB.cols, n)
        ws = torch.zeros(ws_bytes, dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        for call, scale in enumerate((1.0, -1.25)):
            A.values.mul_(scale)
            torch.cuda.synchronize()
            d.compute(A, B, dC, ws)
            d.synchronize()
            want = dC.values[:n].clone()
            out = torch.full((max(n, 1),), float("nan"), dtype=torch.float32, device="cuda")
            assert _call(lib, A, B, dC, out) == L.SUCCESS, f"call {call}"
            torch.cuda.synchronize()
            got = out[:n].cpu().numpy()
            assert np.array_equal(got.view(np.uint32), want.cpu().numpy().view(np.uint32)), \
                f"call {call}"


def test_noalloc_rejects_oversized_b():
    import torch
    lib = L.load()
    hA = gen.random_csr(8, 8, 3, mean_len=2.0)
    A = DeviceCSR.from_host(hA)
    dC = DeviceCSR.empty(8, 8, 16)
    out = torch.zeros(16, dtype=torch.float32, device="cuda")
    too_wide = (16 << 20) // 4 + 1
    assert _call(lib, A, A, dC, out, b_cols=too_wide) == L.ERROR_INVALID_ARGUMENT
    assert lib.rvsp_cuda_numeric_noalloc(None, 8, 8, 8, None, None, None, None, None,
                                         None, None, None, None) == L.ERROR_NULL_POINTER
