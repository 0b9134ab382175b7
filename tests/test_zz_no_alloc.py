"""The numeric entry point that allocates nothing (rvsp_cuda_numeric_noalloc).

It exists for callers that cannot call cudaMalloc when they need C's values
(allocators and memory pools that forbid re-entrant allocation, latency-bound
loops that must not take allocation locks).  Its scratch is a fixed device
array inside the library, so this test checks it through the C-ABI against
the regular device-memory descriptor path and the oracle on two calls in a
row (the second call reuses the array the first one left behind), with the
bit-exact bar of the other parity tests; then at the widest B it accepts
(one accumulator slot, so one block walks every row), with a C structure
that misses a column of the product, and with empty products.

This file is named to be collected last, and it sets up everything it needs,
so it passes in a fresh process or after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from rvsp import Descriptor, DeviceCSR, gen
from rvsp import _lib as L
from rvsp.csr import CSR

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
            ref = oracle.spgemm(hA.with_values(A.values.cpu().numpy()), hB)[2]
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), f"call {call}"


def _widest_b_case(seed):
    """A (300 x 40) times a sparse B of RVSP_NOALLOC_MAX_B_COLS columns."""
    rng = np.random.default_rng(seed)
    max_cols = (16 << 20) // 4
    brows = [np.sort(rng.choice(max_cols, 25, replace=False)) for _ in range(40)]
    brows[3] = np.array([0, max_cols - 1])  # both edges of the accumulator
    brp = np.zeros(41, np.int32)
    brp[1:] = np.cumsum([len(r) for r in brows])
    bci = np.concatenate(brows).astype(np.int32)
    B = CSR(40, max_cols, brp, bci, rng.uniform(-1, 1, bci.size).astype(np.float32))
    A = gen.random_csr(300, 40, seed + 1, mean_len=6.0)
    return A, B


def test_noalloc_widest_b_one_block_all_rows():
    # b_cols == RVSP_NOALLOC_MAX_B_COLS is accepted and leaves room for one
    # accumulator, so a single block computes all 300 rows in turn
    import torch
    lib = L.load()
    hA, hB = _widest_b_case(5)
    rp, ci, want, _ = oracle.spgemm(hA, hB)
    A, B = DeviceCSR.from_host(hA), DeviceCSR.from_host(hB)
    dC = DeviceCSR(hA.rows, hB.cols, torch.from_numpy(rp).cuda(), torch.from_numpy(ci).cuda(),
                   torch.zeros(max(ci.size, 1), dtype=torch.float32, device="cuda"))
    for call in range(2):
        out = torch.full((max(ci.size, 1),), float("nan"), dtype=torch.float32, device="cuda")
        assert _call(lib, A, B, dC, out) == L.SUCCESS
        torch.cuda.synchronize()
        got = out[:ci.size].cpu().numpy()
        assert np.array_equal(got.view(np.uint32), want.view(np.uint32)), f"call {call}"


def test_noalloc_structure_missing_a_column_spoils_only_that_entry():
    # C's structure for row 0 names a column the product does not touch in
    # place of one it does: that entry reads 0, the missing column's partial
    # sum must not leak into the later rows the same (single) block computes
    import torch
    lib = L.load()
    hA, hB = _widest_b_case(9)
    rp, ci, want, _ = oracle.spgemm(hA, hB)
    r0 = int(np.argmax(np.diff(rp) > 0))
    row = set(ci[rp[r0]:rp[r0 + 1]].tolist())
    spare = next(c for c in range(1, hB.cols) if c not in row)
    bad = ci.copy()
    seg = np.sort(np.concatenate([ci[rp[r0]:rp[r0 + 1] - 1], [spare]]))
    bad[rp[r0]:rp[r0 + 1]] = seg
    A, B = DeviceCSR.from_host(hA), DeviceCSR.from_host(hB)
    dC = DeviceCSR(hA.rows, hB.cols, torch.from_numpy(rp).cuda(), torch.from_numpy(bad).cuda(),
                   torch.zeros(max(ci.size, 1), dtype=torch.float32, device="cuda"))
    out = torch.full((max(ci.size, 1),), float("nan"), dtype=torch.float32, device="cuda")
    assert _call(lib, A, B, dC, out) == L.SUCCESS
    torch.cuda.synchronize()
    got = out[:ci.size].cpu().numpy()
    rest = slice(int(rp[r0 + 1]), ci.size)
    assert np.array_equal(got[rest].view(np.uint32), want[rest].view(np.uint32))
    assert np.array_equal(got[:rp[r0]].view(np.uint32), want[:rp[r0]].view(np.uint32))


def test_noalloc_empty_products_are_no_ops():
    import torch
    lib = L.load()
    hA = gen.random_csr(8, 8, 3, mean_len=2.0)
    A = DeviceCSR.from_host(hA)
    dC = DeviceCSR.empty(8, 8, 16)
    out = torch.full((16,), 7.0, dtype=torch.float32, device="cuda")
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    args = (A.row_ptr.data_ptr(), A.col_idx.data_ptr(), A.values.data_ptr(),
            A.row_ptr.data_ptr(), A.col_idx.data_ptr(), A.values.data_ptr(),
            dC.row_ptr.data_ptr(), dC.col_idx.data_ptr(), out.data_ptr())
    assert lib.rvsp_cuda_numeric_noalloc(stream, 0, 8, 8, *args) == L.SUCCESS
    assert lib.rvsp_cuda_numeric_noalloc(stream, 8, 8, 0, *args) == L.SUCCESS
    assert lib.rvsp_cuda_numeric_noalloc(stream, -1, 8, 8, *args) == L.ERROR_INVALID_ARGUMENT
    torch.cuda.synchronize()
    assert torch.all(out == 7.0)


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
