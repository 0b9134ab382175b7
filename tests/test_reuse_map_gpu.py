"""The reuse map (rvsp_cuda_plan_prepare_reuse) through the C-ABI.

Numeric-only repeats of the warp-per-row classes read each product's
position in C's row from the map instead of hashing C's columns.  Bar: the
map covers exactly the products of those rows, and values computed through
it are bit-exact against the oracle, for new values, for a second C buffer
holding the same structure (the map is rebuilt for it), and when built
implicitly by the first numeric-only call.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from rvsp import DeviceCSR, gen
from rvsp import _lib as L

pytestmark = pytest.mark.gpu


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream or 1)


def _symbolic(lib, plan, dA, dB):
    import torch
    rp = torch.zeros(dA.rows + 1, dtype=torch.int32, device="cuda")
    total = C.c_int64()
    L.check(lib.rvsp_cuda_symbolic(plan, _stream(), dA.rows, dB.rows, dB.cols,
                                   dA.row_ptr.data_ptr(), dA.col_idx.data_ptr(),
                                   dB.row_ptr.data_ptr(), dB.col_idx.data_ptr(),
                                   rp.data_ptr(), C.byref(total)), "symbolic")
    return rp, total.value


def _numeric(lib, plan, dA, dB, rp, ci, cv, fill):
    ws_b = max(lib.rvsp_cuda_numeric_workspace_bytes(plan), 256)
    import torch
    ws = torch.zeros(ws_b, dtype=torch.uint8, device="cuda")
    L.check(lib.rvsp_cuda_numeric(plan, _stream(), dA.row_ptr.data_ptr(), dA.col_idx.data_ptr(),
                                  dA.values.data_ptr(), dB.row_ptr.data_ptr(),
                                  dB.col_idx.data_ptr(), dB.values.data_ptr(), rp.data_ptr(),
                                  ci.data_ptr(), cv.data_ptr(), fill, ws.data_ptr(), ws_b),
            "numeric")
    torch.cuda.synchronize()
    L.check(lib.rvsp_cuda_plan_status(plan, _stream()), "status")


def _mapped_ops(A, B, m_rows):
    """Products of the rows the warp classes take (output nnz 33..1024 and more
    than 16 A nonzeros or more than 2048 products, matching classify_row for a
    matrix below the merge-class row count)."""
    ops = oracle.spgemm(A, B)[3]
    return int(ops[(m_rows > 0) & (2 * m_rows <= 2048)].sum())


def test_reuse_map_explicit_and_rebuilt():
    import torch
    lib = L.load()
    A = gen.uniform_rows(3000, 4000, 12, 5)
    B = gen.random_csr(4000, 5000, 6, mean_len=20.0)
    dA, dB = DeviceCSR.from_host(A), DeviceCSR.from_host(B)
    plan = C.c_void_p()
    L.check(lib.rvsp_cuda_plan_create(C.byref(plan)), "plan_create")
    try:
        rp, n = _symbolic(lib, plan, dA, dB)
        ci = torch.zeros(n, dtype=torch.int32, device="cuda")
        cv = torch.zeros(n, dtype=torch.float32, device="cuda")
        _numeric(lib, plan, dA, dB, rp, ci, cv, 1)
        entries = C.c_int64()
        L.check(lib.rvsp_cuda_plan_prepare_reuse(plan, _stream(), dA.row_ptr.data_ptr(),
                                                 dA.col_idx.data_ptr(), dB.row_ptr.data_ptr(),
                                                 dB.col_idx.data_ptr(), rp.data_ptr(),
                                                 ci.data_ptr(), C.byref(entries)),
                "prepare_reuse")
        m_rows = np.diff(rp.cpu().numpy())
        assert entries.value == _mapped_ops(A, B, m_rows) > 0
        for k, scale in enumerate((-0.5, 1.75)):
            A2 = A.with_values((A.values * np.float32(scale)).astype(np.float32))
            dA.values.copy_(torch.from_numpy(A2.values))
            torch.cuda.synchronize()
            cv.zero_()
            _numeric(lib, plan, dA, dB, rp, ci, cv, 0)
            want = oracle.spgemm(A2, B)[2]
            assert np.array_equal(cv.cpu().numpy().view(np.uint32), want.view(np.uint32)), k
        # a second C buffer with the same structure: the map is rebuilt for it
        ci2, cv2 = ci.clone(), torch.zeros_like(cv)
        torch.cuda.synchronize()
        _numeric(lib, plan, dA, dB, rp, ci2, cv2, 0)
        assert np.array_equal(cv2.cpu().numpy().view(np.uint32), want.view(np.uint32))
    finally:
        lib.rvsp_cuda_plan_destroy(plan)


@pytest.mark.parametrize("a_len,b_len,b_cols", [(150, 20, 900), (40, 30, 700), (12, 3, 80)])
def test_reuse_map_stepping_and_tiles(a_len, b_len, b_cols):
    # long B rows step one A nonzero at a time; short ones (3 entries) take
    # flattened tiles with ordered accumulation; 150 x 20 products into 900
    # columns repeat every column many times
    import torch
    lib = L.load()
    A = gen.uniform_rows(1500, 2000, a_len, 7)
    B = gen.uniform_rows(2000, b_cols, b_len, 8)
    dA, dB = DeviceCSR.from_host(A), DeviceCSR.from_host(B)
    plan = C.c_void_p()
    L.check(lib.rvsp_cuda_plan_create(C.byref(plan)), "plan_create")
    try:
        rp, n = _symbolic(lib, plan, dA, dB)
        ci = torch.zeros(n, dtype=torch.int32, device="cuda")
        cv = torch.zeros(n, dtype=torch.float32, device="cuda")
        _numeric(lib, plan, dA, dB, rp, ci, cv, 1)
        for scale in (0.25, -3.0):
            A2 = A.with_values((A.values * np.float32(scale)).astype(np.float32))
            dA.values.copy_(torch.from_numpy(A2.values))
            torch.cuda.synchronize()
            cv.zero_()
            _numeric(lib, plan, dA, dB, rp, ci, cv, 0)
            want = oracle.spgemm(A2, B)[2]
            assert np.array_equal(cv.cpu().numpy().view(np.uint32), want.view(np.uint32))
    finally:
        lib.rvsp_cuda_plan_destroy(plan)


def test_reuse_map_implicit_on_stencil():
    import torch
    lib = L.load()
    A = gen.stencil_3d_27(20)
    dA = DeviceCSR.from_host(A)
    plan = C.c_void_p()
    L.check(lib.rvsp_cuda_plan_create(C.byref(plan)), "plan_create")
    # the reuse map itself: shift classes off (with them, the translated rows
    # never reach the map)
    L.check(lib.rvsp_cuda_plan_set_shift_classes(plan, 0), "set_shift_classes")
    try:
        rp, n = _symbolic(lib, plan, dA, dA)
        ci = torch.zeros(n, dtype=torch.int32, device="cuda")
        cv = torch.zeros(n, dtype=torch.float32, device="cuda")
        _numeric(lib, plan, dA, dA, rp, ci, cv, 1)
        rng = np.random.default_rng(3)
        for _ in range(2):  # the first numeric-only call builds the map
            vals = (A.values + rng.uniform(-0.01, 0.01, A.nnz)).astype(np.float32)
            dA.values.copy_(torch.from_numpy(vals))
            torch.cuda.synchronize()
            _numeric(lib, plan, dA, dA, rp, ci, cv, 0)
            A2 = A.with_values(vals)
            want = oracle.spgemm(A2, A2)[2]
            assert np.array_equal(cv.cpu().numpy().view(np.uint32), want.view(np.uint32))
        # interior rows (at distance >= 2 from every face) repeat one
        # position pattern: all but one of them read a shared map
        shared = C.c_int32()
        L.check(lib.rvsp_cuda_plan_reuse_shared_rows(plan, _stream(), C.byref(shared)),
                "reuse_shared_rows")
        assert shared.value >= (20 - 4) ** 3 - 1
    finally:
        lib.rvsp_cuda_plan_destroy(plan)


def test_reuse_map_shared_patterns_with_distinct_rows():
    # a few row patterns repeated many times, mixed with random rows: the
    # repeats share maps, every value stays bit-exact
    import torch
    from rvsp.csr import CSR
    lib = L.load()
    rng = np.random.default_rng(11)
    B = gen.uniform_rows(3000, 2500, 24, 12)
    pats = [np.sort(rng.choice(3000, 20, replace=False)) for _ in range(3)]
    rows = []
    for i in range(4000):
        rows.append(pats[i % 3] if i % 2 == 0 else np.sort(rng.choice(3000, 20, replace=False)))
    rp = np.zeros(len(rows) + 1, np.int32)
    rp[1:] = np.cumsum([len(r) for r in rows])
    ci = np.concatenate(rows).astype(np.int32)
    A = CSR(len(rows), 3000, rp, ci, rng.uniform(-1, 1, ci.size).astype(np.float32))
    dA, dB = DeviceCSR.from_host(A), DeviceCSR.from_host(B)
    plan = C.c_void_p()
    L.check(lib.rvsp_cuda_plan_create(C.byref(plan)), "plan_create")
    try:
        crp, n = _symbolic(lib, plan, dA, dB)
        cci = torch.zeros(n, dtype=torch.int32, device="cuda")
        cv = torch.zeros(n, dtype=torch.float32, device="cuda")
        _numeric(lib, plan, dA, dB, crp, cci, cv, 1)
        for scale in (0.5, -2.0):
            A2 = A.with_values((A.values * np.float32(scale)).astype(np.float32))
            dA.values.copy_(torch.from_numpy(A2.values))
            torch.cuda.synchronize()
            cv.zero_()
            _numeric(lib, plan, dA, dB, crp, cci, cv, 0)
            want = oracle.spgemm(A2, B)[2]
            assert np.array_equal(cv.cpu().numpy().view(np.uint32), want.view(np.uint32))
        shared = C.c_int32()
        L.check(lib.rvsp_cuda_plan_reuse_shared_rows(plan, _stream(), C.byref(shared)),
                "reuse_shared_rows")
        # 2000 rows repeat 3 patterns; the random rows share nothing
        assert shared.value == 2000 - 3
    finally:
        lib.rvsp_cuda_plan_destroy(plan)


def test_term_tables_need_equal_b_row_lengths():
    # rows of type 1 take B rows of 40 + 40 columns, rows of type 2 B rows of
    # 20 + 60 covering the same 80 columns: the same positions in the same
    # order (one shared map), but the table of the first type names B entries
    # that the second type's rows do not have; those rows must keep the map
    import torch
    from rvsp.csr import CSR
    lib = L.load()
    rng = np.random.default_rng(21)
    brows = [np.arange(0, 40), np.arange(40, 80), np.arange(0, 20), np.arange(20, 80)]
    brp = np.zeros(5, np.int32)
    brp[1:] = np.cumsum([len(r) for r in brows])
    bci = np.concatenate(brows).astype(np.int32)
    B = CSR(4, 80, brp, bci, rng.uniform(-1, 1, bci.size).astype(np.float32))
    arows = [[0, 1] if i % 2 == 0 else [2, 3] for i in range(64)]
    arp = np.zeros(65, np.int32)
    arp[1:] = np.cumsum([len(r) for r in arows])
    aci = np.concatenate(arows).astype(np.int32)
    A = CSR(64, 4, arp, aci, rng.uniform(-1, 1, aci.size).astype(np.float32))
    dA, dB = DeviceCSR.from_host(A), DeviceCSR.from_host(B)
    plan = C.c_void_p()
    L.check(lib.rvsp_cuda_plan_create(C.byref(plan)), "plan_create")
    try:
        crp, n = _symbolic(lib, plan, dA, dB)
        cci = torch.zeros(n, dtype=torch.int32, device="cuda")
        cv = torch.zeros(n, dtype=torch.float32, device="cuda")
        _numeric(lib, plan, dA, dB, crp, cci, cv, 1)
        for scale in (1.5, -0.25):
            A2 = A.with_values((A.values * np.float32(scale)).astype(np.float32))
            dA.values.copy_(torch.from_numpy(A2.values))
            torch.cuda.synchronize()
            cv.zero_()
            _numeric(lib, plan, dA, dB, crp, cci, cv, 0)
            want = oracle.spgemm(A2, B)[2]
            assert np.array_equal(cv.cpu().numpy().view(np.uint32), want.view(np.uint32))
        shared = C.c_int32()
        L.check(lib.rvsp_cuda_plan_reuse_shared_rows(plan, _stream(), C.byref(shared)),
                "reuse_shared_rows")
        assert shared.value == 63  # every row reads row 0's map
    finally:
        lib.rvsp_cuda_plan_destroy(plan)
