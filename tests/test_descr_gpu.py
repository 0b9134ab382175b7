"""Descriptor contracts on the GPU, after tests/test_spgemm_descr_f32.c of the
reference (lifecycle, argument checks at compute, exact nnz and op counts,
the structure-reuse contract, invalidate), plus the device memory space,
caller streams, profiling and the device one-shot."""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from rvsp import CSR, Descriptor, DeviceCSR, gen
from rvsp import _lib as L

pytestmark = pytest.mark.gpu


def test_reference_descriptor_sequence(golden_fixtures):
    lib = L.load()
    _, A, B, Cx = golden_fixtures[0]
    A = A.copy()  # values are mutated below
    a, b = A.struct(), B.struct()
    d = C.c_void_p()
    assert lib.rvsp_spgemm_descr_create(C.byref(d)) == L.SUCCESS
    assert lib.rvsp_spgemm_set_algo(d, L.ALGO_DEFAULT) == L.SUCCESS
    ws_bytes, c_nnz = C.c_size_t(), C.c_int32()
    assert lib.rvsp_spgemm_work_estimation(d, C.byref(a), C.byref(b), C.byref(ws_bytes),
                                           C.byref(c_nnz)) == L.SUCCESS
    assert c_nnz.value == Cx.nnz and ws_bytes.value > 0
    assert lib.rvsp_spgemm_set_algo(d, L.ALGO_DEFAULT) == L.ERROR_INVALID_ARGUMENT
    ops = np.zeros(2, np.int64)
    assert lib.rvsp_spgemm_get_op_counts(d, ops.ctypes.data, 2) == L.SUCCESS
    assert ops.tolist() == [2, 1]
    assert lib.rvsp_spgemm_get_op_counts(d, ops.ctypes.data, 1) == L.ERROR_INVALID_ARGUMENT

    n = c_nnz.value
    rp, ci, cv = np.zeros(A.rows + 1, np.int32), np.zeros(n, np.int32), np.zeros(n, np.float32)
    ws = np.zeros(ws_bytes.value, np.uint8)
    Cm = L.CsrMatrix(A.rows, B.cols, n, rp.ctypes.data, ci.ctypes.data, cv.ctypes.data,
                     L.DTYPE_FP32, L.FORMAT_CSR, 0)
    assert lib.rvsp_spgemm_compute(d, C.byref(a), C.byref(b), C.byref(Cm), None) == L.ERROR_NULL_POINTER
    assert lib.rvsp_spgemm_compute(d, C.byref(a), C.byref(b), None, ws.ctypes.data) == L.ERROR_NULL_POINTER
    small = L.CsrMatrix.from_buffer_copy(Cm)
    small.nnz = n - 1
    assert lib.rvsp_spgemm_compute(d, C.byref(a), C.byref(b), C.byref(small),
                                   ws.ctypes.data) == L.ERROR_INVALID_ARGUMENT
    wrong = L.CsrMatrix.from_buffer_copy(Cm)
    wrong.rows += 1
    assert lib.rvsp_spgemm_compute(d, C.byref(a), C.byref(b), C.byref(wrong),
                                   ws.ctypes.data) == L.ERROR_INVALID_ARGUMENT
    bad_a = L.CsrMatrix.from_buffer_copy(a)
    bad_a.nnz -= 1
    assert lib.rvsp_spgemm_compute(d, C.byref(bad_a), C.byref(b), C.byref(Cm),
                                   ws.ctypes.data) == L.ERROR_INVALID_ARGUMENT

    assert lib.rvsp_spgemm_compute(d, C.byref(a), C.byref(b), C.byref(Cm),
                                   ws.ctypes.data) == L.SUCCESS
    assert Cm.nnz == Cx.nnz
    assert np.array_equal(ci, Cx.col_idx) and np.array_equal(cv, Cx.values)
    # reuse: double A's values, same descriptor and same C, no re-analysis
    A.values *= 2.0
    ci[:] = -7  # a reused structure is not rewritten
    assert lib.rvsp_spgemm_compute(d, C.byref(a), C.byref(b), C.byref(Cm),
                                   ws.ctypes.data) == L.SUCCESS
    assert np.array_equal(cv, 2.0 * Cx.values)
    assert np.all(ci == -7)
    lib.rvsp_spgemm_invalidate_structure(d)
    assert lib.rvsp_spgemm_compute(d, C.byref(a), C.byref(b), C.byref(Cm),
                                   ws.ctypes.data) == L.SUCCESS
    assert np.array_equal(ci, Cx.col_idx)
    lib.rvsp_spgemm_descr_destroy(d)


def reuse_case(seed=5):
    A = gen.random_csr(900, 700, seed, mean_len=12.0, heavy_rows=2, heavy_len=500)
    B = gen.random_csr(700, 800, seed + 1, mean_len=10.0, heavy_rows=2, heavy_len=600)
    return A, B


def test_numeric_only_reuse_host():
    A, B = reuse_case()
    rng = np.random.default_rng(0)
    with Descriptor() as d:
        d.work_estimation(A, B)
        first = d.multiply(A, B)
        rp, ci, _, _ = oracle.spgemm(A, B)
        assert np.array_equal(first.col_idx, ci)
        n = d.c_nnz
        Cm = CSR(A.rows, B.cols, np.zeros(A.rows + 1, np.int32), np.zeros(n, np.int32),
                 np.zeros(n, np.float32))
        ws = np.zeros(d.ws_bytes, np.uint8)
        for it in range(4):
            A2 = A.with_values((A.values + rng.uniform(-0.01, 0.01, A.nnz)).astype(np.float32))
            B2 = B.with_values((B.values * (1 + it)).astype(np.float32))
            d.compute(A2, B2, Cm, ws)
            want = oracle.numeric_f32(A2, B2, rp, ci)
            assert np.array_equal(Cm.col_idx, ci)
            assert np.array_equal(Cm.values.view(np.uint32), want.view(np.uint32))


def test_device_memory_space_and_stream():
    import torch
    A, B = reuse_case(9)
    rp, ci, cv, ops = oracle.spgemm(A, B)
    dA, dB = DeviceCSR.from_host(A), DeviceCSR.from_host(B)
    stream = torch.cuda.Stream()
    with Descriptor(memory=L.MEM_DEVICE, stream=stream, profiling=True) as d:
        ws_bytes, n = d.work_estimation(dA, dB)
        assert n == ci.size
        dC = DeviceCSR.empty(A.rows, B.cols, n)
        ws = torch.zeros(max(ws_bytes, 1), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        d.compute(dA, dB, dC, ws)
        d.synchronize()
        got = dC.to_host(n)
        assert np.array_equal(got.row_ptr, rp) and np.array_equal(got.col_idx, ci)
        assert np.array_equal(got.values.view(np.uint32), cv.view(np.uint32))
        # numeric-only repeats in device memory, values updated on the same stream
        for it in range(3):
            with torch.cuda.stream(stream):
                dA.values.mul_(1.5)
            d.compute(dA, dB, dC, ws)
        d.synchronize()
        A3 = A.with_values(dA.values.cpu().numpy())
        want = oracle.numeric_f32(A3, B, rp, ci)
        assert np.array_equal(dC.values[:n].cpu().numpy().view(np.uint32), want.view(np.uint32))
        times = d.phase_times()
        assert times["symbolic"][0] > 0 and times["numeric"][1] >= 4
        assert np.array_equal(d.get_op_counts(A.rows), ops)


def test_device_oneshot():
    import torch
    A, B = reuse_case(13)
    rp, ci, cv, _ = oracle.spgemm(A, B)
    lib = L.load()
    dA, dB = DeviceCSR.from_host(A), DeviceCSR.from_host(B)
    a, b = dA.struct(), dB.struct()
    c = L.CsrMatrix()
    assert lib.rvsp_spgemm_csr_device(C.byref(a), C.byref(b), C.byref(c), None) == L.SUCCESS
    assert c.owns_data == 2 and c.nnz == ci.size
    n = c.nnz
    h_rp = np.zeros(A.rows + 1, np.int32)
    h_ci = np.zeros(n, np.int32)
    h_cv = np.zeros(n, np.float32)
    torch.cuda.synchronize()
    for dst, src in ((h_rp, c.row_ptr), (h_ci, c.col_idx), (h_cv, c.values)):
        _copy_device_to_host(dst, src, dst.nbytes)
    assert np.array_equal(h_rp, rp) and np.array_equal(h_ci, ci)
    assert np.array_equal(h_cv.view(np.uint32), cv.view(np.uint32))
    lib.rvsp_csr_destroy(C.byref(c))
    assert c.owns_data == 0 and not c.values


def _copy_device_to_host(dst: np.ndarray, src_ptr: int, nbytes: int):
    import cuda.bindings.runtime as rt  # cuda-python
    err, = rt.cudaMemcpy(dst.ctypes.data, src_ptr, nbytes,
                         rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
    assert int(err) == 0


def test_device_chain_keeps_c_on_device():
    # (A B) C with the intermediate product never leaving the device: the
    # first result (owns_data = 2) is the left operand of the second call
    lib = L.load()
    A = gen.uniform_rows(1500, 1200, 9, 31)
    B = gen.uniform_rows(1200, 1300, 7, 32)
    Cm = gen.uniform_rows(1300, 900, 5, 33)
    rp1, ci1, cv1, _ = oracle.spgemm(A, B)
    AB = CSR(A.rows, B.cols, rp1, ci1, cv1)
    rp2, ci2, cv2, _ = oracle.spgemm(AB, Cm)
    dA, dB, dC = DeviceCSR.from_host(A), DeviceCSR.from_host(B), DeviceCSR.from_host(Cm)
    a, b, c3 = dA.struct(), dB.struct(), dC.struct()
    ab = L.CsrMatrix()
    assert lib.rvsp_spgemm_csr_device(C.byref(a), C.byref(b), C.byref(ab), None) == L.SUCCESS
    abc = L.CsrMatrix()
    assert lib.rvsp_spgemm_csr_device(C.byref(ab), C.byref(c3), C.byref(abc), None) == L.SUCCESS
    h_rp = np.zeros(A.rows + 1, np.int32)
    h_ci = np.zeros(abc.nnz, np.int32)
    h_cv = np.zeros(abc.nnz, np.float32)
    for dst, src in ((h_rp, abc.row_ptr), (h_ci, abc.col_idx), (h_cv, abc.values)):
        _copy_device_to_host(dst, src, dst.nbytes)
    assert np.array_equal(h_rp, rp2) and np.array_equal(h_ci, ci2)
    assert np.array_equal(h_cv.view(np.uint32), cv2.view(np.uint32))
    lib.rvsp_csr_destroy(C.byref(ab))
    lib.rvsp_csr_destroy(C.byref(abc))
