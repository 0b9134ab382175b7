"""The C-ABI library loads, exports every function include/*.h declares, and
honours the host-side contracts of the reference API that need no GPU
(argument checks that return before any device work)."""
import ctypes as C
import re
from pathlib import Path

import numpy as np
import pytest

import rvsp
from rvsp import _lib as L

ROOT = Path(__file__).resolve().parents[1]


def declared_functions():
    names = set()
    for h in sorted((ROOT / "include").glob("*.h")):
        text = h.read_text()
        text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)
        text = re.sub(r"//[^\n]*", " ", text)
        for m in re.finditer(r"\b(rvsp_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_reference_api():
    names = set(declared_functions())
    reference_api = {  # include/rv_sparse.h:27-143 of merledu/rv-sparse
        "rvsp_get_version", "rvsp_status_to_string", "rvsp_csr_create",
        "rvsp_csr_validate", "rvsp_csr_destroy", "rvsp_spgemm_csr",
        "rvsp_spgemm_descr_create", "rvsp_spgemm_descr_destroy",
        "rvsp_spgemm_set_algo", "rvsp_spgemm_work_estimation",
        "rvsp_spgemm_compute", "rvsp_spgemm_get_op_counts",
        "rvsp_spgemm_invalidate_structure"}
    assert reference_api <= names


def test_library_exports_every_declared_symbol():
    lib = L.load()
    missing = [n for n in declared_functions() if not hasattr(lib, n)]
    assert not missing, missing


def test_bindings_cover_headers():
    assert set(declared_functions()) == set(L.SIGNATURES)


def test_version_and_strings():
    lib = L.load()
    assert lib.rvsp_get_version() == b"0.1.0"
    expect = {0: b"success", -1: b"null pointer", -2: b"invalid argument",
              -3: b"invalid CSR matrix", -4: b"unsupported data type",
              -5: b"unsupported backend", -6: b"allocation failed",
              -7: b"device error", -99: b"unknown error"}
    for code, s in expect.items():
        assert lib.rvsp_status_to_string(code) == s
    assert lib.rvsp_csr_status_string(0) == b"canonical CSR"
    assert lib.rvsp_csr_status_string(4) == b"duplicate column in row"


def _arr(x, dt):
    return np.ascontiguousarray(np.array(x, dt))


def test_csr_create_and_validate():
    lib = L.load()
    rp, ci, v = _arr([0, 2, 3], np.int32), _arr([0, 1, 1], np.int32), _arr([1, 2, 3], np.float32)
    m = L.CsrMatrix()
    assert lib.rvsp_csr_create(C.byref(m), 2, 2, 3, rp.ctypes.data, ci.ctypes.data,
                               v.ctypes.data, L.DTYPE_FP32) == L.SUCCESS
    assert m.owns_data == 0 and m.nnz == 3
    assert lib.rvsp_csr_create(None, 2, 2, 3, rp.ctypes.data, ci.ctypes.data,
                               v.ctypes.data, L.DTYPE_FP32) == L.ERROR_NULL_POINTER
    assert lib.rvsp_csr_create(C.byref(m), 0, 2, 3, rp.ctypes.data, ci.ctypes.data,
                               v.ctypes.data, L.DTYPE_FP32) == L.ERROR_INVALID_ARGUMENT
    bad = _arr([0, 2, 4], np.int32)  # row_ptr[rows] != nnz
    assert lib.rvsp_csr_create(C.byref(m), 2, 2, 3, bad.ctypes.data, ci.ctypes.data,
                               v.ctypes.data, L.DTYPE_FP32) == L.ERROR_INVALID_CSR
    oor = _arr([0, 1, 5], np.int32)
    assert lib.rvsp_csr_create(C.byref(m), 2, 2, 3, rp.ctypes.data, oor.ctypes.data,
                               v.ctypes.data, L.DTYPE_FP32) == L.ERROR_INVALID_CSR
    # destroy does not free caller arrays, and resets the struct
    lib.rvsp_csr_create(C.byref(m), 2, 2, 3, rp.ctypes.data, ci.ctypes.data,
                        v.ctypes.data, L.DTYPE_FP32)
    lib.rvsp_csr_destroy(C.byref(m))
    assert m.rows == 0 and not m.row_ptr
    lib.rvsp_csr_destroy(None)


def test_csr_check_matches_oracle():
    from oracle import oracle
    lib = L.load()
    cases = [
        (3, 4, [0, 1, 3, 3], [2, 0, 3]),
        (3, 4, [1, 1, 3, 3], [2, 0, 3]),
        (3, 4, [0, 2, 1, 3], [2, 3, 0]),
        (3, 4, [0, 1, 3, 3], [2, 0, 4]),
        (3, 4, [0, 1, 3, 3], [2, 3, 0]),
        (3, 4, [0, 1, 3, 3], [2, 1, 1]),
        (2, 0, [0, 0, 1], [0]),
    ]
    for rows, cols, rp, ci in cases:
        rp, ci = _arr(rp, np.int32), _arr(ci, np.int32)
        bad = C.c_int32()
        code = lib.rvsp_csr_check(rows, cols, rp.ctypes.data, ci.ctypes.data, C.byref(bad))
        assert (code, bad.value) == oracle.csr_check(rows, cols, rp, ci)
    bad = C.c_int32()
    assert lib.rvsp_csr_check(2, 2, None, None, C.byref(bad)) == L.CSR_BAD_ROW_PTR


def test_buffer_size():
    lib = L.load()
    n = C.c_size_t()
    assert lib.rvsp_spgemm_buffer_size(16, C.byref(n)) == L.SUCCESS and n.value > 0
    assert lib.rvsp_spgemm_buffer_size(0, C.byref(n)) == L.ERROR_INVALID_ARGUMENT
    assert lib.rvsp_spgemm_buffer_size(16, None) == L.ERROR_NULL_POINTER


def test_descriptor_contracts_without_device(golden_fixtures):
    """test_spgemm_descr_f32.c:63-103 of the reference: lifecycle, NULL
    handling and ordering rules, all decided before any device work."""
    lib = L.load()
    d = C.c_void_p()
    assert lib.rvsp_spgemm_descr_create(C.byref(d)) == L.SUCCESS and d
    assert lib.rvsp_spgemm_descr_create(None) == L.ERROR_NULL_POINTER
    assert lib.rvsp_spgemm_set_algo(d, L.ALGO_DEFAULT) == L.SUCCESS
    assert lib.rvsp_spgemm_set_algo(d, L.ALGO_CUDA_PLAIN) == L.SUCCESS
    assert lib.rvsp_spgemm_set_algo(None, L.ALGO_DEFAULT) == L.ERROR_NULL_POINTER
    for algo in (L.ALGO_RVV, L.ALGO_CONTIG, L.ALGO_ADAPTIVE, 99):
        assert lib.rvsp_spgemm_set_algo(d, algo) == L.ERROR_UNSUPPORTED_BACKEND
    _, A, B, _ = golden_fixtures[0]
    a, b = A.struct(), B.struct()
    rp = np.zeros(3, np.int32)
    ci = np.zeros(3, np.int32)
    v = np.zeros(3, np.float32)
    Cm = L.CsrMatrix(2, 2, 3, rp.ctypes.data, ci.ctypes.data, v.ctypes.data,
                     L.DTYPE_FP32, L.FORMAT_CSR, 0)
    ws = np.zeros(4096, np.uint8)
    assert lib.rvsp_spgemm_compute(d, C.byref(a), C.byref(b), C.byref(Cm),
                                   ws.ctypes.data) == L.ERROR_INVALID_ARGUMENT
    ops = np.zeros(2, np.int64)
    assert lib.rvsp_spgemm_get_op_counts(d, ops.ctypes.data, 2) == L.ERROR_INVALID_ARGUMENT
    wsb, nnz = C.c_size_t(), C.c_int32()
    assert lib.rvsp_spgemm_work_estimation(d, None, C.byref(b), C.byref(wsb),
                                           C.byref(nnz)) == L.ERROR_NULL_POINTER
    assert lib.rvsp_spgemm_work_estimation(None, C.byref(a), C.byref(b), C.byref(wsb),
                                           C.byref(nnz)) == L.ERROR_NULL_POINTER
    wrong = L.CsrMatrix.from_buffer_copy(b)
    wrong.dtype = L.DTYPE_FP64
    assert lib.rvsp_spgemm_work_estimation(d, C.byref(a), C.byref(wrong), C.byref(wsb),
                                           C.byref(nnz)) == L.ERROR_UNSUPPORTED_DTYPE
    mism = L.CsrMatrix.from_buffer_copy(b)
    mism.rows = 3
    assert lib.rvsp_spgemm_work_estimation(d, C.byref(a), C.byref(mism), C.byref(wsb),
                                           C.byref(nnz)) == L.ERROR_INVALID_ARGUMENT
    assert lib.rvsp_spgemm_set_memory_space(d, 5) == L.ERROR_INVALID_ARGUMENT
    assert lib.rvsp_spgemm_set_memory_space(d, L.MEM_DEVICE) == L.SUCCESS
    assert lib.rvsp_spgemm_compute(None, C.byref(a), C.byref(b), C.byref(Cm),
                                   ws.ctypes.data) == L.ERROR_NULL_POINTER
    lib.rvsp_spgemm_invalidate_structure(None)
    lib.rvsp_spgemm_descr_destroy(None)
    lib.rvsp_spgemm_descr_destroy(d)


def test_oneshot_argument_errors(golden_fixtures):
    """spgemm.c:135-210 and :26-51 of the reference: the errors decided before
    any device work, in the reference's order."""
    lib = L.load()
    _, A, B, _ = golden_fixtures[0]
    a, b = A.struct(), B.struct()
    c = L.CsrMatrix()
    cuda = L.SpgemmOptions(L.BACKEND_CUDA, L.DTYPE_FP32, L.DTYPE_FP32)
    assert lib.rvsp_spgemm_csr(None, C.byref(b), C.byref(c), C.byref(cuda)) == L.ERROR_NULL_POINTER
    for backend in (L.BACKEND_SCALAR, L.BACKEND_SCALAR_UNROLL4, L.BACKEND_RVV_INTRINSICS):
        o = L.SpgemmOptions(backend, L.DTYPE_FP32, L.DTYPE_FP32)
        assert lib.rvsp_spgemm_csr(C.byref(a), C.byref(b), C.byref(c),
                                   C.byref(o)) == L.ERROR_UNSUPPORTED_BACKEND
    # FP64 options reach the FP64 product, whose wrapper refuses FP32 operands
    # with INVALID_ARGUMENT (csr_spgemm_wrappers.c:362-365); INT8 options
    # refuse them with UNSUPPORTED_DTYPE (:43-46); other dtype pairs have no
    # kernel
    o = L.SpgemmOptions(L.BACKEND_CUDA, L.DTYPE_FP64, L.DTYPE_FP64)
    assert lib.rvsp_spgemm_csr(C.byref(a), C.byref(b), C.byref(c),
                               C.byref(o)) == L.ERROR_INVALID_ARGUMENT
    o = L.SpgemmOptions(L.BACKEND_CUDA, L.DTYPE_INT8, L.DTYPE_INT32)
    assert lib.rvsp_spgemm_csr(C.byref(a), C.byref(b), C.byref(c),
                               C.byref(o)) == L.ERROR_UNSUPPORTED_DTYPE
    o = L.SpgemmOptions(L.BACKEND_CUDA, L.DTYPE_FP32, L.DTYPE_FP64)
    assert lib.rvsp_spgemm_csr(C.byref(a), C.byref(b), C.byref(c),
                               C.byref(o)) == L.ERROR_UNSUPPORTED_BACKEND
    f64 = L.CsrMatrix.from_buffer_copy(a)
    f64.dtype = L.DTYPE_FP64
    assert lib.rvsp_spgemm_csr(C.byref(f64), C.byref(b), C.byref(c),
                               C.byref(cuda)) == L.ERROR_UNSUPPORTED_DTYPE
    mism = L.CsrMatrix.from_buffer_copy(b)
    mism.rows = 5
    assert lib.rvsp_spgemm_csr(C.byref(a), C.byref(mism), C.byref(c),
                               C.byref(cuda)) == L.ERROR_INVALID_ARGUMENT
    # row_ptr[0] != 0 is caught on the host, before any upload
    rp_bad = np.array([1, 2, 3], np.int32)
    badm = L.CsrMatrix.from_buffer_copy(a)
    badm.row_ptr = rp_bad.ctypes.data
    assert lib.rvsp_spgemm_csr(C.byref(badm), C.byref(b), C.byref(c),
                               C.byref(cuda)) == L.ERROR_INVALID_CSR
    assert not c.row_ptr and c.nnz == 0 and c.owns_data == 0


def test_checked_symbolic_argument_errors():
    # Argument checks of rvsp_cuda_symbolic_checked come before any use of the
    # plan or the arrays, so stand-in non-null pointers never get read here.
    lib = L.load()
    p = C.c_void_p(16)  # never dereferenced: every call below fails its checks
    arr = C.c_void_p(64)
    total = C.c_int64(0)

    def call(a_rows, a_cols, a_nnz, b_rows, b_cols, b_nnz, plan=p, c_rp=arr):
        return lib.rvsp_cuda_symbolic_checked(plan, None, a_rows, a_cols, a_nnz, b_rows,
                                              b_cols, b_nnz, arr, arr, arr, arr, 1, c_rp,
                                              C.byref(total))
    assert call(4, 3, 5, 3, 2, 4, plan=None) == L.ERROR_NULL_POINTER
    assert call(4, 3, 5, 3, 2, 4, c_rp=None) == L.ERROR_NULL_POINTER
    assert call(0, 3, 5, 3, 2, 4) == L.ERROR_INVALID_ARGUMENT
    assert call(4, 3, -1, 3, 2, 4) == L.ERROR_INVALID_ARGUMENT
    # A's columns must be B's rows: more would index B's row pointers past
    # their end once the check has passed
    assert call(4, 5, 5, 3, 2, 4) == L.ERROR_INVALID_ARGUMENT
    assert call(4, 2, 5, 3, 2, 4) == L.ERROR_INVALID_ARGUMENT
