"""ctypes binding of librvsparse_cuda.so (include/rv_sparse.h, include/rvsp_cuda.h).

The library is the product: every call here goes straight to the C-ABI.  If
the shared library has not been built, loading fails loudly; there is no
fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

PKG_ROOT = Path(__file__).resolve().parent.parent
LIB_PATH = PKG_ROOT / "lib" / "librvsparse_cuda.so"

# ---- enums (include/rv_sparse_types.h) -------------------------------------
SUCCESS = 0
ERROR_NULL_POINTER = -1
ERROR_INVALID_ARGUMENT = -2
ERROR_INVALID_CSR = -3
ERROR_UNSUPPORTED_DTYPE = -4
ERROR_UNSUPPORTED_BACKEND = -5
ERROR_ALLOCATION_FAILED = -6
ERROR_DEVICE = -7

DTYPE_INT8, DTYPE_INT32, DTYPE_BF16, DTYPE_FP32, DTYPE_FP64 = range(5)
FORMAT_CSR = 0
BACKEND_SCALAR, BACKEND_SCALAR_UNROLL4, BACKEND_RVV_INTRINSICS, BACKEND_CUDA = range(4)

ALGO_DEFAULT = 0
ALGO_RVV = 1
ALGO_CONTIG = 2
ALGO_ADAPTIVE = 3
ALGO_CUDA_PLAIN = 16
ALGO_CUDA_LEARNED = 17

MEM_HOST = 0
MEM_DEVICE = 1

PHASES = ("rowstats", "symbolic", "scan", "numeric", "predict", "fused",
          "compact", "copy", "check")
CLASS_NAMES = ("empty", "m4", "m8", "m16", "w64", "w128", "w256", "w512",
               "w1024", "w2048", "b8192", "dense")

CSR_OK, CSR_BAD_ROW_PTR, CSR_COL_OUT_OF_RANGE, CSR_UNSORTED, CSR_DUPLICATE = range(5)


class CsrMatrix(C.Structure):
    """rvsp_csr_matrix_t, field for field."""

    _fields_ = [
        ("rows", C.c_int32),
        ("cols", C.c_int32),
        ("nnz", C.c_int32),
        ("row_ptr", C.c_void_p),
        ("col_idx", C.c_void_p),
        ("values", C.c_void_p),
        ("dtype", C.c_int),
        ("format", C.c_int),
        ("owns_data", C.c_int),
    ]


class SpgemmOptions(C.Structure):
    _fields_ = [("backend", C.c_int), ("input_dtype", C.c_int),
                ("output_dtype", C.c_int)]


_P = C.POINTER
_i32, _i64, _sz, _vp, _int = C.c_int32, C.c_int64, C.c_size_t, C.c_void_p, C.c_int

# name -> (restype, argtypes); every function declared in include/*.h
SIGNATURES = {
    # rv_sparse.h
    "rvsp_get_version": (C.c_char_p, []),
    "rvsp_status_to_string": (C.c_char_p, [_int]),
    "rvsp_csr_create": (_int, [_P(CsrMatrix), _i32, _i32, _i32, _vp, _vp, _vp, _int]),
    "rvsp_csr_validate": (_int, [_P(CsrMatrix)]),
    "rvsp_csr_destroy": (None, [_P(CsrMatrix)]),
    "rvsp_spgemm_csr": (_int, [_P(CsrMatrix), _P(CsrMatrix), _P(CsrMatrix),
                               _P(SpgemmOptions)]),
    "rvsp_spgemm_descr_create": (_int, [_P(_vp)]),
    "rvsp_spgemm_descr_destroy": (None, [_vp]),
    "rvsp_spgemm_set_algo": (_int, [_vp, _int]),
    "rvsp_spgemm_work_estimation": (_int, [_vp, _P(CsrMatrix), _P(CsrMatrix),
                                           _P(_sz), _P(_i32)]),
    "rvsp_spgemm_compute": (_int, [_vp, _P(CsrMatrix), _P(CsrMatrix),
                                   _P(CsrMatrix), _vp]),
    "rvsp_spgemm_get_op_counts": (_int, [_vp, _vp, _i32]),
    "rvsp_spgemm_invalidate_structure": (None, [_vp]),
    "rvsp_csr_check": (_int, [_i32, _i32, _vp, _vp, _P(_i32)]),
    "rvsp_csr_read_mtx": (_int, [C.c_char_p, _int, _P(CsrMatrix)]),
    "rvsp_csr_parse_mtx": (_int, [C.c_char_p, C.c_size_t, _int, _P(CsrMatrix)]),
    "rvsp_csr_copy_arrays": (_int, [_P(CsrMatrix), _P(CsrMatrix)]),
    "rvsp_debug_fail_host_alloc": (None, [_i32]),
    "rvsp_debug_host_allocs": (_i64, []),
    "rvsp_cuda_coo_to_csr": (_int, [_vp, _i32, _i32, _i64, _int, _vp, _vp, _vp, _vp,
                                    _P(_vp), _P(_vp), _P(_i32)]),
    "rvsp_cuda_symbolic_checked": (_int, [_vp, _vp, _i32, _i32, _i32, _i32, _i32, _i32, _vp,
                                          _vp, _vp, _vp, _int, _vp, _P(_i64)]),
    "rvsp_cuda_typed_numeric": (_int, [_vp, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                       _vp, _vp]),
    "rvsp_cuda_drop_zeros": (_int, [_vp, _i32, _i32, _vp, _i64, _vp, _vp, _vp, _sz, _vp,
                                    _vp, _vp, _P(_i32)]),
    "rvsp_cuda_drop_zeros_scratch_bytes": (_sz, [_i64]),
    "rvsp_csr_status_string": (C.c_char_p, [_int]),
    "rvsp_spgemm_buffer_size": (_int, [_i32, _P(_sz)]),
    "rvsp_spgemm_set_memory_space": (_int, [_vp, _int]),
    "rvsp_spgemm_set_stream": (_int, [_vp, _vp]),
    "rvsp_spgemm_set_profiling": (_int, [_vp, _int]),
    "rvsp_spgemm_get_phase_times": (_int, [_vp, _vp, _vp, _i32, _int]),
    "rvsp_spgemm_synchronize": (_int, [_vp]),
    "rvsp_spgemm_get_class_counts": (_int, [_vp, _vp, _vp, _i32]),
    "rvsp_spgemm_csr_device": (_int, [_P(CsrMatrix), _P(CsrMatrix), _P(CsrMatrix),
                                      _P(SpgemmOptions)]),
    # rvsp_cuda.h
    "rvsp_cuda_plan_create": (_int, [_P(_vp)]),
    "rvsp_cuda_plan_destroy": (None, [_vp]),
    "rvsp_cuda_symbolic": (_int, [_vp, _vp, _i32, _i32, _i32, _vp, _vp, _vp, _vp,
                                  _vp, _P(_i64)]),
    "rvsp_cuda_numeric_workspace_bytes": (_sz, [_vp]),
    "rvsp_cuda_numeric": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                 _vp, _int, _vp, _sz]),
    "rvsp_cuda_op_counts": (_int, [_vp, _vp, _vp, _i32]),
    "rvsp_cuda_plan_status": (_int, [_vp, _vp]),
    "rvsp_cuda_csr_check": (_int, [_vp, _vp, _i32, _i32, _vp, _vp, _i32, _P(_i32),
                                   _P(_i32)]),
    "rvsp_cuda_plan_set_profiling": (_int, [_vp, _int]),
    "rvsp_cuda_plan_phase_times": (_int, [_vp, _vp, _vp, _i32, _int]),
    "rvsp_cuda_plan_class_counts": (_int, [_vp, _vp, _vp, _i32]),
    "rvsp_cuda_numeric_noalloc": (_int, [_vp, _i32, _i32, _i32, _vp, _vp, _vp, _vp,
                                         _vp, _vp, _vp, _vp, _vp]),
    "rvsp_mlp_create": (_int, [_P(_vp), C.c_uint64]),
    "rvsp_mlp_destroy": (None, [_vp]),
    "rvsp_mlp_num_params": (_i32, []),
    "rvsp_mlp_get_params": (_int, [_vp, _vp, _i32]),
    "rvsp_mlp_set_params": (_int, [_vp, _vp, _i32]),
    "rvsp_mlp_features": (_int, [_vp, _i32, _i32, _i32, _vp, _vp, _vp, _vp, _vp, _vp]),
    "rvsp_mlp_gradient": (_int, [_vp, _vp, _vp, _vp, _i32, _vp, _P(C.c_float)]),
    "rvsp_mlp_train": (_int, [_vp, _vp, _vp, _vp, _i32, _i32, _i32, C.c_float, _vp]),
    "rvsp_mlp_predict": (_int, [_vp, _vp, _i32, _i32, _i32, _vp, _vp, _vp, _vp, _vp]),
    "rvsp_mlp_save": (_int, [_vp, C.c_char_p]),
    "rvsp_mlp_load": (_int, [_vp, C.c_char_p]),
    "rvsp_cuda_learned_symbolic": (_int, [_vp, _vp, _vp, _i32, _i32, _i32, _vp, _vp, _vp,
                                          _i32, _vp, _vp, _vp, _i32, C.c_float, _vp,
                                          _P(_i64)]),
    "rvsp_cuda_plan_overflow_rows": (_i32, [_vp]),
    "rvsp_cuda_plan_set_merge_policy": (_int, [_vp, _i32]),
    "rvsp_spgemm_set_merge_policy": (_int, [_vp, _i32]),
    "rvsp_spgemm_set_row_tiles": (_int, [_vp, _i32]),
    "rvsp_spgemm_get_tiled_rows": (_int, [_vp, _P(_i32)]),
    "rvsp_cuda_plan_set_row_tiles": (_int, [_vp, _i32]),
    "rvsp_cuda_plan_tiled_rows": (_i32, [_vp]),
    "rvsp_cuda_plan_set_shift_classes": (_int, [_vp, _i32]),
    "rvsp_cuda_plan_shift_rows": (_i32, [_vp]),
    "rvsp_spgemm_set_shift_classes": (_int, [_vp, _i32]),
    "rvsp_cuda_plan_set_persistent": (_int, [_vp, _i32, _i32]),
    "rvsp_cuda_plan_set_pattern_kernels": (_int, [_vp, _i32]),
    "rvsp_cuda_plan_pattern_kernel_rows": (_i32, [_vp]),
    "rvsp_cuda_pattern_kernel_stats": (None, [_P(_i32), _P(C.c_double)]),
    "rvsp_spgemm_set_pattern_kernels": (_int, [_vp, _i32]),
    "rvsp_spgemm_batch_set_persistent": (_int, [_vp, _i32, _i32]),
    "rvsp_spgemm_batch_get_tuning": (_int, [_vp, _P(_i32), _P(_i32), _P(_i32),
                                            _P(C.c_float), _P(_i32)]),
    "rvsp_spgemm_get_shift_rows": (_int, [_vp, _P(_i32)]),
    "rvsp_spgemm_set_model": (_int, [_vp, _vp]),
    "rvsp_spgemm_set_capacity_scale": (_int, [_vp, C.c_float]),
    "rvsp_spgemm_get_overflow_rows": (_int, [_vp, _P(_i32)]),
    "rvsp_spgemm_multiply": (_int, [_vp, _P(CsrMatrix), _P(CsrMatrix), _P(CsrMatrix)]),
    # batches (rv_sparse.h)
    "rvsp_spgemm_batch_create": (_int, [_P(_vp)]),
    "rvsp_spgemm_batch_destroy": (None, [_vp]),
    "rvsp_spgemm_batch_set_memory_space": (_int, [_vp, _int]),
    "rvsp_spgemm_batch_set_stream": (_int, [_vp, _vp]),
    "rvsp_spgemm_batch_set_autotune": (_int, [_vp, _int]),
    "rvsp_spgemm_batch_set_merge_policy": (_int, [_vp, _i32]),
    "rvsp_spgemm_batch_set_group_ops": (_int, [_vp, _i64]),
    "rvsp_spgemm_batch_add": (_int, [_vp, _P(CsrMatrix), _P(CsrMatrix), _P(_i32)]),
    "rvsp_spgemm_batch_work_estimation": (_int, [_vp, _P(_i64)]),
    "rvsp_spgemm_batch_compute": (_int, [_vp]),
    "rvsp_spgemm_batch_synchronize": (_int, [_vp]),
    "rvsp_spgemm_batch_get_nnz": (_int, [_vp, _i32, _P(_i32)]),
    "rvsp_spgemm_batch_get_result": (_int, [_vp, _i32, _P(CsrMatrix)]),
    "rvsp_spgemm_batch_copy_result": (_int, [_vp, _i32, _P(CsrMatrix)]),
    "rvsp_spgemm_batch_get_stats": (_int, [_vp, _P(_i32), _P(_i64), _P(_i32), _P(_i32)]),
    "rvsp_cuda_plan_prepare_reuse": (_int, [_vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
                                            _P(_i64)]),
    "rvsp_cuda_plan_reuse_shared_rows": (_int, [_vp, _vp, _P(_i32)]),
    # batches (rvsp_cuda.h)
    "rvsp_cuda_batch_entries": (_int, [_vp, _vp, _i32]),
    "rvsp_cuda_batch_op_counts": (_int, [_vp, _vp, _i32, _vp, _vp]),
    "rvsp_cuda_batch_pack": (_int, [_vp, _vp, _vp, _i32, _int, _vp, _vp, _vp, _vp, _vp,
                                    _vp, _vp]),
    "rvsp_cuda_batch_views": (_int, [_vp, _vp, _vp, _vp, _i32, _vp, _vp, _vp, _vp]),
}

_lib = None


def lib_path() -> Path:
    override = os.environ.get("RVSP_LIB")
    return Path(override) if override else LIB_PATH


def load() -> C.CDLL:
    """Loads the C-ABI library once; raises if it is missing (no fallback)."""
    global _lib
    if _lib is not None:
        return _lib
    path = lib_path()
    if not path.exists():
        raise RuntimeError(
            f"{path} is not built: run `make -C {PKG_ROOT}` (the CUDA "
            "library is required; there is no CPU fallback)")
    lib = C.CDLL(str(path), mode=C.RTLD_LOCAL)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


class RvspError(RuntimeError):
    def __init__(self, status: int, where: str = ""):
        self.status = status
        msg = load().rvsp_status_to_string(status).decode()
        super().__init__(f"{where}: {msg} ({status})" if where else f"{msg} ({status})")


def check(status: int, where: str = "") -> None:
    if status != SUCCESS:
        raise RvspError(status, where)
