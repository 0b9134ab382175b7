"""CPU oracle for the SpGEMM hot path.  TEST INFRASTRUCTURE ONLY.

Only tests, the smoke check and the CPU-baseline leg of bench.py import this
module, and only as the checker.  The product library never loads it.

Two checkers:
  * liborc.so - a C restatement of the reference scalar backend
    (rvsp_oracle.c; symbolic count, sorted fill, numeric with separately
    rounded multiply and add, plus an FP64 accumulation);
  * librvsp_ref.so - the reference library itself (merledu/rv-sparse),
    compiled from its own sources by oracle/Makefile into oracle/_ref/.
The restatement is pinned against the reference's fixtures
(tests/golden/fixtures.json) and against librvsp_ref.so on seeded inputs
(tests/test_oracle.py).

Matrices are duck-typed: anything with rows, cols, row_ptr (int32),
col_idx (int32) and values (float32) numpy arrays.
"""
from __future__ import annotations

import ctypes as C
import subprocess
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORC_PATH = HERE / "_build" / "liborc.so"
REF_PATH = HERE / "_ref" / "librvsp_ref.so"

_orc = None
_ref = None


def build(with_ref: bool = True) -> None:
    """Compiles the restatement and, when the reference tree exists, the
    reference library (make -C oracle)."""
    target = "all" if with_ref else "orc"
    subprocess.run(["make", "-s", "-C", str(HERE), target], check=True)


def _vp(a: np.ndarray):
    return C.c_void_p(a.ctypes.data) if a is not None else None


def orc() -> C.CDLL:
    global _orc
    if _orc is None:
        if not ORC_PATH.exists():
            build(with_ref=False)
        lib = C.CDLL(str(ORC_PATH), mode=C.RTLD_LOCAL)
        vp, i32 = C.c_void_p, C.c_int32
        lib.orc_csr_check.argtypes = [i32, i32, vp, vp, C.POINTER(i32)]
        lib.orc_csr_check.restype = C.c_int
        lib.orc_symbolic_count.argtypes = [i32, i32, vp, vp, vp, vp, vp, vp,
                                           C.POINTER(C.c_int64)]
        lib.orc_symbolic_count.restype = C.c_int
        lib.orc_symbolic_fill.argtypes = [i32, i32, vp, vp, vp, vp, vp, vp]
        lib.orc_symbolic_fill.restype = None
        lib.orc_numeric_f32.argtypes = [i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        lib.orc_numeric_f32.restype = None
        lib.orc_numeric_f64.argtypes = [i32, i32, vp, vp, vp, vp, vp, vp, vp, vp, vp, vp]
        lib.orc_numeric_f64.restype = None
        lib.orc_numeric_f32_rows.argtypes = [i32, i32, vp, vp, vp, vp, vp, vp, vp, vp,
                                             vp, vp]
        lib.orc_numeric_f32_rows.restype = None
        lib.orc_mtx_to_csr.argtypes = [C.c_char_p, C.c_size_t, C.POINTER(i32), C.POINTER(i32),
                                       C.POINTER(C.c_int64), C.POINTER(vp), C.POINTER(vp),
                                       C.POINTER(vp)]
        lib.orc_mtx_to_csr.restype = C.c_int
        lib.orc_free.argtypes = [vp]
        lib.orc_free.restype = None
        for name in ("orc_spgemm_f64", "orc_spgemm_i8"):
            f = getattr(lib, name)
            f.argtypes = [i32, i32, vp, vp, vp, vp, vp, vp, C.POINTER(vp), C.POINTER(vp),
                          C.POINTER(vp), C.POINTER(C.c_int64)]
            f.restype = C.c_int
        _orc = lib
    return _orc


MTX_ERRORS = {-1: "malformed size line", -2: "index out of range", -3: "out of memory"}


def mtx_to_csr(text: bytes):
    """(rows, cols, row_ptr, col_idx, values) of Matrix Market text, by the
    restatement of the reference reader (mtx_oracle.c)."""
    lib = orc()
    rows, cols, nnz = C.c_int32(), C.c_int32(), C.c_int64()
    rp, ci, cv = C.c_void_p(), C.c_void_p(), C.c_void_p()
    rc = lib.orc_mtx_to_csr(text, len(text), C.byref(rows), C.byref(cols), C.byref(nnz),
                            C.byref(rp), C.byref(ci), C.byref(cv))
    if rc != 0:
        raise ValueError(MTX_ERRORS.get(rc, str(rc)))
    try:
        n, m = rows.value, nnz.value
        row_ptr = np.ctypeslib.as_array(C.cast(rp, C.POINTER(C.c_int32)), (n + 1,)).copy()
        col_idx = (np.ctypeslib.as_array(C.cast(ci, C.POINTER(C.c_int32)), (m,)).copy()
                   if m else np.zeros(0, np.int32))
        values = (np.ctypeslib.as_array(C.cast(cv, C.POINTER(C.c_float)), (m,)).copy()
                  if m else np.zeros(0, np.float32))
    finally:
        for p in (rp, ci, cv):
            lib.orc_free(p)
    return n, cols.value, row_ptr, col_idx, values


MTX_REF_PATH = HERE / "_ref" / "librvsp_mtx_ref.so"
_mtx_ref = None


class _Vec(C.Structure):
    _fields_ = [("data", C.c_void_p), ("size", C.c_size_t), ("capacity", C.c_size_t),
                ("elem_size", C.c_size_t)]


class _RefMtxCsr(C.Structure):
    _fields_ = [("row_ptr", C.POINTER(_Vec)), ("col_ind", C.POINTER(_Vec)),
                ("val", C.POINTER(_Vec))]


def ref_mtx_available() -> bool:
    return MTX_REF_PATH.exists()


def ref_mtx_to_csr(path):
    """(row_ptr, col_idx, values) from the reference's own reader
    (tools/src/mtx_to_csr_formatter.c assemble_csr_matrix, built into
    oracle/_ref/librvsp_mtx_ref.so), or None when it fails."""
    global _mtx_ref
    if _mtx_ref is None:
        lib = C.CDLL(str(MTX_REF_PATH), mode=C.RTLD_LOCAL)
        lib.assemble_csr_matrix.argtypes = [C.c_char_p]
        lib.assemble_csr_matrix.restype = _RefMtxCsr
        lib.vector_free.argtypes = [C.POINTER(_Vec)]
        lib.vector_free.restype = None
        _mtx_ref = lib
    r = _mtx_ref.assemble_csr_matrix(str(path).encode())
    if not r.row_ptr or not r.col_ind or not r.val:
        return None

    def take(v, ctype, dtype):
        n = v.contents.size
        if n == 0:
            return np.zeros(0, dtype)
        return np.ctypeslib.as_array(C.cast(v.contents.data, C.POINTER(ctype)), (n,)).copy()
    try:
        return (take(r.row_ptr, C.c_int32, np.int32), take(r.col_ind, C.c_int32, np.int32),
                take(r.val, C.c_float, np.float32))
    finally:
        for v in (r.row_ptr, r.col_ind, r.val):
            _mtx_ref.vector_free(v)


def _arrs(M):
    return (np.ascontiguousarray(M.row_ptr, np.int32),
            np.ascontiguousarray(M.col_idx, np.int32),
            np.ascontiguousarray(M.values, np.float32))


def csr_check(rows, cols, row_ptr, col_idx):
    """(code, bad_row) with the codes of rvsp_csr_status_t."""
    bad = C.c_int32(-1)
    rp = np.ascontiguousarray(row_ptr, np.int32) if row_ptr is not None else None
    ci = np.ascontiguousarray(col_idx, np.int32) if col_idx is not None else None
    code = orc().orc_csr_check(rows, cols, _vp(rp), _vp(ci), C.byref(bad))
    return code, bad.value


def symbolic(A, B):
    """(row_ptr, col_idx sorted, op_counts) of C = A * B; raises OverflowError
    when nnz(C) > INT32_MAX (the reference's ALLOCATION_FAILED)."""
    arp, aci, _ = _arrs(A)
    brp, bci, _ = _arrs(B)
    crp = np.zeros(A.rows + 1, np.int32)
    ops = np.zeros(max(A.rows, 1), np.int64)
    total = C.c_int64(0)
    st = orc().orc_symbolic_count(A.rows, B.cols, _vp(arp), _vp(aci), _vp(brp),
                                  _vp(bci), _vp(crp), _vp(ops), C.byref(total))
    if st != 0:
        raise OverflowError("nnz(C) exceeds INT32_MAX")
    cci = np.zeros(max(int(total.value), 1), np.int32)
    orc().orc_symbolic_fill(A.rows, B.cols, _vp(arp), _vp(aci), _vp(brp), _vp(bci),
                            _vp(crp), _vp(cci))
    return crp, cci[:int(total.value)], ops[:A.rows]


def numeric_f32(A, B, c_row_ptr, c_col_idx):
    arp, aci, av = _arrs(A)
    brp, bci, bv = _arrs(B)
    out = np.zeros(max(c_col_idx.size, 1), np.float32)
    orc().orc_numeric_f32(A.rows, B.cols, _vp(arp), _vp(aci), _vp(av), _vp(brp),
                          _vp(bci), _vp(bv), _vp(np.ascontiguousarray(c_row_ptr, np.int32)),
                          _vp(np.ascontiguousarray(c_col_idx, np.int32)), _vp(out))
    return out[:c_col_idx.size]


def numeric_f64(A, B, c_row_ptr, c_col_idx):
    """(values, sum of |terms|) per output entry, accumulated in FP64."""
    arp, aci, av = _arrs(A)
    brp, bci, bv = _arrs(B)
    n = max(c_col_idx.size, 1)
    out = np.zeros(n, np.float64)
    mag = np.zeros(n, np.float64)
    orc().orc_numeric_f64(A.rows, B.cols, _vp(arp), _vp(aci), _vp(av), _vp(brp),
                          _vp(bci), _vp(bv), _vp(np.ascontiguousarray(c_row_ptr, np.int32)),
                          _vp(np.ascontiguousarray(c_col_idx, np.int32)), _vp(out),
                          _vp(mag))
    return out[:c_col_idx.size], mag[:c_col_idx.size]


def spgemm(A, B):
    """(row_ptr, col_idx, values f32, op_counts) exactly as the reference
    scalar backend computes them."""
    crp, cci, ops = symbolic(A, B)
    return crp, cci, numeric_f32(A, B, crp, cci), ops


# ---- the reference library itself ----------------------------------------


class _RefCsr(C.Structure):
    _fields_ = [("rows", C.c_int32), ("cols", C.c_int32), ("nnz", C.c_int32),
                ("row_ptr", C.c_void_p), ("col_idx", C.c_void_p),
                ("values", C.c_void_p), ("dtype", C.c_int), ("format", C.c_int),
                ("owns_data", C.c_int)]


class _RefOpts(C.Structure):
    _fields_ = [("backend", C.c_int), ("input_dtype", C.c_int),
                ("output_dtype", C.c_int)]


def ref_available() -> bool:
    return REF_PATH.exists()


def ref() -> C.CDLL:
    global _ref
    if _ref is None:
        if not REF_PATH.exists():
            raise FileNotFoundError(f"{REF_PATH} not built (needs the reference sources)")
        lib = C.CDLL(str(REF_PATH), mode=C.RTLD_LOCAL)
        P = C.POINTER
        lib.rvsp_spgemm_csr.argtypes = [P(_RefCsr), P(_RefCsr), P(_RefCsr), P(_RefOpts)]
        lib.rvsp_spgemm_csr.restype = C.c_int
        lib.rvsp_csr_destroy.argtypes = [P(_RefCsr)]
        lib.rvsp_csr_destroy.restype = None
        lib.rvsp_csr_check.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_void_p,
                                       P(C.c_int32)]
        lib.rvsp_csr_check.restype = C.c_int
        lib.rvsp_spgemm_descr_create.argtypes = [P(C.c_void_p)]
        lib.rvsp_spgemm_descr_create.restype = C.c_int
        lib.rvsp_spgemm_descr_destroy.argtypes = [C.c_void_p]
        lib.rvsp_spgemm_work_estimation.argtypes = [C.c_void_p, P(_RefCsr), P(_RefCsr),
                                                    P(C.c_size_t), P(C.c_int32)]
        lib.rvsp_spgemm_work_estimation.restype = C.c_int
        lib.rvsp_spgemm_compute.argtypes = [C.c_void_p, P(_RefCsr), P(_RefCsr),
                                            P(_RefCsr), C.c_void_p]
        lib.rvsp_spgemm_compute.restype = C.c_int
        lib.rvsp_spgemm_get_op_counts.argtypes = [C.c_void_p, C.c_void_p, C.c_int32]
        lib.rvsp_spgemm_get_op_counts.restype = C.c_int
        _ref = lib
    return _ref


def _ref_struct(M, keep):
    rp, ci, v = _arrs(M)
    keep += [rp, ci, v]
    s = _RefCsr()
    s.rows, s.cols, s.nnz = M.rows, M.cols, int(rp[-1])
    s.row_ptr, s.col_idx, s.values = rp.ctypes.data, ci.ctypes.data, v.ctypes.data
    s.dtype, s.format, s.owns_data = 3, 0, 0  # FP32, CSR
    return s


def ref_spgemm(A, B):
    """rvsp_spgemm_csr(..., RVSP_BACKEND_SCALAR) of the reference library:
    (status, row_ptr, col_idx, values)."""
    keep = []
    a, b = _ref_struct(A, keep), _ref_struct(B, keep)
    c = _RefCsr()
    opts = _RefOpts(0, 3, 3)  # SCALAR, FP32, FP32
    st = ref().rvsp_spgemm_csr(C.byref(a), C.byref(b), C.byref(c), C.byref(opts))
    if st != 0:
        return st, None, None, None
    n = c.nnz
    rp = np.ctypeslib.as_array(C.cast(c.row_ptr, C.POINTER(C.c_int32)),
                               shape=(c.rows + 1,)).copy()
    ci = (np.ctypeslib.as_array(C.cast(c.col_idx, C.POINTER(C.c_int32)), shape=(n,)).copy()
          if n else np.zeros(0, np.int32))
    cv = (np.ctypeslib.as_array(C.cast(c.values, C.POINTER(C.c_float)), shape=(n,)).copy()
          if n else np.zeros(0, np.float32))
    ref().rvsp_csr_destroy(C.byref(c))
    return st, rp, ci, cv


def ref_op_counts(A, B):
    """Per-row op counts from the reference descriptor (get_op_counts)."""
    keep = []
    a, b = _ref_struct(A, keep), _ref_struct(B, keep)
    d = C.c_void_p()
    lib = ref()
    assert lib.rvsp_spgemm_descr_create(C.byref(d)) == 0
    try:
        ws, nnz = C.c_size_t(), C.c_int32()
        st = lib.rvsp_spgemm_work_estimation(d, C.byref(a), C.byref(b), C.byref(ws),
                                             C.byref(nnz))
        if st != 0:
            return st, None
        out = np.zeros(max(A.rows, 1), np.int64)
        st = lib.rvsp_spgemm_get_op_counts(d, out.ctypes.data, A.rows)
        return st, out[:A.rows]
    finally:
        lib.rvsp_spgemm_descr_destroy(d)


def ref_check(rows, cols, row_ptr, col_idx):
    bad = C.c_int32(-1)
    rp = np.ascontiguousarray(row_ptr, np.int32)
    ci = np.ascontiguousarray(col_idx, np.int32)
    code = ref().rvsp_csr_check(rows, cols, rp.ctypes.data, ci.ctypes.data, C.byref(bad))
    return code, bad.value


def time_reference_oneshot(A, B, seconds: float = 10.0, threads: int = 1,
                           max_runs: int = 1000):
    """Times the reference one-shot product on host cores.  Each of `threads`
    Python threads runs independent products (ctypes releases the GIL and the
    reference keeps all state per call).  Returns (runs, elapsed_s)."""
    import threading
    use_ref = ref_available()
    done = [0] * threads
    stop_at = [None]

    def worker(t):
        while True:
            if use_ref:
                ref_spgemm(A, B)
            else:
                spgemm(A, B)
            done[t] += 1
            if time.perf_counter() >= stop_at[0] or sum(done) >= max_runs:
                return

    t0 = time.perf_counter()
    stop_at[0] = t0 + seconds
    ths = [threading.Thread(target=worker, args=(t,)) for t in range(threads)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    return sum(done), time.perf_counter() - t0


def time_reference_batch(products, seconds: float = 10.0, threads: int = 1):
    """Times the reference one-shot product over a list of (A, B) pairs taken
    in order by `threads` Python threads (one product per call, as a CPU
    batch would run), stopping once `seconds` have passed.  Returns (indices
    of the products done, elapsed_s)."""
    import threading
    use_ref = ref_available()
    lock = threading.Lock()
    nxt = [0]
    done = []
    stop_at = time.perf_counter() + seconds

    def worker():
        while True:
            with lock:
                if nxt[0] >= len(products) or time.perf_counter() >= stop_at:
                    return
                i = nxt[0]
                nxt[0] += 1
            A, B = products[i]
            if use_ref:
                ref_spgemm(A, B)
            else:
                spgemm(A, B)
            with lock:
                done.append(i)

    t0 = time.perf_counter()
    ths = [threading.Thread(target=worker) for _ in range(threads)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    return sorted(done), time.perf_counter() - t0


def ref_job(A, B, value_sets=(), keep_first=True, keep_all=False):
    """The reference descriptor's job (spgemm_descr.c:66-380):
    work_estimation(A, B), compute into a caller-owned C (fill + numeric),
    then one numeric-only compute per (a_values, b_values) in value_sets into
    the same C.  Returns (status, row_ptr, col_idx, values after the first
    compute or None, values after the last compute); with keep_all the last
    item is the list of the values after every numeric-only compute."""
    lib = ref()
    keep = []
    a, b = _ref_struct(A, keep), _ref_struct(B, keep)
    d = C.c_void_p()
    assert lib.rvsp_spgemm_descr_create(C.byref(d)) == 0
    try:
        ws_b, nnz = C.c_size_t(), C.c_int32()
        st = lib.rvsp_spgemm_work_estimation(d, C.byref(a), C.byref(b), C.byref(ws_b),
                                             C.byref(nnz))
        if st != 0:
            return st, None, None, None, None
        n = nnz.value
        rp = np.zeros(A.rows + 1, np.int32)
        ci = np.zeros(max(n, 1), np.int32)
        cv = np.zeros(max(n, 1), np.float32)
        ws = np.zeros(max(int(ws_b.value), 1), np.uint8)
        c = _RefCsr()
        c.rows, c.cols, c.nnz = A.rows, B.cols, n
        c.row_ptr, c.col_idx, c.values = rp.ctypes.data, ci.ctypes.data, cv.ctypes.data
        c.dtype, c.format, c.owns_data = 3, 0, 0
        st = lib.rvsp_spgemm_compute(d, C.byref(a), C.byref(b), C.byref(c), ws.ctypes.data)
        if st != 0:
            return st, None, None, None, None
        first = cv[:n].copy() if keep_first else None
        every = []
        for av, bv in value_sets:
            av = np.ascontiguousarray(av, np.float32)
            bv = np.ascontiguousarray(bv, np.float32)
            keep += [av, bv]
            a.values, b.values = av.ctypes.data, bv.ctypes.data
            st = lib.rvsp_spgemm_compute(d, C.byref(a), C.byref(b), C.byref(c),
                                         ws.ctypes.data)
            if st != 0:
                return st, None, None, None, None
            if keep_all:
                every.append(cv[:n].copy())
        return 0, rp, ci[:n], first, (every if keep_all else cv[:n])
    finally:
        lib.rvsp_spgemm_descr_destroy(d)


def time_reference_job(A, B, value_sets, threads: int):
    """The reference's descriptor job on host cores, the rows of A shared out
    as `threads` row panels (each panel times B is a product of its own; the
    panels together are the whole product): each thread runs
    work_estimation + compute + one numeric-only compute per entry of
    value_sets ((A values, B values) of the whole matrices) on its panel.
    Returns elapsed seconds (all threads)."""
    import threading
    use_ref = ref_available()
    bounds = np.linspace(0, A.rows, threads + 1).astype(int)

    def worker(t):
        r0, r1 = int(bounds[t]), int(bounds[t + 1])
        if r1 <= r0:
            return
        P = A.row_panel(r0, r1)
        p0, p1 = int(A.row_ptr[r0]), int(A.row_ptr[r1])
        sets = [(av[p0:p1], bv) for av, bv in value_sets]
        if use_ref:
            ref_job(P, B, sets, keep_first=False)
        else:
            rp, ci, _ = symbolic(P, B)
            numeric_f32(P, B, rp, ci)
            for av, bv in sets:
                numeric_f32(P.with_values(av), B.with_values(bv), rp, ci)

    t0 = time.perf_counter()
    ths = [threading.Thread(target=worker, args=(t,)) for t in range(threads)]
    for th in ths:
        th.start()
    for th in ths:
        th.join()
    return time.perf_counter() - t0


# ---- FP64 and INT8 -> INT32 products (legacy scalar kernels) ----------------

_TYPED = {"f64": (np.float64, np.float64, 4, 4), "i8": (np.int8, np.int32, 0, 1)}


def _take(ptr, ctype, n, dtype):
    if n == 0:
        return np.zeros(0, dtype)
    return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(n,)).copy().view(dtype)


def spgemm_typed(A, B, kind: str):
    """(row_ptr, col_idx, values) of A x B by the restatement of the legacy
    scalar kernel; kind "f64" (float64 values) or "i8" (int8 in, int32 out).
    A and B are (rows, cols, row_ptr, col_idx, values) tuples."""
    vin, vout, _, _ = _TYPED[kind]
    ar, ac, arp, aci, av = A
    br, bc, brp, bci, bv = B
    arp, aci, brp, bci = (np.ascontiguousarray(x, np.int32) for x in (arp, aci, brp, bci))
    av, bv = np.ascontiguousarray(av, vin), np.ascontiguousarray(bv, vin)
    rp, ci, cv, nnz = C.c_void_p(), C.c_void_p(), C.c_void_p(), C.c_int64()
    f = orc().orc_spgemm_f64 if kind == "f64" else orc().orc_spgemm_i8
    rc = f(ar, bc, arp.ctypes.data, aci.ctypes.data, av.ctypes.data, brp.ctypes.data,
           bci.ctypes.data, bv.ctypes.data, C.byref(rp), C.byref(ci), C.byref(cv),
           C.byref(nnz))
    if rc != 0:
        raise MemoryError("oracle out of memory")
    try:
        n = nnz.value
        out_ct = C.c_double if kind == "f64" else C.c_int32
        return (_take(rp, C.c_int32, ar + 1, np.int32), _take(ci, C.c_int32, n, np.int32),
                _take(cv, out_ct, n, vout))
    finally:
        for p in (rp, ci, cv):
            orc().orc_free(p)


def ref_spgemm_typed(A, B, kind: str):
    """rvsp_spgemm_csr of the reference library with RVSP_BACKEND_SCALAR and
    {FP64, FP64} or {INT8, INT32}: (status, row_ptr, col_idx, values)."""
    vin, vout, in_code, out_code = _TYPED[kind]
    keep = []

    def st(M):
        rows, cols, rp, ci, v = M
        rp, ci = np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(ci, np.int32)
        v = np.ascontiguousarray(v, vin)
        keep.extend([rp, ci, v])
        s = _RefCsr()
        s.rows, s.cols, s.nnz = rows, cols, int(rp[-1])
        s.row_ptr, s.col_idx, s.values = rp.ctypes.data, ci.ctypes.data, v.ctypes.data
        s.dtype, s.format, s.owns_data = in_code, 0, 0
        return s
    a, b = st(A), st(B)
    c = _RefCsr()
    status = ref().rvsp_spgemm_csr(C.byref(a), C.byref(b), C.byref(c),
                                   C.byref(_RefOpts(0, in_code, out_code)))
    if status != 0:
        return status, None, None, None
    n = c.nnz
    out_ct = C.c_double if kind == "f64" else C.c_int32
    res = (status, _take(c.row_ptr, C.c_int32, c.rows + 1, np.int32),
           _take(c.col_idx, C.c_int32, n, np.int32), _take(c.values, out_ct, n, vout))
    ref().rvsp_csr_destroy(C.byref(c))
    return res
