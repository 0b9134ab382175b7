"""Python mirror of the rv-sparse C API on the CUDA backend.

Names follow the reference API (include/rv_sparse.h of merledu/rv-sparse):
`spgemm_csr` is rvsp_spgemm_csr, `Descriptor` wraps the rvsp_spgemm_descr_*
sequence (create -> set_algo -> work_estimation -> compute -> get_op_counts ->
invalidate_structure -> destroy).  Errors raise RvspError carrying the
rvsp_status_t code.  Everything calls the C-ABI library; nothing here computes.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L
from .csr import CSR

CUDA_STREAM_LEGACY = 0x1  # cudaStreamLegacy


def spgemm_csr(A: CSR, B: CSR, backend: int | None = L.BACKEND_CUDA) -> CSR:
    """One-shot C = A * B on host arrays (rvsp_spgemm_csr).  backend=None
    passes NULL options."""
    lib = L.load()
    a, b = A.struct(), B.struct()
    c = L.CsrMatrix()
    opts = None
    if backend is not None:
        opts = L.SpgemmOptions(backend, L.DTYPE_FP32, L.DTYPE_FP32)
    st = lib.rvsp_spgemm_csr(C.byref(a), C.byref(b), C.byref(c),
                             C.byref(opts) if opts is not None else None)
    L.check(st, "rvsp_spgemm_csr")
    try:
        n = c.nnz
        rp = np.ctypeslib.as_array(C.cast(c.row_ptr, C.POINTER(C.c_int32)),
                                   shape=(c.rows + 1,)).copy()
        if n > 0:
            ci = np.ctypeslib.as_array(C.cast(c.col_idx, C.POINTER(C.c_int32)),
                                       shape=(n,)).copy()
            cv = np.ctypeslib.as_array(C.cast(c.values, C.POINTER(C.c_float)),
                                       shape=(n,)).copy()
        else:
            ci = np.zeros(0, np.int32)
            cv = np.zeros(0, np.float32)
        return CSR(c.rows, c.cols, rp, ci, cv)
    finally:
        lib.rvsp_csr_destroy(C.byref(c))


_TYPED_CODES = {"f64": (L.DTYPE_FP64, L.DTYPE_FP64, np.float64, np.float64, C.c_double),
                "i8": (L.DTYPE_INT8, L.DTYPE_INT32, np.int8, np.int32, C.c_int32)}


def spgemm_typed(A, B, kind: str, backend: int = L.BACKEND_CUDA):
    """One-shot FP64 (kind "f64") or INT8 -> INT32 (kind "i8") product
    through rvsp_spgemm_csr with options {backend, dtypes}.  A and B are
    (rows, cols, row_ptr, col_idx, values) tuples of host arrays; returns
    (row_ptr, col_idx, values) or raises RvspError."""
    lib = L.load()
    din, dout, vin, vout, ct = _TYPED_CODES[kind]
    keep = []

    def struct(M):
        rows, cols, rp, ci, v = M
        rp, ci = np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(ci, np.int32)
        v = np.ascontiguousarray(v, vin)
        keep.extend([rp, ci, v])
        m = L.CsrMatrix()
        m.rows, m.cols, m.nnz = rows, cols, int(rp[-1]) if rp.size else 0
        m.row_ptr, m.col_idx, m.values = rp.ctypes.data, ci.ctypes.data, v.ctypes.data
        m.dtype, m.format, m.owns_data = din, L.FORMAT_CSR, 0
        return m
    a, b = struct(A), struct(B)
    c = L.CsrMatrix()
    opts = L.SpgemmOptions(backend, din, dout)
    L.check(lib.rvsp_spgemm_csr(C.byref(a), C.byref(b), C.byref(c), C.byref(opts)),
            "rvsp_spgemm_csr")
    try:
        n = c.nnz
        rp = np.ctypeslib.as_array(C.cast(c.row_ptr, C.POINTER(C.c_int32)),
                                   shape=(c.rows + 1,)).copy()
        if n > 0:
            ci = np.ctypeslib.as_array(C.cast(c.col_idx, C.POINTER(C.c_int32)),
                                       shape=(n,)).copy()
            cv = np.ctypeslib.as_array(C.cast(c.values, C.POINTER(ct)), shape=(n,)).copy()
        else:
            ci, cv = np.zeros(0, np.int32), np.zeros(0, vout)
        assert c.dtype == dout
        return rp, ci, cv.astype(vout, copy=False)
    finally:
        lib.rvsp_csr_destroy(C.byref(c))


def read_mtx(source, device: bool = False):
    """A Matrix Market file (path) or its text (bytes) as canonical CSR
    (rvsp_csr_read_mtx / rvsp_csr_parse_mtx): a host CSR, or with
    device=True a DeviceCSR whose tensors hold the library's device result."""
    lib = L.load()
    m = L.CsrMatrix()
    space = L.MEM_DEVICE if device else L.MEM_HOST
    if isinstance(source, (bytes, bytearray)):
        st = lib.rvsp_csr_parse_mtx(bytes(source), len(source), space, C.byref(m))
    else:
        st = lib.rvsp_csr_read_mtx(str(source).encode(), space, C.byref(m))
    L.check(st, "rvsp_csr_read_mtx")
    try:
        if device:
            out = DeviceCSR.empty(m.rows, m.cols, m.nnz)
            L.check(lib.rvsp_csr_copy_arrays(C.byref(m), C.byref(out.struct(m.nnz))),
                    "rvsp_csr_copy_arrays")
            if m.nnz == 0:
                out.col_idx, out.values = out.col_idx[:0], out.values[:0]
            return out
        rp = np.ctypeslib.as_array(C.cast(m.row_ptr, C.POINTER(C.c_int32)),
                                   shape=(m.rows + 1,)).copy()
        if m.nnz > 0:
            ci = np.ctypeslib.as_array(C.cast(m.col_idx, C.POINTER(C.c_int32)),
                                       shape=(m.nnz,)).copy()
            cv = np.ctypeslib.as_array(C.cast(m.values, C.POINTER(C.c_float)),
                                       shape=(m.nnz,)).copy()
        else:
            ci, cv = np.zeros(0, np.int32), np.zeros(0, np.float32)
        return CSR(m.rows, m.cols, rp, ci, cv)
    finally:
        lib.rvsp_csr_destroy(C.byref(m))


class DeviceCSR:
    """CSR arrays in device memory (torch CUDA tensors, used only as storage)."""

    def __init__(self, rows, cols, row_ptr, col_idx, values):
        self.rows, self.cols = int(rows), int(cols)
        self.row_ptr, self.col_idx, self.values = row_ptr, col_idx, values

    @property
    def nnz(self) -> int:
        return int(self.col_idx.numel())

    # Both constructors finish their device work before returning, so the
    # arrays are ready for a descriptor on any stream.
    @staticmethod
    def from_host(M: CSR, device="cuda") -> "DeviceCSR":
        import torch
        out = DeviceCSR(M.rows, M.cols,
                        torch.from_numpy(M.row_ptr).to(device),
                        torch.from_numpy(M.col_idx).to(device),
                        torch.from_numpy(M.values).to(device))
        torch.cuda.synchronize(device)
        return out

    @staticmethod
    def empty(rows, cols, nnz, device="cuda") -> "DeviceCSR":
        import torch
        out = DeviceCSR(rows, cols,
                        torch.zeros(rows + 1, dtype=torch.int32, device=device),
                        torch.zeros(max(nnz, 1), dtype=torch.int32, device=device),
                        torch.zeros(max(nnz, 1), dtype=torch.float32, device=device))
        torch.cuda.synchronize(device)
        return out

    def struct(self, nnz: int | None = None) -> L.CsrMatrix:
        m = L.CsrMatrix()
        m.rows, m.cols = self.rows, self.cols
        m.nnz = self.nnz if nnz is None else nnz
        m.row_ptr = self.row_ptr.data_ptr()
        m.col_idx = self.col_idx.data_ptr()
        m.values = self.values.data_ptr()
        m.dtype, m.format, m.owns_data = L.DTYPE_FP32, L.FORMAT_CSR, 0
        return m

    def to_host(self, nnz: int | None = None) -> CSR:
        n = self.nnz if nnz is None else nnz
        return CSR(self.rows, self.cols, self.row_ptr.cpu().numpy(),
                   self.col_idx[:n].cpu().numpy(), self.values[:n].cpu().numpy())


class Descriptor:
    """rvsp_spgemm_descr_t with its lifecycle in one object."""

    def __init__(self, algo: int = L.ALGO_DEFAULT, memory: int = L.MEM_HOST,
                 stream=None, profiling: bool = False):
        self.lib = L.load()
        self.h = C.c_void_p()
        L.check(self.lib.rvsp_spgemm_descr_create(C.byref(self.h)), "descr_create")
        if algo != L.ALGO_DEFAULT:
            L.check(self.lib.rvsp_spgemm_set_algo(self.h, algo), "set_algo")
        if memory != L.MEM_HOST:
            L.check(self.lib.rvsp_spgemm_set_memory_space(self.h, memory),
                    "set_memory_space")
        if stream is not None:
            ptr = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
            # torch reports the legacy default stream as 0, which the C API
            # reads as "the descriptor's own stream"; name it explicitly.
            ptr = ptr or CUDA_STREAM_LEGACY
            L.check(self.lib.rvsp_spgemm_set_stream(self.h, C.c_void_p(ptr)),
                    "set_stream")
        if profiling:
            L.check(self.lib.rvsp_spgemm_set_profiling(self.h, 1), "set_profiling")
        self.memory = memory
        self.c_nnz = None
        self.ws_bytes = None
        self._keep = []

    def close(self):
        if self.h:
            self.lib.rvsp_spgemm_descr_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def work_estimation(self, A, B):
        a, b = A.struct(), B.struct()
        ws = C.c_size_t()
        nnz = C.c_int32()
        L.check(self.lib.rvsp_spgemm_work_estimation(self.h, C.byref(a), C.byref(b),
                                                     C.byref(ws), C.byref(nnz)),
                "work_estimation")
        self.c_nnz, self.ws_bytes = nnz.value, ws.value
        return ws.value, nnz.value

    def compute(self, A, B, Cm, workspace) -> None:
        a, b = A.struct(), B.struct()
        # an output C advertises its capacity, not its (not yet written) row_ptr
        c = Cm.struct(self.c_nnz) if isinstance(Cm, DeviceCSR) else \
            Cm.struct(nnz=int(Cm.col_idx.size))
        if isinstance(workspace, np.ndarray):
            wptr = workspace.ctypes.data
        elif hasattr(workspace, "data_ptr"):
            wptr = workspace.data_ptr()
        else:
            wptr = workspace
        L.check(self.lib.rvsp_spgemm_compute(self.h, C.byref(a), C.byref(b),
                                             C.byref(c), C.c_void_p(wptr)),
                "compute")

    def multiply(self, A: CSR, B: CSR) -> CSR:
        """Host memory space: estimate (if needed) + allocate C + compute."""
        if self.c_nnz is None:
            self.work_estimation(A, B)
        n = max(self.c_nnz, 1)
        Cm = CSR(A.rows, B.cols, np.zeros(A.rows + 1, np.int32),
                 np.zeros(n, np.int32), np.zeros(n, np.float32))
        ws = np.zeros(max(self.ws_bytes, 1), np.uint8)
        self.compute(A, B, Cm, ws)
        return CSR(Cm.rows, Cm.cols, Cm.row_ptr, Cm.col_idx[:self.c_nnz],
                   Cm.values[:self.c_nnz])

    def get_op_counts(self, n: int) -> np.ndarray:
        out = np.zeros(max(n, 1), np.int64)
        L.check(self.lib.rvsp_spgemm_get_op_counts(self.h, out.ctypes.data, n),
                "get_op_counts")
        return out[:n]

    def class_counts(self):
        sym = np.zeros(len(L.CLASS_NAMES), np.int32)
        num = np.zeros(len(L.CLASS_NAMES), np.int32)
        L.check(self.lib.rvsp_spgemm_get_class_counts(
            self.h, sym.ctypes.data, num.ctypes.data, len(L.CLASS_NAMES)),
            "get_class_counts")
        return dict(zip(L.CLASS_NAMES, sym.tolist())), dict(zip(L.CLASS_NAMES, num.tolist()))

    def phase_times(self, reset: bool = False):
        ms = np.zeros(len(L.PHASES), np.float64)
        ln = np.zeros(len(L.PHASES), np.int64)
        L.check(self.lib.rvsp_spgemm_get_phase_times(
            self.h, ms.ctypes.data, ln.ctypes.data, len(L.PHASES), int(reset)),
            "get_phase_times")
        return {p: (float(ms[i]), int(ln[i])) for i, p in enumerate(L.PHASES)}

    def invalidate_structure(self):
        self.lib.rvsp_spgemm_invalidate_structure(self.h)

    def synchronize(self):
        L.check(self.lib.rvsp_spgemm_synchronize(self.h), "synchronize")

    def set_model(self, model):
        """Row-binning model (rvsp.learn.RowModel) for ALGO_CUDA_LEARNED."""
        self._keep.append(model)
        L.check(self.lib.rvsp_spgemm_set_model(self.h, model.h), "set_model")

    def set_capacity_scale(self, scale: float):
        L.check(self.lib.rvsp_spgemm_set_capacity_scale(self.h, C.c_float(scale)),
                "set_capacity_scale")

    def set_merge_policy(self, policy: int):
        L.check(self.lib.rvsp_spgemm_set_merge_policy(self.h, policy), "set_merge_policy")

    def set_row_tiles(self, enable: bool):
        """Row tiles for numeric-only computes (on by default)."""
        L.check(self.lib.rvsp_spgemm_set_row_tiles(self.h, int(bool(enable))), "set_row_tiles")

    def set_pattern_kernels(self, enable: bool):
        """Compiled kernels for the largest row-tile patterns (on by default)."""
        L.check(self.lib.rvsp_spgemm_set_pattern_kernels(self.h, int(bool(enable))),
                "set_pattern_kernels")

    def set_shift_classes(self, enable):
        """Shift classes in work_estimation: False/0 off, True/1 where they pay
        (the default: large matrices of costly rows), 2 on any matrix whose
        rows are translates."""
        mode = 2 if enable == 2 else int(bool(enable))
        L.check(self.lib.rvsp_spgemm_set_shift_classes(self.h, mode), "set_shift_classes")

    def shift_rows(self) -> int:
        n = C.c_int32()
        L.check(self.lib.rvsp_spgemm_get_shift_rows(self.h, C.byref(n)), "shift_rows")
        return n.value

    def tiled_rows(self) -> int:
        n = C.c_int32()
        L.check(self.lib.rvsp_spgemm_get_tiled_rows(self.h, C.byref(n)), "tiled_rows")
        return n.value

    def overflow_rows(self) -> int:
        n = C.c_int32()
        L.check(self.lib.rvsp_spgemm_get_overflow_rows(self.h, C.byref(n)), "overflow_rows")
        return n.value

    def multiply_once(self, A, B):
        """rvsp_spgemm_multiply: C = A * B in one call.  Host memory space
        returns a host CSR; device memory space returns a DeviceResult."""
        a, b = A.struct(), B.struct()
        c = L.CsrMatrix()
        L.check(self.lib.rvsp_spgemm_multiply(self.h, C.byref(a), C.byref(b), C.byref(c)),
                "multiply")
        if self.memory == L.MEM_DEVICE:
            return DeviceResult(c)
        try:
            n = c.nnz
            rp = np.ctypeslib.as_array(C.cast(c.row_ptr, C.POINTER(C.c_int32)),
                                       shape=(c.rows + 1,)).copy()
            ci = np.ctypeslib.as_array(C.cast(c.col_idx, C.POINTER(C.c_int32)),
                                       shape=(max(n, 1),))[:n].copy()
            cv = np.ctypeslib.as_array(C.cast(c.values, C.POINTER(C.c_float)),
                                       shape=(max(n, 1),))[:n].copy()
            return CSR(c.rows, c.cols, rp, ci, cv)
        finally:
            self.lib.rvsp_csr_destroy(C.byref(c))


class DeviceResult:
    """A C produced in device memory by the library (owns_data = 2)."""

    def __init__(self, c: L.CsrMatrix):
        self.c = c
        self.rows, self.cols, self.nnz = c.rows, c.cols, c.nnz

    def to_host(self) -> CSR:
        import cuda.bindings.runtime as rt
        rp = np.zeros(self.rows + 1, np.int32)
        ci = np.zeros(max(self.nnz, 1), np.int32)
        cv = np.zeros(max(self.nnz, 1), np.float32)
        for dst, src, nb in ((rp, self.c.row_ptr, rp.nbytes),
                             (ci, self.c.col_idx, 4 * self.nnz),
                             (cv, self.c.values, 4 * self.nnz)):
            if nb:
                err, = rt.cudaMemcpy(dst.ctypes.data, src, nb,
                                     rt.cudaMemcpyKind.cudaMemcpyDeviceToHost)
                if int(err) != 0:
                    raise RuntimeError(f"cudaMemcpy failed ({int(err)})")
        return CSR(self.rows, self.cols, rp, ci[:self.nnz], cv[:self.nnz])

    def free(self):
        if self.c.row_ptr:
            L.load().rvsp_csr_destroy(C.byref(self.c))

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class Batch:
    """rvsp_spgemm_batch_t: many independent products computed together.

    Operands are host CSRs (memory=MEM_HOST) or DeviceCSRs (MEM_DEVICE).  The
    batch keeps references to them: change their values in place between
    computes (numeric-only repeats), never their structure."""

    def __init__(self, memory: int = L.MEM_HOST, stream=None, autotune: bool = False,
                 merge_policy: int | None = None, group_ops: int | None = None,
                 persistent: tuple | None = None):
        self.lib = L.load()
        self.h = C.c_void_p()
        L.check(self.lib.rvsp_spgemm_batch_create(C.byref(self.h)), "batch_create")
        if memory != L.MEM_HOST:
            L.check(self.lib.rvsp_spgemm_batch_set_memory_space(self.h, memory),
                    "batch_set_memory_space")
        if stream is not None:
            ptr = stream.cuda_stream if hasattr(stream, "cuda_stream") else stream
            L.check(self.lib.rvsp_spgemm_batch_set_stream(
                self.h, C.c_void_p(ptr or CUDA_STREAM_LEGACY)), "batch_set_stream")
        if autotune:
            L.check(self.lib.rvsp_spgemm_batch_set_autotune(self.h, 1), "batch_set_autotune")
        if merge_policy is not None:
            L.check(self.lib.rvsp_spgemm_batch_set_merge_policy(self.h, merge_policy),
                    "batch_set_merge_policy")
        if group_ops is not None:
            L.check(self.lib.rvsp_spgemm_batch_set_group_ops(self.h, group_ops),
                    "batch_set_group_ops")
        if persistent is not None:  # (merge rows per bin, blocks per SM)
            L.check(self.lib.rvsp_spgemm_batch_set_persistent(self.h, *persistent),
                    "batch_set_persistent")
        self.memory = memory
        self.operands = []
        self.total_nnz = None

    def add(self, A, B) -> int:
        a, b = A.struct(), B.struct()
        idx = C.c_int32()
        L.check(self.lib.rvsp_spgemm_batch_add(self.h, C.byref(a), C.byref(b),
                                               C.byref(idx)), "batch_add")
        self.operands.append((A, B))
        return idx.value

    def work_estimation(self) -> int:
        n = C.c_int64()
        L.check(self.lib.rvsp_spgemm_batch_work_estimation(self.h, C.byref(n)),
                "batch_work_estimation")
        self.total_nnz = n.value
        return n.value

    def compute(self) -> None:
        L.check(self.lib.rvsp_spgemm_batch_compute(self.h), "batch_compute")

    def synchronize(self) -> None:
        L.check(self.lib.rvsp_spgemm_batch_synchronize(self.h), "batch_synchronize")

    def nnz(self, i: int) -> int:
        n = C.c_int32()
        L.check(self.lib.rvsp_spgemm_batch_get_nnz(self.h, i, C.byref(n)), "batch_get_nnz")
        return n.value

    def result(self, i: int) -> CSR:
        """C_i copied to host arrays (rvsp_spgemm_batch_copy_result)."""
        A, B = self.operands[i]
        n = self.nnz(i)
        out = CSR(A.rows, B.cols, np.zeros(A.rows + 1, np.int32),
                  np.zeros(max(n, 1), np.int32), np.zeros(max(n, 1), np.float32))
        c = out.struct(nnz=max(n, 1))
        L.check(self.lib.rvsp_spgemm_batch_copy_result(self.h, i, C.byref(c)),
                "batch_copy_result")
        return CSR(out.rows, out.cols, out.row_ptr, out.col_idx[:n], out.values[:n])

    def copy_result_into(self, i: int, c: L.CsrMatrix) -> None:
        """rvsp_spgemm_batch_copy_result into a caller-built struct."""
        L.check(self.lib.rvsp_spgemm_batch_copy_result(self.h, i, C.byref(c)),
                "batch_copy_result")

    def view(self, i: int) -> L.CsrMatrix:
        """C_i as device arrays owned by the batch (rvsp_spgemm_batch_get_result)."""
        c = L.CsrMatrix()
        L.check(self.lib.rvsp_spgemm_batch_get_result(self.h, i, C.byref(c)),
                "batch_get_result")
        return c

    def stats(self):
        g, ops, pol, nodes = C.c_int32(), C.c_int64(), C.c_int32(), C.c_int32()
        L.check(self.lib.rvsp_spgemm_batch_get_stats(self.h, C.byref(g), C.byref(ops),
                                                     C.byref(pol), C.byref(nodes)),
                "batch_get_stats")
        return {"groups": g.value, "ops": ops.value, "merge_policy": pol.value,
                "graph_nodes": nodes.value}

    def tuning(self):
        """Merge policy, persistent shape and (autotuned) the timed shapes."""
        pol, rows, blocks, n = C.c_int32(), C.c_int32(), C.c_int32(), C.c_int32()
        ms = (C.c_float * 8)()
        L.check(self.lib.rvsp_spgemm_batch_get_tuning(self.h, C.byref(pol), C.byref(rows),
                                                      C.byref(blocks), ms, C.byref(n)),
                "batch_get_tuning")
        shapes = ["per-class", "persistent 128x2", "persistent 256x2", "persistent 256x1",
                  "persistent 64x4"]
        return {"merge_policy": pol.value, "persistent_merge_rows": rows.value,
                "persistent_blocks_per_sm": blocks.value,
                "shape_ms": {shapes[i]: float(ms[i]) for i in range(n.value)}}

    def close(self):
        if self.h:
            self.lib.rvsp_spgemm_batch_destroy(self.h)
            self.h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
