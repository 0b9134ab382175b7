"""Host CSR container and its view as an rvsp_csr_matrix_t."""
from __future__ import annotations

from dataclasses import dataclass

import numpy as np

from . import _lib as L


@dataclass
class CSR:
    """Canonical CSR matrix in host memory (int32 indices, float32 values)."""

    rows: int
    cols: int
    row_ptr: np.ndarray
    col_idx: np.ndarray
    values: np.ndarray

    def __post_init__(self):
        self.row_ptr = np.ascontiguousarray(self.row_ptr, dtype=np.int32)
        self.col_idx = np.ascontiguousarray(self.col_idx, dtype=np.int32)
        self.values = np.ascontiguousarray(self.values, dtype=np.float32)

    @property
    def nnz(self) -> int:
        return int(self.row_ptr[-1]) if self.row_ptr.size else 0

    def struct(self, nnz: int | None = None) -> L.CsrMatrix:
        """An rvsp_csr_matrix_t viewing these arrays (caller keeps self alive).
        nnz defaults to row_ptr[-1]; pass the capacity for an output C."""
        m = L.CsrMatrix()
        m.rows, m.cols = self.rows, self.cols
        m.nnz = self.nnz if nnz is None else nnz
        m.row_ptr = self.row_ptr.ctypes.data
        m.col_idx = self.col_idx.ctypes.data
        m.values = self.values.ctypes.data
        m.dtype, m.format, m.owns_data = L.DTYPE_FP32, L.FORMAT_CSR, 0
        return m

    def row_lengths(self) -> np.ndarray:
        return np.diff(self.row_ptr)

    def copy(self) -> "CSR":
        return CSR(self.rows, self.cols, self.row_ptr.copy(), self.col_idx.copy(),
                   self.values.copy())

    def with_values(self, values: np.ndarray) -> "CSR":
        return CSR(self.rows, self.cols, self.row_ptr, self.col_idx, values)

    def nbytes(self) -> int:
        return self.row_ptr.nbytes + self.col_idx.nbytes + self.values.nbytes

    def to_scipy(self):
        import scipy.sparse as sp
        return sp.csr_matrix((self.values, self.col_idx, self.row_ptr),
                             shape=(self.rows, self.cols))

    @staticmethod
    def from_scipy(m) -> "CSR":
        m = m.tocsr()
        m.sort_indices()
        return CSR(m.shape[0], m.shape[1], m.indptr, m.indices, m.data)

    def row_panel(self, r0: int, r1: int) -> "CSR":
        """Rows [r0, r1) as a CSR of its own (row_ptr rebased to 0)."""
        p0, p1 = int(self.row_ptr[r0]), int(self.row_ptr[r1])
        return CSR(r1 - r0, self.cols, self.row_ptr[r0:r1 + 1] - p0,
                   self.col_idx[p0:p1], self.values[p0:p1])


def intermediate_products(A: CSR, B: CSR) -> np.ndarray:
    """Per-row op counts ops_i = sum over A row i of |B row k| (int64)."""
    blen = np.diff(B.row_ptr).astype(np.int64)
    per_nz = blen[A.col_idx] if A.nnz else np.zeros(0, np.int64)
    out = np.zeros(A.rows, np.int64)
    if A.nnz:
        rows = np.repeat(np.arange(A.rows), np.diff(A.row_ptr))
        np.add.at(out, rows, per_nz)
    return out


def algorithmic_bytes(A: CSR, B: CSR, c_nnz: int) -> int:
    """Compulsory HBM bytes of one product: read A and B, write C."""
    return (4 * (A.rows + 1) + 8 * A.nnz + 4 * (B.rows + 1) + 8 * B.nnz +
            4 * (A.rows + 1) + 8 * int(c_nnz))
