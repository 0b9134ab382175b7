"""Seeded inputs for the FP64 and INT8 -> INT32 parity tests.

Each case is (kind, A, B) with A and B as (rows, cols, row_ptr, col_idx,
values) tuples: "f64" cases carry float64 values, "i8" cases int8 values.
The cases include entries that cancel exactly to zero (the legacy kernels
drop those), empty rows, and rows of B that are empty.
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

sys.path.insert(0, str(Path(__file__).resolve().parents[2] / "rv-sparse_b200"))

from rvsp import gen  # noqa: E402


def _t(M, values):
    return (M.rows, M.cols, M.row_ptr, M.col_idx, values)


def cases() -> dict:
    rng = np.random.default_rng(777)
    out = {}
    A = gen.uniform_rows(300, 200, 8, 11)
    B = gen.uniform_rows(200, 250, 6, 12)
    out["f64_uniform"] = ("f64", _t(A, rng.uniform(-1, 1, A.nnz)),
                          _t(B, rng.uniform(-1, 1, B.nnz)))
    # small integers as doubles: many sums cancel to exactly zero
    out["f64_cancel"] = ("f64", _t(A, rng.integers(-2, 3, A.nnz).astype(np.float64)),
                         _t(B, rng.integers(-2, 3, B.nnz).astype(np.float64)))
    L = gen.laplacian_2d(24)
    out["f64_laplace"] = ("f64", _t(L, L.values.astype(np.float64)),
                          _t(L, L.values.astype(np.float64)))
    P = gen.poisson_rows(500, 6.0, 13)  # empty rows included
    Q = gen.poisson_rows(500, 3.0, 14)
    out["f64_poisson"] = ("f64", _t(P, rng.standard_normal(P.nnz)),
                          _t(Q, rng.standard_normal(Q.nnz)))
    out["i8_uniform"] = ("i8", _t(A, rng.integers(-128, 128, A.nnz).astype(np.int8)),
                         _t(B, rng.integers(-128, 128, B.nnz).astype(np.int8)))
    out["i8_cancel"] = ("i8", _t(A, rng.integers(-1, 2, A.nnz).astype(np.int8)),
                        _t(B, rng.integers(-1, 2, B.nnz).astype(np.int8)))
    out["i8_poisson"] = ("i8", _t(P, rng.integers(-5, 6, P.nnz).astype(np.int8)),
                         _t(Q, rng.integers(-5, 6, Q.nnz).astype(np.int8)))
    return out


def wrap_case():
    """One output entry summing 140,000 products 127 x 127 (2.26e9): past
    INT32_MAX, so the int32 sum wraps."""
    n = 140000
    a = (1, n, np.array([0, n], np.int32), np.arange(n, dtype=np.int32),
         np.full(n, 127, np.int8))
    b = (n, 1, np.arange(n + 1, dtype=np.int32), np.zeros(n, np.int32),
         np.full(n, 127, np.int8))
    return a, b
