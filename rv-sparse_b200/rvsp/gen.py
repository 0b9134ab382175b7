"""Seeded synthetic CSR generators for the benchmark and test workloads.

Every generator is deterministic in its seed (numpy PCG64).  Columns within
a row are distinct and ascending, so every output is canonical CSR.

  uniform_rows     exactly k columns per row, uniform without replacement
  laplacian_2d     5-point Laplacian on a g x g grid (diag 4, off -1)
  stencil_3d_27    27-point stencil on a g^3 grid (diag 26, off -1)
  rmat             R-MAT graph, duplicates merged, values U(0, 1]
  poisson_rows     Poisson(mu) row lengths clipped to [0, n], uniform columns
  batched_products the 512-product batch: n log-uniform in [256, 65536],
                   mu uniform in [8, 32]
  random_csr       small irregular matrices for parity tests
"""
from __future__ import annotations

import numpy as np

from .csr import CSR


def _rng(seed: int) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(seed))


def _distinct_sorted_columns(rng, lengths: np.ndarray, n_cols: int) -> np.ndarray:
    """For each row, lengths[r] distinct columns in [0, n_cols), ascending."""
    lengths = np.asarray(lengths, dtype=np.int64)
    if np.any(lengths > n_cols):
        raise ValueError("row longer than the number of columns")
    total = int(lengths.sum())
    row_of = np.repeat(np.arange(lengths.size, dtype=np.int64), lengths)
    starts = np.concatenate(([0], np.cumsum(lengths)[:-1]))
    cols = np.empty(total, np.int64)
    # Rejection (draw with replacement, redraw rows that drew a repeat) is
    # used only where a row draws no repeat with probability >= ~0.88
    # (k^2 <= n/4); longer rows take the k smallest of n random keys.
    crowded = np.nonzero(lengths * lengths * 4 > n_cols)[0]
    for r in crowded:
        k = int(lengths[r])
        keys = rng.random(n_cols)
        cols[starts[r]:starts[r] + k] = np.sort(np.argpartition(keys, k - 1)[:k])
    todo = np.nonzero((lengths * lengths * 4 <= n_cols) & (lengths > 0))[0]
    while todo.size:
        sel_len = lengths[todo]
        sel_off = np.concatenate(([0], np.cumsum(sel_len)[:-1]))
        idx = (np.repeat(starts[todo], sel_len) +
               np.arange(int(sel_len.sum())) - np.repeat(sel_off, sel_len))
        draw = rng.integers(0, n_cols, size=idx.size, dtype=np.int64)
        key = row_of[idx] * n_cols + draw
        order = np.argsort(key, kind="stable")
        key_sorted = key[order]
        cols[idx] = key_sorted - row_of[idx] * n_cols  # idx is row-ordered
        dup = np.zeros(idx.size, bool)
        dup[1:] = key_sorted[1:] == key_sorted[:-1]
        todo = np.unique(row_of[idx][dup])
    return cols.astype(np.int32)


def uniform_rows(rows: int, cols: int, k: int, seed: int) -> CSR:
    rng = _rng(seed)
    lengths = np.full(rows, k, np.int64)
    col_idx = _distinct_sorted_columns(rng, lengths, cols)
    values = rng.uniform(-1.0, 1.0, size=rows * k).astype(np.float32)
    row_ptr = np.arange(0, rows * k + 1, k, dtype=np.int64)
    return CSR(rows, cols, row_ptr, col_idx, values)


def _stencil(shape, offsets, diag: float, off: float) -> CSR:
    """CSR of a constant-coefficient stencil on a row-major grid; offsets are
    (d0, d1, ...) tuples listed in ascending column order."""
    dims = np.array(shape, np.int64)
    n = int(np.prod(dims))
    idx = np.arange(n, dtype=np.int64)
    coords = np.unravel_index(idx, shape)
    strides = np.array([int(np.prod(dims[i + 1:])) for i in range(len(shape))], np.int64)
    valid = []
    for o in offsets:
        ok = np.ones(n, bool)
        for ax, d in enumerate(o):
            if d:
                c = coords[ax] + d
                ok &= (c >= 0) & (c < dims[ax])
        valid.append(ok)
    counts = np.zeros(n, np.int64)
    for ok in valid:
        counts += ok
    row_ptr = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    nnz = int(row_ptr[-1])
    col_idx = np.empty(nnz, np.int32)
    values = np.empty(nnz, np.float32)
    cursor = row_ptr[:-1].copy()
    for o, ok in zip(offsets, valid):
        delta = int(np.dot(np.array(o, np.int64), strides))
        r = idx[ok]
        pos = cursor[r]
        col_idx[pos] = (r + delta).astype(np.int32)
        values[pos] = diag if delta == 0 else off
        cursor[r] += 1
    return CSR(n, n, row_ptr, col_idx, values)


def laplacian_2d(g: int) -> CSR:
    offs = [(-1, 0), (0, -1), (0, 0), (0, 1), (1, 0)]
    return _stencil((g, g), offs, 4.0, -1.0)


def stencil_3d_27(g: int) -> CSR:
    offs = [(dz, dy, dx) for dz in (-1, 0, 1) for dy in (-1, 0, 1) for dx in (-1, 0, 1)]
    return _stencil((g, g, g), offs, 26.0, -1.0)


def rmat(scale: int, edge_factor: int, probs=(0.57, 0.19, 0.19, 0.05),
         seed: int = 1) -> CSR:
    """R-MAT: each of edge_factor * 2^scale edges picks one quadrant per level."""
    rng = _rng(seed)
    n = 1 << scale
    m = edge_factor * n
    a, b, c, _ = probs
    row = np.zeros(m, np.int64)
    col = np.zeros(m, np.int64)
    for _level in range(scale):
        u = rng.random(m)
        rbit = u >= a + b
        cbit = ((u >= a) & (u < a + b)) | (u >= a + b + c)
        row = (row << 1) | rbit
        col = (col << 1) | cbit
    key = row * n + col
    key.sort()
    if key.size:
        key = key[np.concatenate(([True], key[1:] != key[:-1]))]
    r = key // n
    cl = (key % n).astype(np.int32)
    counts = np.bincount(r, minlength=n)
    row_ptr = np.zeros(n + 1, np.int64)
    np.cumsum(counts, out=row_ptr[1:])
    values = (1.0 - rng.random(key.size)).astype(np.float32)  # U(0, 1]
    return CSR(n, n, row_ptr, cl, values)


def poisson_rows(n: int, mu: float, seed: int, n_cols: int | None = None) -> CSR:
    rng = _rng(seed)
    n_cols = n if n_cols is None else n_cols
    lengths = np.minimum(rng.poisson(mu, size=n), n_cols).astype(np.int64)
    col_idx = _distinct_sorted_columns(rng, lengths, n_cols)
    values = rng.uniform(-1.0, 1.0, size=col_idx.size).astype(np.float32)
    row_ptr = np.zeros(n + 1, np.int64)
    np.cumsum(lengths, out=row_ptr[1:])
    return CSR(n, n_cols, row_ptr, col_idx, values)


def batched_products(count: int = 512, seed: int = 7, n_lo: int = 256,
                     n_hi: int = 65536, mu_lo: float = 8.0, mu_hi: float = 32.0):
    """count square products (A_i, B_i): n log-uniform in [n_lo, n_hi],
    Poisson(mu) row lengths with mu uniform in [mu_lo, mu_hi]."""
    rng = _rng(seed)
    out = []
    for i in range(count):
        n = int(round(float(np.exp(rng.uniform(np.log(n_lo), np.log(n_hi))))))
        mu = float(rng.uniform(mu_lo, mu_hi))
        A = poisson_rows(n, mu, seed * 1_000_003 + 2 * i)
        B = poisson_rows(n, mu, seed * 1_000_003 + 2 * i + 1)
        out.append((A, B))
    return out


def random_csr(rows: int, cols: int, seed: int, mean_len: float = 4.0,
               empty_frac: float = 0.1, heavy_rows: int = 0,
               heavy_len: int = 0, value_kind: str = "uniform") -> CSR:
    """Irregular test matrix: geometric-ish row lengths, some empty rows, and
    optionally a few heavy rows; values uniform[-1, 1] or small integers."""
    rng = _rng(seed)
    lengths = rng.poisson(mean_len, size=rows).astype(np.int64)
    lengths[rng.random(rows) < empty_frac] = 0
    if heavy_rows:
        hr = rng.choice(rows, size=min(heavy_rows, rows), replace=False)
        lengths[hr] = heavy_len
    lengths = np.minimum(lengths, cols)
    col_idx = _distinct_sorted_columns(rng, lengths, cols)
    if value_kind == "int":
        values = rng.integers(-4, 5, size=col_idx.size).astype(np.float32)
    else:
        values = rng.uniform(-1.0, 1.0, size=col_idx.size).astype(np.float32)
    row_ptr = np.zeros(rows + 1, np.int64)
    np.cumsum(lengths, out=row_ptr[1:])
    return CSR(rows, cols, row_ptr, col_idx, values)
