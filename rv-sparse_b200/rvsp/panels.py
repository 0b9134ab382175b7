"""Row panels of A: the unit of work for products whose C does not fit one
call (nnz(C) beyond int32, or beyond one GPU's memory), and the unit of
sharding across GPUs.

C's rows are independent, so C = A x B is the row-wise concatenation of the
panel products A[r0:r1] x B.  A panel is a valid CSR of its own (row_ptr
rebased to 0; CSR.row_panel), and its product's op count bounds its nnz(C),
so panels of at most 2^31 - 1 ops always fit an int32 row_ptr.  Across
ranks, each rank takes whole panels (no data crosses GPUs inside a product;
every rank holds all of B) and the only exchange is one all-gather of each
panel's nnz, from which every rank knows where its rows sit in the global
C.row_ptr.
"""
from __future__ import annotations

import numpy as np


def panel_bounds(ops: np.ndarray, max_ops: int) -> list[tuple[int, int]]:
    """Consecutive row ranges [r0, r1) covering every row, each with at most
    max_ops products (a single row with more gets a panel of its own)."""
    if max_ops <= 0:
        raise ValueError("max_ops must be positive")
    n = int(ops.size)
    bounds = []
    r0, acc = 0, 0
    for r in range(n):
        o = int(ops[r])
        if r > r0 and acc + o > max_ops:
            bounds.append((r0, r))
            r0, acc = r, 0
        acc += o
    if n and r0 < n:
        bounds.append((r0, n))
    return bounds


def panel_bounds_fast(ops: np.ndarray, max_ops: int) -> list[tuple[int, int]]:
    """panel_bounds for long row counts, in O(panels log rows)."""
    if max_ops <= 0:
        raise ValueError("max_ops must be positive")
    cs = np.concatenate([[0], np.cumsum(ops.astype(np.int64))])
    n = int(ops.size)
    bounds = []
    r0 = 0
    while r0 < n:
        # the last r1 with cs[r1] - cs[r0] <= max_ops, at least r0 + 1
        r1 = int(np.searchsorted(cs, cs[r0] + max_ops, side="right")) - 1
        r1 = max(r1, r0 + 1)
        bounds.append((r0, min(r1, n)))
        r0 = min(r1, n)
    return bounds


def assign_panels(bounds: list[tuple[int, int]], ops: np.ndarray,
                  world: int) -> list[list[int]]:
    """Panel indices per rank, balancing op counts (largest panel first to
    the least loaded rank); each rank's list is in row order."""
    cs = np.concatenate([[0], np.cumsum(ops.astype(np.int64))])
    load = [(0, r) for r in range(world)]
    out: list[list[int]] = [[] for _ in range(world)]
    weights = [(int(cs[b] - cs[a]), i) for i, (a, b) in enumerate(bounds)]
    for w, i in sorted(weights, key=lambda x: (-x[0], x[1])):
        load.sort()
        l0, r = load[0]
        out[r].append(i)
        load[0] = (l0 + w, r)
    return [sorted(x) for x in out]


def global_row_ptr(bounds: list[tuple[int, int]], panel_row_ptrs: dict) -> np.ndarray:
    """C.row_ptr of the whole product from every panel's own row_ptr (keyed
    by panel index, e.g. after an all-gather); int64, since the whole C may
    exceed int32."""
    n = bounds[-1][1] if bounds else 0
    out = np.zeros(n + 1, np.int64)
    base = 0
    for i, (r0, r1) in enumerate(bounds):
        rp = np.asarray(panel_row_ptrs[i], np.int64)
        out[r0 + 1:r1 + 1] = base + rp[1:]
        base += int(rp[-1])
    return out
