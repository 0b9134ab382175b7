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

Exchanges (torch.distributed, NCCL on GPUs, gloo on CPU):
  broadcast_csr   B from one rank to all, once: its sizes, then row_ptr,
                  col_idx and values (four broadcasts);
  panel_offsets   one all-reduce of a per-panel nnz vector in which each
                  rank fills its own panels (every panel has one owner), so
                  it carries exactly the all-gather of the panels' nnz; its
                  exclusive scan places each panel in the global C.
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


def broadcast_csr(M, src: int = 0, device="cpu", group=None):
    """Every rank's copy of one CSR (B of a sharded product), sent once from
    rank src.  M is the matrix on rank src (a CSR) and is ignored elsewhere.
    Returns a DeviceCSR whose tensors live on `device` (the rank's GPU under
    NCCL, "cpu" under gloo)."""
    import torch
    import torch.distributed as dist

    from .api import DeviceCSR
    rank = dist.get_rank(group)
    meta = torch.zeros(3, dtype=torch.int64, device=device)
    if rank == src:
        meta[0], meta[1], meta[2] = int(M.rows), int(M.cols), int(M.nnz)
    dist.broadcast(meta, src, group=group)
    rows, cols, nnz = (int(x) for x in meta.tolist())
    if rank == src:
        rp = torch.from_numpy(np.ascontiguousarray(M.row_ptr, np.int32)).to(device)
        ci = torch.from_numpy(np.ascontiguousarray(M.col_idx, np.int32)).to(device)
        v = torch.from_numpy(np.ascontiguousarray(M.values, np.float32)).to(device)
    else:
        rp = torch.empty(rows + 1, dtype=torch.int32, device=device)
        ci = torch.empty(nnz, dtype=torch.int32, device=device)
        v = torch.empty(nnz, dtype=torch.float32, device=device)
    for t in (rp, ci, v):
        if t.numel():  # every rank knows the sizes, so all skip alike
            dist.broadcast(t, src, group=group)
    return DeviceCSR(rows, cols, rp, ci, v)


def panel_offsets(n_panels: int, local_nnz: dict, device="cpu", group=None) -> np.ndarray:
    """Start of every panel's entries in the whole C: int64, n_panels + 1
    entries, the last one nnz(C).  local_nnz maps this rank's panel indices
    to their nnz; every panel must belong to exactly one rank."""
    import torch
    import torch.distributed as dist
    t = torch.zeros(max(n_panels, 1), dtype=torch.int64, device=device)
    for i, n in local_nnz.items():
        t[int(i)] = int(n)
    dist.all_reduce(t, group=group)
    out = np.zeros(n_panels + 1, np.int64)
    np.cumsum(t.cpu().numpy()[:n_panels], out=out[1:])
    return out


def rows_in_global_row_ptr(panel_row_ptr, offset: int) -> np.ndarray:
    """A panel's row_ptr placed in the whole C: entries r0 + 1 .. r1 of the
    global C.row_ptr for the panel's rows [r0, r1) (int64)."""
    return offset + np.asarray(panel_row_ptr, np.int64)[1:]
