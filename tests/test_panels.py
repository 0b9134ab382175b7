"""Row panels (rvsp.panels): the host logic that splits a product whose C
exceeds one call into row panels, and shards panels across ranks.

CPU only.  The two-rank tests run real torch.distributed ranks on the gloo
backend: each rank computes its panels' structure with the oracle, the ranks
all-gather the panels' row pointers (the one exchange the sharding needs),
and every rank must rebuild exactly the whole product's C.row_ptr.  The
exchange test sends B from rank 0 to the other rank (broadcast_csr) and
places each rank's rows in C.row_ptr from one all-reduce of per-panel nnz
(panel_offsets).
"""
import os

import numpy as np
import pytest

from oracle import oracle
from rvsp import gen, intermediate_products
from rvsp.panels import (assign_panels, broadcast_csr, global_row_ptr, panel_bounds,
                         panel_bounds_fast, panel_offsets, rows_in_global_row_ptr)


def test_panel_bounds_cover_rows_within_limit():
    rng = np.random.default_rng(1)
    for trial in range(20):
        ops = rng.integers(0, 50, size=int(rng.integers(1, 400))).astype(np.int64)
        ops[rng.random(ops.size) < 0.05] = 500  # rows above the limit
        limit = int(rng.integers(40, 300))
        b = panel_bounds(ops, limit)
        assert b == panel_bounds_fast(ops, limit), trial
        assert b[0][0] == 0 and b[-1][1] == ops.size
        assert all(x[1] == y[0] for x, y in zip(b, b[1:]))
        for r0, r1 in b:
            assert r1 > r0
            assert ops[r0:r1].sum() <= limit or r1 - r0 == 1


def test_assign_panels_balanced_and_complete():
    ops = np.random.default_rng(2).integers(0, 1000, size=5000).astype(np.int64)
    b = panel_bounds_fast(ops, 20000)
    per = assign_panels(b, ops, 3)
    flat = sorted(i for r in per for i in r)
    assert flat == list(range(len(b)))
    loads = [sum(int(ops[b[i][0]:b[i][1]].sum()) for i in r) for r in per]
    assert max(loads) - min(loads) <= 20000


def test_global_row_ptr_matches_whole_product():
    A = gen.rmat(11, 16, seed=5)
    ops = intermediate_products(A, A)
    b = panel_bounds_fast(ops, int(ops.sum()) // 7)
    rps = {i: oracle.spgemm(A.row_panel(r0, r1), A)[0] for i, (r0, r1) in enumerate(b)}
    assert np.array_equal(global_row_ptr(b, rps), oracle.spgemm(A, A)[0])


def _rank_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        A = gen.rmat(11, 16, seed=6)
        ops = intermediate_products(A, A)
        b = panel_bounds_fast(ops, int(ops.sum()) // 9)
        mine = assign_panels(b, ops, world)[rank]
        local = {i: oracle.spgemm(A.row_panel(*b[i]), A)[0].tolist() for i in mine}
        gathered = [None] * world
        dist.all_gather_object(gathered, local)
        rps = {}
        for g in gathered:
            rps.update({int(k): v for k, v in g.items()})
        full = global_row_ptr(b, rps)
        ok = np.array_equal(full, oracle.spgemm(A, A)[0]) and len(rps) == len(b)
        out.put((rank, bool(ok), len(mine)))
    finally:
        dist.destroy_process_group()


def test_two_rank_panel_sharding_gloo():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0], codes
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert all(ok for _, ok, _ in res), res
    assert all(n > 0 for _, _, n in res)


def _rank_exchange_main(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        src = gen.rmat(11, 16, seed=7) if rank == 0 else None
        B = broadcast_csr(src, src=0, device="cpu").to_host()
        ref = gen.rmat(11, 16, seed=7)  # the checker's own copy
        copy_ok = (B.rows, B.cols) == (ref.rows, ref.cols) and all(
            np.array_equal(x, y) for x, y in ((B.row_ptr, ref.row_ptr),
                                              (B.col_idx, ref.col_idx),
                                              (B.values, ref.values)))
        ops = intermediate_products(B, B)
        b = panel_bounds_fast(ops, int(ops.sum()) // 9)
        mine = assign_panels(b, ops, world)[rank]
        rps = {i: oracle.spgemm(B.row_panel(*b[i]), B)[0] for i in mine}
        offs = panel_offsets(len(b), {i: int(rp[-1]) for i, rp in rps.items()})
        segs = {i: rows_in_global_row_ptr(rp, int(offs[i])).tolist() for i, rp in rps.items()}
        gathered = [None] * world  # checking only: every rank's placed rows
        dist.all_gather_object(gathered, segs)
        full = np.zeros(B.rows + 1, np.int64)
        seen = 0
        for g in gathered:
            for i, seg in g.items():
                r0, r1 = b[int(i)]
                full[r0 + 1:r1 + 1] = seg
                seen += 1
        whole = oracle.spgemm(B, B)[0]
        ok = seen == len(b) and np.array_equal(full, whole) and int(offs[-1]) == int(whole[-1])
        out.put((rank, bool(copy_ok), bool(ok), len(mine)))
    finally:
        dist.destroy_process_group()


def test_two_rank_broadcast_and_panel_offsets_gloo():
    import multiprocessing as mp
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_exchange_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    codes = [p.exitcode for p in procs]
    for p in procs:
        if p.is_alive():
            p.kill()
    assert codes == [0, 0], codes
    res = sorted(q.get(timeout=10) for _ in range(2))
    assert all(copy_ok for _, copy_ok, _, _ in res), res
    assert all(ok for _, _, ok, _ in res), res
    assert all(n > 0 for _, _, _, n in res)
