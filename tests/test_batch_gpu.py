"""Batches of independent products (rvsp_spgemm_batch_*).

Bar: every C_i bit-exact against the oracle's product of its own A_i and
B_i, on the first compute and on numeric-only repeats (graph replays) after
the values change in place; across group boundaries; in both memory spaces;
with the autotuned merge policy; and the same errors as the descriptor API
for invalid operands.
"""
import numpy as np
import pytest

from oracle import oracle
from rvsp import Batch, CSR, DeviceCSR, gen
from rvsp import _lib as L

pytestmark = pytest.mark.gpu


def assert_exact(got: CSR, A: CSR, B: CSR, what: str):
    rp, ci, cv, _ = oracle.spgemm(A, B)
    assert np.array_equal(got.row_ptr, rp), f"row_ptr {what}"
    assert np.array_equal(got.col_idx, ci), f"col_idx {what}"
    assert np.array_equal(got.values.view(np.uint32), cv.view(np.uint32)), f"values {what}"


def uneven_products(count=20, seed=3, n_hi=6000):
    """Mixed sizes, plus one product with long and empty rows."""
    prods = gen.batched_products(count=count, seed=seed, n_lo=16, n_hi=n_hi)
    A = gen.random_csr(700, 500, seed + 1, mean_len=5.0, heavy_rows=4, heavy_len=400)
    B = gen.random_csr(500, 9000, seed + 2, mean_len=30.0, heavy_rows=3, heavy_len=6000)
    prods.insert(count // 2, (A, B))
    return prods


def redraw(M: CSR, rng):
    M.values[:] = rng.uniform(-1.0, 1.0, M.values.size).astype(np.float32)


def test_batch_host_first_and_repeats():
    prods = uneven_products()
    rng = np.random.default_rng(5)
    with Batch() as b:
        for A, B in prods:
            b.add(A, B)
        total = b.work_estimation()
        assert total == sum(int(oracle.spgemm(A, B)[0][-1]) for A, B in prods)
        b.compute()
        for i, (A, B) in enumerate(prods):
            assert_exact(b.result(i), A, B, f"product {i} first compute")
        for rep in range(3):  # numeric-only: capture, then replays
            for A, B in prods:
                redraw(A, rng)
                redraw(B, rng)
            b.compute()
            for i, (A, B) in enumerate(prods):
                assert_exact(b.result(i), A, B, f"product {i} repeat {rep}")
        assert b.stats()["graph_nodes"] > 0


def test_batch_device_memory_and_views():
    import torch
    prods = uneven_products(count=12, seed=7)
    dev = [(DeviceCSR.from_host(A), DeviceCSR.from_host(B)) for A, B in prods]
    with Batch(memory=L.MEM_DEVICE) as b:
        for dA, dB in dev:
            b.add(dA, dB)
        b.work_estimation()
        b.compute()
        b.synchronize()
        for i, (A, B) in enumerate(prods):
            assert_exact(b.result(i), A, B, f"device product {i}")
        v = b.view(3)
        assert v.rows == prods[3][0].rows and v.nnz == b.nnz(3)
        for rep in range(2):
            for (A, B), (dA, dB) in zip(prods, dev):
                A.values[:] = (A.values * np.float32(-1.25)).astype(np.float32)
                dA.values.copy_(torch.from_numpy(A.values))
            torch.cuda.synchronize()
            b.compute()
            b.synchronize()
            for i, (A, B) in enumerate(prods):
                assert_exact(b.result(i), A, B, f"device product {i} repeat {rep}")


def test_batch_groups_split():
    prods = uneven_products(count=16, seed=11, n_hi=3000)
    with Batch(group_ops=200_000) as b:
        for A, B in prods:
            b.add(A, B)
        b.work_estimation()
        assert b.stats()["groups"] > 2
        b.compute()
        for i, (A, B) in enumerate(prods):
            assert_exact(b.result(i), A, B, f"grouped product {i}")


def test_batch_merge_classes_and_autotune():
    # 40 products of 1000 short rows: 40,000 rows in one group, enough for
    # the merge classes under the automatic policy.
    prods = [(gen.poisson_rows(1000, 4.0, 100 + i), gen.poisson_rows(1000, 6.0, 200 + i))
             for i in range(40)]
    with Batch(autotune=True) as b:
        for A, B in prods:
            b.add(A, B)
        b.work_estimation()
        st = b.stats()
        assert st["groups"] == 1 and st["merge_policy"] in (0, 1, 2)
        b.compute()
        b.compute()  # a numeric-only repeat with the chosen policy
        for i, (A, B) in enumerate(prods):
            assert_exact(b.result(i), A, B, f"autotuned product {i}")


def test_batch_errors():
    A = gen.random_csr(50, 40, 1, mean_len=3.0)
    B = gen.random_csr(40, 30, 2, mean_len=3.0)
    with Batch() as b:
        with pytest.raises(L.RvspError) as e:
            b.add(A, gen.random_csr(41, 30, 3))
        assert e.value.status == L.ERROR_INVALID_ARGUMENT
        bad = A.copy()
        r = int(np.argmax(np.diff(bad.row_ptr) >= 2))
        s = bad.row_ptr[r]
        bad.col_idx[s], bad.col_idx[s + 1] = bad.col_idx[s + 1], bad.col_idx[s]
        b.add(A, B)
        b.add(bad, B)
        with pytest.raises(L.RvspError) as e:
            b.work_estimation()
        assert e.value.status == L.ERROR_INVALID_CSR
    with Batch() as b:
        b.add(A, B)
        b.work_estimation()
        with pytest.raises(L.RvspError) as e:
            b.add(A, B)
        assert e.value.status == L.ERROR_INVALID_ARGUMENT
    with Batch() as b:
        with pytest.raises(L.RvspError):
            b.work_estimation()  # empty batch


@pytest.mark.parametrize("shape", [(128, 2), (256, 1), (64, 4)])
def test_batch_persistent_pass(shape):
    # numeric-only repeats through the persistent kernel (one launch pulling
    # row bins from a global queue), captured and replayed: bit-exact
    prods = uneven_products(count=24, seed=41)
    rng = np.random.default_rng(6)
    with Batch(persistent=shape) as b:
        for A, B in prods:
            b.add(A, B)
        b.work_estimation()
        b.compute()
        for rep in range(3):
            for A, B in prods:
                redraw(A, rng)
                redraw(B, rng)
            b.compute()
            for i, (A, B) in enumerate(prods):
                assert_exact(b.result(i), A, B, f"product {i} repeat {rep}")
        t = b.tuning()
        assert t["persistent_merge_rows"] == shape[0]
        assert t["persistent_blocks_per_sm"] == shape[1]


def test_batch_autotune_times_every_shape():
    prods = uneven_products(count=16, seed=43)
    rng = np.random.default_rng(8)
    with Batch(autotune=True) as b:
        for A, B in prods:
            b.add(A, B)
        b.work_estimation()
        t = b.tuning()
        assert len(t["shape_ms"]) == 5 and all(v > 0 for v in t["shape_ms"].values())
        best = min(t["shape_ms"], key=t["shape_ms"].get)
        assert (t["persistent_merge_rows"] == 0) == (best == "per-class")
        b.compute()
        for rep in range(2):
            for A, B in prods:
                redraw(A, rng)
                redraw(B, rng)
            b.compute()
        for i, (A, B) in enumerate(prods):
            assert_exact(b.result(i), A, B, f"product {i}")
