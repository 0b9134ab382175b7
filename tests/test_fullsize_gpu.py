"""Full-size parity on the benchmark configurations.

The reference's bar for a product is an exact structure and its values
(tests/test_spgemm_reference_f32.c:132-150); its reuse contract is that a
numeric-only compute after the values change gives the product of the new
values (tests/test_spgemm_descr_f32.c:196-217).  Here every path the bench
times is held to the reference library itself, bit for bit, at the sizes the
bench runs:

* the 128^3 27-point stencil (n = 2,097,152, nnz(C) = 254,840,104): plain
  and learned full products, then numeric-only repeats with perturbed
  values, through the row tiles and through the term tables;
* all 512 products of the batch, after a numeric-only graph replay;
* the learned path on the 1024^2 Laplacian and the uniform 4096 product.

The reference library (oracle/_ref) is the checker; the C restatement of it
stands in when the library was not built.
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

from oracle import oracle
from rvsp import Batch, Descriptor, DeviceCSR, gen
from rvsp import _lib as L
from rvsp.learn import RowModel, weights_for

pytestmark = [pytest.mark.gpu, pytest.mark.slow]


def _bits(x):
    return np.ascontiguousarray(x, np.float32).view(np.uint32)


def _ref_product(A, B):
    if oracle.ref_available():
        st, rp, ci, cv = oracle.ref_spgemm(A, B)
        assert st == 0
        return rp, ci, cv
    rp, ci, cv, _ = oracle.spgemm(A, B)
    return rp, ci, cv


def _ref_job(A, sets):
    """Reference descriptor: first compute on A's values, then one
    numeric-only compute per value array (B is A)."""
    if oracle.ref_available():
        st, rp, ci, first, every = oracle.ref_job(A, A, [(v, v) for v in sets],
                                                  keep_all=True)
        assert st == 0
        return rp, ci, first, every
    rp, ci, first, _ = oracle.spgemm(A, A)
    every = [oracle.numeric_f32(A.with_values(v), A.with_values(v), rp, ci) for v in sets]
    return rp, ci, first, every


def _assert_same(dC, n, rp, ci, cv, what):
    import torch
    torch.cuda.synchronize()
    assert np.array_equal(dC.row_ptr.cpu().numpy(), rp), f"row_ptr {what}"
    assert np.array_equal(dC.col_idx[:n].cpu().numpy(), ci), f"col_idx {what}"
    got = dC.values[:n].cpu().numpy()
    bad = int((_bits(got) != _bits(cv)).sum())
    assert bad == 0, f"values {what}: {bad} differ"


def test_stencil_128_plain_learned_and_repeats():
    import torch
    A = gen.stencil_3d_27(128)
    rng = np.random.default_rng(2024)
    sets = [(A.values + rng.uniform(-0.01, 0.01, A.nnz)).astype(np.float32) for _ in range(3)]
    rp, ci, first, every = _ref_job(A, sets)
    dA = DeviceCSR.from_host(A)
    model = RowModel(path=weights_for("stencil3d"))
    n = int(rp[-1])
    for algo in (L.ALGO_CUDA_PLAIN, L.ALGO_CUDA_LEARNED):
        with Descriptor(algo=algo, memory=L.MEM_DEVICE) as d:
            if algo == L.ALGO_CUDA_LEARNED:
                d.set_model(model)
            ws_b, nn = d.work_estimation(dA, dA)
            assert nn == n
            dC = DeviceCSR.empty(A.rows, A.cols, n)
            ws = torch.zeros(max(ws_b, 1), dtype=torch.uint8, device="cuda")
            d.compute(dA, dA, dC, ws)
            d.synchronize()
            _assert_same(dC, n, rp, ci, first, f"algo {algo} first compute")
            if algo != L.ALGO_CUDA_LEARNED:
                del dC
                continue
            # numeric-only repeats: two through the row tiles, one through
            # the term tables alone
            for k, v in enumerate(sets):
                d.set_row_tiles(k < 2)
                dA.values.copy_(torch.from_numpy(v))
                torch.cuda.synchronize()
                d.compute(dA, dA, dC, ws)
                d.synchronize()
                if k < 2:
                    assert d.tiled_rows() > 1_900_000
                else:
                    assert d.tiled_rows() == 0
                _assert_same(dC, n, rp, ci, every[k], f"repeat {k}")
            dA.values.copy_(torch.from_numpy(A.values))
            del dC


def test_batch512_every_product_after_graph_replay():
    prods = gen.batched_products(count=512, seed=7)
    rng = np.random.default_rng(17)
    with Batch(autotune=False) as b:
        for A, B in prods:
            b.add(A, B)
        b.work_estimation()
        b.compute()
        for rep in range(2):  # the first numeric-only compute is captured, the next replayed
            for A, B in prods:
                A.values[:] = rng.uniform(-1, 1, A.nnz).astype(np.float32)
                B.values[:] = rng.uniform(-1, 1, B.nnz).astype(np.float32)
            b.compute()
        assert b.stats()["graph_nodes"] > 0
        got = [b.result(i) for i in range(len(prods))]
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 1) as ex:
        want = list(ex.map(lambda p: _ref_product(*p), prods))
    for i, (g, (rp, ci, cv)) in enumerate(zip(got, want)):
        assert np.array_equal(g.row_ptr, rp), f"row_ptr of product {i}"
        assert np.array_equal(g.col_idx, ci), f"col_idx of product {i}"
        assert np.array_equal(_bits(g.values), _bits(cv)), f"values of product {i}"


@pytest.mark.parametrize("workload", ["laplace2d", "uniform4096"])
def test_learned_full_size(workload):
    if workload == "laplace2d":
        A = gen.laplacian_2d(1024)
        B = A
    else:
        A, B = gen.uniform_rows(4096, 4096, 16, 2024), gen.uniform_rows(4096, 4096, 16, 2025)
    rp, ci, cv = _ref_product(A, B)
    model = RowModel(path=weights_for(workload))
    with Descriptor(algo=L.ALGO_CUDA_LEARNED) as d:
        d.set_model(model)
        C_ = d.multiply(A, B)
    assert np.array_equal(C_.row_ptr, rp)
    assert np.array_equal(C_.col_idx, ci)
    assert np.array_equal(_bits(C_.values), _bits(cv))
