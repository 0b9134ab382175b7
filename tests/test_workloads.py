"""The benchmark's synthetic workloads against their published definitions:
row and entry counts, intermediate products, flops and algorithmic bytes of
the 2D Laplacian 1024^2 and the 27-point stencil 128^3 (C = A x A), the
uniform 4096^2 rows, and the batch of 512 products.  CPU only; the
Laplacian's nnz(C) comes from the oracle."""
import numpy as np

from oracle import oracle
from rvsp import algorithmic_bytes, gen, intermediate_products


def _canonical(M):
    d = np.diff(M.row_ptr)
    assert M.row_ptr[0] == 0 and M.row_ptr[-1] == M.nnz and (d >= 0).all()
    rows = np.repeat(np.arange(M.rows), d)
    # strictly increasing columns within each row
    same_row = rows[1:] == rows[:-1]
    assert (np.diff(M.col_idx.astype(np.int64))[same_row] > 0).all()
    assert M.col_idx.min() >= 0 and M.col_idx.max() < M.cols


def test_laplacian_2d_1024():
    A = gen.laplacian_2d(1024)
    assert (A.rows, A.cols, A.nnz) == (1_048_576, 1_048_576, 5_238_784)
    _canonical(A)
    assert set(np.unique(A.values).tolist()) == {4.0, -1.0}
    ops = intermediate_products(A, A)
    assert int(ops.sum()) == 26_177_544 and 2 * int(ops.sum()) == 52_355_088
    rp, _, _, _ = oracle.spgemm(A, A)
    assert int(rp[-1]) == 13_611_012
    assert algorithmic_bytes(A, A, int(rp[-1])) == 205_291_564


def test_stencil_3d_27_128():
    A = gen.stencil_3d_27(128)
    assert (A.rows, A.nnz) == (2_097_152, 55_742_968)
    assert set(np.unique(A.values).tolist()) == {26.0, -1.0}
    ops = intermediate_products(A, A)
    assert int(ops.sum()) == 1_489_355_288 and 2 * int(ops.sum()) == 2_978_710_576
    assert algorithmic_bytes(A, A, 254_840_104) == 2_955_774_156


def test_uniform_4096_rows():
    A = gen.uniform_rows(4096, 4096, 16, 2024)
    B = gen.uniform_rows(4096, 4096, 16, 2025)
    assert (np.diff(A.row_ptr) == 16).all() and A.nnz == 65_536
    _canonical(A)
    _canonical(B)
    assert not np.array_equal(A.col_idx, B.col_idx)  # seeds S and S + 1
    assert int(intermediate_products(A, B).sum()) == 1_048_576
    assert (np.abs(A.values) <= 1.0).all()


def test_batch_of_512():
    prods = gen.batched_products(count=512, seed=7)
    assert len(prods) == 512
    n = np.array([A.rows for A, _ in prods])
    assert n.min() >= 256 and n.max() <= 65536
    for A, B in prods[::64]:
        assert A.cols == B.rows and A.rows == A.cols == B.cols
        _canonical(A)
        _canonical(B)
        mu = A.nnz / A.rows
        assert 4 <= mu <= 40  # Poisson(mu) rows, mu in [8, 32]
