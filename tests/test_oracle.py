"""Pins the CPU oracle before anything is checked against it.

  * the six hand-computed fixtures of the reference suite
    (tests/csr_fixtures.h:42-153, committed as tests/golden/fixtures.json);
  * the reference library's own outputs on seeded irregular inputs
    (tests/golden/ref_random.npz, made by tests/golden/make_golden.py);
  * the reference library run live (oracle/_ref/librvsp_ref.so) on more
    seeded inputs, when it has been built;
  * rvsp_csr_check codes and rows against the reference's check.
"""
import numpy as np
import pytest

from oracle import oracle
from rvsp import CSR, gen, intermediate_products


def test_fixtures_exact(golden_fixtures):
    for name, A, B, Cx in golden_fixtures:
        rp, ci, cv, _ = oracle.spgemm(A, B)
        assert np.array_equal(rp, Cx.row_ptr), name
        assert np.array_equal(ci, Cx.col_idx), name
        # the fixtures are exact small integers
        assert np.array_equal(cv, Cx.values), name


def test_fixture_op_counts_basic(golden_fixtures):
    # test_spgemm_descr_f32.c:123-124: op counts {2, 1} on the basic fixture
    name, A, B, _ = golden_fixtures[0]
    assert name == "basic"
    _, _, _, ops = oracle.spgemm(A, B)
    assert ops.tolist() == [2, 1]


def test_reference_outputs_bit_exact(golden_random):
    for name, A, B, Cx, ops_x in golden_random:
        rp, ci, cv, ops = oracle.spgemm(A, B)
        assert np.array_equal(rp, Cx.row_ptr), name
        assert np.array_equal(ci, Cx.col_idx), name
        assert np.array_equal(cv.view(np.uint32), Cx.values.view(np.uint32)), name
        assert np.array_equal(ops, ops_x), name
        assert np.array_equal(intermediate_products(A, B), ops_x), name


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("seed", range(6))
def test_live_reference_bit_exact(seed):
    A = gen.random_csr(120, 90, 1000 + seed, mean_len=5.0, heavy_rows=2, heavy_len=60)
    B = gen.random_csr(90, 150, 2000 + seed, mean_len=8.0, heavy_rows=1, heavy_len=120)
    st, rp, ci, cv = oracle.ref_spgemm(A, B)
    assert st == 0
    orp, oci, ocv, _ = oracle.spgemm(A, B)
    assert np.array_equal(orp, rp) and np.array_equal(oci, ci)
    assert np.array_equal(ocv.view(np.uint32), cv.view(np.uint32))


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
def test_sequential_rounding_matters():
    """The oracle is not an FMA or reordered sum: on cancelling inputs the
    reference result differs from an FP64 sum rounded once, and the oracle
    still matches the reference bit for bit."""
    A = gen.random_csr(200, 200, 77, mean_len=12.0)
    B = gen.random_csr(200, 200, 78, mean_len=12.0)
    st, rp, ci, cv = oracle.ref_spgemm(A, B)
    _, _, ocv, _ = oracle.spgemm(A, B)
    assert np.array_equal(ocv.view(np.uint32), cv.view(np.uint32))
    v64, _ = oracle.numeric_f64(A, B, rp, ci)
    assert np.any(v64.astype(np.float32) != cv)


def _crafted_checks():
    ok = (3, 4, [0, 1, 3, 3], [2, 0, 3])
    return [
        ok,
        (3, 4, [1, 1, 3, 3], [2, 0, 3]),        # row_ptr[0] != 0
        (3, 4, [0, 2, 1, 3], [2, 3, 0]),        # decreasing row_ptr at row 1
        (3, 4, [0, 1, 3, 3], [2, 0, 4]),        # column out of range
        (3, 4, [0, 1, 3, 3], [2, 3, 0]),        # unsorted
        (3, 4, [0, 1, 3, 3], [2, 1, 1]),        # duplicate
        (3, 4, [0, 2, 4, 4], [1, 0, 3, 3]),     # unsorted row 0 before dup row 1
        (2, 0, [0, 0, 0], []),                  # no columns, empty rows
        (2, 0, [0, 0, 1], [0]),                 # no columns, one entry
    ]


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built")
@pytest.mark.parametrize("case", range(len(_crafted_checks())))
def test_csr_check_matches_reference(case):
    rows, cols, rp, ci = _crafted_checks()[case]
    rp = np.array(rp, np.int32)
    ci = np.array(ci if ci else [0], np.int32)
    assert oracle.csr_check(rows, cols, rp, ci) == oracle.ref_check(rows, cols, rp, ci)


def test_f64_oracle_close_to_f32():
    A = gen.random_csr(50, 40, 5, mean_len=4.0)
    B = gen.random_csr(40, 60, 6, mean_len=4.0)
    rp, ci, cv, _ = oracle.spgemm(A, B)
    v64, mag = oracle.numeric_f64(A, B, rp, ci)
    assert np.all(np.abs(cv - v64) <= 1e-6 * mag + 1e-30)


def test_overflow_reported():
    # nnz(C) > INT32_MAX is detected on the int64 running total; a dense
    # 1 x 2^31-ish product is too big to build, so check the guard's arithmetic
    # on a small case instead: symbolic totals are exact int64 sums.
    A = CSR(2, 3, np.array([0, 3, 3]), np.array([0, 1, 2]), np.ones(3))
    B = CSR(3, 5, np.array([0, 2, 4, 5]), np.array([0, 4, 1, 4, 2]), np.ones(5))
    rp, ci, cv, ops = oracle.spgemm(A, B)
    assert rp.tolist() == [0, 4, 4] and ci.tolist() == [0, 1, 2, 4]
    assert ops.tolist() == [5, 0]
