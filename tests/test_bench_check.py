"""The bench's result check (bench.reference_check / bench.same_csr): a C
that matches the reference library's product bit for bit passes, and a C
with one mistake planted on the CPU (a value's low bit, a column, a row
pointer, a missing entry) fails and is counted.  CPU only; the reference
library stands in for the GPU's C here."""
import numpy as np

import bench
from oracle import oracle
from rvsp import CSR, gen


def _product(seed):
    A = gen.random_csr(300, 200, seed, mean_len=4.0)
    B = gen.random_csr(200, 250, seed + 1, mean_len=3.0)
    rp, ci, cv, _ = oracle.spgemm(A, B)
    return A, B, CSR(A.rows, B.cols, rp, ci, cv)


def _planted(C, kind):
    rp, ci, cv = C.row_ptr.copy(), C.col_idx.copy(), C.values.copy()
    if kind == "value bit":
        cv.view(np.uint32)[7] ^= 1
    elif kind == "column":
        r = next(i for i in range(C.rows) if rp[i + 1] - rp[i] >= 2)
        ci[rp[r]], ci[rp[r] + 1] = ci[rp[r] + 1], ci[rp[r]]
    elif kind == "row_ptr":
        r = next(i for i in range(1, C.rows) if rp[i + 1] > rp[i])
        rp[r] += 1
    else:  # the last entry missing
        rp, ci, cv = rp.copy(), ci[:-1], cv[:-1]
        rp[-1] -= 1
    return CSR(C.rows, C.cols, rp, ci, cv)


def test_matching_product_passes():
    items = [_product(s) for s in (1, 3, 5)]
    res = bench.reference_check(items, "three products")
    assert res["bit_exact"] and res["mismatched"] == 0
    assert res["against"].startswith("reference" if oracle.ref_available() else "port")


def test_planted_mistakes_fail():
    A, B, C = _product(7)
    for kind in ("value bit", "column", "row_ptr", "missing entry"):
        bad = _planted(C, kind)
        res = bench.reference_check([(A, B, C), (A, B, bad)], kind)
        assert not res["bit_exact"] and res["mismatched"] == 1, kind


def test_signed_zero_differs():
    # values are compared as bit patterns: -0.0 is not +0.0
    A = CSR(1, 2, np.array([0, 2]), np.array([0, 1]), np.array([1.0, 1.0], np.float32))
    B = CSR(2, 1, np.array([0, 1, 2]), np.array([0, 0]), np.array([1.0, -1.0], np.float32))
    rp, ci, cv, _ = oracle.spgemm(A, B)
    assert cv[0] == 0.0 and not np.signbit(cv[0])
    flipped = CSR(1, 1, rp, ci, np.array([-0.0], np.float32))
    assert bench.same_csr(CSR(1, 1, rp, ci, cv), rp, ci, cv)
    assert not bench.same_csr(flipped, rp, ci, cv)


def test_panel_rows_cover_every_row_once_by_op_count():
    # the stencil job's row panels: contiguous, disjoint, covering all rows,
    # each near 1/N of the op count (the rows of C are independent)
    from rvsp import intermediate_products
    A = gen.stencil_3d_27(20)
    ops = intermediate_products(A, A)
    for world in (1, 2, 3, 8):
        cuts = [bench.panel_rows(ops, world, r) for r in range(world)]
        assert cuts[0][0] == 0 and cuts[-1][1] == A.rows
        for (a0, a1), (b0, b1) in zip(cuts, cuts[1:]):
            assert a1 == b0 and a0 <= a1
        shares = [int(ops[r0:r1].sum()) for r0, r1 in cuts]
        assert sum(shares) == int(ops.sum())
        assert max(shares) - min(shares) <= 2 * int(ops.max())


def test_job_value_sets_are_seeded_perturbations():
    A = gen.stencil_3d_27(6)
    s1 = bench.job_value_sets_host(A, 2, 5)
    s2 = bench.job_value_sets_host(A, 2, 5)
    for a, b in zip(s1, s2):
        assert np.array_equal(a, b)
        assert a.dtype == np.float32
        assert np.all(np.abs(a - A.values) <= 0.0100001)
    assert not np.array_equal(s1[0], s1[1])


def test_reference_job_matches_the_restatement():
    # the reference descriptor job the bench checks against: first compute,
    # then numeric-only computes with new values, against the oracle
    A = gen.stencil_3d_27(8)
    sets = bench.job_value_sets_host(A, 2, 9)
    st, rp, ci, first, every = oracle.ref_job(A, A, [(v, v) for v in sets], keep_all=True) \
        if oracle.ref_available() else (0, *oracle.spgemm(A, A)[:3], None)
    assert st == 0
    want_rp, want_ci, want_cv, _ = oracle.spgemm(A, A)
    assert np.array_equal(rp, want_rp) and np.array_equal(ci, want_ci)
    assert np.array_equal(first.view(np.uint32), want_cv.view(np.uint32))
    if every is not None:
        for v, got in zip(sets, every):
            A2 = A.with_values(v)
            assert np.array_equal(got.view(np.uint32), oracle.spgemm(A2, A2)[2].view(np.uint32))
