"""Parity of the CUDA path with the reference scalar backend.

Bar: structure (nnz, row_ptr, col_idx) bit-exact, values bit-exact (each
output entry accumulates in A's nonzero order with separately rounded
multiply and add, as the reference does), and per-row op counts exact.
Checked against the hand-computed fixtures, the committed outputs of the
reference library, the CPU oracle on seeded inputs that reach every row
class, and the full-size benchmark workloads.  The FP64 check uses the
tolerance |c - c64| <= 1e-6 * sum_k |a_ik b_kj| (+1e-30).
"""
import numpy as np
import pytest

from oracle import oracle
from rvsp import CSR, Descriptor, gen, spgemm_csr
from rvsp import _lib as L

pytestmark = pytest.mark.gpu


def assert_bit_exact(got: CSR, rp, ci, cv, what=""):
    assert got.nnz == ci.size, what
    assert np.array_equal(got.row_ptr, rp), f"row_ptr {what}"
    assert np.array_equal(got.col_idx, ci), f"col_idx {what}"
    bad = np.nonzero(got.values.view(np.uint32) != cv.view(np.uint32))[0]
    assert bad.size == 0, f"values {what}: {bad.size} differ, first at {bad[:5]}"


def check_against_oracle(A, B, what="", reuse=False):
    """One-shot and descriptor products against the oracle; with reuse, also
    a numeric-only repeat after A's values change."""
    rp, ci, cv, ops = oracle.spgemm(A, B)
    got = spgemm_csr(A, B)
    assert_bit_exact(got, rp, ci, cv, what + " one-shot")
    with Descriptor() as d:
        Cm = d.multiply(A, B)
        assert_bit_exact(Cm, rp, ci, cv, what + " descriptor")
        assert np.array_equal(d.get_op_counts(A.rows), ops), what
        sym, num = d.class_counts()
        if reuse:
            A2 = A.with_values((A.values * -0.75).astype(np.float32))
            _, _, cv2, _ = oracle.spgemm(A2, B)
            d.compute(A2, B, Cm, np.zeros(max(d.ws_bytes, 1), np.uint8))
            assert_bit_exact(Cm, rp, ci, cv2, what + " numeric-only reuse")
    return sym, num


def test_fixtures(golden_fixtures):
    for name, A, B, Cx in golden_fixtures:
        got = spgemm_csr(A, B)
        assert_bit_exact(got, Cx.row_ptr, Cx.col_idx, Cx.values, name)
        with Descriptor() as d:
            assert_bit_exact(d.multiply(A, B), Cx.row_ptr, Cx.col_idx, Cx.values, name)


def test_reference_outputs(golden_random):
    for name, A, B, Cx, ops in golden_random:
        got = spgemm_csr(A, B)
        assert_bit_exact(got, Cx.row_ptr, Cx.col_idx, Cx.values, name)
        with Descriptor() as d:
            d.work_estimation(A, B)
            assert np.array_equal(d.get_op_counts(A.rows), ops), name


def class_probe(seed: int, b_cols: int = 60000):
    """A x B whose rows land in every row class: 200 short B rows (3 columns
    out of the first 20), six groups of 200 rows of 8 columns drawn from
    pools of 20..1024 columns, and 1800 rows of 45 columns over all of B.

    A rows with <= 32 nonzeros give the merge classes; 40 (or 100) rows of
    one 8-column group give > 32 A nonzeros with at most pool-size outputs
    (W64 ... W2048); 45..400 long rows give the block-hash and dense
    classes."""
    rng = np.random.default_rng(seed)
    pools = [20, 64, 128, 256, 512, 1024]
    groups = [(200, 3, 20)] + [(200, 8, p) for p in pools] + [(1800, 45, b_cols)]
    cols, lengths, starts = [], [], []
    first = 0
    for n, ln, pool in groups:
        lens = np.full(n, ln, np.int64)
        cols.append(gen._distinct_sorted_columns(rng, lens, pool))
        lengths.append(lens)
        starts.append(first)
        first += n
    lengths = np.concatenate(lengths)
    cols = np.concatenate(cols)
    nb = lengths.size
    rp = np.zeros(nb + 1, np.int64)
    np.cumsum(lengths, out=rp[1:])
    B = CSR(nb, b_cols, rp, cols, rng.uniform(-1, 1, cols.size).astype(np.float32))

    def pick(group, k):
        n = groups[group][0]
        return starts[group] + rng.choice(n, size=k, replace=False)

    a_rows = [np.zeros(0, np.int64)] * 4
    long_g = len(groups) - 1
    for k in (1, 2, 3, 4, 5, 8, 12, 16, 20, 30, 32):
        a_rows += [pick(long_g, k) for _ in range(6)] + [pick(0, min(k, 12))]
    for g, k in zip(range(1, 7), (40, 40, 40, 40, 40, 100)):
        a_rows += [pick(g, k) for _ in range(8)]
    a_rows += [pick(0, 40) for _ in range(8)]
    for k in (45, 60, 80, 100, 150, 250, 400):
        a_rows += [pick(long_g, k) for _ in range(6)]
    # The merge classes need a matrix of at least 32768 rows: pad with rows of
    # 1..16 A nonzeros (long and short B rows alternately).
    r = 0
    while len(a_rows) < 33000:
        k = 1 + r % 16
        a_rows.append(pick(long_g if r % 3 else 0, min(k, 12) if r % 3 == 0 else k))
        r += 1
    a_rows = [np.sort(x) for x in a_rows]
    lens = np.array([x.size for x in a_rows], np.int64)
    arp = np.zeros(len(a_rows) + 1, np.int64)
    np.cumsum(lens, out=arp[1:])
    aci = np.concatenate(a_rows) if lens.sum() else np.zeros(0, np.int64)
    A = CSR(len(a_rows), nb, arp, aci, rng.uniform(-1, 1, aci.size).astype(np.float32))
    return A, B


def test_every_row_class():
    A, B = class_probe(11)
    sym, num = check_against_oracle(A, B, "class probe", reuse=True)
    for cls in L.CLASS_NAMES:
        assert sym[cls] > 0 or num[cls] > 0, (cls, sym, num)


def test_dense_rows_with_global_bitmap():
    # b_cols beyond the shared-memory bitmap (1.5 Mi columns): dense rows use
    # the global-memory bitmap in both passes.
    A, B = class_probe(12, b_cols=2_000_000)
    sym, num = check_against_oracle(A, B, "wide B", reuse=True)
    assert sym["dense"] > 0 and num["dense"] > 0


def test_dense_rows_wide_smem_bitmap():
    # 2^20 < b_cols <= 1.5 Mi: the block-hash and dense kernels with the
    # bitmap in shared memory and the accumulator in global memory.
    A, B = class_probe(13, b_cols=1_200_000)
    sym, num = check_against_oracle(A, B, "1.2M columns", reuse=True)
    assert sym["dense"] > 0 and num["dense"] > 0


def test_heavy_rows_at_bitmap_limit():
    # b_cols = 2^20, the widest B the heavy-row kernels take: the largest
    # bitmap, and rows whose nnz exceeds the shared-memory accumulator
    # (accumulation in C's value array).
    A, B = class_probe(14, b_cols=1 << 20)
    sym, num = check_against_oracle(A, B, "2^20 columns", reuse=True)
    assert sym["dense"] > 0 and num["dense"] > 0
    nnz = np.diff(spgemm_csr(A, B).row_ptr)
    assert nnz.max() > 12000


def test_rmat_hub_rows():
    # The first rows of an R-MAT matrix are its hubs: thousands of A
    # nonzeros, popular output columns shared by many B rows, and rows of
    # more output nnz than the shared-memory accumulator holds.
    A = gen.rmat(16, 16, seed=1)
    panel = A.row_panel(0, 192)
    check_against_oracle(panel, A, "R-MAT 2^16 hub rows", reuse=True)
    nnz = np.diff(spgemm_csr(panel, A).row_ptr)
    assert nnz.max() > 20000


@pytest.mark.parametrize("seed", range(8))
def test_seeded_irregular(seed):
    A = gen.random_csr(700, 500, 300 + seed, mean_len=3.0 + 3 * (seed % 4),
                       empty_frac=0.1, heavy_rows=seed % 3, heavy_len=200)
    B = gen.random_csr(500, 900, 400 + seed, mean_len=2.0 + 4 * (seed % 3),
                       empty_frac=0.15, heavy_rows=1, heavy_len=300,
                       value_kind="int" if seed % 2 else "uniform")
    check_against_oracle(A, B, f"seed {seed}")


def test_single_merge_class_with_empty_rows():
    # every non-empty row has 3 A nonzeros (one merge class) and a fifth of
    # the rows are empty: the class is run over the whole matrix, no row list
    rng = np.random.default_rng(8)
    n = 40000
    lengths = np.where(rng.random(n) < 0.2, 0, 3).astype(np.int64)
    cols = gen._distinct_sorted_columns(rng, lengths, 5000)
    rp = np.zeros(n + 1, np.int64)
    np.cumsum(lengths, out=rp[1:])
    A = CSR(n, 5000, rp, cols, rng.uniform(-1, 1, cols.size).astype(np.float32))
    B = gen.random_csr(5000, 7000, 9, mean_len=4.0, empty_frac=0.1)
    sym, num = check_against_oracle(A, B, "one merge class")
    assert sym["m4"] > 0 and sym["empty"] > 0


def test_long_a_rows():
    # rows with more A nonzeros than the per-thread rowstats path takes
    A = gen.random_csr(50, 3000, 21, mean_len=5.0, heavy_rows=10, heavy_len=1500)
    B = gen.random_csr(3000, 400, 22, mean_len=2.0, empty_frac=0.5)
    check_against_oracle(A, B, "long A rows")


def test_nnz_beyond_int32_is_allocation_failed():
    # nnz(C) = 65536 x 32768 = 2^31 > INT32_MAX from 98,304 stored entries:
    # every A row selects the one full B row.  The reference's symbolic pass
    # returns ALLOCATION_FAILED on the int64 total (rvsp_symbolic.c:69-72);
    # so must the one-shot call and work_estimation here.
    n, w = 65536, 32768
    A = CSR(n, 1, np.arange(n + 1), np.zeros(n), np.ones(n, np.float32))
    B = CSR(1, w, np.array([0, w]), np.arange(w), np.ones(w, np.float32))
    with pytest.raises(L.RvspError) as e:
        spgemm_csr(A, B)
    assert e.value.status == L.ERROR_ALLOCATION_FAILED
    with Descriptor() as d:
        with pytest.raises(L.RvspError) as e:
            d.work_estimation(A, B)
        assert e.value.status == L.ERROR_ALLOCATION_FAILED


def test_edge_cases():
    one = np.ones(1, np.float32)
    # empty A
    A = CSR(3, 4, np.zeros(4), np.zeros(0), np.zeros(0))
    B = gen.random_csr(4, 5, 1, mean_len=2.0)
    check_against_oracle(A, B, "empty A")
    # all-empty B rows
    A = gen.random_csr(6, 4, 2, mean_len=2.0, empty_frac=0.0)
    B = CSR(4, 7, np.zeros(5), np.zeros(0), np.zeros(0))
    check_against_oracle(A, B, "empty B")
    # 1 x 1
    A = CSR(1, 1, np.array([0, 1]), np.array([0]), one * 3)
    B = CSR(1, 1, np.array([0, 1]), np.array([0]), one * -2)
    check_against_oracle(A, B, "1x1")
    # signed zeros: 0 * -1 = -0, and +0 + -0 = +0 in the accumulator
    A = CSR(1, 2, np.array([0, 2]), np.array([0, 1]), np.array([0.0, -0.0], np.float32))
    B = CSR(2, 2, np.array([0, 2, 4]), np.array([0, 1, 0, 1]),
            np.array([-1.0, 1.0, 1.0, -1.0], np.float32))
    check_against_oracle(A, B, "signed zeros")
    # exact cancellation keeps the structural zero
    A = CSR(1, 2, np.array([0, 2]), np.array([0, 1]), np.array([1.0, 1.0], np.float32))
    B = CSR(2, 1, np.array([0, 1, 2]), np.array([0, 0]), np.array([1.0, -1.0], np.float32))
    got = spgemm_csr(A, B)
    assert got.nnz == 1 and got.values[0] == 0.0
    # inf / nan propagate exactly like the scalar backend
    A = CSR(2, 2, np.array([0, 2, 3]), np.array([0, 1, 1]),
            np.array([np.inf, 1.0, np.nan], np.float32))
    B = CSR(2, 2, np.array([0, 1, 2]), np.array([0, 1]), np.array([0.0, 2.0], np.float32))
    rp, ci, cv, _ = oracle.spgemm(A, B)
    g = spgemm_csr(A, B)
    assert np.array_equal(g.col_idx, ci)
    assert np.array_equal(np.isnan(g.values), np.isnan(cv))
    assert np.array_equal(g.values[~np.isnan(cv)], cv[~np.isnan(cv)])


def test_invalid_csr_rejected():
    A = gen.random_csr(20, 10, 3, mean_len=3.0, empty_frac=0.0)
    B = gen.random_csr(10, 10, 4, mean_len=3.0, empty_frac=0.0)
    for mutate in ("range", "unsorted", "dup", "rowptr"):
        X = A.copy()
        if mutate == "range":
            X.col_idx[5] = 10
        elif mutate == "unsorted":
            r = next(i for i in range(X.rows) if X.row_ptr[i + 1] - X.row_ptr[i] >= 2)
            p = X.row_ptr[r]
            X.col_idx[p], X.col_idx[p + 1] = X.col_idx[p + 1], X.col_idx[p]
        elif mutate == "dup":
            r = next(i for i in range(X.rows) if X.row_ptr[i + 1] - X.row_ptr[i] >= 2)
            p = X.row_ptr[r]
            X.col_idx[p + 1] = X.col_idx[p]
        else:
            X.row_ptr[3] = X.row_ptr[4] + 1
        with pytest.raises(L.RvspError) as e:
            spgemm_csr(X, B)
        assert e.value.status == L.ERROR_INVALID_CSR, mutate


def test_checked_symbolic_merge_rows():
    # With merge classes on (>= 32768 rows) the checked symbolic pass queues
    # the merge rows' count and the scan before the check's verdict reaches
    # the host: a valid structure gives the oracle's row_ptr, with and without
    # warp-class rows beside the merge rows; a structure that fails the check
    # gives INVALID_CSR and the caller's row_ptr is left untouched.  The
    # mutations keep every index in range.
    import ctypes as C
    import torch
    lib = L.load()
    n = 40000
    plan = C.c_void_p()
    L.check(lib.rvsp_cuda_plan_create(C.byref(plan)), "plan_create")
    try:
        B = gen.random_csr(n, n, 41, mean_len=4.0, empty_frac=0.1)
        db = [torch.from_numpy(x).cuda() for x in (B.row_ptr, B.col_idx)]
        plain = gen.random_csr(n, n, 42, mean_len=5.0, empty_frac=0.1)
        mixed = gen.random_csr(n, n, 43, mean_len=5.0, empty_frac=0.1, heavy_rows=40,
                               heavy_len=300)
        cases = [("valid", plain), ("valid+warp rows", mixed)]
        for mutate in ("unsorted", "dup", "rowptr"):
            X = plain.copy()
            r = next(i for i in range(1000, n) if X.row_ptr[i + 1] - X.row_ptr[i] >= 2)
            p = X.row_ptr[r]
            if mutate == "unsorted":
                X.col_idx[p], X.col_idx[p + 1] = X.col_idx[p + 1], X.col_idx[p]
            elif mutate == "dup":
                X.col_idx[p + 1] = X.col_idx[p]
            else:
                X.row_ptr[r] = X.row_ptr[r + 1] + 1
            cases.append((mutate, X))
        for what, X in cases:
            da = [torch.from_numpy(x).cuda() for x in (X.row_ptr, X.col_idx)]
            c_rp = torch.full((n + 1,), -7, dtype=torch.int32, device="cuda")
            total = C.c_int64(-1)
            st = lib.rvsp_cuda_symbolic_checked(
                plan, C.c_void_p(0), n, X.cols, X.nnz, B.rows, B.cols, B.nnz,
                da[0].data_ptr(), da[1].data_ptr(), db[0].data_ptr(), db[1].data_ptr(), 1,
                c_rp.data_ptr(), C.byref(total))
            if what.startswith("valid"):
                assert st == L.SUCCESS, what
                rp, ci, _, _ = oracle.spgemm(X, B)
                assert total.value == ci.size, what
                assert np.array_equal(c_rp.cpu().numpy(), rp.astype(np.int32)), what
            else:
                assert st == L.ERROR_INVALID_CSR, what
                assert bool((c_rp == -7).all()), what
    finally:
        lib.rvsp_cuda_plan_destroy(plan)


def test_device_check_long_rows_matches_oracle():
    # Rows over 256 entries are checked by a warp each: the (code, first bad
    # row) pair must still be the reference's, for violations at chunk
    # boundaries, deep in long rows, and in short rows before or after them.
    import ctypes as C
    import torch
    lib = L.load()
    rng = np.random.default_rng(17)
    base = gen.random_csr(300, 5000, 18, mean_len=8.0, heavy_rows=12, heavy_len=2000)
    long_rows = np.nonzero(np.diff(base.row_ptr) > 256)[0]
    plan = C.c_void_p()
    L.check(lib.rvsp_cuda_plan_create(C.byref(plan)), "plan_create")
    try:
        cases = [None]
        for r in long_rows[:4]:
            for pos in (0, 31, 32, 33, 500, int(base.row_ptr[r + 1] - base.row_ptr[r]) - 1):
                for kind in ("range", "dup", "unsorted"):
                    cases.append((int(r), pos, kind))
        cases.append((int(rng.integers(0, long_rows[0] + 1)), 0, "range"))
        for case in cases:
            X = base.copy()
            if case is not None:
                r, pos, kind = case
                p = int(X.row_ptr[r]) + pos
                if kind == "range":
                    X.col_idx[p] = X.cols
                elif kind == "dup" and pos > 0:
                    X.col_idx[p] = X.col_idx[p - 1]
                elif kind == "unsorted" and pos > 0:
                    X.col_idx[p] = X.col_idx[p - 1] - 1
            rp = torch.from_numpy(X.row_ptr).cuda()
            ci = torch.from_numpy(X.col_idx).cuda()
            code, bad = C.c_int32(), C.c_int32()
            L.check(lib.rvsp_cuda_csr_check(plan, C.c_void_p(0), X.rows, X.cols,
                                            rp.data_ptr(), ci.data_ptr(), X.nnz,
                                            C.byref(code), C.byref(bad)), "csr_check")
            assert (code.value, bad.value) == oracle.csr_check(X.rows, X.cols, X.row_ptr,
                                                               X.col_idx), case
    finally:
        lib.rvsp_cuda_plan_destroy(plan)


def test_fp64_tolerance():
    A = gen.random_csr(400, 300, 31, mean_len=20.0)
    B = gen.random_csr(300, 350, 32, mean_len=20.0)
    got = spgemm_csr(A, B)
    v64, mag = oracle.numeric_f64(A, B, got.row_ptr, got.col_idx)
    assert np.all(np.abs(got.values.astype(np.float64) - v64) <= 1e-6 * mag + 1e-30)


def test_uniform_4096_16_per_row_full():
    # 4096 x 4096, exactly 16 nnz/row, A seed S, B seed S + 1
    A = gen.uniform_rows(4096, 4096, 16, seed=2024)
    B = gen.uniform_rows(4096, 4096, 16, seed=2025)
    st, rp, ci, cv = oracle.ref_spgemm(A, B) if oracle.ref_available() else (0, *oracle.spgemm(A, B)[:3])
    assert st == 0
    assert_bit_exact(spgemm_csr(A, B), rp, ci, cv, "uniform 4096")


def test_laplacian_2d_1024_full():
    A = gen.laplacian_2d(1024)
    assert A.nnz == 5_238_784
    rp, ci, cv, ops = oracle.spgemm(A, A)
    assert ci.size == 13_611_012
    got = spgemm_csr(A, A)
    assert_bit_exact(got, rp, ci, cv, "laplacian 1024")


def test_stencil_3d_27_small():
    A = gen.stencil_3d_27(24)
    check_against_oracle(A, A, "27-point 24^3")


def test_rmat_panel():
    A = gen.rmat(14, 16, seed=3)
    panel = A.row_panel(0, 2048)
    check_against_oracle(panel, A, "R-MAT 2^14 panel")


def test_rmat20_sampled_panels():
    # The power-law configuration runs as row panels (its whole C exceeds
    # int32).  Sampled panels: the hubs (rows of up to ~10^7 products and
    # ~10^5-10^6 outputs, over B's 2^20 columns: the widest heavy-row
    # bitmap and many accumulator windows), a middle block, the last rows;
    # plain and learned paths, and a numeric-only repeat on the hubs.
    from rvsp.learn import DEFAULT_WEIGHTS, RowModel
    A = gen.rmat(20, 16, seed=1)
    model = RowModel(path=DEFAULT_WEIGHTS)
    for r0, r1 in ((0, 32), (500000, 500512), (A.rows - 512, A.rows)):
        P = A.row_panel(r0, r1)
        check_against_oracle(P, A, f"R-MAT 2^20 rows {r0}:{r1}", reuse=(r0 == 0))
        rp, ci, cv, _ = oracle.spgemm(P, A)
        with Descriptor(algo=L.ALGO_CUDA_LEARNED) as d:
            d.set_model(model)
            assert_bit_exact(d.multiply(P, A), rp, ci, cv, f"learned rows {r0}:{r1}")


def test_batched_style_products():
    for i, (A, B) in enumerate(gen.batched_products(count=6, seed=5, n_hi=4096)):
        check_against_oracle(A, B, f"batch {i}")
