"""Shift classes (k_shift.cu): rows that are exact translates of another row.

Such rows take their count, columns (moved by the row distance) and term
table from a canonical row and skip the symbolic pass and the fill.  Bar:
structure and values bit-exact against the oracle (the reference's
rvsp_symbolic_count / rvsp_symbolic_fill / numeric, rvsp_symbolic.c:13-137
and gustavson_core_f32.inc:18-64) with the classes on, with them off, and on
numeric-only repeats; on stencils, Laplacians, banded matrices with far
diagonals, a matrix of translates mixed with random rows, a pattern too
wide for the tables, through the descriptor in both memory spaces, the
learned path (which hands such matrices to this analysis) and the C-ABI
with a caller-given structure.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from rvsp import Descriptor, DeviceCSR, gen
from rvsp import _lib as L
from rvsp.csr import CSR
from rvsp.learn import RowModel, weights_for

pytestmark = pytest.mark.gpu


def _bits(x):
    return np.ascontiguousarray(x, np.float32).view(np.uint32)


def _banded(n, offsets, seed, cols=None):
    cols = n if cols is None else cols
    rows = [[i + o for o in offsets if 0 <= i + o < cols] for i in range(n)]
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum([len(r) for r in rows])
    ci = np.concatenate([np.asarray(r, np.int64) for r in rows]).astype(np.int32)
    rng = np.random.default_rng(seed)
    return CSR(n, cols, rp, ci, rng.uniform(-1, 1, ci.size).astype(np.float32))


def _check(A, B, algo=L.ALGO_CUDA_PLAIN, shift=True, repeats=2, min_shift=1, model=None,
           memory=L.MEM_DEVICE):
    """Full product, then numeric-only repeats with new A values, against the
    oracle; returns the shift rows of the analysis."""
    import torch
    rp, ci, cv, _ = oracle.spgemm(A, B)
    with Descriptor(algo=algo, memory=memory) as d:
        if model is not None:
            d.set_model(model)
        # 2: the analysis runs on these small matrices too (by default it
        # waits for 32768 rows averaging 64 products)
        d.set_shift_classes(2 if shift else 0)
        if memory == L.MEM_DEVICE:
            dA = DeviceCSR.from_host(A)
            dB = dA if B is A else DeviceCSR.from_host(B)
            ws_b, n = d.work_estimation(dA, dB)
            dC = DeviceCSR.empty(A.rows, B.cols, n)
            ws = torch.zeros(max(ws_b, 1), dtype=torch.uint8, device="cuda")
            d.compute(dA, dB, dC, ws)
            d.synchronize()
            got = dC.to_host(n)
        else:
            got = d.multiply(A, B)
        rows = d.shift_rows()
        assert np.array_equal(got.row_ptr, rp), "row_ptr"
        assert np.array_equal(got.col_idx, ci), "col_idx"
        assert np.array_equal(_bits(got.values), _bits(cv)), "values"
        if memory == L.MEM_DEVICE:
            rng = np.random.default_rng(3)
            for r in range(repeats):
                vals = (A.values * np.float32(1 + r) +
                        rng.uniform(-0.01, 0.01, A.nnz)).astype(np.float32)
                dA.values.copy_(torch.from_numpy(vals))
                torch.cuda.synchronize()
                d.compute(dA, dB, dC, ws)
                d.synchronize()
                A2 = A.with_values(vals)
                want = oracle.spgemm(A2, A2 if B is A else B)[2]
                assert np.array_equal(_bits(dC.values[:n].cpu().numpy()), _bits(want)), \
                    f"repeat {r}"
    if shift:
        assert rows >= min_shift, rows
    else:
        assert rows == 0
    return rows


@pytest.mark.parametrize("grid", [20, 32])
def test_stencil_shift_on_and_off(grid):
    A = gen.stencil_3d_27(grid)
    rows = _check(A, A, min_shift=(grid - 4) ** 3)
    assert rows < A.rows
    _check(A, A, shift=False)


def test_laplacian_merge_canonical_rows():
    # 2D 5-point Laplacian on 200^2 (40,000 rows, merge-class rows): the
    # canonical rows are merge rows, so one scan serves the whole analysis
    A = gen.laplacian_2d(200)
    _check(A, A, min_shift=190 * 190)


def test_banded_far_diagonals_a_times_b():
    A = _banded(9000, (-900, -40, -1, 0, 3, 77, 800), 5)
    B = _banded(9000, (-7, 0, 2, 11, 450), 6)
    _check(A, B, min_shift=6000)


def test_translates_mixed_with_random_rows():
    # rows 0..5999 banded, rows 6000..9999 random: most of the probe's
    # samples have translates; only the banded rows join classes
    band = _banded(10000, (-30, -2, 0, 5, 90), 8)
    rnd = gen.random_csr(10000, 10000, 9, mean_len=6.0)
    rows = []
    for i in range(10000):
        src = band if i < 6000 else rnd
        rows.append((src.col_idx[src.row_ptr[i]:src.row_ptr[i + 1]],
                     src.values[src.row_ptr[i]:src.row_ptr[i + 1]]))
    rp = np.zeros(10001, np.int32)
    rp[1:] = np.cumsum([len(c) for c, _ in rows])
    A = CSR(10000, 10000, rp, np.concatenate([c for c, _ in rows]),
            np.concatenate([v for _, v in rows]))
    B = _banded(10000, (-3, 0, 1, 40), 10)
    shifted = _check(A, B, min_shift=5000)
    assert shifted <= 6000


def test_wide_b_rows_take_the_warp_path():
    # B rows of 80 entries: longer than one lane walks, so the whole warp
    # keys them and checks them against their canonical row
    A = _banded(6000, (-2, 0, 1, 3), 21)
    B = _banded(6000, tuple(range(0, 160, 2)), 22, cols=6200)
    _check(A, B, min_shift=5000, repeats=1)


@pytest.mark.parametrize("width", [32, 48])
def test_b_rows_at_the_staging_limit(width):
    # 32-entry B rows: 32 of them fill a warp's staged segment (1024 column
    # indices) exactly, so the warps whose segment starts off a 16-byte
    # boundary read their rows from global memory instead; 48-entry rows
    # never fit, and are walked by one lane each from global memory
    A = _banded(6000, (-1, 0, 2), 23)
    B = _banded(6000, tuple(range(0, 2 * width, 2)), 24, cols=6200)
    _check(A, B, min_shift=5000, repeats=1)


def test_a_segments_too_long_to_stage():
    # every third A row holds 200 random columns: 32 consecutive rows hold
    # more column indices than a warp stages, so the banded rows between
    # them are keyed and checked from global memory
    n = 6000
    band = _banded(n, (-3, 0, 4), 25)
    rng = np.random.default_rng(26)
    rows = []
    for i in range(n):
        if i % 3 == 1:
            c = np.sort(rng.choice(n, 200, replace=False)).astype(np.int32)
        else:
            c = band.col_idx[band.row_ptr[i]:band.row_ptr[i + 1]]
        rows.append(c)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum([len(c) for c in rows])
    ci = np.concatenate(rows).astype(np.int32)
    A = CSR(n, n, rp, ci, rng.uniform(-1, 1, ci.size).astype(np.float32))
    B = _banded(n, (-2, 0, 1, 9), 27)
    shifted = _check(A, B, min_shift=3500, repeats=1)
    assert shifted <= 4000


@pytest.mark.parametrize("off", [1, 2, 3])
def test_column_arrays_off_16_byte_boundaries(off):
    # A's column indices handed over `off` entries into a larger buffer: the
    # key and resolve passes stage them with single loads instead of 16-byte
    # ones
    import torch
    A = gen.stencil_3d_27(16)
    rp, ci, cv, _ = oracle.spgemm(A, A)
    buf = torch.zeros(A.nnz + 4, dtype=torch.int32, device="cuda")
    buf[off:off + A.nnz].copy_(torch.from_numpy(A.col_idx))
    dA = DeviceCSR(A.rows, A.cols, torch.from_numpy(A.row_ptr).cuda(), buf[off:off + A.nnz],
                   torch.from_numpy(A.values).cuda())
    torch.cuda.synchronize()
    with Descriptor(algo=L.ALGO_CUDA_PLAIN, memory=L.MEM_DEVICE) as d:
        d.set_shift_classes(2)
        ws_b, n = d.work_estimation(dA, dA)
        dC = DeviceCSR.empty(A.rows, A.cols, n)
        ws = torch.zeros(max(ws_b, 1), dtype=torch.uint8, device="cuda")
        d.compute(dA, dA, dC, ws)
        d.synchronize()
        got = dC.to_host(n)
        assert d.shift_rows() > 2000
    assert np.array_equal(got.row_ptr, rp)
    assert np.array_equal(got.col_idx, ci)
    assert np.array_equal(_bits(got.values), _bits(cv))


def test_tiles_over_long_chunk_segments():
    # every fourth A row holds 150 random columns, the others a band of 4: a
    # run of 32 rows then holds about 1,300 A entries, more than the tile and
    # record builders stage in shared memory (1,024), so they read those B
    # row starts through the column array; the banded rows still form tiles
    n = 6000
    band = _banded(n, (-3, 0, 1, 4), 51)
    rng = np.random.default_rng(52)
    rows = []
    for i in range(n):
        if i % 4 == 2:
            rows.append(np.sort(rng.choice(n, 150, replace=False)).astype(np.int32))
        else:
            rows.append(band.col_idx[band.row_ptr[i]:band.row_ptr[i + 1]])
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum([len(c) for c in rows])
    ci = np.concatenate(rows).astype(np.int32)
    A = CSR(n, n, rp, ci, rng.uniform(-1, 1, ci.size).astype(np.float32))
    assert int(rp[32] - rp[0]) > 1024
    B = _banded(n, (-2, 0, 1, 9), 53)
    shifted = _check(A, B, min_shift=4000, repeats=1)
    assert shifted <= 4500


def test_random_matrix_has_no_classes():
    A = gen.random_csr(8000, 7000, 12, mean_len=8.0, heavy_rows=3, heavy_len=900)
    B = gen.random_csr(7000, 9000, 13, mean_len=9.0)
    assert _check(A, B, min_shift=0) == 0


def test_pattern_too_wide_for_tables_stays_regular():
    # 32 A nonzeros 64 apart over B rows of 32 columns 2 apart: 1024 products,
    # 1024 distinct outputs per row -- more than the term tables hold, so the
    # rows are translates but keep the regular path
    A = _banded(6000, tuple(range(0, 64 * 32, 64)), 14, cols=6000 + 2048)
    B = _banded(6000 + 2048, tuple(range(0, 64, 2)), 15, cols=6000 + 4096)
    assert _check(A, B, min_shift=0, repeats=1) == 0


def test_learned_path_hands_translates_to_shift_classes():
    A = gen.stencil_3d_27(20)
    model = RowModel(path=weights_for("stencil3d"))
    _check(A, A, algo=L.ALGO_CUDA_LEARNED, model=model, min_shift=16 ** 3)


def test_host_memory_space():
    A = gen.laplacian_2d(100)
    _check(A, A, memory=L.MEM_HOST, min_shift=90 * 90)


def test_tiles_off_uses_the_table_kernel_for_members():
    import torch
    A = gen.stencil_3d_27(18)
    rp, ci, cv, _ = oracle.spgemm(A, A)
    dA = DeviceCSR.from_host(A)
    with Descriptor(memory=L.MEM_DEVICE) as d:
        d.set_shift_classes(2)
        d.set_row_tiles(False)
        ws_b, n = d.work_estimation(dA, dA)
        dC = DeviceCSR.empty(A.rows, A.cols, n)
        ws = torch.zeros(max(ws_b, 1), dtype=torch.uint8, device="cuda")
        d.compute(dA, dA, dC, ws)
        d.synchronize()
        assert d.shift_rows() > 0 and d.tiled_rows() == 0
        got = dC.to_host(n)
    assert np.array_equal(got.col_idx, ci)
    assert np.array_equal(_bits(got.values), _bits(cv))


def test_c_abi_numeric_with_caller_structure():
    # rvsp_cuda_symbolic, then rvsp_cuda_numeric(fill = 0) into a structure
    # the caller copied from the oracle: the member rows' tables come from
    # that structure
    import torch
    lib = L.load()
    A = gen.stencil_3d_27(16)
    rp, ci, cv, _ = oracle.spgemm(A, A)
    dA = DeviceCSR.from_host(A)
    plan = C.c_void_p()
    L.check(lib.rvsp_cuda_plan_create(C.byref(plan)), "plan_create")
    L.check(lib.rvsp_cuda_plan_set_shift_classes(plan, 2), "set_shift_classes")
    try:
        stream = C.c_void_p(torch.cuda.current_stream().cuda_stream or 1)
        crp = torch.zeros(A.rows + 1, dtype=torch.int32, device="cuda")
        total = C.c_int64()
        L.check(lib.rvsp_cuda_symbolic(plan, stream, A.rows, A.rows, A.cols,
                                       dA.row_ptr.data_ptr(), dA.col_idx.data_ptr(),
                                       dA.row_ptr.data_ptr(), dA.col_idx.data_ptr(),
                                       crp.data_ptr(), C.byref(total)), "symbolic")
        assert lib.rvsp_cuda_plan_shift_rows(plan) > 0
        assert np.array_equal(crp.cpu().numpy(), rp)
        cci = torch.from_numpy(ci).cuda()
        cvv = torch.full((ci.size,), float("nan"), dtype=torch.float32, device="cuda")
        ws_b = max(lib.rvsp_cuda_numeric_workspace_bytes(plan), 256)
        ws = torch.zeros(ws_b, dtype=torch.uint8, device="cuda")
        L.check(lib.rvsp_cuda_numeric(plan, stream, dA.row_ptr.data_ptr(), dA.col_idx.data_ptr(),
                                      dA.values.data_ptr(), dA.row_ptr.data_ptr(),
                                      dA.col_idx.data_ptr(), dA.values.data_ptr(),
                                      crp.data_ptr(), cci.data_ptr(), cvv.data_ptr(), 0,
                                      ws.data_ptr(), ws_b), "numeric")
        torch.cuda.synchronize()
        L.check(lib.rvsp_cuda_plan_status(plan, stream), "status")
        assert np.array_equal(_bits(cvv.cpu().numpy()), _bits(cv))
    finally:
        lib.rvsp_cuda_plan_destroy(plan)


def test_default_setting_leaves_cheap_rows_to_the_merge_kernels():
    # a 2D 5-point Laplacian on 300^2 (90,000 rows of 25 products): its rows
    # are translates, but at 25 products a row the default setting keeps the
    # merge kernels (setting 2 takes the classes); both exact
    A = gen.laplacian_2d(300)
    rp, ci, cv, _ = oracle.spgemm(A, A)
    for mode, expect in ((1, False), (2, True)):
        with Descriptor(memory=L.MEM_HOST) as d:
            d.set_shift_classes(mode)
            got = d.multiply(A, A)
            assert (d.shift_rows() > 0) == expect, (mode, d.shift_rows())
        assert np.array_equal(got.col_idx, ci)
        assert np.array_equal(_bits(got.values), _bits(cv))
