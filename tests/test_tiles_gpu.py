"""Row tiles (k_tile.cu) for numeric-only repeats, through the C-ABI.

Runs of consecutive rows that share one term pattern are computed one row
per lane.  Bar: values bit-exact against the oracle (the reference's
numeric-only compute, spgemm_descr.c:330-349, re-running
gustavson_core_f32.inc:31-62 on new values) for stencils, a banded matrix
with far off-diagonals, tiles whose lanes skip rows of another pattern, a B
value array that is not 16-byte aligned (the 4-byte copy path), with tiles
switched off, which must give the same bits, and the compiled pattern
kernels (bulk copies of B ranges, bulk stores of whole tiles) at every
alignment of B's and C's value arrays.
"""
import ctypes as C

import numpy as np
import pytest

from oracle import oracle
from rvsp import DeviceCSR, gen
from rvsp import _lib as L
from rvsp.csr import CSR

pytestmark = pytest.mark.gpu


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream or 1)


class _Plan:
    def __init__(self, lib):
        self.lib = lib
        self.h = C.c_void_p()
        L.check(lib.rvsp_cuda_plan_create(C.byref(self.h)), "plan_create")

    def close(self):
        self.lib.rvsp_cuda_plan_destroy(self.h)

    def symbolic(self, dA, dB):
        import torch
        rp = torch.zeros(dA.rows + 1, dtype=torch.int32, device="cuda")
        total = C.c_int64()
        L.check(self.lib.rvsp_cuda_symbolic(self.h, _stream(), dA.rows, dB.rows, dB.cols,
                                            dA.row_ptr.data_ptr(), dA.col_idx.data_ptr(),
                                            dB.row_ptr.data_ptr(), dB.col_idx.data_ptr(),
                                            rp.data_ptr(), C.byref(total)), "symbolic")
        return rp, total.value

    def numeric(self, dA, dB, rp, ci, cv, fill, b_values_ptr=None, c_values_ptr=None):
        import torch
        ws_b = max(self.lib.rvsp_cuda_numeric_workspace_bytes(self.h), 256)
        ws = torch.zeros(ws_b, dtype=torch.uint8, device="cuda")
        bv = b_values_ptr if b_values_ptr is not None else dB.values.data_ptr()
        cvp = c_values_ptr if c_values_ptr is not None else cv.data_ptr()
        L.check(self.lib.rvsp_cuda_numeric(
            self.h, _stream(), dA.row_ptr.data_ptr(), dA.col_idx.data_ptr(),
            dA.values.data_ptr(), dB.row_ptr.data_ptr(), dB.col_idx.data_ptr(), bv,
            rp.data_ptr(), ci.data_ptr(), cvp, fill, ws.data_ptr(), ws_b), "numeric")
        torch.cuda.synchronize()
        L.check(self.lib.rvsp_cuda_plan_status(self.h, _stream()), "status")


def _bits(x):
    return np.ascontiguousarray(x, np.float32).view(np.uint32)


def _repeats(A, B, seeds, tiles=True, min_tiled=1, same_ab=False, pattern_kernels=True,
             min_jit=0):
    """Fill once, then numeric-only repeats with new A values (and B's when B
    is A); every repeat against the oracle.  Returns the tiled row count and
    the last C values."""
    import torch
    lib = L.load()
    dA = DeviceCSR.from_host(A)
    dB = dA if same_ab else DeviceCSR.from_host(B)
    plan = _Plan(lib)
    try:
        L.check(lib.rvsp_cuda_plan_set_row_tiles(plan.h, 1 if tiles else 0), "set_row_tiles")
        L.check(lib.rvsp_cuda_plan_set_pattern_kernels(plan.h, 1 if pattern_kernels else 0),
                "set_pattern_kernels")
        rp, n = plan.symbolic(dA, dB)
        ci = torch.zeros(max(n, 1), dtype=torch.int32, device="cuda")
        cv = torch.zeros(max(n, 1), dtype=torch.float32, device="cuda")
        plan.numeric(dA, dB, rp, ci, cv, 1)
        last = None
        for seed in seeds:
            rng = np.random.default_rng(seed)
            vals = (A.values + rng.uniform(-0.01, 0.01, A.nnz)).astype(np.float32)
            dA.values.copy_(torch.from_numpy(vals))
            torch.cuda.synchronize()
            cv.fill_(float("nan"))
            plan.numeric(dA, dB, rp, ci, cv, 0)
            A2 = A.with_values(vals)
            want_rp, want_ci, want_cv, _ = oracle.spgemm(A2, A2 if same_ab else B)
            assert np.array_equal(rp.cpu().numpy(), want_rp)
            assert np.array_equal(ci[:n].cpu().numpy(), want_ci)
            got = cv[:n].cpu().numpy()
            assert np.array_equal(_bits(got), _bits(want_cv)), \
                f"{int((_bits(got) != _bits(want_cv)).sum())} values differ"
            last = got
        tiled = lib.rvsp_cuda_plan_tiled_rows(plan.h)
        jit = lib.rvsp_cuda_plan_pattern_kernel_rows(plan.h)
        assert jit >= min_jit if pattern_kernels else jit == 0
        if tiles:
            assert tiled >= min_tiled
        else:
            assert tiled == 0
        return tiled, last
    finally:
        plan.close()


@pytest.mark.parametrize("grid", [16, 24])
def test_row_tiles_stencil_bit_exact(grid):
    A = gen.stencil_3d_27(grid)
    # interior rows (every coordinate in 1..grid-2) share one pattern and
    # come in runs of grid-2 consecutive rows: most of them are tiled
    tiled, on = _repeats(A, A, seeds=(5, 6), min_tiled=(grid - 2) ** 3 // 2, same_ab=True)
    _, off = _repeats(A, A, seeds=(6,), tiles=False, same_ab=True)
    assert np.array_equal(_bits(on), _bits(off))


def _banded(n, offsets, seed):
    rows = []
    for i in range(n):
        c = [i + o for o in offsets if 0 <= i + o < n]
        rows.append(c)
    rp = np.zeros(n + 1, np.int32)
    rp[1:] = np.cumsum([len(r) for r in rows])
    ci = np.concatenate(rows).astype(np.int32)
    rng = np.random.default_rng(seed)
    return CSR(n, n, rp, ci, rng.uniform(-1, 1, ci.size).astype(np.float32))


def test_row_tiles_banded_far_offsets():
    # seven diagonals, two of them far out: every interior row has the same
    # pattern; the B span of one A nonzero is one run of consecutive rows
    A = _banded(6000, (-700, -33, -1, 0, 2, 41, 650), 3)
    B = _banded(6000, (-5, 0, 1, 9, 300), 4)
    _repeats(A, B, seeds=(1, 2), min_tiled=4000)


def test_row_tiles_lanes_skip_other_patterns():
    # even rows take B rows 0 and 1 (40 + 40 columns), odd rows B rows 2 and 3
    # (20 + 60 over the same columns): one shared map, but only the even rows
    # can use its table, so each tile takes every other lane
    rng = np.random.default_rng(21)
    brows = [np.arange(0, 40), np.arange(40, 80), np.arange(0, 20), np.arange(20, 80)]
    brp = np.zeros(5, np.int32)
    brp[1:] = np.cumsum([len(r) for r in brows])
    bci = np.concatenate(brows).astype(np.int32)
    B = CSR(4, 80, brp, bci, rng.uniform(-1, 1, bci.size).astype(np.float32))
    arows = [[0, 1] if i % 2 == 0 else [2, 3] for i in range(640)]
    arp = np.zeros(641, np.int32)
    arp[1:] = np.cumsum([len(r) for r in arows])
    aci = np.concatenate(arows).astype(np.int32)
    A = CSR(640, 4, arp, aci, rng.uniform(-1, 1, aci.size).astype(np.float32))
    tiled, _ = _repeats(A, B, seeds=(7, 8), min_tiled=1)
    assert tiled <= 320


def test_row_tiles_b_values_not_16_byte_aligned():
    # B's values one float into a larger buffer: the stage copies fall back
    # to 4-byte cp.async; the values stay bit-exact
    import torch
    lib = L.load()
    A = gen.stencil_3d_27(14)
    dA = DeviceCSR.from_host(A)
    dB = DeviceCSR.from_host(A)
    shifted = torch.zeros(A.nnz + 1, dtype=torch.float32, device="cuda")
    plan = _Plan(lib)
    try:
        rp, n = plan.symbolic(dA, dB)
        ci = torch.zeros(n, dtype=torch.int32, device="cuda")
        cv = torch.zeros(n, dtype=torch.float32, device="cuda")
        plan.numeric(dA, dB, rp, ci, cv, 1)
        rng = np.random.default_rng(9)
        bvals = (A.values + rng.uniform(-0.01, 0.01, A.nnz)).astype(np.float32)
        shifted[1:].copy_(torch.from_numpy(bvals))
        torch.cuda.synchronize()
        plan.numeric(dA, dB, rp, ci, cv, 0, b_values_ptr=shifted.data_ptr() + 4)
        want = oracle.spgemm(A, A.with_values(bvals))[2]
        assert np.array_equal(_bits(cv.cpu().numpy()), _bits(want))
        assert lib.rvsp_cuda_plan_tiled_rows(plan.h) > 0
    finally:
        plan.close()


def test_descriptor_row_tiles_switch():
    # the descriptor-level switch: the same numeric-only repeat with tiles on
    # and off, bit-identical to each other and to the oracle, and the
    # tiled-row count reported
    import torch
    from rvsp import Descriptor
    A = gen.stencil_3d_27(18)
    scaled = (A.values * np.float32(1.5)).astype(np.float32)
    outs = []
    for tiles in (True, False):
        dA = DeviceCSR.from_host(A)
        with Descriptor(algo=L.ALGO_CUDA_PLAIN, memory=L.MEM_DEVICE) as d:
            d.set_row_tiles(tiles)
            _, n = d.work_estimation(dA, dA)
            dC = DeviceCSR.empty(A.rows, A.cols, n, "cuda")
            ws = torch.zeros(256, dtype=torch.uint8, device="cuda")
            d.compute(dA, dA, dC, ws)
            dA.values.copy_(torch.from_numpy(scaled))
            d.compute(dA, dA, dC, ws)
            d.synchronize()
            outs.append(dC.values.cpu().numpy().copy())
            assert (d.tiled_rows() > 0) == tiles
    assert np.array_equal(_bits(outs[0]), _bits(outs[1]))
    A2 = A.with_values(scaled)
    assert np.array_equal(_bits(outs[0]), _bits(oracle.spgemm(A2, A2)[2]))


@pytest.mark.parametrize("shift", [0, 2])
def test_pattern_kernels_match_table_kernel(shift):
    # the largest pattern of a 24^3 stencil gets a kernel compiled for it
    # (registers for the outputs); its values equal the table kernel's and
    # the oracle's, with the shift classes on (members) and off (shared maps)
    import torch
    lib = L.load()
    A = gen.stencil_3d_27(24)
    outs = []
    for jit in (True, False):
        dA = DeviceCSR.from_host(A)
        plan = _Plan(lib)
        try:
            L.check(lib.rvsp_cuda_plan_set_shift_classes(plan.h, shift), "set_shift_classes")
            L.check(lib.rvsp_cuda_plan_set_pattern_kernels(plan.h, int(jit)),
                    "set_pattern_kernels")
            rp, n = plan.symbolic(dA, dA)
            ci = torch.zeros(n, dtype=torch.int32, device="cuda")
            cv = torch.zeros(n, dtype=torch.float32, device="cuda")
            plan.numeric(dA, dA, rp, ci, cv, 1)
            rng = np.random.default_rng(17)
            vals = (A.values + rng.uniform(-0.01, 0.01, A.nnz)).astype(np.float32)
            dA.values.copy_(torch.from_numpy(vals))
            torch.cuda.synchronize()
            cv.fill_(float("nan"))
            plan.numeric(dA, dA, rp, ci, cv, 0)
            rows = lib.rvsp_cuda_plan_pattern_kernel_rows(plan.h)
            assert (rows > 0) == jit, rows
            outs.append(cv.cpu().numpy())
            A2 = A.with_values(vals)
            assert np.array_equal(_bits(outs[-1]), _bits(oracle.spgemm(A2, A2)[2]))
        finally:
            plan.close()
    assert np.array_equal(_bits(outs[0]), _bits(outs[1]))
    compiles, ms = C.c_int32(), C.c_double()
    lib.rvsp_cuda_pattern_kernel_stats(C.byref(compiles), C.byref(ms))
    assert compiles.value >= 1


@pytest.mark.parametrize("b_off,c_off", [(0, 0), (1, 3), (2, 1), (3, 2)])
def test_pattern_kernels_any_alignment(b_off, c_off):
    # a 40^3 stencil: interior runs of 36 rows, so whole tiles (32 rows of
    # the pattern) exist and their C block goes out by one bulk store; B's
    # and C's values are handed over b_off / c_off floats into larger buffers,
    # so the bulk copies and stores start at every offset within 16 bytes
    import torch
    lib = L.load()
    A = gen.stencil_3d_27(40)
    dA = DeviceCSR.from_host(A)
    plan = _Plan(lib)
    try:
        rp, n = plan.symbolic(dA, dA)
        ci = torch.zeros(n, dtype=torch.int32, device="cuda")
        cv = torch.zeros(n, dtype=torch.float32, device="cuda")
        plan.numeric(dA, dA, rp, ci, cv, 1)
        rng = np.random.default_rng(31 + b_off)
        bvals = (A.values + rng.uniform(-0.01, 0.01, A.nnz)).astype(np.float32)
        bbuf = torch.zeros(A.nnz + 4, dtype=torch.float32, device="cuda")
        bbuf[b_off:b_off + A.nnz].copy_(torch.from_numpy(bvals))
        cbuf = torch.full((n + 4,), float("nan"), dtype=torch.float32, device="cuda")
        torch.cuda.synchronize()
        plan.numeric(dA, dA, rp, ci, cv, 0, b_values_ptr=bbuf.data_ptr() + 4 * b_off,
                     c_values_ptr=cbuf.data_ptr() + 4 * c_off)
        assert lib.rvsp_cuda_plan_pattern_kernel_rows(plan.h) > 0
        got = cbuf.cpu().numpy()
        want = oracle.spgemm(A, A.with_values(bvals))[2]
        assert np.array_equal(_bits(got[c_off:c_off + n]), _bits(want))
        # nothing written outside C's values
        assert np.isnan(got[:c_off]).all() and np.isnan(got[c_off + n:]).all()
    finally:
        plan.close()
