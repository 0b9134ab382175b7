"""The learned path (RVSP_SPGEMM_ALGO_CUDA_LEARNED): MLP-sized single fused
pass with device-side overflow detection and the plain path as fallback.

The bar is the same as the plain path's: structure and values bit-exact
against the oracle, whatever the model predicts.  Overflow is forced by a
small capacity scale and by an untrained model, and values changed between
work_estimation and compute must be seen by compute.  The A/B test reports
what the trained network gains over the plain path on a power-law matrix.
"""
import time

import numpy as np
import pytest

from oracle import oracle
from rvsp import CSR, Descriptor, DeviceCSR, gen
from rvsp import _lib as L

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def model():
    """A model trained in-test on small seeded R-MAT matrices."""
    from rvsp import train
    table = {"k": list(train.K_BINS), "L": list(train.L_BINS),
             "merge_faster": [[True] * len(train.L_BINS)] * len(train.K_BINS)}
    X, T = train.harvest(table, matrices=10, rows_per_matrix=1024, seed=3,
                         scales=(11, 12, 13), workers=2)
    m, hist, summary = train.train(X, T, epochs=25)
    assert hist[-1] < hist[0]
    return m


def learned(model, memory=L.MEM_HOST, scale=None):
    d = Descriptor(algo=L.ALGO_CUDA_LEARNED, memory=memory)
    d.set_model(model)
    if scale is not None:
        d.set_capacity_scale(scale)
    return d


def assert_exact(got, A, B, what):
    rp, ci, cv, _ = oracle.spgemm(A, B)
    assert np.array_equal(got.row_ptr, rp), what
    assert np.array_equal(got.col_idx, ci), what
    assert np.array_equal(got.values.view(np.uint32), cv.view(np.uint32)), what


def test_learned_parity_rmat_host(model):
    A = gen.rmat(14, 16, seed=21)
    with learned(model) as d:
        C = d.multiply(A, A)
        assert_exact(C, A, A, "learned host")
        assert np.array_equal(d.get_op_counts(A.rows), oracle.spgemm(A, A)[3])


def test_learned_parity_rmat_device(model):
    import torch
    A = gen.rmat(14, 16, seed=22)
    B = gen.rmat(14, 16, seed=23)
    dA, dB = DeviceCSR.from_host(A), DeviceCSR.from_host(B)
    with learned(model, memory=L.MEM_DEVICE) as d:
        ws_b, n = d.work_estimation(dA, dB)
        dC = DeviceCSR.empty(A.rows, B.cols, n)
        ws = torch.zeros(max(ws_b, 1), dtype=torch.uint8, device="cuda")
        torch.cuda.synchronize()
        d.compute(dA, dB, dC, ws)
        d.synchronize()
        assert_exact(dC.to_host(n), A, B, "learned device")


@pytest.mark.parametrize("scale", [0.05, 0.5])
def test_learned_forced_overflow(model, scale):
    A = gen.rmat(13, 16, seed=24)
    with learned(model, scale=scale) as d:
        C = d.multiply(A, A)
        assert d.overflow_rows() > 0
        assert_exact(C, A, A, f"overflow scale {scale}")


def test_untrained_model_is_still_exact():
    from rvsp.learn import RowModel
    A = gen.rmat(12, 16, seed=25)
    raw = RowModel(seed=4)
    with learned(raw) as d:
        assert_exact(d.multiply(A, A), A, A, "untrained")


def test_values_changed_between_estimation_and_compute(model):
    A = gen.rmat(13, 16, seed=26)
    B = A.copy()
    with learned(model) as d:
        ws_b, n = d.work_estimation(A, B)
        B.values *= -1.5  # same pattern, new values, before the first compute
        Cm = CSR(A.rows, B.cols, np.zeros(A.rows + 1, np.int32), np.zeros(n, np.int32),
                 np.zeros(n, np.float32))
        d.compute(A, B, Cm, np.zeros(256, np.uint8))
        assert_exact(Cm, A, B, "values changed")
        A2 = A.with_values((A.values * 0.5).astype(np.float32))
        d.compute(A2, B, Cm, np.zeros(256, np.uint8))  # numeric-only reuse
        assert_exact(Cm, A2, B, "reuse after learned")


def test_learned_on_other_structures(model):
    A = gen.laplacian_2d(256)
    with learned(model) as d:
        assert_exact(d.multiply(A, A), A, A, "laplacian")
    A = gen.uniform_rows(2048, 2048, 16, 9)
    B = gen.uniform_rows(2048, 2048, 16, 10)
    with learned(model) as d:
        assert_exact(d.multiply(A, B), A, B, "uniform")
    A = gen.random_csr(3000, 2000, 11, mean_len=6.0, heavy_rows=5, heavy_len=1500)
    B = gen.random_csr(2000, 60000, 12, mean_len=20.0, heavy_rows=5, heavy_len=4000)
    with learned(model) as d:
        assert_exact(d.multiply(A, B), A, B, "irregular + dense rows")


def test_multiply_plain_both_memory_spaces():
    A = gen.random_csr(500, 400, 13, mean_len=5.0)
    B = gen.random_csr(400, 700, 14, mean_len=6.0)
    with Descriptor() as d:
        assert_exact(d.multiply_once(A, B), A, B, "multiply host")
    with Descriptor(memory=L.MEM_DEVICE) as d:
        r = d.multiply_once(DeviceCSR.from_host(A), DeviceCSR.from_host(B))
        assert_exact(r.to_host(), A, B, "multiply device")
        r.free()


def _time(fn, reps=3):
    import torch
    fn()
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        t0 = time.perf_counter()
        fn()
        torch.cuda.synchronize()
        best = min(best, time.perf_counter() - t0)
    return best


def test_learned_vs_plain_on_power_law():
    """A/B with the shipped R-MAT model (weights/rowmlp_rmat.bin): the same
    power-law product with and without the network (device memory, one full
    product per call, best of 5).  Both exact; the learned analysis (one
    fused pass instead of the symbolic pass + the numeric pass) is not
    slower than the plain path, and the times are printed."""
    from rvsp.learn import RowModel, weights_for
    shipped = RowModel(path=weights_for("rmat16"))
    A = gen.rmat(16, 16, seed=27)
    dA = DeviceCSR.from_host(A)
    plain = Descriptor(memory=L.MEM_DEVICE)
    lrn = learned(shipped, memory=L.MEM_DEVICE)
    t_plain = _time(lambda: plain.multiply_once(dA, dA).free(), reps=5)
    t_learned = _time(lambda: lrn.multiply_once(dA, dA).free(), reps=5)
    r = lrn.multiply_once(dA, dA)
    assert_exact(r.to_host(), A, A, "A/B learned")
    r.free()
    print(f"\nR-MAT 2^16 A*A: plain {t_plain * 1e3:.2f} ms, learned {t_learned * 1e3:.2f} ms, "
          f"gain {t_plain / t_learned:.2f}x, overflow rows {lrn.overflow_rows()}")
    assert t_learned <= 1.05 * t_plain