"""The row-binning MLP.

CPU: the FP64 oracle's analytic gradient against central finite differences
(pins the oracle), and its features against a direct per-row loop.
GPU: the CUDA features, gradient, inference and training against the
oracle; save/load round trip.  Gradient tolerance: relative L2 error of the
FP32 kernel gradient against FP64 <= 1e-4.
"""
import numpy as np
import pytest

from oracle import mlp_oracle as M
from rvsp import CSR, gen


def _params(seed=3):
    rng = np.random.default_rng(seed)
    p = np.zeros(M.N_PARAMS)
    p[M.W1:M.B1] = rng.normal(0, 0.5, M.B1 - M.W1)
    p[M.B1:M.W2] = rng.normal(0, 0.1, M.W2 - M.B1)
    p[M.W2:M.B2] = rng.normal(0, 0.25, M.B2 - M.W2)
    p[M.B2:M.W3] = rng.normal(0, 0.1, M.W3 - M.B2)
    p[M.W3:M.B3] = rng.normal(0, 0.25, M.B3 - M.W3)
    p[M.B3:M.N_TRAINED] = rng.normal(0, 0.1, 2)
    p[M.MU:M.INV_SD] = rng.normal(3, 1, 8)
    p[M.INV_SD:] = rng.uniform(0.3, 1.2, 8)
    return p


def _data(n=200, seed=4):
    rng = np.random.default_rng(seed)
    X = rng.normal(3, 2, (n, 8))
    T = np.stack([rng.normal(4, 2, n), (rng.random(n) < 0.4).astype(float)], 1)
    return X, T


def test_oracle_gradient_matches_finite_differences():
    p = _params()
    X, T = _data()
    _, g = M.gradient(p, X, T)
    idx = np.r_[0:6, 250:262, 300:310, 1300:1320, 1340:1350, 1400:1410]
    fd = M.finite_difference(p, X, T, idx)
    assert np.allclose(g[idx], fd, rtol=1e-5, atol=1e-8)


def test_oracle_features_direct_loop():
    A = gen.random_csr(40, 30, 5, mean_len=4.0, empty_frac=0.2)
    B = gen.random_csr(30, 50, 6, mean_len=3.0, empty_frac=0.2)
    F = M.features(A, B)
    for i in range(A.rows):
        ks = A.col_idx[A.row_ptr[i]:A.row_ptr[i + 1]]
        lens = [B.row_ptr[k + 1] - B.row_ptr[k] for k in ks]
        cols = [c for k in ks for c in B.col_idx[B.row_ptr[k]:B.row_ptr[k + 1]]]
        ops = sum(lens)
        span = (max(cols) - min(cols) + 1) if cols else 0
        raw = [len(ks), ops, max(lens, default=0), ops / len(ks) if len(ks) else 0.0,
               span, min(ops, span), B.cols, B.nnz / B.rows]
        assert np.allclose(F[i], np.log2(1.0 + np.array(raw, float))), i


@pytest.mark.gpu
def test_gpu_features_match_oracle():
    from rvsp import DeviceCSR
    from rvsp.learn import features
    A = gen.rmat(12, 8, seed=9)
    feat, ops = features(DeviceCSR.from_host(A), DeviceCSR.from_host(A))
    want = M.features(A, A)
    assert np.allclose(feat.cpu().numpy(), want, rtol=1e-5, atol=1e-5)


@pytest.mark.gpu
def test_gpu_gradient_matches_fp64_oracle():
    import torch
    from rvsp.learn import RowModel
    p = _params(7).astype(np.float32)
    X, T = _data(3000, 8)
    m = RowModel(seed=1)
    m.set_params(p)
    loss, g = m.gradient(torch.from_numpy(X.astype(np.float32)).cuda(),
                         torch.from_numpy(T.astype(np.float32)).cuda())
    want_loss, want = M.gradient(p.astype(np.float64), X.astype(np.float32), T)
    assert abs(loss - want_loss) <= 1e-4 * abs(want_loss)
    assert np.linalg.norm(g - want) <= 1e-4 * np.linalg.norm(want)


@pytest.mark.gpu
def test_gpu_training_reduces_loss_and_predicts_like_oracle(tmp_path):
    import torch
    from rvsp import DeviceCSR
    from rvsp.learn import RowModel, features
    from oracle import oracle
    A = gen.rmat(13, 8, seed=11)
    dA = DeviceCSR.from_host(A)
    feat, _ = features(dA, dA)
    rp, _, _ = oracle.symbolic(A, A)
    m_rows = np.diff(rp)
    t = np.stack([np.log2(1.0 + m_rows), (np.diff(A.row_ptr) <= 4).astype(float)], 1)
    tgt = torch.from_numpy(t.astype(np.float32)).cuda()
    model = RowModel(seed=2)
    f = feat.cpu().numpy()
    model.set_normalization(f.mean(0), f.std(0))
    hist = model.train(feat, tgt, batch=512, epochs=30, lr=3e-3)
    assert hist[-1] < 0.25 * hist[0]
    pred = model.predict(dA, dA).cpu().numpy()
    p64 = model.params().astype(np.float64)
    # FP32 inference against the FP64 forward pass of the same features ...
    *_, y_same = M.forward(p64, f.astype(np.float64))
    assert np.allclose(pred, y_same, rtol=1e-4, atol=1e-3)
    # ... and against the oracle's own FP64 features (outputs reach |y| ~ 20,
    # so FP32 feature rounding moves them by a few 1e-4)
    *_, y = M.forward(p64, M.features(A, A))
    assert np.allclose(pred, y, rtol=1e-3, atol=5e-3)
    path = tmp_path / "m.bin"
    model.save(path)
    other = RowModel(seed=99, path=path)
    assert np.array_equal(other.params(), model.params())
