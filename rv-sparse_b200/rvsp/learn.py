"""The row-binning model: Python wrapper over the rvsp_mlp_* C-ABI.

The network, its training and its inference all run in the library's CUDA
kernels (k_mlp.cu); this module moves arrays and calls them.  Device arrays
are torch CUDA tensors used as storage.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

import numpy as np

from . import _lib as L

N_FEATURES = 8
N_PARAMS = 1426
N_TRAINED = 1410
MU, INV_SD = 1410, 1418
DEFAULT_WEIGHTS = Path(__file__).resolve().parent.parent / "weights" / "rowmlp_rmat.bin"
# Trained on R-MAT plus stencil, Laplacian, uniform and Poisson-row products
# (python -m rvsp.train --families ... --name mixed).
MIXED_WEIGHTS = DEFAULT_WEIGHTS.parent / "rowmlp_mixed.bin"


def weights_for(workload: str) -> Path:
    """The R-MAT model for power-law inputs, the general one otherwise (when
    it exists)."""
    if workload.startswith("rmat") or not MIXED_WEIGHTS.exists():
        return DEFAULT_WEIGHTS
    return MIXED_WEIGHTS


def _stream():
    import torch
    return C.c_void_p(torch.cuda.current_stream().cuda_stream)


def features(A, B):
    """(features float32 [rows, 8] on device, op counts int64 [rows]) of A x B
    for DeviceCSR operands."""
    import torch
    lib = L.load()
    feat = torch.empty((A.rows, N_FEATURES), dtype=torch.float32, device=A.row_ptr.device)
    ops = torch.empty(A.rows, dtype=torch.int64, device=A.row_ptr.device)
    L.check(lib.rvsp_mlp_features(_stream(), A.rows, B.rows, B.cols,
                                  A.row_ptr.data_ptr(), A.col_idx.data_ptr(),
                                  B.row_ptr.data_ptr(), B.col_idx.data_ptr(),
                                  feat.data_ptr(), ops.data_ptr()), "mlp_features")
    return feat, ops


class RowModel:
    """rvsp_mlp_t: 8 -> 32 -> 32 -> 2 row-binning network on the GPU."""

    def __init__(self, seed: int = 0, path: str | Path | None = None):
        self.lib = L.load()
        self.h = C.c_void_p()
        L.check(self.lib.rvsp_mlp_create(C.byref(self.h), C.c_uint64(seed)), "mlp_create")
        if path is not None:
            self.load(path)

    def close(self):
        if self.h:
            self.lib.rvsp_mlp_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        p = np.zeros(N_PARAMS, np.float32)
        L.check(self.lib.rvsp_mlp_get_params(self.h, p.ctypes.data, N_PARAMS), "get_params")
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        L.check(self.lib.rvsp_mlp_set_params(self.h, p.ctypes.data, p.size), "set_params")

    def set_normalization(self, mean, sd) -> None:
        p = self.params()
        p[MU:INV_SD] = np.asarray(mean, np.float32)
        p[INV_SD:N_PARAMS] = 1.0 / np.maximum(np.asarray(sd, np.float32), 1e-3)
        self.set_params(p)

    def gradient(self, feat, target):
        g = np.zeros(N_TRAINED, np.float32)
        loss = C.c_float()
        L.check(self.lib.rvsp_mlp_gradient(self.h, _stream(), feat.data_ptr(),
                                           target.data_ptr(), feat.shape[0],
                                           g.ctypes.data, C.byref(loss)), "mlp_gradient")
        return float(loss.value), g

    def train(self, feat, target, batch: int = 1024, epochs: int = 20,
              lr: float = 3e-3) -> np.ndarray:
        hist = np.zeros(epochs, np.float32)
        L.check(self.lib.rvsp_mlp_train(self.h, _stream(), feat.data_ptr(),
                                        target.data_ptr(), feat.shape[0], batch, epochs,
                                        C.c_float(lr), hist.ctypes.data), "mlp_train")
        return hist

    def predict(self, A, B):
        import torch
        out = torch.empty((A.rows, 2), dtype=torch.float32, device=A.row_ptr.device)
        L.check(self.lib.rvsp_mlp_predict(self.h, _stream(), A.rows, B.rows, B.cols,
                                          A.row_ptr.data_ptr(), A.col_idx.data_ptr(),
                                          B.row_ptr.data_ptr(), B.col_idx.data_ptr(),
                                          out.data_ptr()), "mlp_predict")
        return out

    def save(self, path) -> None:
        L.check(self.lib.rvsp_mlp_save(self.h, str(path).encode()), "mlp_save")

    def load(self, path) -> None:
        L.check(self.lib.rvsp_mlp_load(self.h, str(path).encode()), "mlp_load")
