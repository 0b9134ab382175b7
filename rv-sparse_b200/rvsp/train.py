"""Autotuning and training of the learned row binning.

    python -m rvsp.train [--matrices 200] [--rows-per-matrix 2048] [--out DIR]
    python -m rvsp.train --families rmat,stencil,laplace,uniform,poisson \
        --name mixed --table weights/autotune.json      # the general model

1. autotune(): for a grid of (A nonzeros per row k, B row length L) bins,
   times the same synthetic product with the merge accumulator and with the
   warp hash (plan merge policy 2 against 1), with CUDA events on the
   library's own phase profiler; the table of which accumulator is faster
   per bin is the measured-timing label of the model's second output.
2. harvest(): seeded R-MAT matrices (n = 2^14 .. 2^18, 16 edge draws per row,
   quadrant probabilities (0.57, 0.19, 0.19, 0.05), duplicates merged), C = A x A.
   Per row: the 8 features (GPU kernel), the exact output nnz (GPU symbolic
   pass) and the accumulator label looked up in the autotune table.  With
   --families, products of other seeded families join the R-MAT ones
   (_family_job): the general model the non-power-law workloads use.
3. train(): Adam in the library's GPU kernels; writes the weight file and a
   JSON summary (losses, prediction error, held-out overflow rate).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import multiprocessing as mp
import time
from pathlib import Path

import numpy as np

from . import _lib as L
from . import gen
from .api import Descriptor, DeviceCSR
from .learn import DEFAULT_WEIGHTS, RowModel, features

K_BINS = (1, 2, 4, 8, 12, 16)
L_BINS = (2, 4, 8, 16, 32, 64, 128)
MERGE_MAX_NNZ, MERGE_MAX_OPS = 16, 2048
HASH_MARGIN = 0.9  # the hash labels a bin only when under 90% of the merge time


def _bin(v, edges):
    """Index of the edge nearest to v in log2 space (the bins are powers of
    two or near them, so a row of 5 nonzeros sits with 4, not with 8)."""
    le = np.log2(np.asarray(edges, np.float64))
    lv = np.log2(np.maximum(np.asarray(v, np.float64), 1.0))
    return np.abs(lv[..., None] - le).argmin(axis=-1)


def autotune(n_rows: int = 65536, reps: int = 3, seed: int = 5) -> dict:
    """Per (k, L) bin: product time with merge (policy 2) and with the warp
    hash (policy 1); returns {"k": [...], "L": [...], "merge_ms": [[..]],
    "hash_ms": [[..]], "merge_faster": [[..]]}."""
    import torch
    merge_ms = np.full((len(K_BINS), len(L_BINS)), np.nan)
    hash_ms = np.full_like(merge_ms, np.nan)
    for i, k in enumerate(K_BINS):
        for j, ln in enumerate(L_BINS):
            if k * ln > MERGE_MAX_OPS:
                continue
            A = gen.uniform_rows(n_rows, n_rows, k, seed + 17 * i + j)
            B = gen.uniform_rows(n_rows, n_rows, ln, seed + 1000 + 17 * i + j)
            dA, dB = DeviceCSR.from_host(A), DeviceCSR.from_host(B)
            for policy, out in ((2, merge_ms), (1, hash_ms)):
                with Descriptor(memory=L.MEM_DEVICE, profiling=True) as d:
                    d.set_merge_policy(policy)
                    ws_b, nnz = d.work_estimation(dA, dB)
                    dC = DeviceCSR.empty(A.rows, B.cols, nnz)
                    ws = torch.zeros(max(ws_b, 1), dtype=torch.uint8, device="cuda")
                    torch.cuda.synchronize()
                    d.compute(dA, dB, dC, ws)
                    d.synchronize()
                    d.phase_times(reset=True)
                    for _ in range(reps):
                        d.work_estimation(dA, dB)
                        d.compute(dA, dB, dC, ws)
                    d.synchronize()
                    t = d.phase_times(reset=True)
                    out[i, j] = (t["symbolic"][0] + t["numeric"][0]) / reps
    # merge unless the hash is clearly faster: ties go to the merge, which
    # needs no scratch and has no per-row floor
    faster = np.where(np.isnan(merge_ms), False, hash_ms >= HASH_MARGIN * merge_ms)
    return {"k": list(K_BINS), "L": list(L_BINS), "n_rows": n_rows,
            "merge_ms": np.nan_to_num(merge_ms, nan=-1).tolist(),
            "hash_ms": np.nan_to_num(hash_ms, nan=-1).tolist(),
            "merge_faster": faster.tolist()}


def merge_label(nnz: np.ndarray, ops: np.ndarray, table: dict) -> np.ndarray:
    """1 where the row may merge and the table says merge is faster."""
    if "merge_ms" in table and "hash_ms" in table:
        m = np.asarray(table["merge_ms"], np.float64)
        h = np.asarray(table["hash_ms"], np.float64)
        faster = (m > 0) & (h >= HASH_MARGIN * m)
    else:  # a table given only as the boolean grid
        faster = np.asarray(table["merge_faster"], bool)
    mean_len = np.where(nnz > 0, ops / np.maximum(nnz, 1), 0.0)
    ki = _bin(nnz, table["k"])
    li = _bin(mean_len, table["L"])
    eligible = (nnz <= MERGE_MAX_NNZ) & (ops <= MERGE_MAX_OPS) & (nnz > 0)
    return (eligible & faster[ki, li]).astype(np.float32)


FAMILIES = ("rmat", "stencil", "laplace", "uniform", "poisson")


def _family_job(args):
    """One seeded training product (A, B) of a matrix family, as plain arrays
    (runs in a worker process).  rmat: R-MAT n = 2^scale, 16 edge draws per
    row, C = A x A; stencil: 27-point stencil on g^3, C = A x A; laplace: 2D
    5-point Laplacian on g^2, C = A x A; uniform: n x n, k uniform columns per
    row, A x B; poisson: n log-uniform in [256, 65536], Poisson(mu) rows, mu
    uniform in [8, 32], A x B (the batched products' shape)."""
    family, seed = args
    rng = np.random.default_rng(seed)
    if family == "rmat":
        A = gen.rmat(int(rng.integers(14, 19)), 16, seed=seed)
        B = A
    elif family == "stencil":
        A = gen.stencil_3d_27(int(rng.integers(16, 49)))
        A = A.with_values(rng.uniform(-1, 1, A.nnz).astype(np.float32))
        B = A
    elif family == "laplace":
        A = gen.laplacian_2d(int(rng.integers(128, 1025)))
        B = A
    elif family == "uniform":
        n = int(2 ** rng.uniform(12, 16))
        k = int(rng.integers(4, 33))
        A = gen.uniform_rows(n, n, k, seed)
        B = gen.uniform_rows(n, n, int(rng.integers(4, 33)), seed + 1)
    else:
        n = int(round(float(np.exp(rng.uniform(np.log(256), np.log(65536))))))
        A = gen.poisson_rows(n, float(rng.uniform(8, 32)), seed)
        B = gen.poisson_rows(n, float(rng.uniform(8, 32)), seed + 1)
    pack = lambda M: (M.rows, M.cols, M.row_ptr, M.col_idx, M.values)
    return family, seed, pack(A), (None if B is A else pack(B))


def exact_row_nnz(dA, dB):
    """Per-row output nnz of A x B from the library's GPU symbolic pass."""
    import torch
    lib = L.load()
    plan = C.c_void_p()
    L.check(lib.rvsp_cuda_plan_create(C.byref(plan)), "plan_create")
    try:
        rp = torch.empty(dA.rows + 1, dtype=torch.int32, device="cuda")
        total = C.c_int64()
        L.check(lib.rvsp_cuda_symbolic(plan, C.c_void_p(torch.cuda.current_stream().cuda_stream),
                                       dA.rows, dB.rows, dB.cols, dA.row_ptr.data_ptr(),
                                       dA.col_idx.data_ptr(), dB.row_ptr.data_ptr(),
                                       dB.col_idx.data_ptr(), rp.data_ptr(),
                                       C.byref(total)), "symbolic")
        return (rp[1:] - rp[:-1]).to(torch.int64)
    finally:
        lib.rvsp_cuda_plan_destroy(plan)


def harvest(table: dict, matrices: int = 200, rows_per_matrix: int = 2048,
            seed: int = 1000, scales=(14, 15, 16, 17, 18), workers: int = 8,
            families=("rmat",), extra_per_family: int = 0):
    """(features [N, 8], targets [N, 2]) as numpy arrays.  `matrices` R-MAT
    products cycle through `scales`; every other family in `families` adds
    `extra_per_family` products (see _family_job)."""
    import torch
    from .csr import CSR
    rng = np.random.default_rng(seed)
    jobs = [("rmat-scale", int(scales[i % len(scales)]), seed + i) for i in range(matrices)]
    for fi, fam in enumerate(f for f in families if f != "rmat"):
        jobs += [(fam, 0, seed + 100000 * (fi + 1) + i) for i in range(extra_per_family)]
    feats, targets = [], []
    ctx = mp.get_context("spawn")
    with ctx.Pool(workers) as pool:
        work = [(_rmat_job, (sc, s)) if fam == "rmat-scale" else (_family_job, (fam, s))
                for fam, sc, s in jobs]
        results = [pool.apply_async(fn, (a,)) for fn, a in work]
        for res in results:
            out = res.get()
            if len(out) == 7:  # R-MAT of a given scale
                _, _, rows, cols, rp, ci, v = out
                A = CSR(rows, cols, rp, ci, v)
                B = None
            else:
                _, _, pa, pb = out
                A = CSR(*pa)
                B = None if pb is None else CSR(*pb)
            dA = DeviceCSR.from_host(A)
            dB = dA if B is None else DeviceCSR.from_host(B)
            f, ops = features(dA, dB)
            m = exact_row_nnz(dA, dB)
            take = rng.choice(A.rows, size=min(rows_per_matrix, A.rows), replace=False)
            idx = torch.from_numpy(take).cuda()
            f = f[idx].cpu().numpy()
            ops_h = ops[idx].cpu().numpy().astype(np.float64)
            m_h = m[idx].cpu().numpy().astype(np.float64)
            nnz = np.diff(A.row_ptr)[take].astype(np.float64)
            y0 = np.log2(1.0 + m_h)
            y1 = merge_label(nnz, ops_h, table)
            feats.append(f)
            targets.append(np.stack([y0, y1], 1).astype(np.float32))
            del dA, dB
    X = np.concatenate(feats)
    T = np.concatenate(targets)
    perm = rng.permutation(X.shape[0])
    return X[perm], T[perm]


def _rmat_job(args):
    scale, seed = args
    A = gen.rmat(scale, 16, seed=seed)
    return scale, seed, A.rows, A.cols, A.row_ptr, A.col_idx, A.values


def train(X, T, seed: int = 7, epochs: int = 40, batch: int = 1024, lr: float = 3e-3,
          holdout: float = 0.1):
    import torch
    n = X.shape[0]
    nh = int(n * holdout)
    Xtr, Ttr, Xte, Tte = X[nh:], T[nh:], X[:nh], T[:nh]
    model = RowModel(seed=seed)
    model.set_normalization(Xtr.mean(0), Xtr.std(0))
    hist = model.train(torch.from_numpy(Xtr).cuda(), torch.from_numpy(Ttr).cuda(),
                       batch=batch, epochs=epochs, lr=lr)
    # held-out error of the prediction, evaluated with the FP32 forward pass
    # of the same parameters
    p = model.params().astype(np.float64)
    w1, b1 = p[0:256].reshape(32, 8), p[256:288]
    w2, b2 = p[288:1312].reshape(32, 32), p[1312:1344]
    w3, b3 = p[1344:1408].reshape(2, 32), p[1408:1410]
    x = (Xte - p[1410:1418]) * p[1418:1426]
    y = np.maximum(np.maximum(x @ w1.T + b1, 0) @ w2.T + b2, 0) @ w3.T + b3
    m_true = np.exp2(Tte[:, 0]) - 1
    m_hat = np.exp2(y[:, 0]) - 1
    cap = np.ceil(1.15 * np.maximum(m_hat, 0)) + 16
    summary = {
        "samples": int(n), "train_loss_first": float(hist[0]),
        "train_loss_last": float(hist[-1]),
        "holdout_median_abs_log2_err": float(np.median(np.abs(y[:, 0] - Tte[:, 0]))),
        "holdout_overflow_rate_at_1.15": float(np.mean(m_true > cap)),
        "holdout_class_accuracy": float(np.mean((y[:, 1] > 0) == (Tte[:, 1] > 0.5))),
        "holdout_merge_label_rate": float(np.mean(Tte[:, 1])),
    }
    return model, hist, summary


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--matrices", type=int, default=200)
    ap.add_argument("--rows-per-matrix", type=int, default=2048)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--workers", type=int, default=8)
    ap.add_argument("--out", default=str(DEFAULT_WEIGHTS.parent))
    ap.add_argument("--families", default="rmat",
                    help="comma-separated: rmat plus any of " + ", ".join(FAMILIES[1:]))
    ap.add_argument("--extra-per-family", type=int, default=40)
    ap.add_argument("--name", default="rmat", help="weights written to rowmlp_<name>.bin")
    ap.add_argument("--table", default=None, help="reuse an autotune table (JSON)")
    args = ap.parse_args(argv)
    out = Path(args.out)
    out.mkdir(parents=True, exist_ok=True)
    families = tuple(f for f in args.families.split(",") if f)
    t0 = time.time()
    if args.table:
        table = json.loads(Path(args.table).read_text())
    else:
        table = autotune()
        (out / "autotune.json").write_text(json.dumps(table, indent=1) + "\n")
    t1 = time.time()
    X, T = harvest(table, args.matrices, args.rows_per_matrix, workers=args.workers,
                   families=families, extra_per_family=args.extra_per_family)
    t2 = time.time()
    model, hist, summary = train(X, T, epochs=args.epochs)
    model.save(out / f"rowmlp_{args.name}.bin")
    summary.update({"loss_history": [float(h) for h in hist],
                    "seconds": {"autotune": t1 - t0, "harvest": t2 - t1,
                                "train": time.time() - t2},
                    "matrices": args.matrices, "rows_per_matrix": args.rows_per_matrix,
                    "families": list(families),
                    "extra_per_family": args.extra_per_family if len(families) > 1 else 0})
    (out / f"rowmlp_{args.name}.json").write_text(json.dumps(summary, indent=1) + "\n")
    print(json.dumps({k: v for k, v in summary.items() if k != "loss_history"}))


if __name__ == "__main__":
    main()
