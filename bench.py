#!/usr/bin/env python3
"""SpGEMM benchmark: GFLOP/s (2 x intermediate products / s) and HBM fraction.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--workload NAME]
  python bench.py --impl reference ...      # the reference scalar CPU backend

A step is one pass of the hot path over the workload's input:
  stencil3d_job  (default) the 128^3 27-point stencil's whole job: C = A x A
              by the learned path (work_estimation + compute), then 50
              numeric-only computes with A's values perturbed by
              U[-0.01, 0.01]; plain and learned products and the repeat are
              also reported alone (run_job).
  laplace2d   C = A x A, A the 2D 5-point Laplacian on 1024^2
              (n = 1,048,576, nnz = 5,238,784): one full product
              (work_estimation + compute) with A resident in HBM.
  uniform4096 C = A x B, 4096^2, exactly 16 nnz/row (A seed S, B seed S+1).
  stencil3d   C = A x A, 27-point stencil on 128^3: one full product.
  stencil3d_reuse  the same product, numeric-only compute (structure reused,
              values perturbed by U[-0.01, 0.01] between repeats).

Output: one JSON line (rank 0).  `value` is device-timed throughput of the
whole job with inputs resident in HBM (CUDA events around each step, L2
flushed by a 256 MiB write between steps, max over ranks); `e2e` is the same
metric through the public C API in host memory space (pinned host buffers,
host<->device copies inside the timed region); `roofline` is for the
dominant kernel phase, timed with CUDA events on its own launch stream;
`cpu_baseline` is the reference scalar backend on this host's cores, and
its `check` (and the line's `correct`) says whether the GPU's C of the last
timed step is bit-identical to the reference's product of the same operands
(one product; every 16th of a batch; the last panel), as the reference
bench records `correct` for every timed run.  `correct` is null when the
CPU leg is skipped (--no-cpu-baseline, or more than one rank).

Multi-GPU (torchrun): every rank computes the full workload on its own GPU
(weak scaling: rows of C are independent and no data crosses GPUs).
"""
from __future__ import annotations

import argparse
import gc
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT / "rv-sparse_b200"))

METRIC = "SpGEMM GFLOP/s + HBM % peak: learned-binned/batched vs plain GPU Gustavson"
UNIT = "GFLOP/s"
FALLBACK_HBM_GBS = 6650.0

WORKLOADS = {
    "stencil3d_job": ("3D 27-point stencil 128^3 (n=2,097,152, nnz=55,742,968), C=A*A: the "
                      "first product (learned binning, fused single pass) then 50 numeric-only "
                      "descriptor repeats with A's values perturbed by U[-0.01,0.01]"),
    "laplace2d": "2D 5-point Laplacian 1024x1024 (n=1,048,576, nnz=5,238,784), C=A*A, full product",
    "uniform4096": "4096x4096, exactly 16 nnz/row uniform columns, values U[-1,1], C=A*B, full product",
    "stencil3d": "3D 27-point stencil 128^3 (n=2,097,152, nnz=55,742,968), C=A*A, full product",
    "stencil3d_reuse": "3D 27-point stencil 128^3, C=A*A, numeric-only repeats (values perturbed U[-0.01,0.01])",
    "rmat16": "R-MAT n=2^16, 16 edges/row, (0.57,0.19,0.19,0.05), values U(0,1], C=A*A, full product",
    "rmat18": "R-MAT n=2^18, 16 edges/row, (0.57,0.19,0.19,0.05), values U(0,1], C=A*A, full product",
    "batch512": ("512 independent products C_i=A_i*B_i, n log-uniform in [256, 65536], "
                 "Poisson(mu) row lengths with mu U[8,32], uniform columns, values U[-1,1]; "
                 "one batch analysis + fill, then numeric-only repeats with every value "
                 "redrawn (CUDA graph replay)"),
}

WORKLOADS["mtx_ingest"] = (
    "Matrix Market ingest: the 2D 5-point Laplacian 1024^2 as a symmetric real coordinate "
    "file (lower triangle, 3,143,680 stored entries, 52 MB of text) read into canonical CSR "
    "(5,238,784 entries): host parse on all cores + GPU canonicalisation")
MTX_METRIC = "Matrix Market ingest: stored entries per second"
MTX_UNIT = "Mentries/s"

WORKLOADS["rmat20_panels"] = (
    "R-MAT n=2^20, 16 edges/row, (0.57,0.19,0.19,0.05), values U(0,1], C=A*A as row panels "
    "of A of at most 2^28 products each (nnz(C) ~9e9 exceeds int32), every panel a full "
    "product per step")
PANEL_MAX_OPS = 1 << 28

BATCH_COUNT, BATCH_SEED = 512, 7


def batch_inputs():
    from rvsp import gen
    return gen.batched_products(count=BATCH_COUNT, seed=BATCH_SEED)


def build_inputs(name: str, seed: int = 2024, grid: int = 128):
    from rvsp import gen
    if name == "laplace2d":
        A = gen.laplacian_2d(1024)
        return A, A
    if name == "uniform4096":
        return gen.uniform_rows(4096, 4096, 16, seed), gen.uniform_rows(4096, 4096, 16, seed + 1)
    if name in ("stencil3d", "stencil3d_reuse"):
        A = gen.stencil_3d_27(grid)
        return A, A
    if name.startswith("rmat"):
        A = gen.rmat(int(name[4:]), 16, seed=1)
        return A, A
    raise ValueError(name)


def measured_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d.get("hbm_gbs", FALLBACK_HBM_GBS)), "measured"
    return FALLBACK_HBM_GBS, "fallback"


def committed_traffic(workload: str, phase: str):
    p = ROOT / "profiles" / "traffic.json"
    if not p.exists():
        return None
    d = json.loads(p.read_text())
    return d.get(workload, {}).get(phase)


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms; start()
    returns once the first sample is written, so the timed region that
    follows is covered.  Between start() and stop() Python's garbage
    collector is off (collected once before), so no collection pause lands
    in a timed step."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"rvsp_clocks_{os.getpid()}.csv"

    def start(self):
        gc.collect()
        gc.disable()
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 5.0 and self.proc.poll() is None:
            if self.path.exists() and self.path.stat().st_size > 0:
                break
            time.sleep(0.02)

    def stop(self):
        gc.enable()
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, smax, reasons = [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.path.read_text().splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        self.path.unlink(missing_ok=True)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def mtx_ingest_input():
    """(text, stored entries, (rows, col, val) of the stored entries, 0-based):
    the Laplacian's lower triangle as a symmetric coordinate file."""
    from rvsp import gen
    A = gen.laplacian_2d(1024)
    rows = np.repeat(np.arange(A.rows, dtype=np.int64), np.diff(A.row_ptr))
    keep = rows >= A.col_idx
    r, c, v = rows[keep], A.col_idx[keep].astype(np.int64), A.values[keep]
    body = "\n".join(f"{a} {b} {x:g}" for a, b, x in zip((r + 1).tolist(), (c + 1).tolist(),
                                                        v.tolist()))
    text = (f"%%MatrixMarket matrix coordinate real symmetric\n"
            f"{A.rows} {A.cols} {r.size}\n{body}\n").encode()
    return text, int(r.size), (r.astype(np.int32), c.astype(np.int32), v.astype(np.float32))


def run_mtx_reference(args):
    """The reference's reader (assemble_csr_matrix, oracle/_ref/librvsp_mtx_ref.so)
    on the same file, one thread (the tool is single-threaded); the restatement
    if the reference reader is absent."""
    import tempfile
    sys.path.insert(0, str(ROOT))
    from oracle import oracle
    text, stored, _ = mtx_ingest_input()
    kind = "reference" if oracle.ref_mtx_available() else "port"
    with tempfile.TemporaryDirectory() as tmp:
        path = Path(tmp) / "laplace.mtx"
        path.write_bytes(text)
        times = []
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            if kind == "reference":
                oracle.ref_mtx_to_csr(path)
            else:
                oracle.mtx_to_csr(text)
            if i >= args.warmup:
                times.append(time.perf_counter() - t0)
    el = float(sum(times))
    return stored * len(times) / el / 1e6, el, kind


def run_mtx(args, world, rank, local):
    """mtx_ingest: a step is one rvsp_csr_parse_mtx of the file's text (held
    in host memory) into a device CSR: threaded host parse, the COO upload and
    the GPU canonicalisation, timed on the host clock (the call returns when
    C is complete on the device).  The GPU part alone is timed with CUDA
    events through rvsp_cuda_coo_to_csr on the same entries already on the
    device.  e2e: rvsp_csr_read_mtx from a file into host CSR."""
    import ctypes as C
    import tempfile
    import torch
    from rvsp import _lib as L

    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    lib = L.load()
    text, stored, (r, c, v) = mtx_ingest_input()
    sampler = ClockSampler(local)
    sampler.start()

    def parse_once():
        m = L.CsrMatrix()
        L.check(lib.rvsp_csr_parse_mtx(text, len(text), L.MEM_DEVICE, C.byref(m)), "parse_mtx")
        nnz = m.nnz
        lib.rvsp_csr_destroy(C.byref(m))
        return nnz

    for _ in range(args.warmup):
        nnz = parse_once()
    torch.cuda.synchronize(dev)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        parse_once()
        times.append(time.perf_counter() - t0)
    el = float(sum(times))
    value = stored * args.steps / el / 1e6

    # the GPU canonicalisation alone, on device-resident entries
    dr, dc, dv = (torch.from_numpy(x).to(dev) for x in (r, c, v))
    rp = torch.empty(1024 * 1024 + 1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    gpu_ms = []
    for i in range(args.warmup + args.steps):
        col_p, val_p, n_out = C.c_void_p(), C.c_void_p(), C.c_int32()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        L.check(lib.rvsp_cuda_coo_to_csr(C.c_void_p(stream.cuda_stream), 1024 * 1024,
                                         1024 * 1024, stored, 1, dr.data_ptr(), dc.data_ptr(),
                                         dv.data_ptr(), rp.data_ptr(), C.byref(col_p),
                                         C.byref(val_p), C.byref(n_out)), "coo_to_csr")
        e1.record(stream)
        torch.cuda.synchronize(dev)
        if i >= args.warmup:
            gpu_ms.append(e0.elapsed_time(e1))
        # the output arrays are the caller's (cudaFree): free them through
        # rvsp_csr_destroy of a struct that owns just those two
        out = L.CsrMatrix()
        out.col_idx, out.values, out.owns_data = col_p, val_p, 2
        lib.rvsp_csr_destroy(C.byref(out))
    clocks = sampler.stop()
    g_ms = float(np.mean(gpu_ms))
    # compulsory bytes of the canonicalisation: read the stored entries
    # (row, col, value), write C (row_ptr, columns, values)
    alg = stored * 12 + (1024 * 1024 + 1) * 4 + int(nnz) * 8
    peak, peak_kind = measured_peaks()
    achieved = alg / (g_ms * 1e-3) / 1e9

    with tempfile.TemporaryDirectory() as tmp:
        path = Path(tmp) / "laplace.mtx"
        path.write_bytes(text)
        m = L.CsrMatrix()
        e_times = []
        for i in range(1 + max(1, args.e2e_steps // 5)):
            t0 = time.perf_counter()
            L.check(lib.rvsp_csr_read_mtx(str(path).encode(), L.MEM_HOST, C.byref(m)), "read_mtx")
            if i:
                e_times.append(time.perf_counter() - t0)
            lib.rvsp_csr_destroy(C.byref(m))
    e2e = {"value": stored * len(e_times) / sum(e_times) / 1e6, "unit": MTX_UNIT,
           "h2d_bytes_per_step": stored * 12, "d2h_bytes_per_step": (1024 * 1024 + 1) * 4 + int(nnz) * 8,
           "api": "rvsp_csr_read_mtx (file to host CSR)"}
    cpu = None
    if not args.no_cpu_baseline:
        cv, _, kind = run_mtx_reference(argparse.Namespace(warmup=0, steps=1))
        cpu = {"value": cv, "unit": MTX_UNIT, "cores": 1, "kind": kind,
               "sample": "one read of the same file by the reference reader"}
        # check: the same text through rvsp_csr_parse_mtx into host arrays
        # against the reference reader's CSR, bit for bit
        sys.path.insert(0, str(ROOT))
        from oracle import oracle
        if kind == "reference":
            with tempfile.TemporaryDirectory() as tmp:
                path = Path(tmp) / "laplace.mtx"
                path.write_bytes(text)
                want = oracle.ref_mtx_to_csr(path)
        else:
            want = oracle.mtx_to_csr(text)[2:]
        m = L.CsrMatrix()
        L.check(lib.rvsp_csr_parse_mtx(text, len(text), L.MEM_HOST, C.byref(m)), "parse_mtx")
        n_got = int(m.nnz)

        def take(ptr, ctype, n, dtype):
            if n == 0:
                return np.zeros(0, dtype)
            return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(ctype)), shape=(n,)).copy()
        got = (take(m.row_ptr, C.c_int32, int(m.rows) + 1, np.int32),
               take(m.col_idx, C.c_int32, n_got, np.int32),
               take(m.values, C.c_float, n_got, np.float32))
        lib.rvsp_csr_destroy(C.byref(m))
        same = (want is not None and np.array_equal(got[0], want[0])
                and np.array_equal(got[1], want[1])
                and np.array_equal(got[2].view(np.uint32),
                                   np.ascontiguousarray(want[2], np.float32).view(np.uint32)))
        cpu["check"] = {"bit_exact": bool(same), "mismatched": 0 if same else 1,
                        "against": f"{kind}: the reader's CSR of the same text"}
    line = {"metric": MTX_METRIC, "value": value, "unit": MTX_UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": "mtx_ingest", "description": WORKLOADS["mtx_ingest"],
                       "stored_entries": stored, "nnz": int(nnz), "text_bytes": len(text),
                       "host_threads": os.cpu_count(),
                       "gpu_canonicalise_ms": g_ms,
                       "timing": "host clock around the call (it returns with C complete)"},
            "roofline": {"bound": "hbm", "kernel": "rvsp_cuda_coo_to_csr (all its launches)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                         if peak_kind == "measured" else "fallback 6.65 TB/s",
                         "traffic": None, "algorithmic_bytes_per_launch": alg},
            "clocks": clocks, "e2e": e2e, "gpu_launches": 11 * args.steps,
            "cpu_baseline": cpu,
            "correct": cpu["check"]["bit_exact"] if cpu else None}
    print(json.dumps(line), flush=True)
    return 0


def typed_inputs(args):
    """The workload's matrices with float64 values (the FP32 values widened)
    or int8 values (seeded, in [-8, 8])."""
    A, B = build_inputs(args.workload, grid=args.grid)
    rng = np.random.default_rng(42)

    def vals(M):
        if args.dtype == "f64":
            return M.values.astype(np.float64)
        return rng.integers(-8, 9, M.nnz).astype(np.int8)
    ta = (A.rows, A.cols, A.row_ptr, A.col_idx, vals(A))
    tb = ta if B is A else (B.rows, B.cols, B.row_ptr, B.col_idx, vals(B))
    return A, B, ta, tb


def run_typed(args, world, rank, local):
    """--dtype f64 / i8: a step is one rvsp_spgemm_csr of the workload's
    matrices with {RVSP_BACKEND_CUDA, FP64, FP64} or {.., INT8, INT32}: host
    arrays in, host arrays out (the only form the reference offers for these
    dtypes), timed on the host clock.  The reference's legacy scalar kernel
    on the same inputs, one thread, is the CPU baseline."""
    import torch
    from rvsp import intermediate_products, spgemm_typed
    if rank != 0:
        return 0
    torch.cuda.set_device(local)
    sys.path.insert(0, str(ROOT))
    from oracle import oracle
    A, B, ta, tb = typed_inputs(args)
    flops = 2.0 * float(intermediate_products(A, B).sum())
    sampler = ClockSampler(local)
    sampler.start()
    for _ in range(args.warmup):
        rp, ci, cv = spgemm_typed(ta, tb, args.dtype)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        rp, ci, cv = spgemm_typed(ta, tb, args.dtype)
        times.append(time.perf_counter() - t0)
    clocks = sampler.stop()
    el = float(sum(times))
    value = flops * args.steps / el / 1e9
    cpu = None
    if not args.no_cpu_baseline and oracle.ref_available():
        t0 = time.perf_counter()
        st, rrp, rci, rcv = oracle.ref_spgemm_typed(ta, tb, args.dtype)
        t = time.perf_counter() - t0
        if st == 0:
            same = (np.array_equal(rp, rrp) and np.array_equal(ci, rci)
                    and cv.dtype == rcv.dtype and cv.tobytes() == rcv.tobytes())
            cpu = {"value": flops / t / 1e9, "unit": UNIT, "cores": 1, "kind": "reference",
                   "sample": "one product by the reference's legacy scalar kernel",
                   "check": {"bit_exact": bool(same), "mismatched": 0 if same else 1,
                             "against": "reference: the product of the last timed step"}}
    in_b = sum(x[2].nbytes + x[3].nbytes + x[4].nbytes for x in ((ta, tb) if tb is not ta else (ta,)))
    out_b = rp.nbytes + ci.nbytes + cv.nbytes
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * el / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64" if args.dtype == "f64" else "i8->i32", "data": "synthetic",
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload],
                       "path": f"one-shot {args.dtype} (host arrays)",
                       "products": int(flops / 2), "nnz_c": int(rp[-1]),
                       "timing": "host clock around rvsp_spgemm_csr (host in, host out)"},
            "clocks": clocks,
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": int(in_b),
                    "d2h_bytes_per_step": int(out_b),
                    "api": "rvsp_spgemm_csr {RVSP_BACKEND_CUDA, " +
                           ("FP64, FP64}" if args.dtype == "f64" else "INT8, INT32}")},
            "gpu_launches": None, "cpu_baseline": cpu,
            "correct": cpu["check"]["bit_exact"] if cpu else None}
    print(json.dumps(line), flush=True)
    return 0


def run_reference(args, world, rank):
    """The reference scalar CPU backend (oracle/_ref/librvsp_ref.so, built from
    the reference sources; the C restatement if that is absent) on all host
    threads; rank 0 only."""
    if rank != 0:
        return 0
    sys.path.insert(0, str(ROOT))
    from oracle import oracle
    from rvsp import intermediate_products
    threads = os.cpu_count() or 1
    kind = "reference" if oracle.ref_available() else "port"
    if args.workload == "batch512":
        # each step: the next `threads` products of the batch, one per thread
        prods = batch_inputs()
        pflops = [2.0 * float(intermediate_products(A, B).sum()) for A, B in prods]
        fl, el = 0.0, 0.0
        for i in range(args.warmup + args.steps):
            lo = (i * threads) % len(prods)
            sample = [prods[(lo + j) % len(prods)] for j in range(threads)]
            done, t = oracle.time_reference_batch(sample, seconds=1e9, threads=threads)
            if i >= args.warmup:
                fl += sum(pflops[(lo + j) % len(prods)] for j in done)
                el += t
        value = fl / el / 1e9
        sample = (f"{args.steps * threads} of the {len(prods)} products, one per thread "
                  f"({args.steps} steps x {threads} threads)")
    elif args.workload == "stencil3d_job":
        # each step: the job's first product + JOB_CPU_REPEATS numeric-only
        # repeats (two perturbed value sets alternating), rows of A cut into
        # one panel per thread
        from rvsp import gen
        A = gen.stencil_3d_27(args.grid)
        flops = 2.0 * float(intermediate_products(A, A).sum())
        sets = job_value_sets_host(A, 2, args.seed + 2)
        cpu_sets = [(sets[r % 2], sets[r % 2]) for r in range(JOB_CPU_REPEATS)]
        fl, el = 0.0, 0.0
        for i in range(args.warmup + args.steps):
            t = oracle.time_reference_job(A, A, cpu_sets, threads)
            if i >= args.warmup:
                fl += (1 + JOB_CPU_REPEATS) * flops
                el += t
        value = fl / el / 1e9
        sample = (f"per step the job's first product + {JOB_CPU_REPEATS} of its "
                  f"{args.repeats} numeric-only repeats, rows of A cut into {threads} "
                  f"panels, one per thread ({args.steps} steps)")
    elif args.workload == "rmat20_panels":
        # C does not fit the reference (nnz(C) ~9e9 > INT32_MAX): each step
        # times `threads` panels of 256 rows spread over the matrix, one per
        # thread
        from rvsp import gen
        A = gen.rmat(20, 16, seed=1)
        ops = intermediate_products(A, A)
        starts = np.linspace(0, A.rows - 256, 64).astype(int)
        fl, el = 0.0, 0.0
        for i in range(args.warmup + args.steps):
            rs = [int(starts[(i * threads + j) % len(starts)]) for j in range(threads)]
            sample = [(A.row_panel(r, r + 256), A) for r in rs]
            done, t = oracle.time_reference_batch(sample, seconds=1e9, threads=threads)
            if i >= args.warmup:
                fl += sum(2.0 * float(ops[rs[j]:rs[j] + 256].sum()) for j in done)
                el += t
        value = fl / el / 1e9
        sample = (f"{args.steps * threads} panels of 256 rows spread over the matrix, one "
                  f"per thread ({args.steps} steps x {threads} threads)")
    else:
        A, B = build_inputs(args.workload, grid=args.grid)
        flops = 2.0 * float(intermediate_products(A, B).sum())
        per_step = []
        for i in range(args.warmup + args.steps):
            runs, el = oracle.time_reference_oneshot(A, B, seconds=0.0, threads=threads,
                                                     max_runs=threads)
            if i >= args.warmup:
                per_step.append((runs, el))
        runs = sum(r for r, _ in per_step)
        el = sum(e for _, e in per_step)
        value = flops * runs / el / 1e9
        sample = (f"{runs} full one-shot products of {args.workload} "
                  f"({args.steps} steps x {threads} threads)")
    line = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic",
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload],
                       "grid": args.grid if "stencil" in args.workload else None},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def run_batch(args, world, rank, local):
    """batch512: the batch API in device memory space.  A step is one
    numeric-only compute of all 512 products (the captured graph: value
    refresh + numeric pass of every group) after every value of every A_i and
    B_i was redrawn; the redraw (device copies from pre-drawn pools) and the
    L2 flush happen before each step's start event."""
    import ctypes as C
    import torch
    import rvsp
    from rvsp import Batch, CSR, DeviceCSR, intermediate_products
    from rvsp import _lib as L

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    torch.cuda.set_stream(torch.cuda.Stream(dev))
    stream = torch.cuda.current_stream(dev)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)
        pg = dist

    prods = batch_inputs()
    ops = [int(intermediate_products(A, B).sum()) for A, B in prods]
    flops = 2.0 * float(sum(ops))
    dprods = [(DeviceCSR.from_host(A, dev), DeviceCSR.from_host(B, dev)) for A, B in prods]
    gen_t = torch.Generator(device=dev)
    gen_t.manual_seed(11)
    pools = [[(torch.rand(dA.nnz, generator=gen_t, device=dev) * 2 - 1,
               torch.rand(dB.nnz, generator=gen_t, device=dev) * 2 - 1)
              for dA, dB in dprods] for _ in range(2)]

    def redraw(i):
        for (dA, dB), (va, vb) in zip(dprods, pools[i % 2]):
            dA.values.copy_(va)
            dB.values.copy_(vb)

    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    b = Batch(memory=L.MEM_DEVICE, stream=stream, autotune=True)
    for dA, dB in dprods:
        b.add(dA, dB)
    torch.cuda.synchronize(dev)
    e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    e0.record(stream)
    total_nnz = b.work_estimation()
    e1.record(stream)
    b.compute()  # first compute: columns and values
    e2.record(stream)
    b.synchronize()
    analysis_ms, fill_ms = e0.elapsed_time(e1), e1.elapsed_time(e2)
    nnz = [b.nnz(i) for i in range(len(prods))]
    alg_bytes = sum(rvsp.algorithmic_bytes(A, B, n) for (A, B), n in zip(prods, nnz))

    sampler = ClockSampler(local)
    sampler.start()
    for i in range(args.warmup):
        redraw(i)
        flush.zero_()
        b.compute()
    b.synchronize()
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    for i in range(args.steps):
        redraw(i)
        flush.zero_()
        ev[i][0].record(stream)
        b.compute()
        ev[i][1].record(stream)
    torch.cuda.synchronize(dev)
    b.synchronize()
    clocks = sampler.stop()
    total_ms = float(sum(a.elapsed_time(c) for a, c in ev))
    if pg:
        t = torch.tensor([total_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * flops * args.steps / (total_ms * 1e-3) / 1e9
    stats = b.stats()
    tuning = b.tuning()
    peak, peak_kind = measured_peaks()
    achieved = alg_bytes / (ms_per_step * 1e-3) / 1e9

    # Every 16th product's operands in the last timed step and its C, for the
    # reference check in the CPU baseline leg.
    check_set = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        last = pools[(args.steps - 1) % 2]
        check_set = [(prods[i][0].with_values(last[i][0].cpu().numpy()),
                      prods[i][1].with_values(last[i][1].cpu().numpy()), b.result(i))
                     for i in range(0, len(prods), 16)]

    # End to end: host memory space, pinned operands; each step uploads every
    # value (inside compute) and copies every C_i back (row_ptr, col_idx,
    # values) into one pinned buffer sized for the largest product.
    e2e = None
    if rank == 0 or world > 1:
        def pinned(x):
            return torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy()
        hprods = [(CSR(A.rows, A.cols, pinned(A.row_ptr), pinned(A.col_idx), pinned(A.values)),
                   CSR(B.rows, B.cols, pinned(B.row_ptr), pinned(B.col_idx), pinned(B.values)))
                  for A, B in prods]
        hb = Batch(memory=L.MEM_HOST, merge_policy=stats["merge_policy"],
                   persistent=(tuning["persistent_merge_rows"],
                               tuning["persistent_blocks_per_sm"]))
        for A, B in hprods:
            hb.add(A, B)
        hb.work_estimation()
        mx_rows = max(A.rows for A, _ in prods)
        mx_nnz = max(max(nnz), 1)
        out_rp = pinned(np.zeros(mx_rows + 1, np.int32))
        out_ci = pinned(np.zeros(mx_nnz, np.int32))
        out_v = pinned(np.zeros(mx_nnz, np.float32))

        def e2e_step():
            hb.compute()
            for i, (A, B) in enumerate(hprods):
                c = L.CsrMatrix()
                c.rows, c.cols, c.nnz = A.rows, B.cols, mx_nnz
                c.row_ptr, c.col_idx = out_rp.ctypes.data, out_ci.ctypes.data
                c.values, c.dtype = out_v.ctypes.data, L.DTYPE_FP32
                hb.copy_result_into(i, c)
        e2e_step()
        e2e_step()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        torch.cuda.synchronize(dev)
        el = time.perf_counter() - t0
        h2d = sum(A.values.nbytes + B.values.nbytes for A, B in prods)
        d2h = sum(4 * (A.rows + 1) + 8 * n for (A, _), n in zip(prods, nnz))
        e2e = {"value": world * flops * args.e2e_steps / el / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "steps": args.e2e_steps,
               "api": "rvsp_spgemm_batch_compute + rvsp_spgemm_batch_copy_result per "
                      "product, host memory space (numeric-only repeats)"}
        hb.close()
        del hprods

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        sys.path.insert(0, str(ROOT))
        from oracle import oracle
        threads = os.cpu_count() or 1
        done, el = oracle.time_reference_batch(prods, seconds=12.0, threads=threads)
        cpu = {"value": sum(2.0 * ops[i] for i in done) / el / 1e9, "unit": UNIT,
               "cores": threads, "kind": "reference" if oracle.ref_available() else "port",
               "sample": f"first {len(done)} of {len(prods)} products (one-shot each, "
                         f"one per thread) on {threads} threads in {el:.1f} s"}
        cpu["check"] = reference_check(check_set, f"{len(check_set)} of {len(prods)} "
                                       "products (every 16th) of the last timed step")
        check_set = None

    b.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload],
                       "path": "batch", "products": len(prods), "seed": BATCH_SEED,
                       "rows_total": sum(A.rows for A, _ in prods),
                       "nnz_a_total": sum(A.nnz for A, _ in prods),
                       "nnz_b_total": sum(B.nnz for _, B in prods),
                       "nnz_c_total": int(total_nnz), "intermediate_products": int(sum(ops)),
                       "flops_per_step": flops, "algorithmic_bytes_per_step": alg_bytes,
                       "groups": stats["groups"],
                       "merge_policy_autotuned": stats["merge_policy"],
                       "numeric_shape_autotuned": tuning,
                       "graph_nodes": stats["graph_nodes"],
                       "analysis_ms": analysis_ms, "first_fill_ms": fill_ms,
                       "first_product_gflops": flops / ((analysis_ms + fill_ms) * 1e-3) / 1e9,
                       "l2": "flushed between steps (256 MiB write outside the step events)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU"},
            "hbm_frac": achieved / peak,
            "roofline": {"bound": "hbm", "kernel": "numeric-only batch graph",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                         if peak_kind == "measured" else "fallback 6.65 TB/s",
                         "traffic": committed_traffic(args.workload, "numeric"),
                         "algorithmic_bytes_per_launch": alg_bytes},
            "clocks": clocks, "e2e": e2e, "gpu_launches": stats["graph_nodes"],
            "cpu_baseline": cpu,
            "correct": cpu["check"]["bit_exact"] if cpu else None,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def run_panels(args, world, rank, local):
    """rmat20_panels: C = A x A for R-MAT 2^20 as row panels of A (each a
    full product per step: work_estimation + compute, device memory space).
    With N ranks the panels are shared out by op count (no data crosses GPUs;
    each rank holds all of B), so the total work is fixed: strong scaling."""
    import torch
    import rvsp
    from rvsp import CSR, Descriptor, DeviceCSR, gen, intermediate_products
    from rvsp import _lib as L
    from rvsp.panels import assign_panels, panel_bounds_fast

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    torch.cuda.set_stream(torch.cuda.Stream(dev))
    stream = torch.cuda.current_stream(dev)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=dev)
        pg = dist

    A = gen.rmat(20, 16, seed=1)
    ops = intermediate_products(A, A)
    bounds = panel_bounds_fast(ops, PANEL_MAX_OPS)
    mine = assign_panels(bounds, ops, world)[rank]
    panels = [A.row_panel(*bounds[i]) for i in mine]
    my_ops = int(sum(int(ops[bounds[i][0]:bounds[i][1]].sum()) for i in mine))
    flops_all = 2.0 * float(ops.sum())
    dB = DeviceCSR.from_host(A, dev)
    dP = [DeviceCSR.from_host(P, dev) for P in panels]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)

    model = None
    algo = L.ALGO_CUDA_PLAIN
    if args.path == "learned":
        from rvsp.learn import DEFAULT_WEIGHTS, RowModel
        model = RowModel(path=DEFAULT_WEIGHTS)
        algo = L.ALGO_CUDA_LEARNED
    descs = []
    for _ in dP:
        d = Descriptor(algo=algo, memory=L.MEM_DEVICE, stream=stream, profiling=True)
        if model is not None:
            d.set_model(model)
        descs.append(d)
    nnz = []
    ws_max = 1
    for d, P in zip(descs, dP):
        ws_b, n = d.work_estimation(P, dB)
        nnz.append(n)
        ws_max = max(ws_max, ws_b)
    mx = max(nnz) if nnz else 1
    dC = DeviceCSR.empty(max((P.rows for P in panels), default=1), A.cols, mx, dev)
    ws = torch.zeros(ws_max, dtype=torch.uint8, device=dev)

    def step():
        for d, P, n in zip(descs, dP, nnz):
            C_ = DeviceCSR(P.rows, A.cols, dC.row_ptr[:P.rows + 1], dC.col_idx[:max(n, 1)],
                           dC.values[:max(n, 1)])
            d.work_estimation(P, dB)
            d.compute(P, dB, C_, ws)

    sampler = ClockSampler(local)
    sampler.start()
    for _ in range(args.warmup):
        flush.zero_()
        step()
    torch.cuda.synchronize(dev)
    for d in descs:
        d.synchronize()
        d.phase_times(reset=True)
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        ev[i][0].record(stream)
        step()
        ev[i][1].record(stream)
    torch.cuda.synchronize(dev)
    for d in descs:
        d.synchronize()
    clocks = sampler.stop()
    total_ms = float(sum(a.elapsed_time(c) for a, c in ev))
    if pg:
        t = torch.tensor([total_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = flops_all * args.steps / (total_ms * 1e-3) / 1e9
    # The last panel's C stays in dC after the last step: its operands and C
    # for the reference check in the CPU baseline leg.
    check_set = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline and panels:
        P, n = panels[-1], nnz[-1]
        gC = DeviceCSR(P.rows, A.cols, dC.row_ptr[:P.rows + 1], dC.col_idx[:max(n, 1)],
                       dC.values[:max(n, 1)]).to_host(n)
        check_set = [(P, A, gC)]
    phases = {}
    for d in descs:
        for k, (ms, nl) in d.phase_times(reset=True).items():
            a = phases.setdefault(k, [0.0, 0])
            a[0] += ms
            a[1] += nl
    per_step = {k: (v[0] / args.steps, v[1] / args.steps) for k, v in phases.items() if v[1]}
    alg_bytes = sum(rvsp.algorithmic_bytes(P, A, n) for P, n in zip(panels, nnz))
    peak, peak_kind = measured_peaks()
    dom = max(per_step, key=lambda k: per_step[k][0]) if per_step else "numeric"
    dom_ms = per_step.get(dom, (ms_per_step, 0))[0]
    launches = int(sum(v[1] for v in per_step.values()))
    overflow = sum(d.overflow_rows() for d in descs)

    # End to end: one host-memory-space descriptor, panel by panel, pinned
    # operands and one pinned C buffer of the largest panel.
    e2e = None
    if (rank == 0 or world > 1) and args.e2e_steps > 0:
        def pinned(x):
            return torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy()
        hB = CSR(A.rows, A.cols, pinned(A.row_ptr), pinned(A.col_idx), pinned(A.values))
        hP = [CSR(P.rows, P.cols, pinned(P.row_ptr), pinned(P.col_idx), pinned(P.values))
              for P in panels]
        hC = CSR(max(P.rows for P in panels), A.cols, pinned(np.zeros(max(P.rows for P in panels) + 1, np.int32)),
                 pinned(np.zeros(mx, np.int32)), pinned(np.zeros(mx, np.float32)))
        he = Descriptor(algo=algo, memory=L.MEM_HOST)
        if model is not None:
            he.set_model(model)

        def e2e_step():
            for P, n in zip(hP, nnz):
                he.work_estimation(P, hB)
                C_ = CSR(P.rows, A.cols, hC.row_ptr[:P.rows + 1], hC.col_idx[:max(n, 1)],
                         hC.values[:max(n, 1)])
                he.compute(P, hB, C_, np.zeros(256, np.uint8))
        e2e_step()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        torch.cuda.synchronize(dev)
        el = time.perf_counter() - t0
        h2d = sum(P.nbytes() + A.nbytes() for P in panels)
        d2h = sum(4 * (P.rows + 1) + 8 * n for P, n in zip(panels, nnz))
        e2e_val = 2.0 * my_ops * args.e2e_steps / el / 1e9
        if pg:
            t = torch.tensor([el], device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            e2e_val = flops_all * args.e2e_steps / float(t.item()) / 1e9
        e2e = {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "steps": args.e2e_steps,
               "api": "rvsp_spgemm_work_estimation + rvsp_spgemm_compute per panel, "
                      "host memory space (B uploaded with every panel)"}
        he.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the reference on a bounded sample: small panels spread over the rows
        sys.path.insert(0, str(ROOT))
        from oracle import oracle
        threads = os.cpu_count() or 1
        rows = np.linspace(0, A.rows - 256, 64).astype(int)
        sample = [(A.row_panel(int(r), int(r) + 256), A) for r in rows]
        sops = [int(ops[int(r):int(r) + 256].sum()) for r in rows]
        done, el = oracle.time_reference_batch(sample, seconds=20.0, threads=threads)
        cpu = {"value": sum(2.0 * sops[i] for i in done) / el / 1e9, "unit": UNIT,
               "cores": threads, "kind": "reference" if oracle.ref_available() else "port",
               "sample": f"{len(done)} panels of 256 rows spread over the matrix, one-shot "
                         f"each, on {threads} threads in {el:.1f} s"}
        if check_set:
            cpu["check"] = reference_check(check_set, "the last panel of the last timed step")
            check_set = None

    for d in descs:
        d.close()
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload],
                       "path": args.path, "rows": A.rows, "nnz_a": A.nnz,
                       "panels": len(bounds), "panels_this_rank": len(mine),
                       "panel_max_ops": PANEL_MAX_OPS, "overflow_rows": overflow,
                       "nnz_c_this_rank": int(sum(nnz)), "products": int(ops.sum()),
                       "flops_per_step": flops_all, "algorithmic_bytes_per_step": alg_bytes,
                       "l2": "flushed between steps (256 MiB write outside the step events)",
                       "parallelism": f"panels over {world} GPUs" if world > 1 else "single GPU"},
            "hbm_frac": alg_bytes / (ms_per_step * 1e-3) / 1e9 / peak,
            "phase_ms_per_step": {k: v[0] for k, v in per_step.items()},
            "roofline": {"bound": "hbm", "kernel": f"{dom} phase",
                         "achieved": alg_bytes / (dom_ms * 1e-3) / 1e9, "peak": peak,
                         "unit": "GB/s", "frac": alg_bytes / (dom_ms * 1e-3) / 1e9 / peak,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                         if peak_kind == "measured" else "fallback 6.65 TB/s",
                         "traffic": committed_traffic(args.workload, dom),
                         "algorithmic_bytes_per_launch": alg_bytes},
            "clocks": clocks, "e2e": e2e, "gpu_launches": launches, "cpu_baseline": cpu,
            "correct": cpu["check"]["bit_exact"] if cpu and "check" in cpu else None,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


JOB_REPEATS = 50     # numeric-only repeats of the stencil job
JOB_CPU_REPEATS = 8  # repeats in the reference's bounded sample of the job


def panel_rows(ops: np.ndarray, world: int, rank: int):
    """Rank's contiguous row range [r0, r1) when the rows are cut into
    `world` panels of about equal op count (rows of C are independent)."""
    if world <= 1:
        return 0, int(ops.size)
    cum = np.concatenate([[0], np.cumsum(ops, dtype=np.int64)])
    cuts = [int(np.searchsorted(cum, cum[-1] * k / world)) for k in range(world + 1)]
    cuts[0], cuts[-1] = 0, int(ops.size)
    for k in range(1, world + 1):
        cuts[k] = max(cuts[k], cuts[k - 1])
    return cuts[rank], cuts[rank + 1]


def job_value_sets_host(A, n: int, seed: int):
    """n host copies of A's values perturbed by U[-0.01, 0.01] (seeded)."""
    rng = np.random.default_rng(seed)
    return [(A.values + rng.uniform(-0.01, 0.01, A.nnz)).astype(np.float32) for _ in range(n)]


def run_job(args, world, rank, local):
    """stencil3d_job (default): the 128^3 27-point stencil's whole job.  A
    step is C = A x A through the descriptor API in device memory space --
    work_estimation + compute on the learned path (fused single pass, or the
    plain two-pass path with --path plain) -- then JOB_REPEATS numeric-only
    computes into the same C, each with A's values (B is A) perturbed by
    U[-0.01, 0.01] (pre-drawn on the device, one array per repeat).  The
    first numeric-only compute builds the reuse structures (map, term
    tables, row tiles) inside the step.  value = (1 + JOB_REPEATS) products'
    flops per step time.  Beside it, timed separately on the same inputs:
    the plain and the learned full products alone, and the numeric-only
    repeat alone (read from the job's own per-compute events).  With N ranks
    the rows of A are cut into N panels of equal op count (each rank holds all
    of B and runs the job on its panel): strong scaling."""
    import torch
    import rvsp
    from rvsp import CSR, Descriptor, DeviceCSR, gen, intermediate_products
    from rvsp import _lib as L
    from rvsp.learn import RowModel, weights_for

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    torch.cuda.set_stream(torch.cuda.Stream(dev))
    stream = torch.cuda.current_stream(dev)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=dev)
        pg = dist
    R = args.repeats
    A = gen.stencil_3d_27(args.grid)
    ops = intermediate_products(A, A)
    flops_all = 2.0 * float(ops.sum())
    r0, r1 = panel_rows(ops, world, rank)
    p0, p1 = int(A.row_ptr[r0]), int(A.row_ptr[r1])
    P = A if world == 1 else A.row_panel(r0, r1)
    my_flops = 2.0 * float(ops[r0:r1].sum())
    dA = DeviceCSR.from_host(A, dev)
    dP = dA if world == 1 else DeviceCSR.from_host(P, dev)
    gen_t = torch.Generator(device=dev)
    gen_t.manual_seed(args.seed)
    vals = [dA.values + (torch.rand(A.nnz, generator=gen_t, device=dev) * 0.02 - 0.01)
            for _ in range(R)]
    views_b = [DeviceCSR(A.rows, A.cols, dA.row_ptr, dA.col_idx, v) for v in vals]
    views_p = views_b if world == 1 else [
        DeviceCSR(P.rows, P.cols, dP.row_ptr, dP.col_idx, v[p0:p1]) for v in vals]
    torch.cuda.synchronize(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    model_file = weights_for("stencil3d")
    model = RowModel(path=model_file)

    def make_descr(algo, memory=L.MEM_DEVICE, **kw):
        dd = Descriptor(algo=algo, memory=memory, **kw)
        if algo == L.ALGO_CUDA_LEARNED:
            dd.set_model(model)
        return dd

    algo = L.ALGO_CUDA_LEARNED if args.path == "learned" else L.ALGO_CUDA_PLAIN
    d = make_descr(algo, stream=stream, profiling=True)
    ws_bytes, c_nnz = d.work_estimation(dP, dA)
    dC = DeviceCSR.empty(P.rows, A.cols, c_nnz, dev)
    ws = torch.zeros(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    alg_bytes = rvsp.algorithmic_bytes(P, A, c_nnz)

    def job(ev=None):
        d.work_estimation(dP, dA)
        d.compute(dP, dA, dC, ws)
        if ev is not None:
            ev[0].record(stream)
        for r in range(R):
            d.compute(views_p[r], views_b[r], dC, ws)
            if ev is not None:
                ev[r + 1].record(stream)

    sampler = ClockSampler(local)
    sampler.start()
    for _ in range(args.warmup):
        flush.zero_()
        job()
    torch.cuda.synchronize(dev)
    d.synchronize()
    d.phase_times(reset=True)
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    E = torch.cuda.Event
    starts = [E(enable_timing=True) for _ in range(args.steps)]
    evs = [[E(enable_timing=True) for _ in range(R + 1)] for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        starts[i].record(stream)
        job(evs[i])
    torch.cuda.synchronize(dev)
    d.synchronize()
    if pg:
        pg.barrier()
    clocks = sampler.stop()
    step_ms = [starts[i].elapsed_time(evs[i][R]) for i in range(args.steps)]
    first_ms = [starts[i].elapsed_time(evs[i][0]) for i in range(args.steps)]
    rep_ms = [[evs[i][r].elapsed_time(evs[i][r + 1]) for r in range(R)]
              for i in range(args.steps)]
    phases = d.phase_times(reset=True)
    total_ms = float(sum(step_ms))
    if pg:
        t = torch.tensor([total_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = (1 + R) * flops_all * args.steps / (total_ms * 1e-3) / 1e9
    steady = [x for row in rep_ms for x in row[1:]]
    repeat_ms = float(np.median(steady)) if steady else float(np.mean([r[0] for r in rep_ms]))
    prep_ms = float(np.mean([r[0] for r in rep_ms])) - repeat_ms
    peak, peak_kind = measured_peaks()
    peak_src = (f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6.65 TB/s")
    repeat_gbs = alg_bytes / (repeat_ms * 1e-3) / 1e9
    tiled = d.tiled_rows()
    overflow = d.overflow_rows()
    per_step = {k: v[0] / args.steps for k, v in phases.items() if v[1]}
    launches = int(sum(v[1] for v in phases.values()) / args.steps)
    last_vals = vals[R - 1]

    # The full products alone, plain and learned, on the unperturbed values.
    def product_ms(pa, keep):
        dd = make_descr(pa, stream=stream)
        wsb, n = dd.work_estimation(dP, dA)
        cc = DeviceCSR.empty(P.rows, A.cols, n, dev)
        w = torch.zeros(max(wsb, 1), dtype=torch.uint8, device=dev)
        for _ in range(args.warmup):
            flush.zero_()
            dd.work_estimation(dP, dA)
            dd.compute(dP, dA, cc, w)
        torch.cuda.synchronize(dev)
        if pg:
            pg.barrier()
        es = [(E(enable_timing=True), E(enable_timing=True)) for _ in range(args.steps)]
        for i in range(args.steps):
            flush.zero_()
            es[i][0].record(stream)
            dd.work_estimation(dP, dA)
            dd.compute(dP, dA, cc, w)
            es[i][1].record(stream)
        torch.cuda.synchronize(dev)
        dd.synchronize()
        ms = float(sum(a.elapsed_time(b) for a, b in es)) / args.steps
        if pg:
            t = torch.tensor([ms], device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            ms = float(t.item())
        host = cc.to_host(n) if keep else None
        dd.close()
        del cc
        return ms, host
    keep = rank == 0 and world == 1 and not args.no_cpu_baseline
    plain_ms, plain_c = product_ms(L.ALGO_CUDA_PLAIN, keep)
    learned_ms, learned_c = product_ms(L.ALGO_CUDA_LEARNED, keep)
    job_c = dC.to_host(c_nnz) if keep else None
    last_host = last_vals.cpu().numpy() if keep else None
    d.close()

    # End to end through the public C API in host memory space: pinned host
    # operands, the job's first product and every repeat with host values
    # (two pinned perturbed arrays, alternating), C copied back each compute.
    e2e = None
    if args.e2e_steps > 0:
        def pinned(x):
            return torch.from_numpy(np.ascontiguousarray(x)).pin_memory().numpy()
        hA = CSR(A.rows, A.cols, pinned(A.row_ptr), pinned(A.col_idx), pinned(A.values))
        hP = hA if world == 1 else CSR(P.rows, P.cols, pinned(P.row_ptr), pinned(P.col_idx),
                                       pinned(P.values))
        hv = [pinned(v) for v in job_value_sets_host(A, 2, args.seed + 1)]
        hvb = [hA.with_values(v) for v in hv]
        hvp = hvb if world == 1 else [hP.with_values(v[p0:p1]) for v in hv]
        n = max(c_nnz, 1)
        hC = CSR(P.rows, A.cols, pinned(np.zeros(P.rows + 1, np.int32)),
                 pinned(np.zeros(n, np.int32)), pinned(np.zeros(n, np.float32)))
        hws = np.zeros(256, np.uint8)
        he = make_descr(algo, memory=L.MEM_HOST)

        def e2e_step():
            he.work_estimation(hP, hA)
            he.compute(hP, hA, hC, hws)
            for r in range(R):
                he.compute(hvp[r % 2], hvb[r % 2], hC, hws)
        e2e_step()
        torch.cuda.synchronize(dev)
        if pg:
            pg.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            e2e_step()
        torch.cuda.synchronize(dev)
        el = time.perf_counter() - t0
        if pg:
            t = torch.tensor([el], device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            el = float(t.item())
        h2d = P.nbytes() + (0 if world == 1 else A.nbytes()) + R * (
            P.values.nbytes + (0 if world == 1 else A.values.nbytes))
        d2h = (4 * (P.rows + 1) + 8 * c_nnz) + R * (4 * (P.rows + 1) + 4 * c_nnz)
        e2e = {"value": (1 + R) * flops_all * args.e2e_steps / el / 1e9, "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "steps": args.e2e_steps,
               "api": "rvsp_spgemm_work_estimation + rvsp_spgemm_compute, then "
                      f"{R} numeric-only rvsp_spgemm_compute, host memory space"}
        he.close()
        del hA, hP, hv, hvb, hvp, hC

    cpu, checks = None, None
    if keep:
        sys.path.insert(0, str(ROOT))
        from oracle import oracle
        threads = os.cpu_count() or 1
        sets = job_value_sets_host(A, 2, args.seed + 2)
        cpu_sets = [(sets[r % 2], sets[r % 2]) for r in range(JOB_CPU_REPEATS)]
        el = oracle.time_reference_job(A, A, cpu_sets, threads)
        kind = "reference" if oracle.ref_available() else "port"
        cpu = {"value": (1 + JOB_CPU_REPEATS) * flops_all / el / 1e9, "unit": UNIT,
               "cores": threads, "kind": kind,
               "sample": f"the job with {JOB_CPU_REPEATS} of its {R} numeric-only repeats "
                         f"(first product + {JOB_CPU_REPEATS} repeats, two perturbed value "
                         f"sets alternating), rows of A cut into {threads} panels, one per "
                         f"thread, in {el:.1f} s"}
        # Bit-exact checks of every measured path against the reference
        # library's descriptor: its first compute (unperturbed values) for the
        # plain and learned products, and a numeric-only compute with the last
        # repeat's values for the job's C.
        if oracle.ref_available():
            st, rp, ci, first, last = oracle.ref_job(A, A, [(last_host, last_host)])
        else:
            rp, ci, first, _ = oracle.spgemm(A, A)
            last = oracle.numeric_f32(A.with_values(last_host), A.with_values(last_host),
                                      rp, ci)
            st = 0
        checks = {}
        for name, got, want in (("plain", plain_c, first), ("learned", learned_c, first),
                                ("job", job_c, last)):
            checks[name] = bool(st == 0 and same_csr(got, rp, ci, want))
        cpu["check"] = {"bit_exact": all(checks.values()),
                        "mismatched": sum(not v for v in checks.values()),
                        "paths": checks,
                        "against": f"{kind}: descriptor first compute (plain, learned) and a "
                                   "numeric-only compute with the last repeat's values (job)"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "strong" if world > 1 else "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "stencil3d_job", "description": WORKLOADS["stencil3d_job"],
                       "path": args.path, "model": model_file.name, "grid": args.grid,
                       "rows": A.rows, "nnz_a": A.nnz, "nnz_c": int(c_nnz) if world == 1 else None,
                       "products": int(ops.sum()), "repeats": R, "seed": args.seed,
                       "flops_per_product": flops_all,
                       "algorithmic_bytes_per_product": rvsp.algorithmic_bytes(A, A, c_nnz)
                       if world == 1 else None,
                       "l2": "flushed between steps (256 MiB write outside the step events); "
                             "every repeat reads its own 223 MB value array",
                       "parallelism": f"row panels over {world} GPUs" if world > 1
                       else "single GPU",
                       "overflow_rows": overflow, "tiled_rows": tiled},
            "hbm_frac": (1 + R) * alg_bytes / (ms_per_step * 1e-3) / 1e9 / peak,
            "job": {"first_product_ms": float(np.mean(first_ms)),
                    "reuse_prep_ms": prep_ms, "repeat_ms": repeat_ms,
                    "repeat_gflops": my_flops / (repeat_ms * 1e-3) / 1e9,
                    "repeat_hbm_frac": repeat_gbs / peak},
            "plain": {"product_ms": plain_ms,
                      "gflops": flops_all / (plain_ms * 1e-3) / 1e9},
            "learned": {"product_ms": learned_ms,
                        "gflops": flops_all / (learned_ms * 1e-3) / 1e9},
            "learned_vs_plain": plain_ms / learned_ms,
            "job_vs_plain_job": ((plain_ms + prep_ms + R * repeat_ms) /
                                 (float(np.mean(first_ms)) + prep_ms + R * repeat_ms)),
            "phase_ms_per_step": per_step,
            "roofline": {"bound": "hbm",
                         "kernel": "numeric-only repeat: rvsp_pattern_tiles (kernels compiled "
                                   "per term pattern, the interior one persistent over every "
                                   "SM) on the caller's stream, the table tiles, leftover rows "
                                   "and class kernels on six side streams joined back into it; "
                                   "one launch = one numeric-only compute, timed by CUDA "
                                   "events on the caller's stream",
                         "achieved": repeat_gbs, "peak": peak, "unit": "GB/s",
                         "frac": repeat_gbs / peak, "peak_source": peak_src,
                         "traffic": committed_traffic("stencil3d_job", "repeat"),
                         "traffic_source": "committed: profiles/traffic.json stencil3d_job "
                                           "(DRAM bytes of every kernel of one repeat, one ncu "
                                           "capture named there), not measured in this run",
                         "algorithmic_bytes_per_launch": alg_bytes},
            "clocks": clocks, "e2e": e2e, "gpu_launches": launches,
            "cpu_baseline": cpu,
            "correct": cpu["check"]["bit_exact"] if cpu else None,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


def same_csr(got, rp, ci, cv) -> bool:
    """Bit-identical structure and values (values compared as bit patterns)."""
    return (np.array_equal(got.row_ptr, rp) and np.array_equal(got.col_idx, ci)
            and np.array_equal(got.values.view(np.uint32), cv.view(np.uint32)))


def cpu_baseline(A, B, flops, seconds=12.0, check=None):
    """The reference library timed on all host cores.  check = (A, B, C): the
    operands of the GPU's last timed step and the C it wrote; the reference
    computes that product once more and `check.bit_exact` says whether the
    GPU's C is bit-identical to it (the reference bench's `correct` column)."""
    sys.path.insert(0, str(ROOT))
    from oracle import oracle
    threads = os.cpu_count() or 1
    runs, el = oracle.time_reference_oneshot(A, B, seconds=seconds, threads=threads,
                                             max_runs=400)
    kind = "reference" if oracle.ref_available() else "port"
    out = {"value": flops * runs / el / 1e9, "unit": UNIT, "cores": threads, "kind": kind,
           "sample": f"{runs} full one-shot products on {threads} threads in {el:.1f} s"}
    if check is not None:
        out["check"] = reference_check([check], "one product of the last timed step")
    return out


def reference_check(items, what: str) -> dict:
    """items: (A, B, C) triples, C the GPU's product; each is recomputed by
    the reference library (the oracle port when the library is absent) and
    compared bit for bit."""
    sys.path.insert(0, str(ROOT))
    from oracle import oracle
    ref = oracle.ref_available()
    bad = 0
    for cA, cB, gC in items:
        if ref:
            st, rp, ci, cv = oracle.ref_spgemm(cA, cB)
        else:
            st, (rp, ci, cv, _) = 0, oracle.spgemm(cA, cB)
        bad += 0 if st == 0 and same_csr(gC, rp, ci, cv) else 1
    return {"bit_exact": bad == 0, "mismatched": bad,
            "against": f"{'reference' if ref else 'port'}: {what}"}


def launch_ranks(n: int) -> int:
    """--gpus N without a launcher: run this same command as N ranks (one per
    GPU) under torch.distributed.run on 127.0.0.1, and return its status."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1",
           f"--nproc-per-node={n}", "--master-addr=127.0.0.1", f"--master-port={port}",
           str(Path(__file__).resolve())] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None,
                    help="timed steps (default: 1500 for the sub-millisecond laplace2d and "
                         "uniform4096 steps, so the timed region lasts long enough for the "
                         "clock samples; 40 otherwise; 3 for --impl reference)")
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--workload", default="stencil3d_job", choices=sorted(WORKLOADS))
    ap.add_argument("--impl", default="ours", choices=("ours", "reference"))
    ap.add_argument("--path", default=None, choices=("plain", "learned"),
                    help="plain GPU Gustavson, or the learned (MLP-binned, fused) path "
                         "(default: learned for stencil3d_job, plain otherwise)")
    ap.add_argument("--repeats", type=int, default=JOB_REPEATS,
                    help="stencil3d_job: numeric-only repeats per job")
    ap.add_argument("--seed", type=int, default=11,
                    help="stencil3d_job: seed of the value perturbations")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--grid", type=int, default=128,
                    help="stencil workloads: grid edge (128 is the benchmark; smaller "
                         "grids are for profiler captures)")
    ap.add_argument("--e2e-steps", type=int, default=None,
                    help="end-to-end steps (default 2 for stencil3d_job, 10 otherwise)")
    ap.add_argument("--dtype", default="f32", choices=("f32", "f64", "i8"),
                    help="f64 / i8: the FP64 or INT8->INT32 one-shot product of the "
                         "workload's matrices (host arrays in and out)")
    args = ap.parse_args()
    if args.steps is None:
        if args.impl == "reference":
            args.steps = 3  # each step is seconds of CPU work
        elif args.workload == "stencil3d_job":
            args.steps = 10
        else:
            args.steps = 1500 if args.workload in ("laplace2d", "uniform4096") else 40
    if args.path is None:
        args.path = "learned" if args.workload == "stencil3d_job" else "plain"
    if args.e2e_steps is None:
        args.e2e_steps = 2 if args.workload == "stencil3d_job" else 10
    args.repeats = max(args.repeats, 1)
    args.warmup = max(args.warmup, 3)
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        return launch_ranks(args.gpus)
    world, rank, local = dist_setup()

    if args.impl == "reference" and args.workload == "mtx_ingest":
        if rank != 0:
            return 0
        value, el, kind = run_mtx_reference(args)
        print(json.dumps({
            "metric": MTX_METRIC, "value": value, "unit": MTX_UNIT, "impl": "reference",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * el / max(args.steps, 1), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": "mtx_ingest", "description": WORKLOADS["mtx_ingest"]},
            "cpu_baseline": {"value": value, "unit": MTX_UNIT, "cores": 1, "kind": kind,
                             "sample": f"{args.steps} reads of the file"},
            "e2e": {"value": value, "unit": MTX_UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}), flush=True)
        return 0
    if args.impl == "reference":
        return run_reference(args, world, rank)
    if args.workload == "mtx_ingest":
        return run_mtx(args, world, rank, local)
    if args.dtype != "f32":
        return run_typed(args, world, rank, local)
    if args.workload == "batch512":
        return run_batch(args, world, rank, local)
    if args.workload == "rmat20_panels":
        return run_panels(args, world, rank, local)
    if args.workload == "stencil3d_job":
        return run_job(args, world, rank, local)

    import torch
    import rvsp
    from rvsp import CSR, Descriptor, DeviceCSR, intermediate_products
    from rvsp import _lib as L

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    # One dedicated stream carries the L2 flush, the step events and every
    # kernel of the library (the descriptor is bound to it below).
    torch.cuda.set_stream(torch.cuda.Stream(dev))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)
        pg = dist

    A, B = build_inputs(args.workload, grid=args.grid)
    ops = intermediate_products(A, B)
    flops = 2.0 * float(ops.sum())
    dA = DeviceCSR.from_host(A, dev)
    dB = dA if B is A else DeviceCSR.from_host(B, dev)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    reuse = args.workload.endswith("_reuse")

    model = None
    model_file = None
    algo = L.ALGO_CUDA_PLAIN
    if args.path == "learned":
        from rvsp.learn import RowModel, weights_for
        model_file = weights_for(args.workload)
        model = RowModel(path=model_file)
        algo = L.ALGO_CUDA_LEARNED

    def make_descr(memory, **kw):
        dd = Descriptor(algo=algo, memory=memory, **kw)
        if model is not None:
            dd.set_model(model)
        return dd

    d = make_descr(L.MEM_DEVICE, stream=stream, profiling=True)
    ws_bytes, c_nnz = d.work_estimation(dA, dB)
    dC = DeviceCSR.empty(A.rows, B.cols, c_nnz, dev)
    ws = torch.zeros(max(ws_bytes, 1), dtype=torch.uint8, device=dev)
    alg_bytes = rvsp.algorithmic_bytes(A, B, c_nnz)
    rng = np.random.default_rng(1)
    perturb = None
    if reuse:
        d.compute(dA, dB, dC, ws)  # fill once; repeats are numeric-only
        base = dA.values.clone()
        perturb = [base + torch.from_numpy(rng.uniform(-0.01, 0.01, A.nnz).astype(np.float32)).to(dev)
                   for _ in range(2)]

    def step(i):
        if reuse:
            dA.values.copy_(perturb[i % 2])
            d.compute(dA, dB, dC, ws)
        else:
            d.work_estimation(dA, dB)
            d.compute(dA, dB, dC, ws)

    sampler = ClockSampler(local)
    sampler.start()
    for i in range(args.warmup):
        flush.zero_()
        step(i)
    torch.cuda.synchronize(dev)
    d.synchronize()
    d.phase_times(reset=True)
    if pg:
        pg.barrier()
    torch.cuda.synchronize(dev)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    for i in range(args.steps):
        flush.zero_()
        ev[i][0].record(stream)
        step(i)
        ev[i][1].record(stream)
    torch.cuda.synchronize(dev)
    d.synchronize()
    if pg:
        pg.barrier()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(sum(step_ms))
    phases = d.phase_times(reset=True)
    clocks = sampler.stop()
    if pg:
        t = torch.tensor([total_ms], device=dev)
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        total_ms = float(t.item())
    ms_per_step = total_ms / args.steps
    value = world * flops * args.steps / (total_ms * 1e-3) / 1e9

    # Dominant phase and its roofline (algorithmic bytes of one product).
    per_step = {k: (v[0] / args.steps, v[1] / args.steps) for k, v in phases.items() if v[1]}
    dom = max(per_step, key=lambda k: per_step[k][0])
    peak, peak_kind = measured_peaks()
    dom_ms = per_step[dom][0]
    achieved = alg_bytes / (dom_ms * 1e-3) / 1e9
    launches = int(sum(v[1] for v in phases.values()))
    traffic = committed_traffic(args.workload, dom)

    # The last timed step's operands and result, for the reference check in
    # the CPU baseline leg (in the reuse steps A's values, and B's when B is
    # A, are the last perturbation).
    check = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        A_last = A.with_values(dA.values.cpu().numpy())
        check = (A_last, A_last if B is A else B, dC.to_host(c_nnz))

    # End to end through the public API, host memory space, pinned buffers.
    e2e = None
    if rank == 0 or world > 1:
        def pinned(x):
            t = torch.from_numpy(np.ascontiguousarray(x)).pin_memory()
            return t.numpy()
        hA = CSR(A.rows, A.cols, pinned(A.row_ptr), pinned(A.col_idx), pinned(A.values))
        hB = hA if B is A else CSR(B.rows, B.cols, pinned(B.row_ptr), pinned(B.col_idx),
                                   pinned(B.values))
        n = max(c_nnz, 1)
        hC = CSR(A.rows, B.cols, pinned(np.zeros(A.rows + 1, np.int32)),
                 pinned(np.zeros(n, np.int32)), pinned(np.zeros(n, np.float32)))
        hws = np.zeros(256, np.uint8)
        he = make_descr(L.MEM_HOST)
        he.work_estimation(hA, hB)
        he.compute(hA, hB, hC, hws)
        if reuse:
            vals = [pinned(p.cpu().numpy()) for p in perturb]

        def e2e_step(i):
            if reuse:
                he.compute(hA.with_values(vals[i % 2]), hB, hC, hws)
            else:
                he.work_estimation(hA, hB)
                he.compute(hA, hB, hC, hws)
        for i in range(3):
            e2e_step(i)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        for i in range(args.e2e_steps):
            e2e_step(i)
        torch.cuda.synchronize(dev)
        el = time.perf_counter() - t0
        if reuse:
            h2d = A.values.nbytes + (0 if B is A else B.values.nbytes)
            d2h = 4 * (A.rows + 1) + 4 * c_nnz
        else:
            h2d = A.nbytes() + (0 if B is A else B.nbytes())
            d2h = 4 * (A.rows + 1) + 8 * c_nnz
        e2e_val = world * flops * args.e2e_steps / el / 1e9
        if pg:
            t = torch.tensor([el], device=dev)
            pg.all_reduce(t, op=pg.ReduceOp.MAX)
            e2e_val = world * flops * args.e2e_steps / float(t.item()) / 1e9
        e2e = {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "steps": args.e2e_steps,
               "api": "rvsp_spgemm_work_estimation + rvsp_spgemm_compute, host memory space"}
        he.close()

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(A, B, flops, check=check)
        check = None

    d.close()
    if rank == 0:
        sym, num = {}, {}
        with make_descr(L.MEM_DEVICE, stream=stream) as dd:
            dd.work_estimation(dA, dB)
            sym, num = dd.class_counts()
            overflow = dd.overflow_rows()
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_per_step,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic",
            "config": {"workload": args.workload, "description": WORKLOADS[args.workload],
                       "path": args.path,
                       "model": model_file.name if model_file is not None else None,
                       "grid": args.grid if "stencil" in args.workload else None,
                       "rows": A.rows, "nnz_a": A.nnz, "nnz_b": B.nnz,
                       "overflow_rows": overflow,
                       "nnz_c": c_nnz, "products": int(ops.sum()),
                       "flops_per_step": flops, "algorithmic_bytes_per_step": alg_bytes,
                       "l2": "flushed between steps (256 MiB write outside the step events)",
                       "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                       "step_hbm_frac": alg_bytes / (ms_per_step * 1e-3) / 1e9 / peak,
                       "row_classes_symbolic": sym, "row_classes_numeric": num},
            "hbm_frac": alg_bytes / (ms_per_step * 1e-3) / 1e9 / peak,
            "phase_ms_per_step": {k: v[0] for k, v in per_step.items()},
            "roofline": {"bound": "hbm", "kernel": f"{dom} phase", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"
                         if peak_kind == "measured" else "fallback 6.65 TB/s",
                         "traffic": traffic,
                         "algorithmic_bytes_per_launch": alg_bytes},
            "clocks": clocks, "e2e": e2e, "gpu_launches": launches,
            "cpu_baseline": cpu,
            "correct": cpu["check"]["bit_exact"] if cpu and "check" in cpu else None,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
