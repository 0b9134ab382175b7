"""Concurrency: descriptors on several host threads and streams, and one-shot
calls from several threads at once.

The reference keeps all of a product's state in its descriptor
(src/core/spgemm_descr.c:19-37), so products on different threads are
independent.  Here each descriptor owns its plan and stream, and each host
thread keeps its own one-shot context (csrc/host/spgemm.c).  Bar: every
product computed concurrently is bit-exact against the oracle.
"""
import threading

import numpy as np
import pytest

from oracle import oracle
from rvsp import Descriptor, DeviceCSR, gen
from rvsp import _lib as L

pytestmark = pytest.mark.gpu


def _bits(x):
    return np.ascontiguousarray(x, np.float32).view(np.uint32)


def _run_threads(fns):
    errors = []

    def wrap(f):
        try:
            f()
        except BaseException as e:  # noqa: BLE001 - reported below
            errors.append(e)
    ths = [threading.Thread(target=wrap, args=(f,)) for f in fns]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    if errors:
        raise errors[0]


def test_descriptors_on_two_threads_and_streams():
    import torch
    cases = [
        (gen.random_csr(3000, 2500, 31, mean_len=10.0, heavy_rows=3, heavy_len=1500),
         gen.random_csr(2500, 2800, 32, mean_len=12.0, heavy_rows=2, heavy_len=2000)),
        (gen.stencil_3d_27(14), None),
    ]
    want = {}
    for i, (A, B) in enumerate(cases):
        B = A if B is None else B
        want[i] = []
        for s in (1.0, -0.5, 2.0):
            As = A.with_values((A.values * np.float32(s)).astype(np.float32))
            # B is A itself when the case has no B (the device arrays alias)
            want[i].append(oracle.spgemm(As, As if B is A else B))
    got = {}

    def worker(i):
        A, B = cases[i]
        B = A if B is None else B
        stream = torch.cuda.Stream()
        dA = DeviceCSR.from_host(A)
        dB = dA if B is A else DeviceCSR.from_host(B)
        outs = []
        with torch.cuda.stream(stream):
            with Descriptor(algo=L.ALGO_CUDA_PLAIN, memory=L.MEM_DEVICE, stream=stream) as d:
                for rep in range(4):  # estimate + fill, then numeric-only repeats
                    for s in (1.0, -0.5, 2.0):
                        vals = (A.values * np.float32(s)).astype(np.float32)
                        dA.values.copy_(torch.from_numpy(vals).to(dA.values.device),
                                        non_blocking=False)
                        stream.synchronize()
                        if rep == 0 and s == 1.0:
                            ws_b, n = d.work_estimation(dA, dB)
                            dC = DeviceCSR.empty(A.rows, B.cols, n)
                            ws = torch.zeros(max(ws_b, 1), dtype=torch.uint8, device="cuda")
                        d.compute(dA, dB, dC, ws)
                        d.synchronize()
                        outs.append((s, dC.to_host(n)))
        got[i] = outs

    _run_threads([lambda i=i: worker(i) for i in range(len(cases))])
    for i in range(len(cases)):
        for s, C_ in got[i]:
            rp, ci, cv, _ = want[i][(1.0, -0.5, 2.0).index(s)]
            assert np.array_equal(C_.row_ptr, rp)
            assert np.array_equal(C_.col_idx, ci)
            assert np.array_equal(_bits(C_.values), _bits(cv))


def test_one_shot_calls_from_four_threads():
    import rvsp
    pairs = [(gen.random_csr(900 + 50 * t, 800, 40 + t, mean_len=8.0, heavy_rows=2,
                             heavy_len=600),
              gen.random_csr(800, 1000 + 30 * t, 60 + t, mean_len=9.0)) for t in range(4)]
    want = [oracle.spgemm(A, B) for A, B in pairs]
    got = [[] for _ in pairs]

    def worker(t):
        A, B = pairs[t]
        for _ in range(5):
            got[t].append(rvsp.spgemm_csr(A, B))

    _run_threads([lambda t=t: worker(t) for t in range(len(pairs))])
    for t in range(len(pairs)):
        rp, ci, cv, _ = want[t]
        for C_ in got[t]:
            assert np.array_equal(C_.row_ptr, rp)
            assert np.array_equal(C_.col_idx, ci)
            assert np.array_equal(_bits(C_.values), _bits(cv))
