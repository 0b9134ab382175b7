"""FP64 and INT8 -> INT32 one-shot products on the GPU.

rvsp_spgemm_csr with {RVSP_BACKEND_CUDA, FP64, FP64} or {.., INT8, INT32}
must give the legacy scalar kernels' results bit for bit: the reference's
own outputs (tests/golden/ref_typed.npz) and the oracle's on larger inputs
-- uniform, Laplacian, R-MAT hub rows (the heavy classes), 3D stencil,
entries cancelling to zero, an int32 sum that wraps.  Argument errors follow
the reference wrappers; unsorted input is refused with INVALID_CSR.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from rvsp import _lib as L
from rvsp import gen, spgemm_typed

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from typed_cases import cases, wrap_case  # noqa: E402

pytestmark = pytest.mark.gpu
GOLDEN = np.load(Path(__file__).resolve().parent / "golden" / "ref_typed.npz")
CASES = cases()


def same(got, want):
    for g, w in zip(got, want):
        assert g.dtype == w.dtype and g.shape == w.shape
        assert g.tobytes() == w.tobytes()


@pytest.mark.parametrize("name", sorted(CASES))
def test_golden(name):
    kind, A, B = CASES[name]
    same(spgemm_typed(A, B, kind),
         tuple(GOLDEN[f"{name}.{k}"] for k in ("row_ptr", "col_idx", "values")))


def _t(M, v):
    return (M.rows, M.cols, M.row_ptr, M.col_idx, v)


@pytest.mark.parametrize("kind", ["f64", "i8"])
@pytest.mark.parametrize("which", ["rmat", "stencil", "uniform_big"])
def test_larger_against_oracle(kind, which):
    rng = np.random.default_rng(5)
    if which == "rmat":
        A = gen.rmat(12, 16, seed=3)
        B = A
    elif which == "stencil":
        A = gen.stencil_3d_27(16)
        B = A
    else:
        A = gen.uniform_rows(40000, 40000, 12, 8)
        B = gen.uniform_rows(40000, 30000, 10, 9)

    def vals(n):
        if kind == "f64":
            return rng.uniform(-1, 1, n)
        return rng.integers(-3, 4, n).astype(np.int8)
    ta = _t(A, vals(A.nnz))
    tb = ta if B is A else _t(B, vals(B.nnz))
    same(spgemm_typed(ta, tb, kind), oracle.spgemm_typed(ta, tb, kind))


def test_int32_wrap():
    a, b = wrap_case()
    got = spgemm_typed(a, b, "i8")
    same(got, oracle.spgemm_typed(a, b, "i8"))
    assert int(got[2][0]) == 140000 * 127 * 127 - (1 << 32)


def test_f64_empty_rows_product():
    a = (0, 3, np.zeros(1, np.int32), np.zeros(0, np.int32), np.zeros(0))
    b = (3, 4, np.zeros(4, np.int32), np.zeros(0, np.int32), np.zeros(0))
    rp, ci, cv = spgemm_typed(a, b, "f64")
    assert rp.tolist() == [0] and ci.size == 0


@pytest.mark.parametrize("kind,mutate,status", [
    ("f64", "cols", L.ERROR_INVALID_ARGUMENT),   # A.cols != B.rows
    ("i8", "cols", L.ERROR_INVALID_ARGUMENT),
    ("i8", "rows0", L.ERROR_INVALID_ARGUMENT),   # the i8 kernel wants rows > 0
    ("f64", "unsorted", L.ERROR_INVALID_CSR),
    ("i8", "unsorted", L.ERROR_INVALID_CSR),
])
def test_errors(kind, mutate, status):
    kind_, A, B = CASES["f64_uniform" if kind == "f64" else "i8_uniform"]
    A = list(A)
    B = list(B)
    if mutate == "cols":
        A[1] += 1
    elif mutate == "rows0":
        A = [0, A[1], np.zeros(1, np.int32), np.zeros(0, np.int32), A[4][:0]]
    else:
        ci = A[3].copy()
        ci[0], ci[1] = ci[1], ci[0]
        A[3] = ci
    with pytest.raises(L.RvspError) as e:
        spgemm_typed(tuple(A), tuple(B), kind)
    assert e.value.status == status
