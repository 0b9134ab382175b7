"""FP64 and INT8 -> INT32 products: the oracle pinned to the reference.

oracle/typed_oracle.c restates the legacy scalar kernels
(src/kernels/spgemm/legacy/csr_scalar_f64.c, csr_scalar_i8.c).  It must give
the reference library's own outputs (tests/golden/ref_typed.npz, made by
tests/golden/make_typed_golden.py) bit for bit -- structure after entries
that cancel to zero are dropped, and every value -- and agree with the live
reference library where it is built, including an int32 sum that wraps.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from typed_cases import cases, wrap_case  # noqa: E402

GOLDEN = np.load(Path(__file__).resolve().parent / "golden" / "ref_typed.npz")
CASES = cases()


def bits_equal(a, b):
    return a.dtype == b.dtype and a.shape == b.shape and np.array_equal(
        a.view(np.uint64 if a.dtype.itemsize == 8 else np.uint32),
        b.view(np.uint64 if b.dtype.itemsize == 8 else np.uint32))


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_golden(name):
    kind, A, B = CASES[name]
    rp, ci, cv = oracle.spgemm_typed(A, B, kind)
    assert np.array_equal(rp, GOLDEN[f"{name}.row_ptr"])
    assert np.array_equal(ci, GOLDEN[f"{name}.col_idx"])
    assert bits_equal(cv, GOLDEN[f"{name}.values"])


def test_cancel_cases_drop_entries():
    # the fixtures must exercise the dropping: fewer entries than the
    # structural union of the products
    for name in ("f64_cancel", "i8_cancel"):
        kind, A, B = CASES[name]
        rp, _, cv = oracle.spgemm_typed(A, B, kind)
        ones = (A[0], A[1], A[2], A[3], np.ones(A[3].size, np.float64 if kind == "f64" else np.int8))
        pos = (B[0], B[1], B[2], B[3], np.ones(B[3].size, np.float64 if kind == "f64" else np.int8))
        full = oracle.spgemm_typed(ones, pos, kind)[0]
        assert rp[-1] < full[-1]
        assert np.all(cv != 0)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference library not built here")
def test_oracle_matches_live_reference_including_wrap():
    a, b = wrap_case()
    st, rp, ci, cv = oracle.ref_spgemm_typed(a, b, "i8")
    mine = oracle.spgemm_typed(a, b, "i8")
    assert st == 0
    assert np.array_equal(rp, mine[0]) and np.array_equal(ci, mine[1])
    assert np.array_equal(cv, mine[2])
    assert int(cv[0]) == int(np.int64(140000 * 127 * 127) - (1 << 32))
