"""Matrix Market reader: the oracle pinned to the reference's own reader.

The oracle (oracle/mtx_oracle.c) restates assemble_csr_matrix
(tools/src/mtx_to_csr_formatter.c).  It must reproduce, bit for bit, the
outputs of the reference reader itself committed in tests/golden/mtx_ref.npz
(tests/golden/make_mtx_golden.py), and, where the reference reader is built
here (oracle/_ref), its live outputs on larger seeded files.  The library's
exports are checked by test_abi.py; the GPU reader is checked against this
oracle in test_mtx_gpu.py.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from mtx_cases import big_case, cases  # noqa: E402

GOLDEN = np.load(Path(__file__).resolve().parent / "golden" / "mtx_ref.npz")
CASES = cases()


def same(a, b):
    return a.shape == b.shape and np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_matches_reference_golden(name):
    rows, cols, rp, ci, cv = oracle.mtx_to_csr(CASES[name])
    assert np.array_equal(rp, GOLDEN[f"{name}.row_ptr"])
    assert np.array_equal(ci, GOLDEN[f"{name}.col_idx"])
    assert same(cv, GOLDEN[f"{name}.values"])


def test_repeats_are_order_sensitive():
    # the fixture must actually pin the summation order: summing the repeated
    # cell in another order gives different bits
    rows, cols, rp, ci, cv = oracle.mtx_to_csr(CASES["repeats"])
    text = CASES["repeats"].decode().splitlines()[2:]
    vals = [np.float32(float(line.split()[2])) for line in text if line.split()[:2] == ["1", "1"]]
    fwd = vals[0]
    for v in vals[1:]:
        fwd = np.float32(fwd + v)
    rev = vals[-1]
    for v in reversed(vals[:-1]):
        rev = np.float32(rev + v)
    assert fwd.view(np.uint32) == cv[0].view(np.uint32)
    assert fwd.view(np.uint32) != rev.view(np.uint32)


def test_oracle_rejects_out_of_range_and_bad_size_line():
    with pytest.raises(ValueError):
        oracle.mtx_to_csr(b"%%MatrixMarket matrix coordinate real general\n3 3 1\n4 1 1.0\n")
    with pytest.raises(ValueError):
        oracle.mtx_to_csr(b"%%MatrixMarket matrix coordinate real symmetric\n3 2 1\n3 1 1.0\n")
    with pytest.raises(ValueError):
        oracle.mtx_to_csr(b"%%MatrixMarket matrix coordinate real general\nnot a size\n")


@pytest.mark.skipif(not oracle.ref_mtx_available(), reason="reference reader not built here")
@pytest.mark.parametrize("symmetric", [False, True])
def test_oracle_matches_live_reference_on_larger_files(tmp_path, symmetric):
    text = big_case(3000, 3000, 60000, seed=5 + symmetric, symmetric=symmetric, long_rows=1)
    path = tmp_path / "m.mtx"
    path.write_bytes(text)
    want = oracle.ref_mtx_to_csr(path)
    rows, cols, rp, ci, cv = oracle.mtx_to_csr(text)
    assert np.array_equal(rp, want[0]) and np.array_equal(ci, want[1]) and same(cv, want[2])
