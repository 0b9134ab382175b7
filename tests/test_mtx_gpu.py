"""Matrix Market reader on the GPU (rvsp_csr_read_mtx / rvsp_csr_parse_mtx).

Bar: for every case the library's CSR -- host and device memory space, text
and file input -- equals the oracle's (which tests/test_mtx.py pins to the
reference's own reader) bit for bit: row pointers, columns and the bits of
every value, repeated entries summed in file order.  Large files take the
threaded parser and every sort size (warp rows, block rows, rows past 4096
entries); a large file with a token that converts only in part takes the
sequential fallback.  Out-of-range indices and a bad size line are errors.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

from oracle import oracle
from rvsp import _lib as L
from rvsp import read_mtx

sys.path.insert(0, str(Path(__file__).resolve().parent / "golden"))
from mtx_cases import big_case, cases  # noqa: E402

pytestmark = pytest.mark.gpu
CASES = cases()


def check_equal(got, text):
    rows, cols, rp, ci, cv = oracle.mtx_to_csr(text)
    assert (got.rows, got.cols) == (rows, cols)
    assert np.array_equal(np.asarray(got.row_ptr), rp)
    assert np.array_equal(np.asarray(got.col_idx)[:rp[-1]], ci)
    assert np.array_equal(np.asarray(got.values)[:rp[-1]].view(np.uint32), cv.view(np.uint32))


@pytest.mark.parametrize("name", sorted(CASES))
def test_cases_host_and_device(name):
    text = CASES[name]
    check_equal(read_mtx(text), text)
    d = read_mtx(text, device=True)
    check_equal(d.to_host(), text)


def test_file_input(tmp_path):
    p = tmp_path / "a.mtx"
    p.write_bytes(CASES["symmetric_repeats"])
    check_equal(read_mtx(p), CASES["symmetric_repeats"])


@pytest.mark.parametrize("symmetric", [False, True])
def test_large_threaded_all_sort_sizes(symmetric):
    # about 9 MB of text (threaded parser); uniform rows (warp sort), rows of
    # 6000 entries (global sort), and mid-size rows from the repeats
    text = big_case(200000, 200000, 400000, seed=11 + symmetric, symmetric=symmetric,
                    long_rows=3)
    assert len(text) > (4 << 20)
    got = read_mtx(text)
    check_equal(got, text)
    lens = np.diff(got.row_ptr)
    assert lens.max() > 4096


def test_block_sort_rows():
    rng = np.random.default_rng(3)
    r = np.repeat(np.arange(1, 51), 500)  # 50 rows of 500 entries (block sort)
    c = rng.integers(1, 400, r.size)      # many repeats inside each row
    v = rng.uniform(-1, 1, r.size).astype(np.float32)
    text = ("%%MatrixMarket matrix coordinate real general\n50 400 %d\n" % r.size +
            "".join(f"{a} {b} {x:.7g}\n" for a, b, x in zip(r, c, v))).encode()
    check_equal(read_mtx(text), text)


def test_large_partial_token_falls_back():
    text = big_case(50000, 50000, 300000, seed=4)
    lines = text.split(b"\n")
    mid = len(lines) // 2
    lines[mid] = b"7.5 " + lines[mid].split(b" ", 1)[1]  # "7.5": 7, then ".5" fails
    text = b"\n".join(lines)
    got = read_mtx(text)
    check_equal(got, text)
    assert got.row_ptr[-1] < 300000


@pytest.mark.parametrize("text,status", [
    (b"%%MatrixMarket matrix coordinate real general\n3 3 1\n4 1 1.0\n", L.ERROR_INVALID_CSR),
    (b"%%MatrixMarket matrix coordinate real general\n3 3 1\n1 0 1.0\n", L.ERROR_INVALID_CSR),
    (b"%%MatrixMarket matrix coordinate real symmetric\n3 2 1\n3 1 1.0\n", L.ERROR_INVALID_CSR),
    (b"%%MatrixMarket matrix coordinate real general\nnot a size\n", L.ERROR_INVALID_ARGUMENT),
])
def test_errors(text, status):
    with pytest.raises(L.RvspError) as e:
        read_mtx(text)
    assert e.value.status == status


def test_missing_file(tmp_path):
    with pytest.raises(L.RvspError) as e:
        read_mtx(tmp_path / "none.mtx")
    assert e.value.status == L.ERROR_INVALID_ARGUMENT
