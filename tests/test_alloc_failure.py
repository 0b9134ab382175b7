"""Host allocation failures, injected through the library's allocator hook
(rvsp_debug.h): every host allocation a call makes is failed in turn, and
each failure must come back as RVSP_ERROR_ALLOCATION_FAILED with the output
matrix left empty.  No GPU fault is provoked.  Without a GPU the calls stop at
their first device step (after their host allocations); with one they run to
the end, and the host copies of C are failed too."""
import ctypes as C

import pytest

from rvsp import _lib as L

TEXT = (b"%%MatrixMarket matrix coordinate real general\n"
        b"% a comment line\n"
        b"4 5 6\n"
        b"1 1 1.5\n2 3 -2.0\n4 5 3.25\n1 2 0.5\n3 3 1.0\n1 1 2.0\n")


@pytest.fixture
def lib():
    lib = L.load()
    yield lib
    lib.rvsp_debug_fail_host_alloc(-1)


def _empty(m):
    return (m.rows, m.cols, m.nnz, m.owns_data) == (0, 0, 0, 0) and not m.row_ptr \
        and not m.col_idx and not m.values


def _walk(lib, call):
    """Fails each host allocation of call() in turn; returns how many."""
    out = L.CsrMatrix()
    before = lib.rvsp_debug_host_allocs()
    base = call(out)
    allocs = lib.rvsp_debug_host_allocs() - before
    assert base in (L.SUCCESS, L.ERROR_UNSUPPORTED_BACKEND, L.ERROR_DEVICE), base
    if base == L.SUCCESS:
        lib.rvsp_csr_destroy(C.byref(out))
    assert allocs >= 1
    for k in range(allocs):
        out = L.CsrMatrix()
        out.rows, out.nnz, out.row_ptr = 7, 9, 1234  # stale contents to clear
        lib.rvsp_debug_fail_host_alloc(k)
        st = call(out)
        assert st == L.ERROR_ALLOCATION_FAILED, (k, st)
        assert _empty(out), k
    lib.rvsp_debug_fail_host_alloc(-1)
    return allocs


def test_parse_mtx_each_host_allocation_fails_cleanly(lib):
    for space in (L.MEM_HOST, L.MEM_DEVICE):
        n = _walk(lib, lambda m: lib.rvsp_csr_parse_mtx(TEXT, len(TEXT), space, C.byref(m)))
        assert n >= 4  # the text copy and the three COO arrays


def test_read_mtx_each_host_allocation_fails_cleanly(lib, tmp_path):
    path = tmp_path / "m.mtx"
    path.write_bytes(TEXT)
    n = _walk(lib, lambda m: lib.rvsp_csr_read_mtx(str(path).encode(), L.MEM_HOST,
                                                   C.byref(m)))
    assert n >= 5  # the file buffer, then the parse's own


def test_hook_fails_once_then_turns_off(lib):
    lib.rvsp_debug_fail_host_alloc(0)
    m = L.CsrMatrix()
    assert lib.rvsp_csr_parse_mtx(TEXT, len(TEXT), L.MEM_HOST, C.byref(m)) == \
        L.ERROR_ALLOCATION_FAILED
    st = lib.rvsp_csr_parse_mtx(TEXT, len(TEXT), L.MEM_HOST, C.byref(m))
    assert st != L.ERROR_ALLOCATION_FAILED
    if st == L.SUCCESS:
        lib.rvsp_csr_destroy(C.byref(m))
