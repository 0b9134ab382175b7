"""Host logic of the MLP's training labels (rvsp.train): the log2-nearest
binning of a row's A nonzeros and mean B-row length, and the accumulator
label (merge or warp hash) a row gets from the autotuned timing table.  CPU
only: the table is written by hand here."""
import numpy as np

from rvsp import train


def test_bin_is_nearest_in_log2():
    k = train.K_BINS  # 1, 2, 4, 8, 12, 16
    got = train._bin(np.array([0, 1, 2, 3, 5, 6, 7, 10, 11, 14, 40]), k)
    # in log2: 0 counts as 1; 3 (1.58) is nearer 4 (2) than 2 (1); 5 (2.32)
    # -> 4; 6 (2.58) -> 8; 10 (3.32) is nearer 12 (3.58) than 8 (3); 14
    # (3.81) -> 16 (4) rather than 12; 40 -> 16, the last edge
    assert [k[i] for i in got] == [1, 1, 2, 4, 4, 8, 8, 12, 12, 16, 16]


def _table(merge_ms, hash_ms):
    return {"k": list(train.K_BINS), "L": list(train.L_BINS),
            "merge_ms": merge_ms, "hash_ms": hash_ms}


def test_merge_label_from_timings():
    nk, nl = len(train.K_BINS), len(train.L_BINS)
    m = np.ones((nk, nl))
    h = np.ones((nk, nl))
    h[1, 2] = 0.5   # k = 2, L = 8: the hash clearly faster
    h[2, 2] = 0.95  # k = 4, L = 8: within the margin, the merge keeps it
    m[3, 6] = -1    # k = 8, L = 128: no merge timing (over the op limit)
    t = _table(m.tolist(), h.tolist())
    nnz = np.array([2, 4, 8, 0, 17, 16, 1])
    ops = np.array([16, 32, 1024, 0, 17 * 8, 16 * 200, 8])
    lab = train.merge_label(nnz, ops, t)
    # 2 x 8: hash faster -> 0; 4 x 8: tie -> 1; 8 x 128: no merge timing -> 0;
    # empty row -> 0; 17 nonzeros -> not eligible; 3200 ops -> not eligible;
    # 1 x 8 -> merge
    assert lab.tolist() == [0.0, 1.0, 0.0, 0.0, 0.0, 0.0, 1.0]
    assert lab.dtype == np.float32


def test_merge_label_from_boolean_grid():
    nk, nl = len(train.K_BINS), len(train.L_BINS)
    grid = np.ones((nk, nl), bool)
    grid[0, :] = False  # one-nonzero rows: hash
    t = {"k": list(train.K_BINS), "L": list(train.L_BINS), "merge_faster": grid.tolist()}
    lab = train.merge_label(np.array([1, 2, 16]), np.array([4, 8, 2048]), t)
    assert lab.tolist() == [0.0, 1.0, 1.0]
