"""Seeded Matrix Market texts for the reader's parity tests.

Each case exercises one behaviour of the reference reader
(tools/src/mtx_to_csr_formatter.c of merledu/rv-sparse): general real and
integer files, pattern files (values 1.0), symmetric files (mirrored
off-diagonals), repeated entries whose sum depends on the order, comments,
blank lines and irregular spacing, a file shorter than its size line, an
entry that stops converting mid-file, empty rows and an empty matrix.
"""
from __future__ import annotations

import numpy as np


def _fmt_entries(r, c, v=None, sep=" "):
    if v is None:
        return "".join(f"{a}{sep}{b}\n" for a, b in zip(r, c))
    return "".join(f"{a}{sep}{b}{sep}{x}\n" for a, b, x in zip(r, c, v))


def _floats(rng, n):
    # a mix of magnitudes, so that the order of a sum shows in its bits
    mag = 10.0 ** rng.integers(-3, 9, n)
    return [repr(float(np.float32(x))) for x in rng.uniform(-1, 1, n) * mag]


def cases() -> dict[str, bytes]:
    rng = np.random.default_rng(20240611)
    out: dict[str, bytes] = {}

    n = 40
    r = rng.integers(1, 31, n)
    c = rng.integers(1, 26, n)
    out["general_real"] = (b"%%MatrixMarket matrix coordinate real general\n"
                           b"% generated\n" + f"30 25 {n}\n".encode() +
                           _fmt_entries(r, c, _floats(rng, n)).encode())

    r = rng.integers(1, 9, 30)
    c = rng.integers(1, 9, 30)
    out["integer_values"] = (b"%%MatrixMarket matrix coordinate integer general\n"
                             b"8 8 30\n" +
                             _fmt_entries(r, c, rng.integers(-50, 50, 30)).encode())

    r = rng.integers(1, 21, 60)
    c = rng.integers(1, 21, 60)
    out["pattern_general"] = (b"%%MatrixMarket matrix coordinate pattern general\n"
                              b"20 20 60\n" + _fmt_entries(r, c).encode())

    # symmetric: lower triangle with a diagonal, some repeats
    rr, cc = [], []
    for _ in range(80):
        a, b = sorted(rng.integers(1, 26, 2))
        rr.append(b)
        cc.append(a)
    out["symmetric_real"] = (b"%%MatrixMarket matrix coordinate real symmetric\n"
                             b"% lower triangle\n" + f"25 25 {len(rr)}\n".encode() +
                             _fmt_entries(rr, cc, _floats(rng, len(rr))).encode())
    out["symmetric_pattern"] = (b"%%MatrixMarket matrix coordinate pattern symmetric\n"
                                b"25 25 40\n" + _fmt_entries(rr[:40], cc[:40]).encode())

    # heavy repeats: 3 cells hit 100 times each with values whose sum is
    # order-sensitive in FP32
    cells = [(1, 1), (2, 3), (4, 2)]
    rr, cc = [], []
    for k in range(300):
        a, b = cells[k % 3]
        rr.append(a)
        cc.append(b)
    out["repeats"] = (b"%%MatrixMarket matrix coordinate real general\n"
                      b"4 4 300\n" + _fmt_entries(rr, cc, _floats(rng, 300)).encode())
    out["symmetric_repeats"] = (b"%%MatrixMarket matrix coordinate real symmetric\n"
                                b"4 4 300\n" +
                                _fmt_entries([max(a, b) for a, b in zip(rr, cc)],
                                             [min(a, b) for a, b in zip(rr, cc)],
                                             _floats(rng, 300)).encode())

    # comments, blank line, tabs and extra spaces
    out["spacing"] = (b"%%MatrixMarket matrix coordinate real general\n"
                      b"%\n% a comment\n%another\n"
                      b"5 6 4\n"
                      b"1\t2\t0.5\n  3   4   -1.25e-3\n\n5 6 7\n2 2 +3.0\n")

    # fewer entries than the size line announces
    out["short_file"] = (b"%%MatrixMarket matrix coordinate real general\n"
                         b"6 6 10\n1 1 1.0\n2 2 2.0\n3 3 3.0\n")
    # an entry that does not convert ends the reading
    out["stops_early"] = (b"%%MatrixMarket matrix coordinate real general\n"
                          b"6 6 5\n1 1 1.0\n2 2 2.0\nx 3 3.0\n4 4 4.0\n5 5 5.0\n")
    # a row index given as "2.5": fscanf reads 2, then ".5" as the column
    out["partial_token"] = (b"%%MatrixMarket matrix coordinate real general\n"
                            b"6 6 3\n1 1 1.0\n2.5 3 3.0\n4 4 4.0\n")
    # empty rows at the start and end
    out["empty_rows"] = (b"%%MatrixMarket matrix coordinate real general\n"
                         b"7 3 3\n3 1 1.0\n3 3 2.0\n4 2 -1.0\n")
    out["empty_matrix"] = (b"%%MatrixMarket matrix coordinate real general\n"
                           b"5 5 0\n")
    # no banner: the first line is taken as the banner and lost
    out["no_banner"] = b"% only a comment\n3 3 2\n1 1 1.0\n2 2 2.0\n"
    return out


def big_case(rows: int, cols: int, entries: int, seed: int, symmetric: bool = False,
             long_rows: int = 0) -> bytes:
    """A large coordinate file: uniform entries with about 1% repeats, plus
    `long_rows` rows of 6000 entries (past the block sort's 4096)."""
    rng = np.random.default_rng(seed)
    r = rng.integers(1, rows + 1, entries)
    c = rng.integers(1, cols + 1, entries)
    rep = rng.integers(0, entries, entries // 100)
    r = np.concatenate([r, r[rep]])
    c = np.concatenate([c, c[rep]])
    for k in range(long_rows):
        row = 1 + (k * 7919) % rows
        r = np.concatenate([r, np.full(6000, row)])
        c = np.concatenate([c, rng.integers(1, cols + 1, 6000)])
    if symmetric:
        r, c = np.maximum(r, c), np.minimum(r, c)
    v = rng.uniform(-1, 1, r.size).astype(np.float32)
    head = (f"%%MatrixMarket matrix coordinate real {'symmetric' if symmetric else 'general'}\n"
            f"{rows} {cols} {r.size}\n")
    body = "\n".join(f"{a} {b} {x:.7g}" for a, b, x in zip(r.tolist(), c.tolist(),
                                                          v.tolist()))
    return (head + body + "\n").encode()
