"""Regenerates the golden fixtures under tests/golden/.

  fixtures.json    the six hand-verified (A, B, C) triples of the reference
                   test suite, read as text from tests/csr_fixtures.h:42-153
                   of merledu/rv-sparse;
  ref_random.npz   seeded irregular inputs and the outputs of the reference
                   library itself (oracle/_ref/librvsp_ref.so, compiled from
                   the reference sources by oracle/Makefile): structure,
                   values and per-row op counts.

Run from the repository root, in a container where the reference tree is
mounted:  python tests/golden/make_golden.py [--ref-root PATH]
The GPU tests only read the committed outputs.
"""
from __future__ import annotations

import argparse
import os
import json
import re
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "rv-sparse_b200"))

from oracle import oracle  # noqa: E402
from rvsp import gen  # noqa: E402

ARRAY_RE = re.compile(
    r"static\s+const\s+(int32_t|float)\s+(\w+)\[\]\s*=\s*\{([^}]*)\};", re.S)
TRIPLE = r"\{\s*(\d+)\s*,\s*(\d+)\s*,\s*(\d+)\s*,\s*(\w+)\s*,\s*(\w+)\s*,\s*(\w+)\s*\}"
PAIR_RE = re.compile(r'\{\s*"([^"]+)"\s*,\s*"([^"]+)"\s*,\s*' + TRIPLE + r"\s*,\s*" +
                     TRIPLE + r"\s*,\s*" + TRIPLE + r"\s*\}", re.S)


def parse_fixtures(header: Path):
    text = header.read_text()
    arrays = {}
    for kind, name, body in ARRAY_RE.findall(text):
        vals = [v.strip().rstrip("f") for v in body.replace("\n", " ").split(",")
                if v.strip()]
        arrays[name] = [int(v) for v in vals] if kind == "int32_t" else [float(v) for v in vals]
    out = []
    for m in PAIR_RE.findall(text):
        name, targets = m[0], m[1]
        mats = []
        for k in range(3):
            rows, cols, nnz, rp, ci, v = m[2 + 6 * k: 8 + 6 * k]
            mats.append({"rows": int(rows), "cols": int(cols), "nnz": int(nnz),
                         "row_ptr": arrays[rp], "col_idx": arrays[ci],
                         "values": arrays[v]})
        out.append({"name": name, "targets": targets, "a": mats[0], "b": mats[1],
                    "c": mats[2]})
    return out


RANDOM_CASES = [
    # (name, A args, B args) for gen.random_csr(rows, cols, seed, mean_len, empty_frac, heavy_rows, heavy_len, value_kind)
    ("small_int", (12, 9, 101, 2.0, 0.2, 0, 0, "int"), (9, 11, 102, 2.0, 0.2, 0, 0, "int")),
    ("small_uniform", (40, 30, 103, 3.0, 0.1, 0, 0, "uniform"), (30, 50, 104, 3.0, 0.1, 0, 0, "uniform")),
    ("esc_edge", (64, 64, 105, 5.0, 0.05, 0, 0, "uniform"), (64, 64, 106, 6.0, 0.0, 0, 0, "uniform")),
    ("hash_rows", (80, 500, 107, 12.0, 0.05, 0, 0, "uniform"), (500, 700, 108, 20.0, 0.05, 0, 0, "uniform")),
    ("heavy_rows", (60, 400, 109, 3.0, 0.1, 3, 300, "uniform"), (400, 3000, 110, 15.0, 0.1, 4, 2500, "uniform")),
    ("cancel_int", (50, 50, 111, 6.0, 0.1, 0, 0, "int"), (50, 50, 112, 6.0, 0.1, 0, 0, "int")),
    ("wide_cols", (30, 200, 113, 40.0, 0.0, 0, 0, "uniform"), (200, 20000, 114, 60.0, 0.0, 0, 0, "uniform")),
    ("all_empty_b", (20, 10, 115, 3.0, 0.0, 0, 0, "uniform"), (10, 10, 116, 0.0, 1.0, 0, 0, "uniform")),
]


def make_random():
    arrays = {}
    for name, aa, ba in RANDOM_CASES:
        A = gen.random_csr(*aa[:3], mean_len=aa[3], empty_frac=aa[4], heavy_rows=aa[5],
                           heavy_len=aa[6], value_kind=aa[7])
        B = gen.random_csr(*ba[:3], mean_len=ba[3], empty_frac=ba[4], heavy_rows=ba[5],
                           heavy_len=ba[6], value_kind=ba[7])
        st, rp, ci, cv = oracle.ref_spgemm(A, B)
        assert st == 0, (name, st)
        st, ops = oracle.ref_op_counts(A, B)
        assert st == 0, (name, st)
        for tag, M in (("a", A), ("b", B)):
            arrays[f"{name}/{tag}_shape"] = np.array([M.rows, M.cols], np.int64)
            arrays[f"{name}/{tag}_row_ptr"] = M.row_ptr
            arrays[f"{name}/{tag}_col_idx"] = M.col_idx
            arrays[f"{name}/{tag}_values"] = M.values
        arrays[f"{name}/c_row_ptr"] = rp
        arrays[f"{name}/c_col_idx"] = ci
        arrays[f"{name}/c_values"] = cv
        arrays[f"{name}/op_counts"] = ops
    return arrays


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref-root", default=os.environ.get(
        "RVSP_REFERENCE_ROOT", str(Path(__file__).resolve().parents[3] / "reference")),
        help="the reference tree (default: RVSP_REFERENCE_ROOT, else a checkout named "
             "'reference' beside this repository)")
    args = ap.parse_args()
    here = Path(__file__).resolve().parent
    fx = parse_fixtures(Path(args.ref_root) / "tests" / "csr_fixtures.h")
    assert len(fx) == 6, len(fx)
    (here / "fixtures.json").write_text(json.dumps(
        {"source": "merledu/rv-sparse tests/csr_fixtures.h:42-153", "fixtures": fx},
        indent=1) + "\n")
    oracle.build(with_ref=True)
    np.savez_compressed(here / "ref_random.npz", **make_random())
    print("wrote", here / "fixtures.json", "and", here / "ref_random.npz")


if __name__ == "__main__":
    main()
