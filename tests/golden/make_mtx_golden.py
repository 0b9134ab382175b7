"""Regenerates tests/golden/mtx_ref.npz: the reference's own Matrix Market
reader (assemble_csr_matrix of tools/src/mtx_to_csr_formatter.c, compiled
from the reference sources into oracle/_ref/librvsp_mtx_ref.so by
oracle/Makefile) run on every case of mtx_cases.py.  For each case NAME the
archive holds NAME.row_ptr, NAME.col_idx and NAME.values.

Run from the repository root, in a container where the reference tree is
mounted:  python tests/golden/make_mtx_golden.py
The tests only read the committed archive.
"""
from __future__ import annotations

import sys
import tempfile
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE))

from oracle import oracle  # noqa: E402
from mtx_cases import cases  # noqa: E402


def main() -> int:
    oracle.build(with_ref=True)
    if not oracle.ref_mtx_available():
        print("reference reader not built (no reference tree)", file=sys.stderr)
        return 1
    out = {}
    with tempfile.TemporaryDirectory() as tmp:
        for name, text in cases().items():
            path = Path(tmp) / f"{name}.mtx"
            path.write_bytes(text)
            res = oracle.ref_mtx_to_csr(path)
            if res is None:
                print(f"{name}: the reference reader failed", file=sys.stderr)
                return 1
            out[f"{name}.row_ptr"], out[f"{name}.col_idx"], out[f"{name}.values"] = res
    np.savez_compressed(HERE / "mtx_ref.npz", **out)
    print(f"wrote {len(out) // 3} cases to {HERE / 'mtx_ref.npz'}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
