"""Regenerates tests/golden/ref_typed.npz: the reference library's own FP64
and INT8 -> INT32 products (rvsp_spgemm_csr with RVSP_BACKEND_SCALAR, which
runs src/kernels/spgemm/legacy/csr_scalar_f64.c and csr_scalar_i8.c; built
into oracle/_ref/librvsp_ref.so by oracle/Makefile) on every case of
typed_cases.py: NAME.row_ptr, NAME.col_idx, NAME.values.

Run from the repository root where the reference tree is mounted:
    python tests/golden/make_typed_golden.py
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE.parents[1]))
sys.path.insert(0, str(HERE))

from oracle import oracle  # noqa: E402
from typed_cases import cases  # noqa: E402


def main() -> int:
    oracle.build(with_ref=True)
    if not oracle.ref_available():
        print("reference library not built (no reference tree)", file=sys.stderr)
        return 1
    out = {}
    for name, (kind, A, B) in cases().items():
        st, rp, ci, cv = oracle.ref_spgemm_typed(A, B, kind)
        if st != 0:
            print(f"{name}: status {st}", file=sys.stderr)
            return 1
        out[f"{name}.row_ptr"], out[f"{name}.col_idx"], out[f"{name}.values"] = rp, ci, cv
    np.savez_compressed(HERE / "ref_typed.npz", **out)
    print(f"wrote {len(out) // 3} cases")
    return 0


if __name__ == "__main__":
    sys.exit(main())
