"""The reference's own programs, compiled unchanged against this library.

oracle/Makefile (`make progs`) compiles the reference's examples
(examples/spgemm_csr_f32.c, spgemm_csr_descr_f32.c, spgemm_csr_reuse_f32.c)
and its descriptor and fixture tests (tests/test_spgemm_descr_f32.c,
tests/test_spgemm_reference_f32.c) twice: against include/ and
librvsparse_cuda.so (<name>_cuda) and against the reference library itself
(<name>_ref).  examples/spgemm_csr_f32.c asks for the scalar CPU backend on
its options line (:63-68), which this library does not provide; its _cuda
build gets the one documented change of that line to RVSP_BACKEND_CUDA.

Bar: each _cuda program exits 0 and prints exactly what its _ref twin
prints (the reference's tests print PASS with the same check counts).
"""
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PROGS = ROOT / "oracle" / "_ref" / "progs"
NAMES = ["spgemm_csr_f32", "spgemm_csr_descr_f32", "spgemm_csr_reuse_f32",
         "test_spgemm_descr_f32", "test_spgemm_reference_f32"]

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", NAMES)
def test_reference_program_runs_unchanged(name):
    cuda, ref = PROGS / f"{name}_cuda", PROGS / f"{name}_ref"
    if not (cuda.exists() and ref.exists()):
        pytest.skip("reference programs not built (needs the reference sources at build time)")
    want = subprocess.run([str(ref)], capture_output=True, text=True, timeout=120)
    got = subprocess.run([str(cuda)], capture_output=True, text=True, timeout=120)
    assert want.returncode == 0, want.stdout + want.stderr
    assert got.returncode == 0, got.stdout + got.stderr
    assert got.stdout == want.stdout
    if name.startswith("test_"):
        assert ": PASS" in got.stdout
