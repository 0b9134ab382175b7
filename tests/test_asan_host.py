"""The C host layer under AddressSanitizer: `make asan` builds the library
with its host C files instrumented, tests/asan_host.c drives the host layer
through the paths that need no GPU (argument errors, the Matrix Market
reader with every host allocation failed in turn, the one-shot, descriptor
and batch entry points up to their first device step), and the run must
report no memory error and no leak.  CPU; valid with a GPU present too."""
import os
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "rv-sparse_b200"


def _libasan() -> bool:
    out = subprocess.run(["gcc", "-print-file-name=libasan.so"], capture_output=True,
                         text=True).stdout.strip()
    return os.path.isabs(out) and os.path.exists(out)


@pytest.mark.skipif(not _libasan(), reason="gcc without libasan")
def test_host_layer_clean_under_asan(tmp_path):
    subprocess.run(["make", "-s", "-j8", "-C", str(PKG), "asan"], check=True, timeout=1200)
    exe = tmp_path / "asan_host"
    subprocess.run(["gcc", "-std=c11", "-O1", "-g", "-fsanitize=address",
                    "-fno-omit-frame-pointer", "-D_POSIX_C_SOURCE=200809L",
                    f"-I{ROOT / 'include'}", str(ROOT / "tests" / "asan_host.c"),
                    f"-L{PKG / 'lib'}", "-lrvsparse_cuda_asan",
                    f"-Wl,-rpath,{PKG / 'lib'}", "-o", str(exe)], check=True, timeout=300)
    env = dict(os.environ, ASAN_OPTIONS="detect_leaks=1:protect_shadow_gap=0")
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "all checks passed" in r.stdout
