import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "rv-sparse_b200"))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")
    config.addinivalue_line("markers", "slow: full-size workloads")


def _has_gpu() -> bool:
    try:
        import torch
        if not torch.cuda.is_available():
            return False
        return torch.cuda.get_device_capability(0) == (10, 0)
    except Exception:
        return False


HAS_GPU = _has_gpu()


def pytest_collection_modifyitems(config, items):
    if HAS_GPU:
        return
    skip = pytest.mark.skip(reason="no sm_100 GPU in this container")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def golden_fixtures():
    from rvsp import CSR
    data = json.loads((GOLDEN / "fixtures.json").read_text())["fixtures"]
    out = []
    for f in data:
        mats = []
        for k in ("a", "b", "c"):
            m = f[k]
            mats.append(CSR(m["rows"], m["cols"], np.array(m["row_ptr"]),
                            np.array(m["col_idx"]), np.array(m["values"])))
        out.append((f["name"], *mats))
    return out


@pytest.fixture(scope="session")
def golden_random():
    from rvsp import CSR
    z = np.load(GOLDEN / "ref_random.npz")
    names = sorted({k.split("/")[0] for k in z.files})
    out = []
    for n in names:
        def mat(tag):
            r, c = z[f"{n}/{tag}_shape"]
            return CSR(int(r), int(c), z[f"{n}/{tag}_row_ptr"], z[f"{n}/{tag}_col_idx"],
                       z[f"{n}/{tag}_values"])
        A, B = mat("a"), mat("b")
        Cm = CSR(A.rows, B.cols, z[f"{n}/c_row_ptr"], z[f"{n}/c_col_idx"],
                 z[f"{n}/c_values"])
        out.append((n, A, B, Cm, z[f"{n}/op_counts"]))
    return out
