import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)

GOLDEN = os.path.join(ROOT, "tests", "golden")
GOLDEN_CASES = ["t_au13", "t_au55w", "t_2np", "t_water", "c1", "c1_field"]


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs an sm_100 GPU and the built CUDA library")


def golden_paths(case: str) -> dict:
    d = os.path.join(GOLDEN, case)
    return {"gro": os.path.join(d, "init.gro"), "par": os.path.join(d, "param.txt"),
            "mds": os.path.join(d, "mdset.txt")}


def golden_ref(case: str) -> dict:
    with np.load(os.path.join(GOLDEN, case, "ref.npz")) as z:
        return {k: z[k] for k in z.files}


def rel_err(a, b) -> float:
    """max |a - b| / max |b| (normwise relative error)."""
    a, b = np.asarray(a, dtype=np.float64), np.asarray(b, dtype=np.float64)
    if b.size == 0:
        return 0.0
    scale = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / scale) if scale > 0 else float(np.max(np.abs(a)))


def slot_rel_err(a, b) -> float:
    """Largest relative error over the non-zero potential slots."""
    a, b = np.asarray(a), np.asarray(b)
    m = np.abs(b) > 0
    if not m.any():
        return float(np.max(np.abs(a)))
    return float(np.max(np.abs(a[m] - b[m]) / np.abs(b[m])))


@pytest.fixture(scope="session")
def gpu_available() -> bool:
    try:
        import torch
        if not torch.cuda.is_available():
            return False
        return torch.cuda.get_device_capability(0)[0] == 10
    except Exception:
        return False
