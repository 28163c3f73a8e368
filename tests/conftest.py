import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))

from __graft_entry__ import load_package  # noqa: E402

GOLDEN = ROOT / "tests" / "golden"
REF_DATA = Path("/root/reference/mriData")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200)")


@pytest.fixture(scope="session")
def pkg():
    return load_package()


@pytest.fixture(scope="session")
def synth(pkg):
    from impatient_mri_b200 import synth as s
    return s


def golden(name: str) -> dict:
    z = np.load(GOLDEN / f"{name}.npz")
    case = {k: z[k] for k in z.files}
    case["dims"] = tuple(int(v) for v in case["dims"])
    case.setdefault("opts", dict(use_z=0))
    return case


def has_cuda() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False
