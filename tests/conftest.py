"""Shared test setup: the ``gpu`` marker, golden-vector loading, repo paths."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


def golden(name: str):
    return np.load(GOLDEN / f"{name}.npz", allow_pickle=False)


TRANSPORT_CASES = ("c20mev", "si50mev", "stack10mev", "si30kev", "sio2_300kev")
LUT_CASES = ("c20mev", "stack10mev", "si30kev", "sio2_300kev")
CXR_CASES = ("hopg20", "si50")


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)
