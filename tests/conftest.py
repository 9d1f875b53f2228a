import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def pytest_collection_modifyitems(config, items):
    import torch
    if torch.cuda.is_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(autouse=True)
def _poison_workspace(monkeypatch):
    """Every propagation in the tests runs on a workspace filled with NaN
    bytes, so a read of scratch that a call never wrote fails its test instead
    of passing on whatever an earlier allocation left behind."""
    monkeypatch.setenv("SWEEP_B200_POISON_WORKSPACE", "1")
