"""Shared fixtures: the golden files, the package loader and the ``gpu`` marker."""

from __future__ import annotations

import importlib
import json
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = Path(__file__).resolve().parent / "golden"
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


@pytest.fixture(scope="session")
def golden_values() -> dict:
    return json.loads((GOLDEN / "reference_values.json").read_text())


@pytest.fixture(scope="session")
def golden_arrays():
    with np.load(GOLDEN / "reference_fixtures.npz") as data:
        return {k: data[k] for k in data.files}


@pytest.fixture(scope="session")
def pkg():
    """The product package (its directory name is not a Python identifier)."""
    import __graft_entry__

    return __graft_entry__.package()


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
