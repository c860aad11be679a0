"""Shared fixtures: the golden slab vectors, the oracle and (on a GPU host) the CUDA backend."""

from __future__ import annotations

import importlib
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).resolve().parent / "golden" / "slab.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def slab():
    """The reference's slab fixture, as extracted by tests/golden/make_golden.py."""
    with np.load(GOLDEN) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def oracle():
    return importlib.import_module("oracle")


def package():
    """The product package (its directory name carries a hyphen, so it is imported by name)."""
    return importlib.import_module("sherd-refit_b200")


@pytest.fixture(scope="session")
def sherd():
    return package()


@pytest.fixture(scope="session")
def gpu_ctx(sherd):
    import torch

    if not torch.cuda.is_available():
        pytest.fail("the gpu tests need a CUDA device")
    return sherd.Context(0)
