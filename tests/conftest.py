"""Shared test set-up: the ``gpu`` marker (tests that need a B200) and the repository on sys.path."""

import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (a B200) and the built engine")


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False


@pytest.fixture(scope="session")
def built():
    """The engine library, built in-tree (nvcc cross-compiles without a GPU)."""
    from lumen_b200 import make as build

    return build.build()


@pytest.fixture(scope="session", autouse=True)
def checker_built():
    """The CPU checker (oracle/), rebuilt by make when a source is newer than its library."""
    import oracle

    oracle.build()
