"""Shared test setup: markers, paths, and the session-wide builds.

``gpu``-marked tests need a CUDA device and run the libgsolve kernels; everything else runs
on the CPU (oracle pins, ABI/symbol checks, host logic, gloo multi-process tests).
"""
from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); runs the CUDA kernels")
    config.addinivalue_line("markers", "slow: long-running")


def load_golden(name: str) -> dict:
    with np.load(GOLDEN / f"{name}.npz") as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as O

    O.build()
    return O


@pytest.fixture(scope="session")
def gslib():
    from gradsolve_b200.csrc import build as B

    B.build()
    from gradsolve_b200 import _lib

    return _lib


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("gpu-marked test needs a CUDA device and none is visible")
    return torch.device("cuda:0")
