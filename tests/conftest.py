"""Shared fixtures.  Tests marked `gpu` need a CUDA device (a B200) and the built library;
everything else runs on CPU."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
GOLDEN = ROOT / "tests" / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU and the built libprc_b200.so")


def _cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def nrmse(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.sqrt(np.mean((a - b) ** 2)) / np.sqrt(np.mean(b ** 2)))


@pytest.fixture(scope="session")
def ref_golden():
    """Outputs of the reference executable (prc.cu built for sm_100a) on a B200."""
    return np.load(GOLDEN / "ref_outputs.npz")


@pytest.fixture(scope="session")
def fixture72():
    from prc_mlem_b200 import phantoms
    return phantoms.solver_fixture()


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle
    return oracle
