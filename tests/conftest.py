"""Shared fixtures. GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""
import os
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


@pytest.fixture(scope="session")
def of():
    import openfusion_b200
    return openfusion_b200


@pytest.fixture(scope="session")
def ora():
    from oracle import Oracle
    return Oracle("f64")


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")


def pose_error(P, G):
    """(rotation angle rad, translation mm) between two 4x4 poses."""
    R = np.asarray(P)[:3, :3].T @ np.asarray(G)[:3, :3]
    c = np.clip((np.trace(R) - 1.0) / 2.0, -1.0, 1.0)
    return float(np.arccos(c)), float(np.linalg.norm(np.asarray(P)[:3, 3] - np.asarray(G)[:3, 3]))
