"""Test configuration: the `gpu` marker, golden fixtures and the oracle build."""

from pathlib import Path

import numpy as np
import pytest

GOLDEN = Path(__file__).resolve().parent / "golden"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (sm_100a) and the built library")


@pytest.fixture(scope="session")
def argon():
    return dict(np.load(GOLDEN / "argon_512.npz"))


@pytest.fixture(scope="session")
def argon_md():
    return dict(np.load(GOLDEN / "argon_512_md.npz"))


@pytest.fixture(scope="session")
def lj_frames():
    return dict(np.load(GOLDEN / "lj_frames_4.npz"))


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda", 0)
