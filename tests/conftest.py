import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests" / "golden"))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the built libgann.so")


def gpu_available() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    # a GPU test that stops making progress ends the run instead of holding the box
    for item in items:
        if "gpu" in item.keywords and item.get_closest_marker("timeout") is None:
            item.add_marker(pytest.mark.timeout(600, method="thread"))
    if gpu_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)


@pytest.fixture(scope="session")
def golden(tmp_path_factory):
    """Unpacked golden fixtures: name -> metadata dict with file paths."""
    from make_fixtures import FIXTURES, unpack

    base = tmp_path_factory.mktemp("golden")
    return {name: unpack(name, base / name) for name in FIXTURES}


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import oracle

    return oracle
