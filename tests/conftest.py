"""Shared pytest configuration.

Markers
  gpu   -- needs a CUDA device (run with ``-m gpu`` on a B200)
  slow  -- takes more than a few seconds of CPU time
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: test needs a CUDA GPU")
    config.addinivalue_line("markers", "slow: test takes more than a few seconds")


def _has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def gpu_available():
    return _has_gpu()


@pytest.fixture(scope="session", autouse=True)
def built_libraries():
    """Build the product library and the oracle once per session (nvcc and
    gcc are present here and on the GPU box; an up-to-date build is a no-op)."""
    from openswpc_b200 import build as pbuild

    pbuild.build()
    sys.path.insert(0, str(ROOT))
    import importlib.util

    spec = importlib.util.spec_from_file_location("build_oracle", ROOT / "oracle" / "build_oracle.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    mod.build()
    yield


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
