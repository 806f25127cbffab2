"""Test configuration: the `gpu` marker, import paths and shared fixtures.

Tests marked `gpu` call the engine through its C ABI on a CUDA device; every other test runs
on the CPU (the oracle, the reference's own exact path built under oracle/_ref, the Python
host layer and the library's exported symbols).
"""
import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT / "tsne-h2pack-python_b200", ROOT / "oracle", ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))

os.environ.setdefault("TSNE_H2PACK_NO_PROXY_CACHE", "1")


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the engine)")
    config.addinivalue_line("markers", "slow: long-running")


def _cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _cuda_available():
        return
    skip = pytest.mark.skip(reason="no CUDA device in this environment")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
