import os
import sys

import pytest

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200, sm_100a)")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


def reference_dir():
    """Location of a reference checkout: $SPECTRAL_REFERENCE_DIR, else a
    checkout named ``reference`` beside this repository (None if absent)."""
    d = os.environ.get("SPECTRAL_REFERENCE_DIR") or os.path.join(
        os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__)))), "reference")
    return d if os.path.isfile(os.path.join(d, "main.py")) else None


@pytest.fixture
def reference_tree():
    d = reference_dir()
    if d is None:
        pytest.skip("reference checkout not present (set SPECTRAL_REFERENCE_DIR)")
    return d
