import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
for p in (ROOT, ROOT / "tests"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (runs the CUDA path)")


@pytest.fixture(autouse=True)
def _per_step_march_for_small_3d(monkeypatch, request):
    """Small 3D grids would otherwise march all their steps in one cooperative launch
    (march3d_kernel); the parity tests are written against the per-step kernels (the
    blocked 3D step, the TMA row step), so they keep those, and tests/test_gpu_march3d.py
    covers the cooperative march on its own."""
    if "march3d" not in request.node.nodeid:
        monkeypatch.setenv("CWB_MARCH3D", "0")


def pytest_collection_modifyitems(config, items):
    try:
        import torch

        has_gpu = torch.cuda.is_available()
    except Exception:
        has_gpu = False
    if has_gpu:
        return
    skip = pytest.mark.skip(reason="no CUDA device")
    for item in items:
        if "gpu" in item.keywords:
            item.add_marker(skip)
