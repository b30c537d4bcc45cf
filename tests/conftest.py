"""Shared fixtures.  Tests marked `gpu` need a CUDA device; everything else runs on CPU."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


@pytest.fixture(scope="session", autouse=True)
def _built():
    """Build the library and the checker once per session (no-op when up to date)."""
    from culda_cgs_b200 import build

    build.build_library()
    build.build_cli()
    from oracle import build_oracle

    build_oracle.build_oracle_lib()


@pytest.fixture(scope="session")
def has_gpu() -> bool:
    try:
        import torch

        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(autouse=True)
def _gpu_guard(request, has_gpu):
    if request.node.get_closest_marker("gpu") and not has_gpu:
        pytest.skip("no CUDA device")
