"""Shared test setup: import paths, the gpu marker, lazy builds."""
from __future__ import annotations

import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
for p in (ROOT, ROOT / "gpu-sims_b200"):
    if str(p) not in sys.path:
        sys.path.insert(0, str(p))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200); run with -m gpu")


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def lbm_lib():
    """The CUDA library (built in-tree if missing)."""
    import lbm
    if not lbm.LIB_PATH.exists():
        sys.path.insert(0, str(ROOT / "gpu-sims_b200"))
        import build as _b
        _b.build()
    lbm.load()
    return lbm


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o
    if not o.LIB.exists():
        o.build()
    o.lib()
    return o


@pytest.fixture(scope="session")
def golden():
    import json
    return json.loads((ROOT / "tests" / "golden" / "d3q19_equilibrium.json").read_text())


@pytest.fixture
def gpu(lbm_lib):
    if not cuda_available():
        pytest.fail("test marked gpu needs a CUDA device")
    return lbm_lib
