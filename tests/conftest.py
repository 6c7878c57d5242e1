"""Shared test setup: import paths, the `gpu` marker, native builds.

CPU tests (-m "not gpu") exercise the oracle against golden vectors, the host
topology/index code and the C-ABI surface of libcmfb200 without launching any
kernel.  GPU tests (-m gpu) compare the CUDA path with the oracle.
"""
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
PKG = ROOT / "cama-flood-gpu_b200"
for p in (str(ROOT), str(PKG), str(ROOT / "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200)")


def _ensure_built():
    sys.path.insert(0, str(PKG))
    import build as pkg_build  # cama-flood-gpu_b200/build.py
    pkg_build.build()
    from oracle import oracle as orc
    orc.build()


_ensure_built()


def cuda_available() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def device():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch.device("cuda:0")
