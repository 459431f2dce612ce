"""Shared fixtures.  GPU tests are marked `gpu`; everything else runs on CPU."""
from __future__ import annotations

import os
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent
sys.path.insert(0, str(ROOT))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")
    config.addinivalue_line("markers", "slow: long-running parity run")


def has_gpu() -> bool:
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


@pytest.fixture(scope="session")
def oracle_mod():
    from oracle import pyoracle
    pyoracle.build()
    return pyoracle


@pytest.fixture(scope="session")
def lib():
    from bgk_pcm_b200 import build as b
    b.build()
    from bgk_pcm_b200 import capi
    return capi.load()


def small_params(Nx=16, Ny=12, **kw):
    """A small cavity with the benchmark's physics (cavity256 mapping)."""
    from bgk_pcm_b200 import inputs
    d = inputs.workload_params(Nx=Nx, Ny=Ny, iter=100, Ra=1e5)
    d.update(kw)
    return d
