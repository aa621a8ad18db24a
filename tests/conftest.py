"""Shared pytest setup.

* registers the ``gpu`` marker (tests that need a B200; run with ``-m gpu``);
* puts the repo root (for the ``oracle`` checker package) and
  ``stokesflow.jl_b200`` (for the ``stokesflow_b200`` product package) on sys.path;
* builds the oracle and the CUDA library once per session if they are missing.
"""
import os
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "stokesflow.jl_b200")
for p in (ROOT, PKG, os.path.join(ROOT, "tests")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200, sm_100a)")


@pytest.fixture(scope="session")
def oracle_lib():
    import oracle
    oracle.build()
    return oracle


@pytest.fixture(scope="session")
def sf():
    """The product package with its CUDA library loaded (GPU tests only)."""
    import torch
    if not torch.cuda.is_available():
        pytest.fail("GPU test collected without a CUDA device")
    import stokesflow_b200
    stokesflow_b200.build()
    stokesflow_b200.lib()
    return stokesflow_b200
