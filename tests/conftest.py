"""Shared fixtures. GPU tests are marked ``gpu``; everything else runs on CPU."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a B200 (sm_100a) GPU")


def _has_gpu():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:
        return False


def pytest_collection_modifyitems(config, items):
    if _has_gpu():
        return
    skip = pytest.mark.skip(reason="no GPU in this environment")
    for it in items:
        if "gpu" in it.keywords:
            it.add_marker(skip)


@pytest.fixture(scope="session")
def orc():
    from oracle import oracle
    oracle.lib()
    return oracle


@pytest.fixture(scope="session")
def geo():
    import geo_simulator_b200 as g
    return g


def thermal_problem(n, orc, lx=1000.0, ly=1000.0, lz=600.0, nz=None):
    """The 1D thermal benchmark set-up (thermal_1d_improved_mesh.rs:18-52)."""
    xyz, conn = orc.generate_cube(n, n, nz or n, lx, ly, lz)
    mask, vals = orc.thermal_bc(xyz, lz)
    return xyz, conn, mask, vals

