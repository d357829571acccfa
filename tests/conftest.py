"""Shared fixtures.  ``gpu``-marked tests need a CUDA device and the built library."""

from __future__ import annotations

import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "optimode.jl_b200")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and libomb200.so")


def gaussian_epsinv(p, Dx=6.0, Dy=4.0, Nx=24, Ny=16):
    """Isotropic Gaussian index bump (``ME/test/runtests.jl:29-41``), reference-indexed
    ``(3, 3, Nx, Ny)`` inverse permittivity."""
    ec, eb, wx, wy = p
    x = -Dx / 2 + np.arange(Nx) * (Dx / Nx)
    y = -Dy / 2 + np.arange(Ny) * (Dy / Ny)
    X, Y = np.meshgrid(x, y, indexing="ij")  # (Nx, Ny)
    eps = eb + (ec - eb) * np.exp(-(X ** 2 / wx ** 2 + Y ** 2 / wy ** 2))
    ei = np.zeros((3, 3, Nx, Ny))
    for a in range(3):
        ei[a, a] = 1.0 / eps
    return ei


P_WG = (4.2, 2.1, 1.0, 0.6)
OMEGA0 = 1.0 / 1.55


@pytest.fixture(scope="session")
def gauss_case():
    import oracle as O
    grid = O.Grid(6.0, 4.0, 24, 16)
    return grid, gaussian_epsinv(P_WG)


@pytest.fixture(scope="session")
def cuda_available():
    try:
        import torch
        return torch.cuda.is_available()
    except Exception:  # pragma: no cover
        return False
