"""The C-ABI library builds, loads and exports every symbol its header declares; without a
GPU it refuses to run instead of falling back to the CPU.  No GPU needed."""

from __future__ import annotations

import ctypes
import os
import re
import subprocess

import pytest

from conftest import ROOT

HEADER = os.path.join(ROOT, "include", "omb200.h")


def _ensure_built():
    from omb200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        subprocess.run(["make", "-C", os.path.join(ROOT, "optimode.jl_b200"), "-j8"], check=True,
                       stdout=subprocess.DEVNULL)
    return _lib


def _declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(omb_[a-zA-Z0-9_]+)\s*\(", src)))


def test_header_declares_what_the_binding_exports():
    from omb200 import _lib
    assert sorted(_lib.EXPORTS) == _declared_functions()


def test_library_exports_every_declared_symbol():
    _lib = _ensure_built()
    lib = ctypes.CDLL(_lib.LIB_PATH)
    for name in _declared_functions():
        assert hasattr(lib, name), name


def test_library_metadata_without_gpu():
    _lib = _ensure_built()
    lib = _lib.load()
    assert lib.omb_version() >= 100
    for n in (8, 12, 16, 20, 24, 128, 192, 256, 512):
        assert lib.omb_fft_size_supported(n) == 1
    for n in (7, 14, 1000, 0, -4):
        assert lib.omb_fft_size_supported(n) == 0


def test_no_cpu_fallback_without_gpu(cuda_available):
    if cuda_available:
        pytest.skip("a GPU is present")
    _lib = _ensure_built()
    with pytest.raises(_lib.OmbError) as ei:
        _lib.Context(0)
    assert "CUDA" in str(ei.value)


def test_smoothing_needs_the_gpu(cuda_available):
    """The device smoothing has no CPU fallback either."""
    if cuda_available:
        pytest.skip("a GPU is present")
    _ensure_built()
    import numpy as np
    import omb200
    square = np.array([[-0.5, -0.5], [0.5, -0.5], [0.5, 0.5], [-0.5, 0.5]])
    with pytest.raises(omb200.OmbError) as ei:
        omb200.SmoothingPlan([square], [0, 1], omb200.Grid(2.0, 2.0, 8, 8))
    assert "CUDA" in str(ei.value)


def test_smoothing_argument_checks_without_gpu():
    """Host-side argument checks of the smoothing binding run before any device call."""
    import numpy as np
    import omb200
    g = omb200.Grid(2.0, 2.0, 8, 8)
    square = np.array([[-0.5, -0.5], [0.5, -0.5], [0.5, 0.5], [-0.5, 0.5]])
    with pytest.raises(ValueError):
        omb200.SmoothingPlan([square], [0, 1], g, fill="area")
    with pytest.raises(ValueError):
        omb200.SmoothingPlan([square], [0], g)
    with pytest.raises(ValueError):
        omb200.material_column(np.eye(2))
    col = omb200.material_column(np.diag([1.0, 2.0, 3.0]), np.eye(3))
    assert col.shape == (27,) and col[4] == 2.0 and col[9] == 1.0 and col[18:].sum() == 0.0
    # clockwise outlines are stored counter-clockwise
    p = omb200.Polygon(square[::-1])
    assert np.array_equal(p.vertices, square)
