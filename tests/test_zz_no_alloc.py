"""The allocation-free operator entry point (``omb_apply_M_noalloc``) against the regular
one (``omb_apply``) and the FP64 oracle, through the C ABI.

``omb_apply_M_noalloc`` serves callers that cannot allocate device memory when they need
the operator: a host framework that owns the whole device pool (a Julia or PyTorch caching
allocator that forbids foreign cudaMalloc/cudaFree), a caller with a device-memory budget
fixed up front, or a hot loop that must not pay the latency and implicit synchronisation of
cudaMalloc/cudaFree.  It takes caller-owned device buffers and keeps its scratch in a fixed
static device array.  The test owns its device buffers (allocated with torch, as such a
caller would), calls the entry point twice in a row on the same scratch for each shape, and
compares each result with ``omb_apply`` in FP32 and with the oracle at the FP32 operator
tolerance used by the other parity tests (relative L2 ≤ 3e-6).  Shapes: the bench grid with
4 columns, the 512×512×1 size limit (Stockham passes), non-square two-level grids and radix
3/5 lengths.  This file is collected last so a failure here cannot hide the other tests'
results.
"""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu

TOL_FP32 = 3e-6


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _eps(g, which):
    from omb200 import geometry as G
    from oracle import smoothing as OS
    if which == "ridge":
        shapes, bg = G.ln_ridge_shapes(g, top_width=1.5)
    else:
        shapes, bg = G.si3n4_rect_shapes()
    return OS.smooth_epsinv_constant(shapes, bg, g)


@pytest.mark.parametrize("Nx,Ny,Dx,Dy,ncol,which", [
    (256, 256, 8.0, 5.0, 4, "ridge"),   # the bench grid, two-level passes
    (512, 512, 8.0, 5.0, 1, "ridge"),   # the size limit, Stockham passes
    (192, 128, 6.0, 4.0, 2, "rect"),    # non-square, radix 3
    (320, 192, 8.0, 5.0, 2, "ridge"),   # Stockham rows, two-level columns
    (24, 40, 6.0, 4.0, 3, "rect"),      # small, radix 3 and 5
])
def test_noalloc_apply_matches_apply_twice(Nx, Ny, Dx, Dy, ncol, which):
    import torch

    import omb200
    from omb200 import _lib

    lib = _lib.load()
    g = omb200.Grid(Dx, Dy, Nx, Ny)
    og = O.Grid(Dx, Dy, Nx, Ny)
    ei = _eps(g, which)
    k = 1.3
    rng = np.random.default_rng(21 + Nx + Ny + ncol)
    e_dev = torch.from_numpy(np.asfortranarray(ei).ravel(order="F").astype(np.float32)).cuda()
    op = O.Operator(k, ei, og)
    for call in range(2):
        H = rng.standard_normal((2 * g.N, ncol)) + 1j * rng.standard_normal((2 * g.N, ncol))
        H = H.astype(np.complex64).astype(np.complex128)  # exact in FP32
        ref = omb200.apply_M(k, ei, g, H, precision="fp32")
        h_dev = torch.from_numpy(np.asfortranarray(H.astype(np.complex64)).ravel(order="F").view(np.float32)).cuda()
        o_dev = torch.full_like(h_dev, float("nan"))
        torch.cuda.synchronize()
        rc = lib.omb_apply_M_noalloc(g.Nx, g.Ny, g.Dx, g.Dy, k, e_dev.data_ptr(), ncol, h_dev.data_ptr(),
                                     o_dev.data_ptr(), None)
        _lib.check(rc)
        torch.cuda.synchronize()
        got = o_dev.cpu().numpy().view(np.complex64).reshape(ncol, 2 * g.N).T.astype(np.complex128)
        err = _rel(got, ref)
        assert err < TOL_FP32, f"call {call}: rel err vs omb_apply {err:.3e}"
        exact = np.stack([op.M(H[:, j]) for j in range(ncol)], axis=1)
        err_o = _rel(got, exact)
        assert err_o < TOL_FP32, f"call {call}: rel err vs oracle {err_o:.3e}"


def test_noalloc_rejects_blocks_above_its_scratch():
    import torch

    from omb200 import _lib

    lib = _lib.load()
    # 512×512 with 2 columns exceeds the fixed scratch (262144 pixel-columns); the check runs
    # before any device work, so the buffers are never touched
    dummy = torch.zeros(8, device="cuda")
    rc = lib.omb_apply_M_noalloc(512, 512, 8.0, 8.0, 1.3, dummy.data_ptr(), 2, dummy.data_ptr(),
                                 dummy.data_ptr(), None)
    assert rc == 1
    assert "exceeds its fixed scratch" in lib.omb_last_error().decode()
