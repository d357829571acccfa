"""The allocation-free operator entry point (``omb_apply_M_noalloc``) against the regular
one (``omb_apply``), through the C ABI.

``omb_apply_M_noalloc`` serves callers that cannot allocate device memory when they need
the operator (inside a stream capture, under a framework that owns the device pool, or in
a hot loop that must not pay allocation latency): it takes caller-owned device buffers and
keeps its scratch in a fixed static device array.  The test owns its device buffers
(allocated with torch, as such a caller would), calls the entry point twice in a row on
the same scratch, and compares each result with ``omb_apply`` at the FP32 operator
tolerance used by the other parity tests (relative L2 ≤ 3e-6).  This file is collected
last so a failure here cannot hide the other tests' results.
"""

from __future__ import annotations

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

TOL_FP32 = 3e-6


def _rel(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_noalloc_apply_matches_apply_twice():
    import torch

    import omb200
    from omb200 import _lib
    from omb200 import geometry as G

    lib = _lib.load()
    g = omb200.Grid(8.0, 5.0, 256, 256)
    ei = G.ln_ridge(g, top_width=1.5)
    k = 1.3
    ncol = 4
    rng = np.random.default_rng(21)
    e_dev = torch.from_numpy(np.asfortranarray(ei).ravel(order="F").astype(np.float32)).cuda()
    outs = []
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
        assert err < TOL_FP32, f"call {call}: rel err {err:.3e}"
        outs.append(err)
    assert len(outs) == 2


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
