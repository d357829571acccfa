"""Parity of the fused operator kernels (M̂, P̂, HMₖH, E) with the FP64 oracle, through the
C ABI.  Tolerances: relative L2 ≤ 1e-12 in FP64 and ≤ 3e-6 in FP32."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from conftest import gaussian_epsinv, P_WG

pytestmark = pytest.mark.gpu

TOL = {"fp64": 1e-12, "fp32": 3e-6}

# (Nx, Ny, Dx, Dy): non-square, radix-2/3/5, the bench sizes and the largest size
GRIDS = [(24, 16, 6.0, 4.0), (12, 8, 3.0, 2.0), (20, 40, 2.0, 4.0), (128, 128, 6.0, 4.0),
         (192, 128, 6.0, 4.0), (256, 192, 8.0, 5.0), (256, 256, 8.0, 5.0), (512, 512, 8.0, 8.0)]


def random_epsinv(Nx, Ny, seed=0):
    """Random anisotropic symmetric positive-definite ε per pixel, inverted."""
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((Nx, Ny, 3, 3)))
    d = rng.uniform(1.0, 12.0, (Nx, Ny, 3))
    eps = np.einsum("xyab,xyb,xycb->xyac", Q, d, Q)
    ei = np.linalg.inv(eps)
    ei = 0.5 * (ei + np.swapaxes(ei, -1, -2))
    return np.ascontiguousarray(np.transpose(ei, (2, 3, 0, 1)))


def rand_block(n, m, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def omb():
    import omb200
    return omb200


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("Nx,Ny,Dx,Dy", GRIDS)
def test_apply_M_and_P(omb, prec, Nx, Ny, Dx, Dy):
    g = omb.Grid(Dx, Dy, Nx, Ny)
    og = O.Grid(Dx, Dy, Nx, Ny)
    ei = random_epsinv(Nx, Ny, seed=Nx + Ny)
    k = 1.37
    H = rand_block(2 * g.N, 3, seed=1)
    op = O.Operator(k, ei, og)
    out = omb.apply_M(k, ei, g, H, precision=prec)
    ref = op.M_block(H)
    assert rel(out, ref) < TOL[prec]
    outp = omb.apply_P(k, ei, g, H, precision=prec)
    assert rel(outp, op.P_block(H)) < TOL[prec]
    outd = omb.apply_P(k, ei, g, H, precision=prec, kind="diag")
    assert rel(outd, op.P_block(H, "diag")) < TOL[prec]


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("Nx,Ny,Dx,Dy", GRIDS[:5])
def test_HMkH_and_Efield(omb, prec, Nx, Ny, Dx, Dy):
    g = omb.Grid(Dx, Dy, Nx, Ny)
    og = O.Grid(Dx, Dy, Nx, Ny)
    ei = random_epsinv(Nx, Ny, seed=3)
    k = 1.1
    H = rand_block(2 * g.N, 2, seed=2)
    H /= np.linalg.norm(H, axis=0)
    op = O.Operator(k, ei, og)
    got = omb.HMkH(k, ei, g, H, precision=prec)
    ref = np.array([op.HMkH(H[:, j]) for j in range(2)])
    assert np.allclose(got, ref, rtol=10 * TOL[prec], atol=0)
    E = omb.E_field(k, ei, g, H[:, 0], precision=prec)
    assert rel(E, O.E_field(k, H[:, 0], ei, og)) < TOL[prec]


def test_hermitian_fp64(omb):
    # ME/test/runtests.jl:50-58, rtol 1e-9
    g = omb.Grid(6.0, 4.0, 24, 16)
    ei = gaussian_epsinv(P_WG)
    k0 = O.k_guess(1 / 1.55, ei)
    V = rand_block(2 * g.N, 2, seed=9)
    MV = omb.apply_M(k0, ei, g, V)
    a = np.vdot(V[:, 1], MV[:, 0])
    b = np.conj(np.vdot(V[:, 0], MV[:, 1]))
    assert np.isclose(a, b, rtol=1e-9)


def test_uniform_medium_is_diagonal(omb):
    g = omb.Grid(6.0, 4.0, 24, 16)
    ei = np.zeros((3, 3, 24, 16))
    for a in range(3):
        ei[a, a] = 1 / 2.5
    op = O.Operator(1.3, ei, O.Grid(6.0, 4.0, 24, 16))
    v = rand_block(2 * g.N, 1, 4)[:, 0]
    assert rel(omb.apply_M(1.3, ei, g, v), np.repeat((op.mag ** 2 / 2.5).reshape(-1), 2) * v) < 1e-13


def test_rejects_bad_input(omb):
    g = omb.Grid(6.0, 4.0, 24, 16)
    ei = gaussian_epsinv(P_WG)
    bad = ei.copy()
    bad[0, 1, 3, 3] = 0.3  # asymmetric
    with pytest.raises(omb.OmbError, match="symmetric"):
        omb.apply_M(1.2, bad, g, np.ones(2 * g.N, complex))
    with pytest.raises(omb.OmbError, match="unsupported grid"):
        omb.apply_M(1.2, np.zeros((3, 3, 14, 16)), omb.Grid(6.0, 4.0, 14, 16), np.ones(2 * 14 * 16, complex))
    nan = ei.copy()
    nan[1, 1, 0, 0] = np.nan
    with pytest.raises(omb.OmbError, match="non-finite"):
        omb.apply_M(1.2, nan, g, np.ones(2 * g.N, complex))


def test_hfield_matches_oracle():
    """omb_hfield: fft2(h1 m̂ + h2 n̂) (``fields.jl:125-126`` with ``tc``) against the oracle's
    basis and FFT, FP64, relative L2 ≤ 1e-12, on a non-square radix-3 grid."""
    import omb200
    g = omb200.Grid(6.0, 4.0, 48, 32)
    og = O.Grid(6.0, 4.0, 48, 32)
    k = 1.7
    rng = np.random.default_rng(4)
    H = rng.standard_normal((2 * g.N, 2)) + 1j * rng.standard_normal((2 * g.N, 2))
    got = omb200.H_field(k, g, H)
    mag, m, n = O.mag_mn(k, og)
    for j in range(2):
        h = H[:, j].reshape(g.Ny, g.Nx, 2)
        cart = h[..., 0:1] * m + h[..., 1:2] * n
        ref = O.maxwell.fft2(cart).reshape(-1)
        assert np.linalg.norm(got[j] - ref) / np.linalg.norm(ref) < 1e-12


@pytest.mark.parametrize("n2,n", [(131072, 12), (65536 * 3, 15), (4096, 36)])
def test_gram_blocks_accuracy(n2, n):
    """The eigensolver's streaming Gram kernel on FP32-exact random blocks against the exact
    (FP64) products: FP32 with compensated tile sums within 5e-7·‖z_a‖‖z_b‖ (the FP32 rounding
    of one tile's partial sums), FP64 within 1e-13."""
    import omb200
    from omb200.ops import gram_blocks
    rng = np.random.default_rng(n2 + n)
    Z = (rng.standard_normal((n2, n)) + 1j * rng.standard_normal((n2, n))).astype(np.complex64).astype(np.complex128)
    AZ = (rng.standard_normal((n2, n)) + 1j * rng.standard_normal((n2, n))).astype(np.complex64).astype(np.complex128)
    Ge, Se = Z.conj().T @ Z, Z.conj().T @ AZ
    nz, naz = np.linalg.norm(Z, axis=0), np.linalg.norm(AZ, axis=0)
    # the kernel computes the upper triangles (a ≤ b) and mirrors them: in the solver both
    # products are Hermitian; here AZ is random, so only the upper triangle of S is compared
    up = np.triu(np.ones((n, n), dtype=bool))
    for prec, tol in (("fp32", 5e-7), ("fp64", 1e-13)):
        G, S = gram_blocks(Z, AZ, prec)
        eg = np.max(np.abs(G - Ge) / np.outer(nz, nz))
        es = np.max((np.abs(S - Se) / np.outer(nz, naz))[up])
        assert eg < tol and es < tol, (prec, eg, es)


@pytest.mark.parametrize("Nx,Ny", [(24, 16), (40, 24), (12, 8), (128, 128), (192, 128), (256, 192)])
def test_component_parallel_passes_match_oracle(omb, Nx, Ny):
    """The component-parallel FP32 passes (row variant 3, column variants 3 and 4) against the
    FP64 oracle at the FP32 tolerance, on radix-2/3/5 and non-square grids."""
    import torch

    from omb200 import ops
    name = torch.cuda.get_device_name(0)
    g = omb.Grid(6.0, 4.0, Nx, Ny)
    og = O.Grid(6.0, 4.0, Nx, Ny)
    ei = random_epsinv(Nx, Ny, seed=3)
    H = rand_block(2 * g.N, 3, seed=Nx + Ny)
    op = O.Operator(1.3, ei, og)
    ref = np.stack([op.M(H[:, j]) for j in range(3)], axis=1)
    try:
        for r, c in ((3, 3), (4, 4), (3, 1), (4, 5), (1, 3)):
            ops.tune_set(name, Nx, Ny, r, c, 0)
            got = omb.apply_M(1.3, ei, g, H, precision="fp32")
            assert rel(got, ref) <= TOL["fp32"], (r, c)
    finally:
        ops.tune_set(name, Nx, Ny, 1, 1, 0)


def test_tile_variants_agree_and_autotune_picks_one():
    """Every tile variant of the FP32 M̂ passes gives the default tiles' result (the per-pixel
    arithmetic does not depend on the tiling); the wave variants (several launches per pass,
    which only the batched engine's many units reach) give the same eigensolves; the
    autotuner times every combination (the one-kernel cluster apply once) and keeps the
    fastest."""
    import torch

    import omb200
    from omb200 import ops
    from omb200.geometry import ln_ridge_shapes
    from oracle import smoothing as OS
    name = torch.cuda.get_device_name(0)
    for (Nx, Ny) in ((256, 256), (192, 128)):
        g = omb200.Grid(8.0, 5.0, Nx, Ny)
        shapes, bg = ln_ridge_shapes(g, top_width=1.5)
        ei = OS.smooth_epsinv_constant(shapes, bg, g)
        rng = np.random.default_rng(Nx)
        H = rng.standard_normal((2 * g.N, 3)) + 1j * rng.standard_normal((2 * g.N, 3))
        ops.tune_set(name, Nx, Ny, 1, 1, 0)
        ref = omb200.apply_M(1.3, ei, g, H, precision="fp32")
        for r in range(7):
            for c in range(6):
                ops.tune_set(name, Nx, Ny, r, c, 0)
                got = omb200.apply_M(1.3, ei, g, H, precision="fp32")
                assert np.linalg.norm(got - ref) / np.linalg.norm(ref) < 1e-6, (Nx, Ny, r, c)
        probs = [{"omega": w, "eps_inv": ei, "grid": g, "nev": 3} for w in (0.62, 0.64, 0.66, 0.68)]
        ks = []
        for r, c, w in ((1, 1, 0), (1, 1, 1), (1, 1, 3), (3, 3, 0), (4, 4, 2), (4, 5, 0), (5, 1, 0), (6, 1, 0)):
            ops.tune_set(name, Nx, Ny, r, c, w)
            res = omb200.solve_k_batch(probs, omb200.B200Solver(precision="mixed"))
            ks.append(np.array([km for km, _ in res]))
        for kv in ks[1:]:
            assert np.allclose(kv, ks[0], rtol=1e-10)
        r, c, w, t = ops.autotune(g)
        timed = t[t >= 0]
        assert np.all(timed > 0) and t[r, c, w] == timed.min()
        # each cluster apply is timed once (its column and wave slots are not separate kernels)
        for rc in (5, 6):
            assert (t[rc] >= 0).sum() == (1 if (Nx, Ny) == (256, 256) else 0)
        assert ops.tune_get(name, Nx, Ny) == (r, c, w)
