"""Parity of the z-periodic (3D) device path with the FP64 oracle (``oracle.periodic``), through
the C ABI: the 3D M̂ / P̂ / HMₖH applications, ``solve_k_periodic`` and its pull-back (ω̄, ε̄⁻¹
and the period cotangent Λ̄, ``lib/MaxwellEigenmodes/src/grads/period.jl:136-200``).

Tolerances: operator applications relative L2 ≤ 1e-12 (FP64) and ≤ 3e-6 (FP32); k relative
≤ 1e-9 at k_tol = eig_tol = 1e-11; modes |⟨h_dev, h_oracle⟩| ≥ 1 − 1e-9; pull-backs (both
computed on the device's own modes) relative ≤ 1e-7 for ω̄ and Λ̄ and relative L2 ≤ 1e-6 for ε̄⁻¹
(the adjoint MINRES stops at 1e-12)."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from oracle import periodic as OP

pytestmark = pytest.mark.gpu

OMEGA = 1 / 1.55
TOL = {"fp64": 1e-12, "fp32": 3e-6}


def grating(Nx=24, Ny=16, Nz=8, depth=0.3, Dx=6.0, Dy=4.0, shift=(0.13, 0.07)):
    """A Gaussian-core guide (off-centre, so no mirror symmetry ties the phase pixel) whose
    core index is modulated along z over one period: a Bragg grating, ε⁻¹ (3, 3, Nx, Ny, Nz)."""
    x = -Dx / 2 + np.arange(Nx) * Dx / Nx - shift[0]
    y = -Dy / 2 + np.arange(Ny) * Dy / Ny - shift[1]
    z = np.arange(Nz) / Nz
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    core = np.exp(-(X ** 2 / 1.0 + Y ** 2 / 0.36))
    eps = 2.1 + (4.2 - 2.1) * core * (1 + depth * np.cos(2 * np.pi * Z))
    ei = np.zeros((3, 3, Nx, Ny, Nz))
    for a in range(3):
        ei[a, a] = 1 / eps
    return ei


def rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.fixture(scope="module")
def omb():
    import omb200
    return omb200


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("dims", [(24, 16, 8), (32, 24, 12), (64, 48, 16)])
def test_apply3_and_HMkH3_match_oracle(omb, prec, dims):
    Nx, Ny, Nz = dims
    L = 0.25
    ei = grating(Nx, Ny, Nz)
    g = omb.Grid3(6.0, 4.0, L, Nx, Ny, Nz)
    op = OP.Operator3(1.3, ei, OP.Grid3(6.0, 4.0, L, Nx, Ny, Nz))
    rng = np.random.default_rng(5)
    H = rng.standard_normal((op.size, 2)) + 1j * rng.standard_normal((op.size, 2))
    for name, f in (("M", op.M), ("P", op.P)):
        got = omb.apply3(name, 1.3, ei, g, H, precision=prec)
        for j in range(2):
            assert rel(got[:, j], f(H[:, j])) <= TOL[prec], (name, j)
    hm = omb.HMkH3(1.3, ei, g, H, precision=prec)
    for j in range(2):
        ref = op.HMkH(H[:, j])
        assert abs(hm[j] - ref) <= 10 * TOL[prec] * np.linalg.norm(H[:, j]) ** 2 * 1.3


def test_apply3_hermitian(omb):
    """⟨a|M̂b⟩ = conj⟨b|M̂a⟩ on the 3D operator (``ME/test/runtests.jl:58``)."""
    ei = grating()
    g = omb.Grid3(6.0, 4.0, 0.25, 24, 16, 8)
    rng = np.random.default_rng(2)
    n = 2 * g.N
    a = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    b = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    Ma, Mb = omb.apply3("M", 1.1, ei, g, a), omb.apply3("M", 1.1, ei, g, b)
    assert abs(np.vdot(a, Mb) - np.conj(np.vdot(b, Ma))) <= 1e-12 * abs(np.vdot(a, Mb))


@pytest.fixture(scope="module")
def solved(omb):
    ei = grating()
    L = 0.25
    g = omb.Grid3(6.0, 4.0, L, 24, 16, 8)
    km, kv, info = omb.solve_k_periodic(OMEGA, ei, L, g, nev=2, k_tol=1e-11, eig_tol=1e-11, return_info=True)
    return ei, L, g, km, kv, info


def test_solve_k_periodic_matches_oracle(solved):
    ei, L, g, km, kv, info = solved
    assert np.all(info["status"] == 0)
    og = OP.Grid3(6.0, 4.0, L, 24, 16, 8)
    kr, vr = OP.solve_k_periodic(OMEGA, ei, L, og, nev=2, k_tol=1e-12, eig_tol=1e-11)
    assert np.allclose(km, kr, rtol=1e-9, atol=0)
    for j in range(2):
        assert abs(abs(np.vdot(kv[j], vr[j])) - 1) <= 1e-9
        # the residual of the device mode under the oracle's operator
        op = OP.Operator3(km[j], ei, og)
        r = op.M(kv[j]) - OMEGA ** 2 * kv[j]
        assert np.linalg.norm(r) <= 1e-8 * OMEGA ** 2
        # ∂ω²/∂k reported with the solve
        assert np.isclose(info["dw2dk"][j], 2 * op.HMkH(kv[j]), rtol=1e-9)
    # phase canonicalisation: the same field, not just the same ray
    assert rel(kv[0], vr[0]) <= 1e-6


def test_z_invariant_cell_matches_2d_solve(omb):
    ei3 = grating(depth=0.0)
    g3 = omb.Grid3(6.0, 4.0, 0.25, 24, 16, 8)
    k3, _ = omb.solve_k_periodic(OMEGA, ei3, 0.25, g3, nev=2, k_tol=1e-11, eig_tol=1e-11)
    k2, _ = omb.solve_k(OMEGA, ei3[..., 0], omb.Grid(6.0, 4.0, 24, 16), nev=2, k_tol=1e-11, eig_tol=1e-11)
    assert np.allclose(k3, k2, rtol=1e-10)


def test_pullback_periodic_matches_oracle(omb, solved):
    ei, L, g, km, kv, _ = solved
    og = OP.Grid3(6.0, 4.0, L, 24, 16, 8)
    rng = np.random.default_rng(11)
    c = rng.standard_normal(kv[0].size) + 1j * rng.standard_normal(kv[0].size)
    cases = [([1.0, 0.5], None), (None, [c, None]), ([0.3, -0.2], [0.1 * c, c])]
    for kbar, evbar in cases:
        wb, eib, Lb = omb.solve_k_periodic_pullback(OMEGA, ei, L, g, km, kv, kbar, evbar)
        wr, eir, Lr = OP.solve_k_periodic_pullback(OMEGA, ei, L, og, km, kv, kbar, evbar)
        assert np.isclose(wb, wr, rtol=1e-7), (kbar is None, evbar is None)
        assert np.isclose(Lb, Lr, rtol=1e-7), (kbar is None, evbar is None)
        assert rel(eib, eir) <= 1e-6


def test_period_cotangent_against_device_finite_differences(omb, solved):
    """Λ̄ for k̄ = (1, 0) is dk₁/dΛ: central differences of re-solved k on the device."""
    ei, L, g, km, kv, _ = solved
    _, _, Lb = omb.solve_k_periodic_pullback(OMEGA, ei, L, g, km, kv, kbar=[1.0, 0.0])
    h = 1e-4

    def k1(LL):
        return omb.solve_k_periodic(OMEGA, ei, LL, g, nev=1, k_tol=1e-12, eig_tol=1e-12)[0][0]

    fd = (k1(L + h) - k1(L - h)) / (2 * h)
    assert np.isclose(Lb, fd, rtol=1e-5)


def test_rrule_and_invalid_inputs(omb, solved):
    ei, L, g, km, kv, _ = solved
    (k2, v2), pb = omb.solve_k_periodic_rrule(OMEGA, ei, L, g, nev=1, k_tol=1e-11, eig_tol=1e-11)
    assert np.isclose(k2[0], km[0], rtol=1e-9)
    wb, eib, Lb = pb(([1.0], None))
    assert wb > 0 and np.isfinite(Lb) and eib.shape == (3, 3, 24, 16, 8)
    with pytest.raises(omb.OmbError):  # Nz below the 8 slabs a periodic cell needs
        omb.solve_k_periodic(OMEGA, ei[..., :4], L, omb.Grid3(6.0, 4.0, L, 24, 16, 4))
    with pytest.raises(ValueError):
        omb.solve_k_periodic(OMEGA, ei, L, g, omb.B200Solver(newton="outer"))
