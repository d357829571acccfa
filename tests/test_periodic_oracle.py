"""The z-periodic (3D) oracle (``oracle.periodic``), pinned like the 2D one by invariants the
reference's tests use and by finite differences:

* Hermitian M̂ and ⟨H|M̂|H⟩ real (``ME/test/runtests.jl:58``);
* a uniform medium's fundamental band: k = ω√ε;
* a z-invariant cell reproduces the 2D oracle's k (its lowest bands have g_z = 0);
* ``HMₖH_weighted`` with weight 1 equals ``HMₖH``;
* the pull-back (``period.jl:136-200``): ω̄ against d k/dω, Λ̄ against d k/dΛ and a diagonal
  ε̄⁻¹ direction against central differences of re-solved k, and the eigenvector channel
  against central differences of a linear functional of the (phase-canonical) mode."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from oracle import periodic as P

OMEGA = 1 / 1.55


def _grating(Nx=12, Ny=8, Nz=4, depth=0.3):
    """A Gaussian-core guide whose core index is modulated along z (a Bragg grating)."""
    x = -3.0 + np.arange(Nx) * 6.0 / Nx
    y = -2.0 + np.arange(Ny) * 4.0 / Ny
    z = np.arange(Nz) / Nz
    X, Y, Z = np.meshgrid(x, y, z, indexing="ij")
    core = np.exp(-(X ** 2 / 1.0 + Y ** 2 / 0.36))
    eps = 2.1 + (4.2 - 2.1) * core * (1 + depth * np.cos(2 * np.pi * Z))
    ei = np.zeros((3, 3, Nx, Ny, Nz))
    for a in range(3):
        ei[a, a] = 1 / eps
    return ei


def test_hermitian_and_uniform_medium():
    g = P.Grid3(6.0, 4.0, 0.25, 12, 8, 4)
    ei = _grating()
    op = P.Operator3(1.3, ei, g)
    rng = np.random.default_rng(1)
    a = rng.standard_normal(op.size) + 1j * rng.standard_normal(op.size)
    b = rng.standard_normal(op.size) + 1j * rng.standard_normal(op.size)
    assert abs(np.vdot(a, op.M(b)) - np.conj(np.vdot(b, op.M(a)))) <= 1e-9 * abs(np.vdot(a, op.M(b)))
    assert np.isclose(op.HMkH_weighted(a, np.ones((4, 8, 12))), op.HMkH(a), rtol=1e-13)
    u = np.zeros_like(ei)
    for c in range(3):
        u[c, c] = 1 / 2.5
    # (the period keeps k = ω√ε inside the first Brillouin zone, |k| < 1/(2Λ) = 2 μm⁻¹)
    km, _ = P.solve_k_periodic(OMEGA, u, 0.25, g, nev=1, k_tol=1e-12, eig_tol=1e-11)
    assert np.isclose(km[0], OMEGA * np.sqrt(2.5), rtol=1e-10)
    # the MPB-style P̂ inverts M̂ exactly in a uniform medium
    opu = P.Operator3(1.3, u, g)
    assert np.allclose(opu.P(opu.M(a)), a, rtol=0, atol=1e-12 * np.linalg.norm(a))


def test_z_invariant_cell_matches_2d_oracle():
    ei3 = _grating(depth=0.0)
    g3 = P.Grid3(6.0, 4.0, 0.25, 12, 8, 4)
    km3, kv3 = P.solve_k_periodic(OMEGA, ei3, 0.25, g3, nev=2, k_tol=1e-12, eig_tol=1e-11)
    km2, _ = O.solve_k(OMEGA, ei3[..., 0], O.Grid(6.0, 4.0, 12, 8), nev=2, k_tol=1e-12, eig_tol=1e-11)
    assert np.allclose(km3, km2, rtol=1e-10)


def _fd(f, x, h):
    return (f(x - 2 * h) - 8 * f(x - h) + 8 * f(x + h) - f(x + 2 * h)) / (12 * h)


@pytest.fixture(scope="module")
def grating_case():
    ei = _grating()
    L = 0.25
    g = P.Grid3(6.0, 4.0, L, 12, 8, 4)
    km, kv = P.solve_k_periodic(OMEGA, ei, L, g, nev=1, k_tol=1e-13, eig_tol=1e-12)
    return ei, L, g, km, kv


def test_pullback_k_channel_against_finite_differences(grating_case):
    ei, L, g, km, kv = grating_case
    wb, eib, Lb = P.solve_k_periodic_pullback(OMEGA, ei, L, g, km, kv, kbar=[1.0])
    solve = lambda w=OMEGA, e=ei, LL=L: P.solve_k_periodic(w, e, LL, g, nev=1, k_tol=1e-13, eig_tol=1e-12)[0][0]
    assert np.isclose(wb, _fd(lambda w: solve(w=w), OMEGA, 1e-3), rtol=1e-6)
    assert np.isclose(Lb, _fd(lambda LL: solve(LL=LL), L, 1e-3), rtol=1e-6)
    rng = np.random.default_rng(3)
    dirn = np.zeros_like(ei)
    for a in range(3):
        dirn[a, a] = rng.standard_normal(ei.shape[2:]) * 1e-2
    fd = _fd(lambda t: solve(e=ei + t * dirn), 0.0, 1e-2)
    assert np.isclose(np.sum(eib * dirn), fd, rtol=1e-5)


def test_pullback_eigenvector_channel_against_finite_differences(grating_case):
    """A linear functional Re⟨c, h⟩ of the phase-canonical mode: ē = c (the reference's
    convention ē = ∂L/∂conj(h) for L = Re⟨c, h⟩ up to the factor the pull-back expects)."""
    ei, L, g, km, kv = grating_case
    rng = np.random.default_rng(7)
    c = rng.standard_normal(kv[0].size) + 1j * rng.standard_normal(kv[0].size)

    def f(w=OMEGA, LL=L):
        _, v = P.solve_k_periodic(w, ei, LL, g, nev=1, k_tol=1e-13, eig_tol=1e-12)
        return float(np.real(np.vdot(c, v[0])))

    wb, _, Lb = P.solve_k_periodic_pullback(OMEGA, ei, L, g, km, kv, evbar=[c])
    assert np.isclose(wb, _fd(lambda w: f(w=w), OMEGA, 1e-3), rtol=1e-4)
    assert np.isclose(Lb, _fd(lambda LL: f(LL=LL), L, 1e-3), rtol=1e-4)
