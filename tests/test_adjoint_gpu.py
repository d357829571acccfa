"""The device adjoint pull-back (``omb_pullback``) against the FP64 oracle on identical
inputs, and the reference's finite-difference checks (``ME/test/runtests.jl:91-110``) run
through the GPU solver.  Tolerances: ω̄ rtol 1e-7 and ε̄⁻¹ relative L2 1e-6 vs the oracle
(both solve the adjoint system to ~1e-11); FD checks at the reference's rtol 1e-4 (dk/dω)
and 1e-3 (diagonal ε⁻¹ direction)."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from conftest import OMEGA0, P_WG, gaussian_epsinv

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def omb():
    import omb200
    return omb200


@pytest.fixture(scope="module")
def case():
    grid = O.Grid(6.0, 4.0, 24, 16)
    ei = gaussian_epsinv(P_WG)
    km, kv = O.solve_k(OMEGA0, ei, grid, nev=2, k_tol=1e-12, eig_tol=1e-11)
    return grid, ei, km, kv


def _rel(a, b):
    return np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("which", ["k", "ev", "both"])
def test_pullback_parity_with_oracle(omb, case, which):
    grid, ei, km, kv = case
    g = omb.Grid(6.0, 4.0, 24, 16)
    rng = np.random.default_rng(17)
    kbar = rng.standard_normal(2) if which in ("k", "both") else None
    evbar = None
    if which in ("ev", "both"):
        evbar = [rng.standard_normal(2 * g.N) + 1j * rng.standard_normal(2 * g.N) for _ in range(2)]
    wb, eib, info = omb.pullback(OMEGA0, ei, g, km, kv, kbar, evbar, return_info=True)
    wr, eir = O.solve_k_pullback(OMEGA0, ei, grid, km, kv, kbar=kbar, evbar=evbar)
    assert np.isclose(wb, wr, rtol=1e-7, atol=0), (wb, wr)
    assert _rel(eib, eir) < 1e-6
    if evbar is not None:
        assert np.all(info["iterations"] > 0)


def test_pullback_zero_band_cotangent(omb, case):
    # an all-zero ē column stands for the reference's AbstractZero band
    grid, ei, km, kv = case
    g = omb.Grid(6.0, 4.0, 24, 16)
    rng = np.random.default_rng(3)
    ev1 = rng.standard_normal(2 * g.N) + 1j * rng.standard_normal(2 * g.N)
    wb, eib = omb.pullback(OMEGA0, ei, g, km, kv, [0.5, None], [None, ev1])
    wr, eir = O.solve_k_pullback(OMEGA0, ei, grid, km, kv, kbar=[0.5, None], evbar=[None, ev1])
    assert np.isclose(wb, wr, rtol=1e-7)
    assert _rel(eib, eir) < 1e-6


def test_eps_bar_through_sliceinv(omb, case):
    grid, ei, km, kv = case
    g = omb.Grid(6.0, 4.0, 24, 16)
    wb, eib, eb = omb.pullback(OMEGA0, ei, g, km, kv, [1.0, -0.3], None, want_eps_bar=True)
    assert _rel(eb, O.sliceinv_3x3_pullback(ei, eib)) < 1e-12


def _fd5(f, x, h):
    return (f(x - 2 * h) - 8 * f(x - h) + 8 * f(x + h) - f(x + 2 * h)) / (12 * h)


def test_dk_domega_vs_fd_through_gpu_solver(omb, case):
    # ME/test/runtests.jl:91-96
    _, ei, _, _ = case
    g = omb.Grid(6.0, 4.0, 24, 16)
    s = omb.B200Solver(precision="fp64")
    f = lambda om: omb.solve_k(om, ei, g, s, nev=1, k_tol=1e-12, eig_tol=1e-11)[0][0]
    fd = _fd5(f, OMEGA0, 1e-4)
    (km, kv), pb = omb.solve_k_rrule(OMEGA0, ei, g, s, nev=1, k_tol=1e-12, eig_tol=1e-11)
    wb, _ = pb(([1.0], None))
    assert np.isclose(wb, fd, rtol=1e-4)
    assert np.sqrt(P_WG[1]) < wb < 1.5 * np.sqrt(P_WG[0])


def test_epsinv_diagonal_direction_vs_fd_through_gpu_solver(omb, case):
    # ME/test/runtests.jl:98-110
    _, ei, _, _ = case
    g = omb.Grid(6.0, 4.0, 24, 16)
    s = omb.B200Solver(precision="fp64")
    rng = np.random.default_rng(7)
    dirn = np.zeros_like(ei)
    for a in range(3):
        dirn[a, a] = rng.standard_normal((g.Nx, g.Ny)) * 1e-3
    f = lambda t: omb.solve_k(OMEGA0, ei + t * dirn, g, s, nev=1, k_tol=1e-12, eig_tol=1e-11)[0][0]
    fd = _fd5(f, 0.0, 1e-2)
    (km, kv), pb = omb.solve_k_rrule(OMEGA0, ei, g, s, nev=1, k_tol=1e-12, eig_tol=1e-11)
    _, eib = pb(([1.0], None))
    assert np.isclose(np.sum(eib * dirn), fd, rtol=1e-3)


def test_pullback_config1_rectangle(omb):
    # 128² Si₃N₄ rectangle, 2 bands, seeded random cotangent on (k, H)
    from omb200 import geometry as G
    g = omb.Grid(6.0, 4.0, 128, 128)
    og = O.Grid(6.0, 4.0, 128, 128)
    ei = G.si3n4_rect(g)
    km, kv = O.solve_k(OMEGA0, ei, og, nev=2, k_tol=1e-12, eig_tol=1e-10)
    rng = np.random.default_rng(0)
    kbar = rng.standard_normal(2)
    evbar = [rng.standard_normal(2 * g.N) + 1j * rng.standard_normal(2 * g.N) for _ in range(2)]
    wb, eib = omb.pullback(OMEGA0, ei, g, km, kv, kbar, evbar)
    wr, eir = O.solve_k_pullback(OMEGA0, ei, og, km, kv, kbar=kbar, evbar=evbar)
    assert np.isclose(wb, wr, rtol=1e-6)
    assert _rel(eib, eir) < 1e-5
