"""The FP64 oracle against every invariant the reference's own tests assert for this path
(``ME/test/runtests.jl``) plus analytic known answers.  CPU only."""

from __future__ import annotations

import os
import numpy as np
import pytest

import oracle as O
from conftest import OMEGA0, P_WG, gaussian_epsinv


def _rand(n, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(n) + 1j * rng.standard_normal(n)


def test_operator_hermitian_and_HMH(gauss_case):
    # ME/test/runtests.jl:50-61
    grid, ei = gauss_case
    k0 = O.k_guess(OMEGA0, ei)
    op = O.Operator(k0, ei, grid)
    v, w = _rand(2 * grid.N, 0), _rand(2 * grid.N, 1)
    assert np.isclose(np.vdot(w, op.M(v)), np.conj(np.vdot(v, op.M(w))), rtol=1e-9)
    assert np.isclose(op.HMH(v), np.real(np.vdot(v, op.M(v))), rtol=1e-6)
    # the preconditioner is Hermitian positive definite
    assert np.isclose(np.vdot(w, op.P(v)), np.conj(np.vdot(v, op.P(w))), rtol=1e-9)
    assert np.real(np.vdot(v, op.P(v))) > 0


def test_uniform_medium_known_answer():
    # uniform ε: M̂ is diagonal with entries |k+G|²/ε, so the lowest band is k = ω√ε
    grid = O.Grid(6.0, 4.0, 24, 16)
    eps = 2.5
    ei = np.zeros((3, 3, grid.Nx, grid.Ny))
    for a in range(3):
        ei[a, a] = 1.0 / eps
    op = O.Operator(1.3, ei, grid)
    v = _rand(2 * grid.N, 3)
    diag = np.repeat((op.mag ** 2 / eps).reshape(-1), 2)
    assert np.allclose(op.M(v), diag * v, rtol=1e-12, atol=1e-12)
    # ∂M̂/∂k = diag(2k/ε), so ⟨v|∂M̂/∂k|v⟩/2 = k/ε for any unit v
    assert np.isclose(op.HMkH(v / np.linalg.norm(v)), 1.3 / eps, rtol=1e-12)
    km, _ = O.solve_k(OMEGA0, ei, grid, nev=2)
    assert np.allclose(km, OMEGA0 * np.sqrt(eps), rtol=1e-12)


def test_solve_omega2_residual_and_bounds(gauss_case):
    # ME/test/runtests.jl:64-82
    grid, ei = gauss_case
    k0 = O.k_guess(OMEGA0, ei)
    evals, evecs, info = O.solve_omega2(k0, ei, grid, nev=2)
    assert info["converged"] and np.all(evals > 0)
    op = O.Operator(k0, ei, grid)
    for a, v in zip(evals, evecs):
        assert np.linalg.norm(op.M(v) - a * v) / np.linalg.norm(v) < 1e-8
    kmags, _ = O.solve_k(OMEGA0, ei, grid, nev=1)
    neff = kmags[0] / OMEGA0
    assert np.sqrt(P_WG[1]) < neff < np.sqrt(P_WG[0])
    ev2, _, _ = O.solve_omega2(kmags[0], ei, grid, nev=1)
    assert np.isclose(ev2[0], OMEGA0 ** 2, rtol=1e-6)


def test_solve_k_modes_are_eigenvectors(gauss_case):
    grid, ei = gauss_case
    kmags, evecs = O.solve_k(OMEGA0, ei, grid, nev=2, k_tol=1e-11, eig_tol=1e-10)
    for k, v in zip(kmags, evecs):
        op = O.Operator(k, ei, grid)
        assert np.isclose(np.linalg.norm(v), 1.0, rtol=1e-12)
        assert np.linalg.norm(op.M(v) - OMEGA0 ** 2 * v) < 1e-8
        # canonical phase: the largest E component is real and positive
        E = O.E_field(k, v, ei, grid)
        e = E[np.argmax(np.abs(E))]
        assert abs(np.imag(e)) < 1e-12 * abs(e) and np.real(e) > 0


def _fd5(f, x, h):
    return (f(x - 2 * h) - 8 * f(x - h) + 8 * f(x + h) - f(x + 2 * h)) / (12 * h)


def test_adjoint_dk_domega_vs_fd(gauss_case):
    # ME/test/runtests.jl:91-96 (rtol 1e-4)
    grid, ei = gauss_case
    f = lambda om: O.solve_k(om, ei, grid, nev=1, k_tol=1e-12, eig_tol=1e-11)[0][0]
    fd = _fd5(f, OMEGA0, 1e-4)
    km, kv = O.solve_k(OMEGA0, ei, grid, nev=1, k_tol=1e-12, eig_tol=1e-11)
    wb, _ = O.solve_k_pullback(OMEGA0, ei, grid, km, kv, kbar=[1.0])
    assert np.isclose(wb, fd, rtol=1e-4)
    assert np.sqrt(P_WG[1]) < wb < 1.5 * np.sqrt(P_WG[0])


def test_adjoint_epsinv_diagonal_direction_vs_fd(gauss_case):
    # ME/test/runtests.jl:98-110 (rtol 1e-3)
    grid, ei = gauss_case
    rng = np.random.default_rng(7)
    dirn = np.zeros_like(ei)
    for a in range(3):
        dirn[a, a] = rng.standard_normal((grid.Nx, grid.Ny)) * 1e-3
    f = lambda t: O.solve_k(OMEGA0, ei + t * dirn, grid, nev=1, k_tol=1e-12, eig_tol=1e-11)[0][0]
    fd = _fd5(f, 0.0, 1e-2)
    km, kv = O.solve_k(OMEGA0, ei, grid, nev=1, k_tol=1e-12, eig_tol=1e-11)
    _, eib = O.solve_k_pullback(OMEGA0, ei, grid, km, kv, kbar=[1.0])
    assert np.isclose(np.sum(eib * dirn), fd, rtol=1e-3)


def test_adjoint_field_cotangent_vs_fd(gauss_case):
    # gauge-invariant objective Σ w|H|² exercises the eig_adjt branch of the pull-back
    grid, ei = gauss_case
    wt = np.random.default_rng(3).random(2 * grid.N)

    def fH(om):
        _, kv = O.solve_k(om, ei, grid, nev=1, k_tol=1e-13, eig_tol=1e-12)
        return float(np.sum(wt * np.abs(kv[0]) ** 2))

    km, kv = O.solve_k(OMEGA0, ei, grid, nev=1, k_tol=1e-13, eig_tol=1e-12)
    wb, _ = O.solve_k_pullback(OMEGA0, ei, grid, km, kv, kbar=[0.0], evbar=[2 * wt * kv[0]])
    fd = (fH(OMEGA0 + 1e-4) - fH(OMEGA0 - 1e-4)) / 2e-4
    assert np.isclose(wb, fd, rtol=1e-5)


def test_dense_eig_adjt():
    # ME/test/runtests.jl:267-285 (rtol 1e-6)
    rng = np.random.default_rng(11)
    n = 40
    A0 = rng.standard_normal((n, n))
    A = (A0 + A0.T) / 2
    lam, V = np.linalg.eigh(A)
    al, v = lam[0], V[:, 0]
    B0 = rng.standard_normal((n, n))
    B = (B0 + B0.T) / 2
    l = O.eig_adjt(A, al, v.astype(complex), 0.0, (2 * B @ v).astype(complex))
    dA0 = rng.standard_normal((n, n))
    dA = (dA0 + dA0.T) / 2 * 1e-2

    def fv(t):
        _, VV = np.linalg.eigh(A + t * dA)
        vt = VV[:, 0] * np.sign(VV[:, 0] @ v)
        return vt @ B @ vt

    assert np.isclose(-np.real(np.vdot(l, dA @ v)), _fd5(fv, 0.0, 1e-3), rtol=1e-6)


def test_sliceinv_pullback_vs_fd():
    rng = np.random.default_rng(5)
    A = rng.standard_normal((3, 3, 4, 3))
    A = A + np.transpose(A, (1, 0, 2, 3)) + 6 * np.eye(3)[:, :, None, None]
    Y = O.sliceinv_3x3(A)
    Ybar = rng.standard_normal(Y.shape)
    Abar = O.sliceinv_3x3_pullback(Y, Ybar)
    dA = rng.standard_normal(A.shape)
    f = lambda t: np.sum(Ybar * O.sliceinv_3x3(A + t * dA))
    assert np.isclose(np.sum(Abar * dA), _fd5(f, 0.0, 1e-4), rtol=1e-8)


def _dispersive_case():
    from conftest import P_WG, gaussian_epsinv
    g = O.Grid(6.0, 4.0, 24, 16)
    ei0 = gaussian_epsinv(P_WG)
    eps0 = np.zeros_like(ei0)
    for a in range(3):
        eps0[a, a] = 1.0 / ei0[a, a]
    x = -3 + np.arange(24) * 0.25
    y = -2 + np.arange(16) * 0.25
    X, Y = np.meshgrid(x, y, indexing="ij")
    bump = np.exp(-(X ** 2 / 1.0 + Y ** 2 / 0.36))
    deps = np.zeros_like(eps0)
    for a in range(3):
        deps[a, a] = 0.8 * bump + 0.1
    deps[0, 1] = deps[1, 0] = 0.05 * bump
    return g, eps0, deps


def _epsinv_at(eps0, deps, w, w0):
    e = eps0 + deps * (w - w0)
    return np.moveaxis(np.linalg.inv(np.moveaxis(e, (0, 1), (-2, -1))), (-2, -1), (0, 1))


def test_group_index_matches_finite_difference():
    """n_g = dk/dω (lib/ModeAnalysis/src/group_index.jl:21-29) against central differences
    of solve_k with ε(ω) = ε₀ + (∂ε/∂ω)(ω − ω₀) (the reference's dk/dω check,
    ME/test/runtests.jl:94, rtol 1e-4; here it holds to ~1e-9)."""
    g, eps0, deps = _dispersive_case()
    w0, h = 1 / 1.55, 1e-4
    km, kv = O.solve_k(w0, _epsinv_at(eps0, deps, w0, w0), g, nev=2, k_tol=1e-13, eig_tol=1e-12)
    kp = O.solve_k(w0 + h, _epsinv_at(eps0, deps, w0 + h, w0), g, nev=2, k_tol=1e-13, eig_tol=1e-12)[0]
    kmn = O.solve_k(w0 - h, _epsinv_at(eps0, deps, w0 - h, w0), g, nev=2, k_tol=1e-13, eig_tol=1e-12)[0]
    for b in range(2):
        ng = O.group_index(km[b], kv[b], w0, _epsinv_at(eps0, deps, w0, w0), deps, g)
        fd = (kp[b] - kmn[b]) / (2 * h)
        assert abs(ng - fd) / fd < 1e-7
        # without dispersion the formula reduces to 2ω/(∂ω²/∂k)
        ng0 = O.group_index(km[b], kv[b], w0, _epsinv_at(eps0, deps, w0, w0), None, g)
        assert ng0 < ng


def _dispersive2_case():
    g, eps0, deps = _dispersive_case()
    dd = np.zeros_like(deps)
    for a in range(3):
        dd[a, a] = 0.3 * deps[a, a] - 0.05
    dd[0, 1] = dd[1, 0] = 0.02
    return g, eps0, deps, dd


def _epsinv_at2(eps0, deps, dd, w, w0):
    d = w - w0
    e = eps0 + deps * d + dd * d * d / 2
    return np.moveaxis(np.linalg.inv(np.moveaxis(e, (0, 1), (-2, -1))), (-2, -1), (0, 1))


def test_ng_gvd_matches_finite_difference():
    """GVD = ∂n_g/∂ω (ng_gvd, lib/ModeAnalysis/src/group_index.jl:112-168) against central
    differences of n_g(ω) from modes re-solved with ε(ω) = ε₀ + ∂ε δ + ∂²ε δ²/2; the
    difference shrinks 4× per halving of the step (truncation), ~1e-7 at h = 2.5e-4."""
    from oracle.analysis import ng_gvd
    g, eps0, deps, dd = _dispersive2_case()
    w0, h = 1 / 1.55, 2.5e-4
    km, kv = O.solve_k(w0, _epsinv_at2(eps0, deps, dd, w0, w0), g, nev=1, k_tol=1e-13, eig_tol=1e-12)
    ng, gvd = ng_gvd(w0, km[0], kv[0], _epsinv_at2(eps0, deps, dd, w0, w0), deps, dd, g)
    assert ng == pytest.approx(O.group_index(km[0], kv[0], w0, _epsinv_at2(eps0, deps, dd, w0, w0), deps, g),
                               rel=1e-13)
    ngs = []
    for w in (w0 + h, w0 - h):
        k2, v2 = O.solve_k(w, _epsinv_at2(eps0, deps, dd, w, w0), g, nev=1, k_tol=1e-13, eig_tol=1e-12)
        ngs.append(O.group_index(k2[0], v2[0], w, _epsinv_at2(eps0, deps, dd, w, w0), deps + dd * (w - w0), g))
    fd = (ngs[0] - ngs[1]) / (2 * h)
    assert gvd == pytest.approx(fd, rel=5e-7)


def test_golden_config1_reproduced_by_oracle():
    """The committed config-1 fixture (128² Si₃N₄ rectangle, 2 bands) is what the oracle
    computes now: k to 1e-12, n_g to 1e-10, field probes to 1e-8 (the fixture generator
    itself is ``tests/golden/make_golden.py``)."""
    import json

    from golden.make_golden import OMEGA, config_inputs, epsinv_checksum, field_probes
    gold = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "solve_k_configs.json")))["config1"]
    g, nev, ei = config_inputs("config1")
    assert np.allclose(epsinv_checksum(ei), gold["epsinv_checksum"], rtol=1e-12)
    og = O.Grid(g.Dx, g.Dy, g.Nx, g.Ny)
    km, kv = O.solve_k(OMEGA, ei, og, nev=nev, k_tol=1e-12, eig_tol=1e-11)
    assert np.allclose(km, gold["kmags"], rtol=1e-12, atol=0)
    pr = field_probes(2 * g.N)
    for b in range(nev):
        d = 2 * O.Operator(km[b], ei, og).HMkH(kv[b])
        assert abs(2 * OMEGA / d - gold["n_g"][b]) <= 1e-10 * gold["n_g"][b]
        ref = np.array([complex(*p) for p in gold["field_probes"][b]])
        assert np.max(np.abs(pr.conj() @ kv[b] - ref) / np.linalg.norm(pr, axis=1)) < 1e-8
