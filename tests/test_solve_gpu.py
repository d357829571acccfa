"""Parity of the device eigensolves (solve_ω², solve_k) with the FP64 oracle, through the
C ABI, on the reference's own test fixture (``ME/test/runtests.jl:29-45``) and analytic
known answers.

Tolerances: eigenvalue / k relative error ≤ 1e-9 (the target after the FP64 polish),
residual ‖M̂h − ω²h‖ ≤ 1e-8 of the converged unit eigenvector (plus the |Δk| < k_tol
offset of the final Newton update), FP32-only runs at the reference's FP32 tolerance 1e-5
(``ME/test/runtests.jl:205-218``)."""

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


def _resid(k, ei, grid, h, w2):
    return np.linalg.norm(O.Operator(k, ei, grid).M(h) - w2 * h)


def _overlap(a, b):
    return abs(np.vdot(a, b)) / (np.linalg.norm(a) * np.linalg.norm(b))


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_solve_omega2_parity(omb, case, prec):
    grid, ei, _, _ = case
    g = omb.Grid(6.0, 4.0, 24, 16)
    k0 = O.k_guess(OMEGA0, ei)
    ref, refv, _ = O.solve_omega2(k0, ei, grid, nev=3, tol=1e-11)
    ev, evecs, info = omb.solve_omega2(k0, ei, g, omb.B200Solver(precision=prec), nev=3, return_info=True)
    assert np.all(info["status"] == 0)
    assert np.allclose(ev, ref, rtol=1e-9, atol=0)
    for a, v in zip(ev, evecs):
        assert np.isclose(np.linalg.norm(v), 1.0, rtol=1e-10)
        assert _resid(k0, ei, grid, v, a) < 1.5e-8


@pytest.mark.parametrize("prec,precond,newton", [
    ("mixed", "mpb", "inner"), ("fp64", "mpb", "inner"), ("mixed", "diag", "inner"),
    ("fp64", "mpb", "outer"), ("fp64", "diag", "outer"),
])
def test_solve_k_parity(omb, case, prec, precond, newton):
    grid, ei, km_ref, kv_ref = case
    g = omb.Grid(6.0, 4.0, 24, 16)
    solver = omb.B200Solver(precision=prec, preconditioner=precond, newton=newton)
    km, kv, info = omb.solve_k(OMEGA0, ei, g, solver, nev=2, return_info=True)
    assert np.all(info["status"] == 0), info
    assert np.allclose(km, km_ref, rtol=1e-9, atol=0), (km, km_ref)
    for k, h, href in zip(km, kv, kv_ref):
        assert np.isclose(np.linalg.norm(h), 1.0, rtol=1e-10)
        assert _resid(k, ei, grid, h, OMEGA0 ** 2) < 5e-8
        assert _overlap(h, href) > 1 - 1e-8
        E = O.E_field(k, h, ei, grid)
        e = E[np.argmax(np.abs(E))]
        assert abs(e.imag) <= 1e-9 * abs(e) and e.real > 0
    # n_g from the adjoint slope: ∂ω²/∂k = 2⟨h|∂M̂/∂k|h⟩
    for k, h, d in zip(km, kv, info["dw2dk"]):
        assert np.isclose(d, 2 * O.Operator(k, ei, grid).HMkH(h), rtol=1e-6)


def test_solve_k_fp32(omb, case):
    grid, ei, km_ref, _ = case
    g = omb.Grid(6.0, 4.0, 24, 16)
    km, kv = omb.solve_k(OMEGA0, ei, g, omb.B200Solver(precision="fp32"), nev=2)
    assert np.allclose(km, km_ref, rtol=1e-5)


def test_uniform_medium_known_answer(omb):
    g = omb.Grid(6.0, 4.0, 24, 16)
    eps = 2.5
    ei = np.zeros((3, 3, 24, 16))
    for a in range(3):
        ei[a, a] = 1 / eps
    km, _ = omb.solve_k(OMEGA0, ei, g, nev=2)
    assert np.allclose(km, OMEGA0 * np.sqrt(eps), rtol=1e-10)


def test_round_trip_and_bounds(omb, case):
    # ME/test/runtests.jl:76-82
    grid, ei, _, _ = case
    g = omb.Grid(6.0, 4.0, 24, 16)
    km, _ = omb.solve_k(OMEGA0, ei, g, nev=1)
    assert np.sqrt(P_WG[1]) < km[0] / OMEGA0 < np.sqrt(P_WG[0])
    ev, _ = omb.solve_omega2(km[0], ei, g, nev=1)
    assert np.isclose(ev[0], OMEGA0 ** 2, rtol=1e-9)


def test_batch_matches_single(omb, case):
    grid, ei, _, _ = case
    g = omb.Grid(6.0, 4.0, 24, 16)
    omegas = [1 / 1.45, 1 / 1.55, 1 / 1.65]
    batch = omb.solve_k_batch([{"omega": w, "eps_inv": ei, "grid": g, "nev": 2} for w in omegas])
    for w, (km, kv) in zip(omegas, batch):
        ref, _ = O.solve_k(w, ei, grid, nev=2, k_tol=1e-12, eig_tol=1e-11)
        assert np.allclose(km, ref, rtol=1e-9)


def test_warm_start_guess(omb, case):
    grid, ei, km_ref, kv_ref = case
    g = omb.Grid(6.0, 4.0, 24, 16)
    ret, info = omb.solve_k_batch([{"omega": OMEGA0, "eps_inv": ei, "grid": g, "nev": 2,
                                    "kguess": km_ref[0], "Hguess": kv_ref}], return_info=True)
    km = ret[0][0]
    assert np.allclose(km, km_ref, rtol=1e-9)
    _, info0 = omb.solve_k_batch([{"omega": OMEGA0, "eps_inv": ei, "grid": g, "nev": 2}],
                                 return_info=True)
    assert info[0]["iterations"].sum() < info0[0]["iterations"].sum()


@pytest.mark.parametrize("newton", ["inner", "outer"])
def test_sweep_warm_start(omb, case, newton):
    """A frequency sweep in one batch (OMB_WARM_SWEEP): the same k as independent solves
    (and the oracle), and the members started from the solved neighbour need fewer
    iterations than their cold solves."""
    grid, ei, _, _ = case
    g = omb.Grid(6.0, 4.0, 24, 16)
    omegas = [1 / 1.50, 1 / 1.53, 1 / 1.56, 1 / 1.59]
    probs = [{"omega": w, "eps_inv": ei, "grid": g, "nev": 2} for w in omegas]
    prec = "fp64" if newton == "outer" else "mixed"
    cold, info_c = omb.solve_k_batch(probs, omb.B200Solver(precision=prec, newton=newton), return_info=True)
    warm, info_w = omb.solve_k_batch(probs, omb.B200Solver(precision=prec, newton=newton, warm_start="sweep"),
                                     return_info=True)
    for w, (kc, _), (kw, vw), iw in zip(omegas, cold, warm, info_w):
        assert np.all(iw["status"] == 0)
        assert np.allclose(kw, kc, rtol=1e-9)
        ref, _ = O.solve_k(w, ei, grid, nev=2, k_tol=1e-12, eig_tol=1e-11)
        assert np.allclose(kw, ref, rtol=1e-9)
        for b in range(2):
            assert _resid(kw[b], ei, grid, vw[b], w * w) < 2e-8
    # the anchor is the ω nearest the mean (index 1 or 2); the other three start warm
    it_c = np.array([i["iterations"].sum() for i in info_c])
    it_w = np.array([i["iterations"].sum() for i in info_w])
    assert it_w.sum() < it_c.sum()


def test_cells_warm_start(omb):
    """A taper of cross-sections at one ω in one batch (OMB_WARM_CELLS, the batched form of
    eme(...; warmstart=true)): every cell matches its own oracle solve, and the cells started
    from the middle one need fewer iterations than their cold solves."""
    from conftest import gaussian_epsinv
    grid = O.Grid(6.0, 4.0, 24, 16)
    g = omb.Grid(6.0, 4.0, 24, 16)
    cells = [gaussian_epsinv((4.2, 2.1, 1.0 + 0.04 * c, 0.6)) for c in range(5)]
    probs = [{"omega": OMEGA0, "eps_inv": e, "grid": g, "nev": 2} for e in cells]
    cold, info_c = omb.solve_k_batch(probs, omb.B200Solver(), return_info=True)
    warm, info_w = omb.solve_k_batch(probs, omb.B200Solver(warm_start="cells"), return_info=True)
    for e, (kc, _), (kw, vw), iw in zip(cells, cold, warm, info_w):
        assert np.all(iw["status"] == 0)
        assert np.allclose(kw, kc, rtol=1e-9)
        ref, _ = O.solve_k(OMEGA0, e, grid, nev=2, k_tol=1e-12, eig_tol=1e-11)
        assert np.allclose(kw, ref, rtol=1e-9)
        for b in range(2):
            assert _resid(kw[b], e, grid, vw[b], OMEGA0 ** 2) < 2e-8
    it_c = np.array([i["iterations"].sum() for i in info_c])
    it_w = np.array([i["iterations"].sum() for i in info_w])
    assert it_w.sum() < it_c.sum()


def test_kguess_bands(omb, case):
    """Per-band Newton starts reach the same k."""
    grid, ei, km_ref, _ = case
    g = omb.Grid(6.0, 4.0, 24, 16)
    ret = omb.solve_k_batch([{"omega": OMEGA0, "eps_inv": ei, "grid": g, "nev": 2,
                              "kguess_bands": km_ref * 1.01}])
    assert np.allclose(ret[0][0], km_ref, rtol=1e-9)


def test_uneven_batch(omb):
    """One batch mixing grids, cells, frequencies and band counts (the shape of the
    uneven-grid sweep): every instance matches its own oracle solve."""
    specs = [  # (Nx, Ny, Dx, Dy, ω, nev, bump)
        (24, 16, 6.0, 4.0, 1 / 1.55, 2, P_WG),
        (32, 24, 6.0, 4.5, 1 / 1.45, 3, (4.6, 2.1, 1.1, 0.7)),
        (20, 20, 5.0, 5.0, 1 / 1.60, 1, (3.98, 2.09, 0.9, 0.9)),
        (24, 16, 6.0, 4.0, 1 / 1.50, 3, P_WG),
        (48, 32, 6.0, 4.0, 1 / 1.55, 2, P_WG),
    ]
    probs, refs = [], []
    for Nx, Ny, Dx, Dy, w, nev, p in specs:
        ei = gaussian_epsinv(p, Dx, Dy, Nx, Ny)
        probs.append({"omega": w, "eps_inv": ei, "grid": omb.Grid(Dx, Dy, Nx, Ny), "nev": nev})
        refs.append(O.solve_k(w, ei, O.Grid(Dx, Dy, Nx, Ny), nev=nev, k_tol=1e-12, eig_tol=1e-11)[0])
    for warm in ("none", "sweep"):
        out, info = omb.solve_k_batch(probs, omb.B200Solver(warm_start=warm), return_info=True)
        for (km, kv), i, ref, pr in zip(out, info, refs, probs):
            assert np.all(i["status"] == 0)
            assert np.allclose(km, ref, rtol=1e-9)
            assert len(kv) == pr["nev"] and all(v.shape == (2 * pr["grid"].N,) for v in kv)
