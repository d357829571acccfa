"""``solve_ω²`` and ``solve_k`` (oracle; test infrastructure).

``solve_omega2`` follows ``ME/src/solve.jl:38-63`` with the LOBPCG backend
(``ME/src/solvers/dftk.jl:32-37``).  ``solve_k`` follows ``ME/src/solve.jl:104-115,
182-210``: bands are solved one after another, each by a Newton iteration on
Δω²(k) = ω²_band(k) − ω² with slope ∂ω²/∂k = 2⟨H|∂M̂/∂k|H⟩; each Newton step is one
block eigensolve warm-started from the previous one, band b+1 starts from band b's final
k, and the loop stops once |Δk| < k_tol (the explicit loop of
``ME/src/solvers/gpu.jl:222-237``; the returned k is the one after the last update).
Eigenvectors are phase-canonicalised (``ME/src/fields.jl:258-260``).
"""

from __future__ import annotations

import numpy as np

from .lobpcg import lobpcg
from .maxwell import Grid, Operator, canonicalize_phase, k_guess


def random_block(n: int, m: int, seed: int = 0) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.standard_normal((n, m)) + 1j * rng.standard_normal((n, m))


def _apply_Hguess(X: np.ndarray, Hguess) -> np.ndarray:
    """``_apply_Hguess!`` (``ME/src/solve.jl:201-210``): copy matching-length columns."""
    if Hguess is None:
        return X
    cols = [Hguess] if np.ndim(Hguess) == 1 else (
        list(np.asarray(Hguess).T) if isinstance(Hguess, np.ndarray) else list(Hguess))
    for j, h in enumerate(cols):
        if j >= X.shape[1]:
            break
        h = np.asarray(h)
        if h.shape[0] == X.shape[0]:
            X[:, j] = h
    return X


def solve_omega2(k: float, epsinv, grid: Grid, nev: int = 1, tol: float = 1e-8,
                 maxiter: int = 300, X0=None, seed: int = 0, precond: str = "mpb"):
    """Lowest ``nev`` eigenpairs (ω², H) of M̂(k).  Returns ``(evals, evecs, info)``."""
    op = Operator(k, epsinv, grid)
    X = random_block(op.size, nev, seed) if X0 is None else np.array(X0, dtype=np.complex128)
    prec = (lambda R: op.P_block(R, precond)) if precond else None
    lam, X, info = lobpcg(op.M_block, X, prec, tol=tol, maxiter=maxiter)
    return lam.copy(), [X[:, j].copy() for j in range(nev)], info


def solve_k(omega: float, epsinv, grid: Grid, nev: int = 1, max_eigsolves: int = 60,
            maxiter: int = 300, k_tol: float = 1e-8, eig_tol: float = 1e-8, kguess=None,
            Hguess=None, seed: int = 0, precond: str = "mpb", canonicalize: bool = True,
            return_info: bool = False):
    """Propagation constants and modes of the lowest ``nev`` bands at frequency ω.

    Returns ``(kmags, evecs)`` (plus per-band info when ``return_info``).
    """
    epsinv = np.asarray(epsinv, dtype=np.float64)
    k = float(kguess) if kguess is not None else k_guess(omega, epsinv)
    op = Operator(k, epsinv, grid)
    X = _apply_Hguess(random_block(op.size, nev, seed), Hguess)
    prec = (lambda R: op.P_block(R, precond)) if precond else None
    kmags, evecs, infos = [], [], []
    for band in range(nev):
        steps, iters = 0, 0
        ev = None
        for _ in range(max_eigsolves):
            op.set_k(k)
            lam, X, info = lobpcg(op.M_block, X, prec, tol=eig_tol, maxiter=maxiter)
            steps += 1
            iters += info["iterations"]
            ev = X[:, band].copy()
            dw2 = lam[band] - omega ** 2
            dw2dk = 2.0 * op.HMkH(ev)
            dk = dw2 / dw2dk
            k -= dk
            if abs(dk) < k_tol:
                break
        kmags.append(k)
        evecs.append(canonicalize_phase(ev, k, epsinv, grid) if canonicalize else ev)
        infos.append({"newton_steps": steps, "lobpcg_iterations": iters,
                      "resid": float(info["resid"][band])})
    if return_info:
        return np.array(kmags), evecs, infos
    return np.array(kmags), evecs
