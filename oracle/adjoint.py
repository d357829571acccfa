"""Adjoint pull-back of ``solve_k`` (oracle; test infrastructure).

Restates ``ME/src/solve.jl:213-289`` (the generic ``rrule(solve_k)``), ``eig_adjt``
(``ME/src/grads/solve.jl:96-113``), the 2D ``ε⁻¹_bar`` (``ME/src/grads/solve.jl:490-515``),
``∇ₖmag_m_n`` (``ME/src/maxwell.jl:560-566``) and the ``sliceinv_3x3`` pull-back
(``ME/src/grads/linalg.jl:40-47``).  The adjoint linear system (the reference's
``my_linsolve``, ``ME/src/grads/solve.jl:56-66``: IterativeSolvers ``gmres`` with ``Pl = P̂``)
is solved to rounding here, by a different route on purpose: exactly through the dense
eigendecomposition of the deflated operator when the system is small, otherwise by MINRES
on the deflated system with a symmetric positive-definite preconditioner, and in both cases
the true residual is checked.  Every converged solver returns the same λ.
"""

from __future__ import annotations

import numpy as np
import scipy.sparse.linalg as spla

from .maxwell import Grid, Operator, bfft2, eid, fft2, kx_tc

DENSE_MAX = 4096


def _deflated_solve(apply_A, x: np.ndarray, b: np.ndarray, apply_P=None, rtol: float = 1e-13):
    """λ ⟂ x with (A)λ = b on x⊥, b ⟂ x, for Hermitian A (already shifted)."""
    n = b.shape[0]
    proj = lambda v: v - x * np.vdot(x, v)
    if n <= DENSE_MAX:
        Am = np.stack([apply_A(c) for c in np.eye(n, dtype=np.complex128)], axis=1)
        Am = 0.5 * (Am + Am.conj().T)
        Q = np.eye(n, dtype=np.complex128) - np.outer(x, x.conj())
        w, V = np.linalg.eigh(Q @ Am @ Q)
        c = V.conj().T @ b
        # the deflated direction x has eigenvalue 0 and carries no part of b
        keep = np.abs(c) > 0
        scale = np.max(np.abs(w))
        keep &= np.abs(w) > 1e-13 * scale
        lam = V[:, keep] @ (c[keep] / w[keep])
    else:
        Aop = spla.LinearOperator((n, n), matvec=lambda v: proj(apply_A(proj(v))), dtype=np.complex128)
        Mop = spla.LinearOperator((n, n), matvec=lambda v: proj(apply_P(proj(v))), dtype=np.complex128) \
            if apply_P else None
        lam, info = spla.minres(Aop, b, M=Mop, rtol=rtol, maxiter=50 * n)
    lam = proj(lam)
    r = np.linalg.norm(proj(apply_A(lam)) - b) / np.linalg.norm(b)
    if not r < 1e-9:
        raise RuntimeError(f"adjoint solve did not converge (relative residual {r:.2e})")
    return lam


def eig_adjt(A, alpha: float, x: np.ndarray, alpha_bar: float, x_bar, P=None,
             rtol: float = 1e-13) -> np.ndarray:
    """Adjoint vector λ = λₓ + ᾱ x, (A − αI) λₓ = x̄ − x⟨x, x̄⟩, λₓ ⟂ x.

    ``A`` is a dense matrix or a callable; ``P`` an optional symmetric positive-definite
    preconditioner callable (used by the iterative route only).
    """
    if x_bar is None or not np.any(x_bar):
        return np.zeros_like(x) if alpha_bar == 0 else alpha_bar * x
    apply = (lambda v: A @ v - alpha * v) if isinstance(A, np.ndarray) else (lambda v: A(v) - alpha * v)
    x = np.asarray(x, dtype=np.complex128)
    b = x_bar - x * np.vdot(x, x_bar)
    lx = _deflated_solve(apply, x, b, P, rtol=rtol)
    return lx + alpha_bar * x


def epsinv_bar(d: np.ndarray, ld: np.ndarray, grid: Grid) -> np.ndarray:
    """2D ``ε⁻¹_bar(d, λd)``: diagonal −Re(λd_a d̄_a); off-diagonal
    −Re(conj(λd_b) d_a + λd_a conj(d_b)) mirrored.  Inputs are ``(Ny, Nx, 3)`` fields;
    returns the reference-indexed ``(3, 3, Nx, Ny)`` array."""
    out = np.zeros((grid.Ny, grid.Nx, 3, 3))
    for a in range(3):
        out[..., a, a] = np.real(-ld[..., a] * np.conj(d[..., a]))
    for a, b in ((0, 1), (1, 2), (0, 2)):
        v = np.real(-np.conj(ld[..., b]) * d[..., a] - ld[..., a] * np.conj(d[..., b]))
        out[..., a, b] = v
        out[..., b, a] = v
    return np.transpose(out, (2, 3, 1, 0)).copy()


def grad_k_mag_m_n(magbar, mbar, nbar, mag, m, n) -> float:
    """``∇ₖmag_m_n`` with dk̂ = ẑ: k̄ from the sensitivities of (|k+G|, m̂, n̂)."""
    dk = np.array([0.0, 0.0, 1.0])
    kpg_over_mag = np.cross(m, n) / mag[..., None]
    kbar_mag = np.sum(magbar * (kpg_over_mag @ dk) * mag)
    q = np.cross(kpg_over_mag, np.broadcast_to(dk, kpg_over_mag.shape))
    kbar_m = -np.sum(mbar * np.cross(m, q))
    kbar_n = -np.sum(nbar * np.cross(n, q))
    return float(kbar_mag + kbar_m + kbar_n)


def solve_k_pullback(omega: float, epsinv, grid: Grid, kmags, evecs, kbar=None, evbar=None,
                     precond: str = "diag", rtol: float = 1e-14):
    """Pull (k̄, ē) back to (ω̄, ε̄⁻¹) for the modes ``(kmags, evecs)`` of ``solve_k``.

    ``kbar``/``evbar`` may be ``None`` (a zero cotangent) as a whole or per band.
    Returns ``(omega_bar, epsinv_bar)`` with ``epsinv_bar`` shaped ``(3, 3, Nx, Ny)``.
    """
    epsinv = np.asarray(epsinv, dtype=np.float64)
    nev = len(kmags)
    kbar = [None] * nev if kbar is None else list(kbar)
    evbar = [None] * nev if evbar is None else list(evbar)
    ei_bar = np.zeros_like(epsinv)
    omega_bar = 0.0
    Ninv = 1.0 / grid.N
    for j in range(nev):
        k, ev = float(kmags[j]), np.asarray(evecs[j], dtype=np.complex128)
        op = Operator(k, epsinv, grid)
        dw2dk = 2.0 * op.HMkH(ev)
        kb = 0.0 if kbar[j] is None else float(kbar[j])
        ebar = evbar[j]
        evg = ev.reshape(grid.Ny, grid.Nx, 2)
        if ebar is not None and np.any(ebar):
            P = (lambda v: op.P(v)) if precond == "mpb" else (
                (lambda v: op.P_diag(v)) if precond == "diag" else None)
            lam = eig_adjt(op.M, omega ** 2, ev, 0.0, np.asarray(ebar, dtype=np.complex128), P, rtol)
            lam = lam - np.vdot(ev, lam) * ev
            lg = lam.reshape(grid.Ny, grid.Nx, 2)
            d = fft2(kx_tc(evg * Ninv, op.mag, op.m, op.n))
            ld = fft2(kx_tc(lg, op.mag, op.m, op.n))
            ei_bar += epsinv_bar(d, ld, grid)
            ld = ld * Ninv
            le = bfft2(eid(op.E, ld, transpose=True))
            e = bfft2(eid(op.E, d, transpose=True))
            kxbar_m = np.real(le * np.conj(evg[..., 1:2]) + e * np.conj(lg[..., 1:2]))
            kxbar_n = -np.real(le * np.conj(evg[..., 0:1]) + e * np.conj(lg[..., 0:1]))
            magbar = np.sum(op.n * kxbar_n, axis=-1) + np.sum(op.m * kxbar_m, axis=-1)
            kbar_h = -grad_k_mag_m_n(magbar, kxbar_m * op.mag[..., None],
                                     kxbar_n * op.mag[..., None], op.mag, op.m, op.n)
        else:
            kbar_h = 0.0
        scale = (kb + kbar_h) / dw2dk
        lam2 = scale * evg
        d = fft2(kx_tc(evg * Ninv, op.mag, op.m, op.n))
        ld = fft2(kx_tc(lam2, op.mag, op.m, op.n))
        ei_bar += epsinv_bar(d, ld, grid)
        omega_bar += 2.0 * omega * scale
    return omega_bar, ei_bar


def sliceinv_3x3(A: np.ndarray) -> np.ndarray:
    """Per-pixel 3×3 inverse of a ``(3, 3, Nx, Ny)`` array (ε ⇄ ε⁻¹)."""
    M = np.transpose(A, (2, 3, 0, 1))
    return np.transpose(np.linalg.inv(M), (2, 3, 0, 1)).copy()


def sliceinv_3x3_pullback(Y: np.ndarray, Ybar: np.ndarray) -> np.ndarray:
    """Ā = −Yᵀ Ȳ Yᵀ per pixel, with Y = sliceinv_3x3(A) (``ME/src/grads/linalg.jl:40-47``)."""
    Yp = np.transpose(Y, (2, 3, 0, 1))
    Yb = np.transpose(Ybar, (2, 3, 0, 1))
    YT = np.swapaxes(Yp, -1, -2)
    return np.transpose(-(YT @ Yb @ YT), (2, 3, 0, 1)).copy()
