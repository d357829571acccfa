"""Block LOBPCG (oracle; test infrastructure).

Restated from the published method -- A. V. Knyazev, SIAM J. Sci. Comput. 23 (2001);
U. Hetmaniuk & R. Lehoucq, J. Comput. Phys. 218 (2006) (orthogonal basis, P built in
coefficient space); J. A. Duersch, M. Shao, C. Yang & M. Gu, SIAM J. Sci. Comput. 40
(2018) (Gram-based Rayleigh–Ritz, stable orthonormalisation) -- keeping the semantics of
the reference's vendored solver ``ME/src/solvers/dftk.jl:304-506``:

* ``tol`` is an absolute bound on the 2-norm of the residual ``A x − λ x`` of a unit
  vector (``dftk.jl:381-386, 396-409``);
* vectors lock in order, lowest first, and only from iteration ``miniter`` = 1 on;
* the preconditioner acts on the residual block (``dftk.jl:389-394``);
* the incoming block is the warm start and is orthonormalised first (``dftk.jl:317``).

The orthonormalisation is SVQB (Stathopoulos & Wu, SIAM J. Sci. Comput. 23 (2002)),
applied twice, dropping directions whose Gram eigenvalue falls below a relative floor.
"""

from __future__ import annotations

import numpy as np
import scipy.linalg as sla


def _svqb(W: np.ndarray, drop: float = 1e-14) -> np.ndarray:
    """Orthonormalise the columns of W (twice), dropping numerically dependent ones."""
    for _ in range(2):
        if W.shape[1] == 0:
            return W
        G = W.conj().T @ W
        G = 0.5 * (G + G.conj().T)
        dg = np.sqrt(np.maximum(np.real(np.diag(G)), np.finfo(float).tiny))
        Gs = G / np.outer(dg, dg)
        th, V = np.linalg.eigh(Gs)
        keep = th > drop * max(th.max(), 1.0)
        V = V[:, keep] / np.sqrt(th[keep])
        W = (W / dg) @ V
    return W


def _project_out(W: np.ndarray, Z: np.ndarray) -> np.ndarray:
    if Z is None or Z.shape[1] == 0:
        return W
    for _ in range(2):
        W = W - Z @ (Z.conj().T @ W)
    return W


def lobpcg(A, X0: np.ndarray, Prec=None, tol: float = 1e-8, maxiter: int = 300,
           miniter: int = 1):
    """Smallest eigenpairs of the Hermitian operator ``A`` (block callable).

    Returns ``(lam, X, info)`` with ``info = {"iterations", "n_matvec", "resid",
    "converged"}``.
    """
    n, M = X0.shape
    X = _svqb(np.array(X0, dtype=np.complex128))
    if X.shape[1] < M:  # degenerate warm start: refill with random directions
        rng = np.random.default_rng(12345)
        extra = rng.standard_normal((n, M - X.shape[1])) + 1j * rng.standard_normal((n, M - X.shape[1]))
        X = _svqb(np.concatenate([X, _project_out(extra, X)], axis=1))
    AX = A(X)
    n_matvec = M
    # initial Rayleigh–Ritz on X so the block starts as Ritz pairs
    S = X.conj().T @ AX
    lam, C = np.linalg.eigh(0.5 * (S + S.conj().T))
    X, AX = X @ C, AX @ C
    P = AP = None
    nlocked = 0
    resid = np.full(M, np.inf)
    it = 0
    converged = False
    while True:
        R = AX - X * lam[None, :]
        resid = np.linalg.norm(R, axis=0)
        prev = nlocked
        if it >= miniter:
            while nlocked < M and resid[nlocked] < tol:
                nlocked += 1
        if nlocked >= M:
            converged = True
            break
        if it >= maxiter:
            break
        if P is not None and nlocked > prev:
            P, AP = P[:, nlocked - prev:], AP[:, nlocked - prev:]
        a = slice(nlocked, M)
        ma = M - nlocked
        W = R[:, a] if Prec is None else Prec(R[:, a])
        Z = X if P is None else np.concatenate([X, P], axis=1)
        W = _svqb(_project_out(W, Z))
        AW = A(W) if W.shape[1] else W
        n_matvec += W.shape[1]
        blocks_Y = [X[:, a], W] + ([P] if P is not None else [])
        blocks_AY = [AX[:, a], AW] + ([AP] if P is not None else [])
        Y = np.concatenate(blocks_Y, axis=1)
        AY = np.concatenate(blocks_AY, axis=1)
        G = Y.conj().T @ Y
        S = Y.conj().T @ AY
        G = 0.5 * (G + G.conj().T)
        S = 0.5 * (S + S.conj().T)
        theta, Cfull = sla.eigh(S, G)
        C = Cfull[:, :ma]
        # P direction in coefficient space: (Ritz vector − old X), made G-orthogonal to
        # the new Ritz vectors and G-orthonormal (Hetmaniuk–Lehoucq)
        cP = C.copy()
        cP[:ma, :] -= np.eye(ma)
        cP = cP - C @ (C.conj().T @ (G @ cP))
        GP = cP.conj().T @ G @ cP
        GP = 0.5 * (GP + GP.conj().T)
        th, V = np.linalg.eigh(GP)
        keep = th > 1e-14 * max(th.max(), 1e-300)
        cP = cP @ (V[:, keep] / np.sqrt(th[keep])) if keep.any() else cP[:, :0]
        X[:, a] = Y @ C
        AX[:, a] = AY @ C
        lam[a] = theta[:ma]
        P, AP = (Y @ cP, AY @ cP) if cP.shape[1] else (None, None)
        it += 1
    return lam, X, {"iterations": it, "n_matvec": n_matvec, "resid": resid,
                    "converged": converged}
