"""CPU restatement (FP64, NumPy) of the modal group index — test infrastructure only.

``group_index(k, evec, ω, ε⁻¹, ∂ε/∂ω, grid)`` follows
``lib/ModeAnalysis/src/group_index.jl:21-29``:

    n_g = (ω + HMH(evec, ε⁻¹·∂ε/∂ω·ε⁻¹)/2) / HMₖH(evec, ε⁻¹)

with HMH (``ME/src/maxwell.jl:288-290``) and HMₖH (``ME/src/maxwell.jl:267-269``) as in
``oracle.maxwell``; ``∂ε/∂ω = None`` is the non-dispersive case n_g = ω/HMₖH
(= 2ω/(∂ω²/∂k), ``ME/src/solve.jl:82``).  The formula is pinned here against its physics
(n_g = dk/dω by central differences of ``solve_k`` with ε(ω) = ε₀ + (∂ε/∂ω)(ω − ω₀), the
reference's own check at ``ME/test/runtests.jl:94``) in ``tests/test_oracle.py``."""

from __future__ import annotations

import numpy as np

from .maxwell import Grid, Operator


def tensor_product(a: np.ndarray, b: np.ndarray, c: np.ndarray) -> np.ndarray:
    """Per-pixel 3×3 product a·b·c of reference-indexed (3, 3, Nx, Ny) tensors
    (``_dot(ε⁻¹, ∂ε_∂ω, ε⁻¹)``)."""
    return np.einsum("ab...,bc...,cd...->ad...", a, b, c)


def group_index(k: float, evec: np.ndarray, omega: float, epsinv: np.ndarray, deps_domega, grid: Grid) -> float:
    hmkh = Operator(k, epsinv, grid).HMkH(evec)
    if deps_domega is None:
        return float(omega / hmkh)
    T = tensor_product(epsinv, deps_domega, epsinv)
    hmh = Operator(k, T, grid).HMH(evec)
    return float((omega + hmh / 2.0) / hmkh)


def _richardson(f, k: float, h: float):
    """df/dk by central differences with one Richardson step (error O(h⁴))."""
    d1 = (f(k + h) - f(k - h)) / (2 * h)
    d2 = (f(k + h / 2) - f(k - h / 2)) / h
    return (4 * d2 - d1) / 3


def _sym(t):
    return 0.5 * (t + np.swapaxes(t, 0, 1))


def sym_contract(a: np.ndarray, t: np.ndarray) -> float:
    """⟨a, t⟩ for a ε⁻¹-cotangent ``a`` whose off-diagonal entries hold the summed (i,j)+(j,i)
    sensitivity (the pull-back's convention) and a symmetric direction ``t``: the diagonal
    once, each off-diagonal pair once."""
    s = sum(float(np.sum(a[i, i] * t[i, i])) for i in range(3))
    for i, j in ((0, 1), (0, 2), (1, 2)):
        s += float(np.sum(a[i, j] * t[i, j]))
    return s


def ng_gvd(omega: float, k: float, evec: np.ndarray, epsinv: np.ndarray, deps_domega: np.ndarray,
           d2eps_domega2: np.ndarray, grid: Grid, rtol: float = 1e-14):
    """(n_g, GVD = ∂n_g/∂ω) of one converged mode, the quantities of ``ng_gvd``
    (``lib/ModeAnalysis/src/group_index.jl:112-168``).

    The reference differentiates n_g = (ω + A/2)/B, A = ⟨H|M̂[ε⁻¹∂εε⁻¹]|H⟩,
    B = HMₖH(H, ε⁻¹), by one adjoint solve.  Here the same total derivative is written as a
    chain rule around the ``solve_k`` pull-back: with T = ε⁻¹∂εε⁻¹ (dε⁻¹/dω = −T),
    T₂ = ε⁻¹∂²εε⁻¹ and T₃ = T∂εε⁻¹,

      k̄ = HMₖH(H, T)/B − (n_g/B)·∂B/∂k,   ēv = M̂[T]H/B − (n_g/B)·(∂M̂/∂k)H,
      (ω̄, ε̄⁻¹) = pull-back of solve_k at (k̄, ēv),
      GVD = 1/B + ω̄ − ⟨ε̄⁻¹, T⟩ − A₃/B + n_g·HMₖH(H, T)/B + A₂/(2B),

    where the explicit k-derivatives at fixed coefficients H (∂B/∂k and (∂M̂/∂k)H) are
    central differences with a Richardson step (error ~1e-12).  Pinned against
    central differences of n_g(ω) from re-solved modes in ``tests/test_oracle.py``."""
    from .adjoint import solve_k_pullback
    H = np.asarray(evec, dtype=np.complex128).reshape(-1)
    ei = np.asarray(epsinv, dtype=np.float64)
    d1 = np.asarray(deps_domega, dtype=np.float64)
    d2 = np.asarray(d2eps_domega2, dtype=np.float64)
    B = Operator(k, ei, grid).HMkH(H)
    T = _sym(tensor_product(ei, d1, ei))
    opT = Operator(k, T, grid)
    MT_H = opT.M(H)
    A = float(np.real(np.vdot(H, MT_H)))
    ng = (omega + A / 2.0) / B
    A2 = Operator(k, _sym(tensor_product(ei, d2, ei)), grid).HMH(H)
    A3 = Operator(k, _sym(tensor_product(T, d1, ei)), grid).HMH(H)
    BT = opT.HMkH(H)
    h = 1e-3 * k
    dB = _richardson(lambda kk: Operator(kk, ei, grid).HMkH(H), k, h)
    dMH = _richardson(lambda kk: Operator(kk, ei, grid).M(H), k, h)
    kbar = BT / B - ng / B * dB
    ebar = MT_H / B - (ng / B) * dMH
    wbar, eib = solve_k_pullback(omega, ei, grid, [k], [H], kbar=[kbar], evbar=[ebar], rtol=rtol)
    gvd = 1.0 / B + wbar - sym_contract(eib, T) - A3 / B + ng * BT / B + A2 / (2.0 * B)
    return float(ng), float(gvd)
