"""Post-processing of converged modes on the device: the modal group index.

``group_index(k, evec, ω, ε⁻¹, grid, ∂ε/∂ω)`` mirrors the reference's
``group_index(k, evec, ω, ε⁻¹, ∂ε_∂ω, grid)`` (``lib/ModeAnalysis/src/group_index.jl:21-29``):

    n_g = (ω + ⟨evec|M̂[ε⁻¹·∂ε/∂ω·ε⁻¹]|evec⟩/2) / ⟨evec|∂M̂/∂k|evec⟩

Both brackets run on the GPU through the fused operator passes (FP64): the HMₖH pass,
and M̂ applied with the pixelwise tensor ε⁻¹·∂ε/∂ω·ε⁻¹.  That tensor need not be positive
(∂ε/∂ω vanishes in air), while the library's cell upload requires a positive ε⁻¹, so the
apply uses T + c·I and removes c·⟨evec|M̂[I]|evec⟩ exactly (HMH is linear in the tensor).
Without dispersion (``deps_domega=None``) n_g = ω/HMₖH = 2ω/(∂ω²/∂k).

``ng_gvd(k, evec, ω, ε⁻¹, grid, ∂ε/∂ω, ∂²ε/∂ω²)`` adds the group-velocity dispersion
GVD = ∂n_g/∂ω (``ng_gvd``, ``lib/ModeAnalysis/src/group_index.jl:112-168``): the total
ω-derivative of n_g through the mode (k, H) and the material data, by one device adjoint
solve (the ``solve_k`` pull-back) — see :func:`ng_gvd`.
"""

from __future__ import annotations

import numpy as np

from .grid import Grid
from .ops import HMkH, apply_M


def _tensor_product(a, b, c):
    return np.einsum("ab...,bc...,cd...->ad...", a, b, c)


def _hmh(k, tensor, grid: Grid, H, device):
    out = apply_M(k, tensor, grid, H, precision="fp64", device=device)
    return float(np.real(np.vdot(H, out)))


def group_index(k: float, evec, omega: float, eps_inv, grid: Grid, deps_domega=None, device: int = 0) -> float:
    """Modal group index n_g = d|k|/dω of one converged mode (``evec`` of unit norm, as
    returned by ``solve_k``), optionally with the material dispersion ∂ε/∂ω given as a
    reference-indexed ``(3, 3, Nx, Ny)`` array."""
    H = np.asarray(evec, dtype=np.complex128).reshape(-1)
    hmkh = float(HMkH(k, eps_inv, grid, H, precision="fp64", device=device))
    if deps_domega is None:
        return float(omega / hmkh)
    ei = np.asarray(eps_inv, dtype=np.float64)
    T = _tensor_product(ei, np.asarray(deps_domega, dtype=np.float64), ei)
    T = 0.5 * (T + np.swapaxes(T, 0, 1))  # symmetric to rounding
    c = float(np.max(np.abs(T))) + 1.0
    eye = np.zeros_like(T)
    for a in range(3):
        eye[a, a] = 1.0
    hmh = _hmh(k, T + c * eye, grid, H, device) - c * _hmh(k, eye, grid, H, device)
    return float((omega + 0.5 * hmh) / hmkh)


def _shifted(tensor):
    """T + c·I with c making the diagonal positive, and c."""
    c = float(np.max(np.abs(tensor))) + 1.0
    out = tensor.copy()
    for a in range(3):
        out[a, a] += c
    return out, c


def _eye(grid: Grid):
    e = np.zeros((3, 3, grid.Nx, grid.Ny))
    for a in range(3):
        e[a, a] = 1.0
    return e


def _sym_contract(a, t) -> float:
    s = sum(float(np.sum(a[i, i] * t[i, i])) for i in range(3))
    for i, j in ((0, 1), (0, 2), (1, 2)):
        s += float(np.sum(a[i, j] * t[i, j]))
    return s


def _richardson(f, k: float, h: float):
    d1 = (f(k + h) - f(k - h)) / (2 * h)
    d2 = (f(k + h / 2) - f(k - h / 2)) / h
    return (4 * d2 - d1) / 3


def ng_gvd(k: float, evec, omega: float, eps_inv, grid: Grid, deps_domega, d2eps_domega2, solver=None,
           device: int = 0):
    """(n_g, GVD) of one converged mode of ``solve_k`` (unit ``evec``), with the smoothed
    material dispersion ∂ε/∂ω and ∂²ε/∂ω² as reference-indexed (3, 3, Nx, Ny) arrays.

    With T = ε⁻¹∂εε⁻¹ (so dε⁻¹/dω = −T), T₂ = ε⁻¹∂²εε⁻¹, T₃ = T∂εε⁻¹, A = ⟨H|M̂[T]|H⟩,
    B = HMₖH(H) and n_g = (ω + A/2)/B:

      k̄ = HMₖH(H; T)/B − (n_g/B)·∂B/∂k,   ēv = M̂[T]H/B − (n_g/B)·(∂M̂/∂k)H,
      (ω̄, ε̄⁻¹) = the device ``solve_k`` pull-back (one adjoint MINRES solve),
      GVD = 1/B + ω̄ − ⟨ε̄⁻¹, T⟩ − ⟨H|M̂[T₃]|H⟩/B + n_g·HMₖH(H; T)/B + ⟨H|M̂[T₂]|H⟩/(2B).

    Every operator product runs on the GPU in FP64 (M̂ and HMₖH with a pixel tensor use the
    T + c·I shift of :func:`group_index`); the explicit k-derivatives at fixed coefficients
    (∂B/∂k, (∂M̂/∂k)H) are central differences of device evaluations with a Richardson step
    (error ~1e-12)."""
    from .adjoint import pullback
    from .solver import B200Solver
    H = np.asarray(evec, dtype=np.complex128).reshape(-1)
    ei = np.asarray(eps_inv, dtype=np.float64)
    d1 = np.asarray(deps_domega, dtype=np.float64)
    d2 = np.asarray(d2eps_domega2, dtype=np.float64)
    eye = _eye(grid)

    def M_of(tensor):  # M̂[tensor]·H for a symmetric tensor of any sign
        ts, c = _shifted(tensor)
        return (apply_M(k, ts, grid, H, precision="fp64", device=device)
                - c * apply_M(k, eye, grid, H, precision="fp64", device=device))

    def hmkh_of(tensor):
        ts, c = _shifted(tensor)
        return (float(HMkH(k, ts, grid, H, precision="fp64", device=device))
                - c * float(HMkH(k, eye, grid, H, precision="fp64", device=device)))

    B = float(HMkH(k, ei, grid, H, precision="fp64", device=device))
    T = _tensor_product(ei, d1, ei)
    T = 0.5 * (T + np.swapaxes(T, 0, 1))
    MT_H = M_of(T)
    A = float(np.real(np.vdot(H, MT_H)))
    ng = (omega + A / 2.0) / B
    T2 = _tensor_product(ei, d2, ei)
    T3 = _tensor_product(T, d1, ei)
    A2 = float(np.real(np.vdot(H, M_of(0.5 * (T2 + np.swapaxes(T2, 0, 1))))))
    A3 = float(np.real(np.vdot(H, M_of(0.5 * (T3 + np.swapaxes(T3, 0, 1))))))
    BT = hmkh_of(T)
    h = 1e-3 * k
    dB = _richardson(lambda kk: float(HMkH(kk, ei, grid, H, precision="fp64", device=device)), k, h)
    dMH = _richardson(lambda kk: apply_M(kk, ei, grid, H, precision="fp64", device=device), k, h)
    kbar = BT / B - ng / B * dB
    ebar = MT_H / B - (ng / B) * dMH
    wbar, eib = pullback(omega, ei, grid, [k], [H], kbar=[kbar], evbar=[ebar],
                         solver=solver or B200Solver(device=device))
    gvd = 1.0 / B + wbar - _sym_contract(eib, T) - A3 / B + ng * BT / B + A2 / (2.0 * B)
    return float(ng), float(gvd)
