"""Post-processing of converged modes on the device: the modal group index.

``group_index(k, evec, ω, ε⁻¹, grid, ∂ε/∂ω)`` mirrors the reference's
``group_index(k, evec, ω, ε⁻¹, ∂ε_∂ω, grid)`` (``lib/ModeAnalysis/src/group_index.jl:21-29``):

    n_g = (ω + ⟨evec|M̂[ε⁻¹·∂ε/∂ω·ε⁻¹]|evec⟩/2) / ⟨evec|∂M̂/∂k|evec⟩

Both brackets run on the GPU through the fused operator passes (FP64): the HMₖH pass,
and M̂ applied with the pixelwise tensor ε⁻¹·∂ε/∂ω·ε⁻¹.  That tensor need not be positive
(∂ε/∂ω vanishes in air), while the library's cell upload requires a positive ε⁻¹, so the
apply uses T + c·I and removes c·⟨evec|M̂[I]|evec⟩ exactly (HMH is linear in the tensor).
Without dispersion (``deps_domega=None``) n_g = ω/HMₖH = 2ω/(∂ω²/∂k).
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
