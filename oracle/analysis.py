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
