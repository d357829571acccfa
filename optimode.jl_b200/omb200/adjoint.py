"""Adjoint pull-back of ``solve_k`` through the C ABI (``omb_pullback``), mirroring the
reference's ``rrule(solve_k, ω, ε⁻¹, grid, solver)`` (``lib/MaxwellEigenmodes/src/solve.jl:213-289``):
``solve_k_rrule`` returns ``((kmags, evecs), pullback)`` and ``pullback((k̄, ē))`` returns
``(ω̄, ε̄⁻¹)``."""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .grid import Grid
from .ops import epsinv_host
from .solver import B200Solver, solve_k


def pullback(omega: float, eps_inv, grid: Grid, kmags, evecs, kbar=None, evbar=None,
             solver: B200Solver | None = None, want_eps_bar=False, return_info=False):
    """(ω̄, ε̄⁻¹[, ε̄]) for cotangents ``kbar`` (nev values or None) and ``evbar`` (nev vectors,
    None entries or None for zero) of the outputs ``(kmags, evecs)`` of ``solve_k``."""
    solver = solver or B200Solver()
    lib = _lib.load()
    ctx = _lib.context(solver.device)
    e = epsinv_host(eps_inv, grid)
    nev = len(kmags)
    n2 = 2 * grid.N
    km = np.ascontiguousarray(np.asarray(kmags, dtype=np.float64))
    V = np.asfortranarray(np.stack([np.asarray(v, dtype=np.complex128) for v in evecs], axis=1))
    kb = None if kbar is None else np.ascontiguousarray(
        np.array([0.0 if x is None else float(x) for x in kbar], dtype=np.float64))
    if evbar is None:
        EB = None
    else:
        EB = np.zeros((n2, nev), dtype=np.complex128, order="F")
        for j, x in enumerate(evbar):
            if x is not None:
                EB[:, j] = np.asarray(x, dtype=np.complex128)
    wbar = np.zeros(1)
    eib = np.zeros((3, 3, grid.Nx, grid.Ny), order="F")
    ebar = np.zeros((3, 3, grid.Nx, grid.Ny), order="F") if want_eps_bar else None
    iters = np.zeros(nev, dtype=np.int32)
    opt = solver.options()
    null = ctypes.cast(None, _lib._dp)
    _lib.check(lib.omb_pullback(ctx.handle, ctypes.byref(grid.c()), float(omega), _lib.dptr(e), nev,
                                _lib.dptr(km), _lib.dptr(V), _lib.dptr(kb) if kb is not None else null,
                                _lib.dptr(EB) if EB is not None else null, ctypes.byref(opt),
                                _lib.dptr(wbar), _lib.dptr(eib), _lib.dptr(ebar) if ebar is not None else null,
                                iters.ctypes.data_as(_lib._ip)))
    out = (float(wbar[0]), np.ascontiguousarray(eib))
    if want_eps_bar:
        out = out + (np.ascontiguousarray(ebar),)
    if return_info:
        out = out + ({"iterations": iters},)
    return out


def solve_k_rrule(omega: float, eps_inv, grid: Grid, solver: B200Solver | None = None, nev: int = 1, **kw):
    """``((kmags, evecs), pullback)``; ``pullback((kbar, evbar)) -> (omega_bar, epsinv_bar)``."""
    kmags, evecs = solve_k(omega, eps_inv, grid, solver, nev=nev, **kw)

    def _pullback(cot):
        kbar, evbar = cot
        return pullback(omega, eps_inv, grid, kmags, evecs, kbar, evbar, solver)

    return (kmags, evecs), _pullback
