"""3D waveguides periodic along ẑ (Bragg and photonic-crystal-defect guides) through the C ABI:
``omb_apply3`` / ``omb_HMkH3`` (the 3D M̂, P̂ and ⟨H|∂M̂/∂k|H⟩), ``omb_solve_k_periodic`` and
``omb_pullback_periodic``.

Mirrors the reference's ``solve_k_periodic(ω, ε⁻¹, Λ, grid, solver; nev)`` and its reverse-mode
rule (``lib/MaxwellEigenmodes/src/grads/period.jl:108-112, 136-200``): the solve runs on the
grid whose z-extent is the period Λ (``_grid_with_period``, ``period.jl:125-128``), with ε⁻¹
held fixed in index space, and the pull-back returns (ω̄, ε̄⁻¹, Λ̄).

Layouts are the reference's column-major ones: a field is a flat complex vector ordered
``(2, Nx, Ny, Nz)``; ε⁻¹ is ``(3, 3, Nx, Ny, Nz)``.
"""

from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import _lib
from .ops import block_host
from .solver import B200Solver


@dataclasses.dataclass(frozen=True)
class Grid3:
    """Dx × Dy × Dz μm cell on Nx × Ny × Nz pixels (the reference's ``Grid{3}``); Dz is the period."""

    Dx: float
    Dy: float
    Dz: float
    Nx: int
    Ny: int
    Nz: int

    @property
    def N(self) -> int:
        return self.Nx * self.Ny * self.Nz

    def with_period(self, L: float) -> "Grid3":
        """The same cell with z-extent ``L`` (``_grid_with_period``)."""
        return Grid3(self.Dx, self.Dy, float(L), self.Nx, self.Ny, self.Nz)

    def c(self) -> "c_grid3":
        return c_grid3(int(self.Nx), int(self.Ny), int(self.Nz), float(self.Dx), float(self.Dy), float(self.Dz))


class c_grid3(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int32), ("Ny", ctypes.c_int32), ("Nz", ctypes.c_int32),
                ("Dx", ctypes.c_double), ("Dy", ctypes.c_double), ("Dz", ctypes.c_double)]


def _declare(lib):
    vp, dp, ip, d = ctypes.c_void_p, _lib._dp, _lib._ip, ctypes.c_double
    gp = ctypes.POINTER(c_grid3)
    op = ctypes.POINTER(_lib.c_options)
    sig = {
        "omb_apply3": [vp, ctypes.c_int, ctypes.c_int, gp, d, dp, ctypes.c_int, dp, dp],
        "omb_HMkH3": [vp, ctypes.c_int, gp, d, dp, ctypes.c_int, dp, dp],
        "omb_solve_k_periodic": [vp, gp, d, dp, ctypes.c_int, d, op, dp, dp, dp, dp, ip, ip],
        "omb_pullback_periodic": [vp, gp, d, dp, ctypes.c_int, dp, dp, dp, dp, op, dp, dp, dp, ip],
    }
    for name, args in sig.items():
        f = getattr(lib, name)
        f.restype = ctypes.c_int
        f.argtypes = args


_lib.EXPORTS = _lib.EXPORTS + ("omb_apply3", "omb_HMkH3", "omb_solve_k_periodic", "omb_pullback_periodic")
_lib._DECLARERS.append(_declare)
if _lib._lib is not None:  # the library was loaded before this module was imported
    _declare(_lib._lib)

_NULL_D = ctypes.cast(None, _lib._dp)
_NULL_I = ctypes.cast(None, _lib._ip)


def epsinv_host3(epsinv, grid: Grid3) -> np.ndarray:
    """``(3, 3, Nx, Ny, Nz)`` ε⁻¹ as the column-major Float64 memory the C ABI reads."""
    e = np.asarray(epsinv, dtype=np.float64)
    if e.shape != (3, 3, grid.Nx, grid.Ny, grid.Nz):
        raise ValueError(f"epsinv must have shape (3, 3, {grid.Nx}, {grid.Ny}, {grid.Nz}), got {e.shape}")
    return np.asfortranarray(e)


def apply3(op: str, k: float, epsinv, grid: Grid3, H, precision: str = "fp64", device: int = 0):
    """``op`` ∈ {"M", "P"} on a z-periodic cell, one field or a block of columns."""
    lib = _lib.load()
    ctx = _lib.context(device)
    e = epsinv_host3(epsinv, grid)
    B, ncol, vec = block_host(H, 2 * grid.N)
    out = np.empty_like(B, order="F")
    _lib.check(lib.omb_apply3(ctx.handle, _lib.OPS[op], _lib.PREC[precision], ctypes.byref(grid.c()), float(k),
                              _lib.dptr(e), ncol, _lib.dptr(B), _lib.dptr(out)))
    return out[:, 0].copy() if vec else out


def HMkH3(k: float, epsinv, grid: Grid3, H, precision: str = "fp64", device: int = 0):
    """⟨H|∂M̂/∂k|H⟩ per column on a z-periodic cell (a float for a single vector)."""
    lib = _lib.load()
    ctx = _lib.context(device)
    e = epsinv_host3(epsinv, grid)
    B, ncol, vec = block_host(H, 2 * grid.N)
    out = np.empty(ncol)
    _lib.check(lib.omb_HMkH3(ctx.handle, _lib.PREC[precision], ctypes.byref(grid.c()), float(k), _lib.dptr(e),
                             ncol, _lib.dptr(B), _lib.dptr(out)))
    return float(out[0]) if vec else out


def solve_k_periodic(omega: float, eps_inv, L: float, grid: Grid3, solver: B200Solver | None = None, nev: int = 1,
                     k_tol=1e-8, eig_tol=1e-8, max_eigsolves=60, maxiter=None, kguess=None, canonicalize=True,
                     return_info=False):
    """k and phase-canonical unit modes of the lowest ``nev`` Bloch bands at ω and period ``L``
    (``solve_k_periodic``, ``period.jl:108-112``).  Uses the inner Newton iteration."""
    solver = solver or B200Solver()
    if solver.newton != "inner":
        raise ValueError("z-periodic cells use the inner Newton iteration (newton='inner')")
    lib = _lib.load()
    ctx = _lib.context(solver.device)
    g = grid.with_period(L)
    e = epsinv_host3(eps_inv, g)
    n2 = 2 * g.N
    kmags = np.zeros(nev)
    evecs = np.zeros((n2, nev), dtype=np.complex128, order="F")
    resid = np.zeros(nev)
    dw2dk = np.zeros(nev)
    status = np.zeros(nev, dtype=np.int32)
    iters = np.zeros(nev, dtype=np.int32)
    opt = solver.options(k_tol, eig_tol, max_eigsolves, maxiter, canonicalize)
    rc = lib.omb_solve_k_periodic(ctx.handle, ctypes.byref(g.c()), float(omega), _lib.dptr(e), int(nev),
                                  float(kguess) if kguess else 0.0, ctypes.byref(opt), _lib.dptr(kmags),
                                  _lib.dptr(evecs), _lib.dptr(resid), _lib.dptr(dw2dk),
                                  status.ctypes.data_as(_lib._ip), iters.ctypes.data_as(_lib._ip))
    if rc != _lib.OMB_OK and not (return_info and rc == 3):
        _lib.check(rc)
    out = (kmags, [evecs[:, j].copy() for j in range(nev)])
    if return_info:
        return out + ({"residuals": resid, "dw2dk": dw2dk, "status": status, "iterations": iters},)
    return out


def solve_k_periodic_pullback(omega: float, eps_inv, L: float, grid: Grid3, kmags, evecs, kbar=None, evbar=None,
                              solver: B200Solver | None = None, return_info=False):
    """(ω̄, ε̄⁻¹, Λ̄) for cotangents ``kbar`` (nev values or None) and ``evbar`` (nev vectors,
    None entries or None for zero) of ``solve_k_periodic``'s outputs (``_solve_k_period_grads``,
    ``period.jl:136-200``)."""
    solver = solver or B200Solver()
    lib = _lib.load()
    ctx = _lib.context(solver.device)
    g = grid.with_period(L)
    e = epsinv_host3(eps_inv, g)
    nev = len(kmags)
    n2 = 2 * g.N
    km = np.ascontiguousarray(np.asarray(kmags, dtype=np.float64))
    V = np.asfortranarray(np.stack([np.asarray(v, dtype=np.complex128) for v in evecs], axis=1))
    kb = None if kbar is None else np.ascontiguousarray(
        np.array([0.0 if x is None else float(x) for x in kbar], dtype=np.float64))
    EB = None
    if evbar is not None:
        EB = np.zeros((n2, nev), dtype=np.complex128, order="F")
        for j, x in enumerate(evbar):
            if x is not None:
                EB[:, j] = np.asarray(x, dtype=np.complex128)
    wbar, Lbar = np.zeros(1), np.zeros(1)
    eib = np.zeros((3, 3, g.Nx, g.Ny, g.Nz), order="F")
    iters = np.zeros(nev, dtype=np.int32)
    opt = solver.options()
    _lib.check(lib.omb_pullback_periodic(ctx.handle, ctypes.byref(g.c()), float(omega), _lib.dptr(e), nev,
                                         _lib.dptr(km), _lib.dptr(V), _lib.dptr(kb) if kb is not None else _NULL_D,
                                         _lib.dptr(EB) if EB is not None else _NULL_D, ctypes.byref(opt),
                                         _lib.dptr(wbar), _lib.dptr(eib), _lib.dptr(Lbar),
                                         iters.ctypes.data_as(_lib._ip)))
    out = (float(wbar[0]), np.ascontiguousarray(eib), float(Lbar[0]))
    if return_info:
        out = out + ({"iterations": iters},)
    return out


def solve_k_periodic_rrule(omega: float, eps_inv, L: float, grid: Grid3, solver: B200Solver | None = None,
                           nev: int = 1, **kw):
    """``((kmags, evecs), pullback)``; ``pullback((kbar, evbar)) -> (omega_bar, epsinv_bar, L_bar)``
    (the reference's ``rrule(solve_k_periodic, ω, ε⁻¹, Λ, grid, solver)``)."""
    kmags, evecs = solve_k_periodic(omega, eps_inv, L, grid, solver, nev=nev, **kw)

    def _pullback(cot):
        kbar, evbar = cot
        return solve_k_periodic_pullback(omega, eps_inv, L, grid, kmags, evecs, kbar, evbar, solver)

    return (kmags, evecs), _pullback
