"""Single operator evaluations through the C ABI (``omb_apply``, ``omb_HMkH``,
``omb_efield``).  These mirror the reference's ``HelmholtzMap`` / ``HelmholtzPreconditioner``
application, ``HMₖH`` and ``E⃗`` (``lib/MaxwellEigenmodes/src/maxwell.jl``,
``src/fields.jl``) and are what the parity tests call."""

from __future__ import annotations

import ctypes

import numpy as np

from . import _lib
from .grid import Grid


def epsinv_host(epsinv, grid: Grid) -> np.ndarray:
    """Reference-indexed ``(3, 3, Nx, Ny)`` ε⁻¹ as the column-major Float64 memory the C ABI
    reads."""
    e = np.asarray(epsinv, dtype=np.float64)
    if e.shape != (3, 3, grid.Nx, grid.Ny):
        raise ValueError(f"epsinv must have shape (3, 3, {grid.Nx}, {grid.Ny}), got {e.shape}")
    return np.asfortranarray(e)


def block_host(H, n: int):
    """Complex block → (column-major complex128 array of shape (n, ncol), ncol, was_vector)."""
    H = np.asarray(H)
    vec = H.ndim == 1
    B = H.reshape(n, 1) if vec else H
    if B.shape[0] != n:
        raise ValueError(f"field length must be {n}, got {B.shape[0]}")
    return np.asfortranarray(B.astype(np.complex128, copy=False)), B.shape[1], vec


def _dptr(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def apply(op: str, k: float, epsinv, grid: Grid, H, precision: str = "fp64", device: int = 0):
    """``op`` ∈ {"M", "P", "P_diag"} applied to one field or a block of columns."""
    lib = _lib.load()
    ctx = _lib.context(device)
    e = epsinv_host(epsinv, grid)
    B, ncol, vec = block_host(H, 2 * grid.N)
    out = np.empty_like(B, order="F")
    _lib.check(lib.omb_apply(ctx.handle, _lib.OPS[op], _lib.PREC[precision], ctypes.byref(grid.c()),
                             float(k), _dptr(e), ncol, _dptr(B), _dptr(out)))
    return out[:, 0].copy() if vec else out


def apply_M(k, epsinv, grid, H, precision="fp64", device=0):
    return apply("M", k, epsinv, grid, H, precision, device)


def apply_P(k, epsinv, grid, H, precision="fp64", kind="mpb", device=0):
    return apply("P" if kind == "mpb" else "P_diag", k, epsinv, grid, H, precision, device)


def HMkH(k, epsinv, grid, H, precision="fp64", device=0):
    """⟨H|∂M̂/∂k|H⟩ per column (a float for a single vector)."""
    lib = _lib.load()
    ctx = _lib.context(device)
    e = epsinv_host(epsinv, grid)
    B, ncol, vec = block_host(H, 2 * grid.N)
    out = np.empty(ncol)
    _lib.check(lib.omb_HMkH(ctx.handle, _lib.PREC[precision], ctypes.byref(grid.c()), float(k),
                            _dptr(e), ncol, _dptr(B), _dptr(out)))
    return float(out[0]) if vec else out


def E_field(k, epsinv, grid, H, precision="fp64", device=0):
    """Un-normalised E = ε⁻¹·fft(kx_tc H) as a flat ``(3, Nx, Ny)`` column-major vector."""
    lib = _lib.load()
    ctx = _lib.context(device)
    e = epsinv_host(epsinv, grid)
    B, ncol, vec = block_host(H, 2 * grid.N)
    if ncol != 1:
        raise ValueError("E_field takes one column")
    out = np.empty(3 * grid.N, dtype=np.complex128)
    _lib.check(lib.omb_efield(ctx.handle, _lib.PREC[precision], ctypes.byref(grid.c()), float(k),
                              _dptr(e), _dptr(B), _dptr(out)))
    return out


def H_field(k, grid, H, device=0):
    """Real-space Cartesian H = fft(h1 m̂ + h2 n̂) per column (``omb_hfield``), shaped
    ``(ncol, 3·Nx·Ny)`` (each row a flat ``(3, Nx, Ny)`` column-major field), FP64."""
    lib = _lib.load()
    ctx = _lib.context(device)
    B, ncol, vec = block_host(H, 2 * grid.N)
    out = np.empty((ncol, 3 * grid.N), dtype=np.complex128)
    _lib.check(lib.omb_hfield(ctx.handle, ctypes.byref(grid.c()), float(k), int(ncol), _dptr(B), _dptr(out)))
    return out[0] if vec else out


def profile_apply(op: str, k, epsinv, grid: Grid, ncol: int, nbatch: int, reps: int = 20,
                  precision: str = "fp32", device: int = 0) -> float:
    """Mean device seconds of one application of ``op`` ("M" or "P") to ``ncol`` columns on
    each of ``nbatch`` device-resident copies of the cell (``omb_profile_apply``)."""
    lib = _lib.load()
    ctx = _lib.context(device)
    e = epsinv_host(epsinv, grid)
    out = np.zeros(1)
    _lib.check(lib.omb_profile_apply(ctx.handle, _lib.OPS[op], _lib.PREC[precision], ctypes.byref(grid.c()),
                                     float(k), _dptr(e), int(ncol), int(nbatch), int(reps), _dptr(out)))
    return float(out[0])


def gram_blocks(Z, AZ, precision: str = "fp32", device: int = 0):
    """(G, S) = (ZᴴZ, ZᴴAZ) from the eigensolver's streaming Gram kernel (``omb_gram_blocks``)
    for complex blocks Z, AZ of shape (n2, n)."""
    lib = _lib.load()
    ctx = _lib.context(device)
    Z = np.asfortranarray(np.asarray(Z, dtype=np.complex128))
    AZ = np.asfortranarray(np.asarray(AZ, dtype=np.complex128))
    n2, n = Z.shape
    G = np.zeros((n, n), dtype=np.complex128, order="F")
    S = np.zeros((n, n), dtype=np.complex128, order="F")
    _lib.check(lib.omb_gram_blocks(ctx.handle, _lib.PREC[precision], int(n2), int(n), _dptr(Z), _dptr(AZ),
                                   _dptr(G), _dptr(S)))
    return G, S


# ---- operator-tile autotuning -------------------------------------------------------------

def autotune(grid, ncol: int = 4, device: int = 0):
    """Tune the FP32 operator tiles of `grid` now (``omb_autotune``): returns
    ``(row_variant, col_variant, wave_variant, seconds[7][6][4])`` (-1 where a combination
    is not timed: the cluster applies' column and wave slots, or grids without them)."""
    lib = _lib.load()
    ctx = _lib.context(device)
    r, c, w = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    t = np.zeros(168)
    _lib.check(lib.omb_autotune(ctx.handle, ctypes.byref(grid.c()), int(ncol), ctypes.byref(r), ctypes.byref(c),
                                ctypes.byref(w), _dptr(t)))
    return r.value, c.value, w.value, t.reshape(7, 6, 4)


def tune_set(device_name: str, Nx: int, Ny: int, row: int, col: int, wave: int = 0) -> None:
    _lib.check(_lib.load().omb_tune_set(device_name.encode(), Nx, Ny, row, col, wave))


def tune_get(device_name: str, Nx: int, Ny: int):
    r, c, w = ctypes.c_int32(), ctypes.c_int32(), ctypes.c_int32()
    _lib.check(_lib.load().omb_tune_get(device_name.encode(), Nx, Ny, ctypes.byref(r), ctypes.byref(c),
                                        ctypes.byref(w)))
    return r.value, c.value, w.value


def tune_clear() -> None:
    _lib.check(_lib.load().omb_tune_clear())


def tune_save(path: str) -> None:
    _lib.check(_lib.load().omb_tune_save(path.encode()))


def tune_load(path: str) -> int:
    n = ctypes.c_int32()
    _lib.check(_lib.load().omb_tune_load(path.encode(), ctypes.byref(n)))
    return n.value
