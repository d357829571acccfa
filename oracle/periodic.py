"""3D z-periodic waveguides (oracle; test infrastructure).

Restates, in FP64 NumPy, the reference's periodic-along-ẑ solve and its period adjoint
(``ME/src/grads/period.jl``): ``solve_k_periodic`` (``:108-112``, ``solve_k`` on the grid
whose z-extent is the period Λ), ``gz_field`` / ``period_weight`` (``:36-58``),
``HMₖH_weighted`` (``:69-74``), ``_wbar_z`` (``:113-117``) and the pull-back
``_solve_k_period_grads`` (``:136-200``), with the 3D operator of ``ME/src/maxwell.jl``
(``kx_tc``/``kx_ct`` on (3, Nx, Ny, Nz) fields, ``_M!`` with 3D FFTs, ``mag_mn`` with
w = k ẑ − G, G = (gx, gy, gz) in cycles/μm).

Arrays follow the reference's column-major layout: a field H is a flat vector ordered as
``(2, Nx, Ny, Nz)``, ε⁻¹ is ``(3, 3, Nx, Ny, Nz)``; internally fields are ``(Nz, Ny, Nx, c)``.
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np
import scipy.fft as sfft

from . import maxwell as _mx
from .adjoint import eig_adjt
from .lobpcg import lobpcg
from .solve import _apply_Hguess, random_block


@dataclass(frozen=True)
class Grid3:
    """Dx × Dy × Dz μm cell on Nx × Ny × Nz pixels (``Grid{3}``); Dz is the period Λ."""
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
        """``_grid_with_period`` (``period.jl:125-128``)."""
        return Grid3(self.Dx, self.Dy, float(L), self.Nx, self.Ny, self.Nz)


def _freq(n: int, d: float) -> np.ndarray:
    i = np.arange(n)
    return np.where(i < (n + 1) // 2, i, i - n) / d


def g_vectors(grid: Grid3):
    return _freq(grid.Nx, grid.Dx), _freq(grid.Ny, grid.Dy), _freq(grid.Nz, grid.Dz)


def mag_mn(k: float, grid: Grid3):
    """(mag, m̂, n̂) per plane wave, arrays (Nz, Ny, Nx[, 3]); w = k ẑ − G."""
    gx, gy, gz = g_vectors(grid)
    GZ, GY, GX = np.meshgrid(gz, gy, gx, indexing="ij")
    w = np.stack([-GX, -GY, float(k) - GZ], axis=-1)
    mag = np.sqrt(np.sum(w * w, axis=-1))
    zxw = np.stack([GY, -GX, np.zeros_like(GX)], axis=-1)  # ẑ × w = (gy, −gx, 0)
    perp = np.sqrt(zxw[..., 0] ** 2 + zxw[..., 1] ** 2)
    with np.errstate(invalid="ignore", divide="ignore"):
        n = np.where((perp > 0)[..., None], zxw / perp[..., None], np.array([0.0, 1.0, 0.0]))
    m = np.cross(n, w)
    m = m / np.sqrt(np.sum(m * m, axis=-1))[..., None]
    return mag, m, n


def gz_field(grid: Grid3) -> np.ndarray:
    """g_z = m/Λ per plane wave, (Nz, Ny, Nx) (``gz_field``, ``period.jl:48-58``)."""
    gz = _freq(grid.Nz, grid.Dz)
    return np.broadcast_to(gz[:, None, None], (grid.Nz, grid.Ny, grid.Nx)).copy()


def period_weight(grid: Grid3) -> np.ndarray:
    """g_z/Λ (``period_weight``, ``period.jl:36-39``)."""
    return gz_field(grid) / grid.Dz


def fft3(a):
    return sfft.fftn(a, axes=(0, 1, 2), workers=_mx.FFT_WORKERS)


def bfft3(a):
    return sfft.ifftn(a, axes=(0, 1, 2), norm="forward", workers=_mx.FFT_WORKERS)


def _field(v, grid: Grid3, c: int):
    return np.asarray(v).reshape(grid.Nz, grid.Ny, grid.Nx, c)


def _epsinv_internal(epsinv):
    e = np.asarray(epsinv, dtype=np.float64)
    assert e.ndim == 5 and e.shape[:2] == (3, 3)
    return np.ascontiguousarray(np.transpose(e, (4, 3, 2, 0, 1)))  # (Nz, Ny, Nx, a, b)


def kx_tc(H, mag, m, n):
    return (H[..., 0:1] * n - H[..., 1:2] * m) * (-mag)[..., None]


def kx_ct(e, mag, m, n, scale):
    s = mag * scale
    return np.stack([-np.sum(e * n, axis=-1) * s, np.sum(e * m, axis=-1) * s], axis=-1)


def zx_tc(H, m, n):
    d1 = -(H[..., 0] * m[..., 1] + H[..., 1] * n[..., 1])
    d2 = H[..., 0] * m[..., 0] + H[..., 1] * n[..., 0]
    return np.stack([d1, d2, np.zeros_like(d1)], axis=-1)


class Operator3:
    """M̂(k), P̂(k) and HMₖH on a z-periodic cell (the 3D forms of ``ME/src/maxwell.jl``)."""

    def __init__(self, k: float, epsinv, grid: Grid3):
        self.grid = grid
        self.E = _epsinv_internal(epsinv)
        self.eps_ave = 3.0 / (self.E[..., 0, 0] + self.E[..., 1, 1] + self.E[..., 2, 2])
        self.set_k(k)

    def set_k(self, k: float) -> None:
        self.k = float(k)
        self.mag, self.m, self.n = mag_mn(self.k, self.grid)

    @property
    def size(self) -> int:
        return 2 * self.grid.N

    def _eid(self, d, transpose=True):
        sub = "zyxlh,zyxl->zyxh" if transpose else "zyxab,zyxb->zyxa"
        return np.einsum(sub, self.E, d)

    def M(self, Hv):
        H = _field(Hv, self.grid, 2)
        d = fft3(kx_tc(H, self.mag, self.m, self.n))
        e = bfft3(self._eid(d))
        return kx_ct(e, self.mag, self.m, self.n, 1.0 / self.grid.N).reshape(-1)

    def P(self, Hv):
        """MPB-style preconditioner (``_P!``, ``ME/src/maxwell.jl:430-469``) on 3D fields:
        e = (H₁n − H₂m)/mag → bfft → ε_ave·e → fft → H₁ = (d·n)/(mag N), H₂ = −(d·m)/(mag N)."""
        H = _field(Hv, self.grid, 2)
        e = (H[..., 0:1] * self.n - H[..., 1:2] * self.m) / self.mag[..., None]
        d = fft3(bfft3(e) * self.eps_ave[..., None])
        s = 1.0 / (self.mag * self.grid.N)
        return np.stack([np.sum(d * self.n, axis=-1) * s, -np.sum(d * self.m, axis=-1) * s], axis=-1).reshape(-1)

    def P_diag(self, Hv):
        H = _field(Hv, self.grid, 2)
        scale = float(np.mean(self.eps_ave)) / self.mag ** 2
        return (H * scale[..., None]).reshape(-1)

    def M_block(self, X):
        return np.stack([self.M(X[:, j]) for j in range(X.shape[1])], axis=1)

    def P_block(self, X, kind="diag"):
        return np.stack([self.P_diag(X[:, j]) for j in range(X.shape[1])], axis=1)

    def HMkH_weighted(self, Hv, wt=None) -> float:
        """⟨H|∂M̂|H⟩ with the ẑ× action weighted per plane wave by `wt` (``HMₖH_weighted``,
        ``period.jl:69-74``); wt = 1 is ``HMₖH``."""
        H = _field(Hv, self.grid, 2)
        zxh = zx_tc(H, self.m, self.n)
        if wt is not None:
            zxh = zxh * wt[..., None]
        e = bfft3(self._eid(fft3(zxh), transpose=False)) / self.grid.N
        out = kx_ct(e, self.mag, self.m, self.n, 1.0)
        return float(-np.real(np.vdot(H.reshape(-1), out.reshape(-1))))

    def HMkH(self, Hv) -> float:
        return self.HMkH_weighted(Hv, None)


def E_field(k, Hv, epsinv, grid: Grid3):
    op = Operator3(k, epsinv, grid)
    H = _field(Hv, grid, 2)
    return op._eid(fft3(kx_tc(H, op.mag, op.m, op.n)), transpose=False).reshape(-1)


def canonicalize_phase(Hv, k, epsinv, grid: Grid3):
    E = E_field(k, Hv, epsinv, grid)
    idx = int(np.argmax(np.abs(E) ** 2))
    return np.asarray(Hv) * np.exp(-1j * np.angle(E[idx]))


def solve_k_periodic(omega: float, epsinv, L: float, grid: Grid3, nev: int = 1, max_eigsolves: int = 60,
                     maxiter: int = 300, k_tol: float = 1e-8, eig_tol: float = 1e-8, kguess=None, Hguess=None,
                     seed: int = 0, canonicalize: bool = True):
    """k and modes of the lowest `nev` Bloch bands at ω and period Λ = `L` (``solve_k_periodic``,
    ``period.jl:108-112``): the band-by-band Newton ``solve_k`` (``ME/src/solve.jl:104-115``)
    on ``grid.with_period(L)``, diagonal (k+G)² preconditioner."""
    g = grid.with_period(L)
    epsinv = np.asarray(epsinv, dtype=np.float64)
    k = float(kguess) if kguess is not None else _mx.k_guess(omega, epsinv)
    op = Operator3(k, epsinv, g)
    X = _apply_Hguess(random_block(op.size, nev, seed), Hguess)
    kmags, evecs = [], []
    for band in range(nev):
        ev = None
        for _ in range(max_eigsolves):
            op.set_k(k)
            lam, X, _ = lobpcg(op.M_block, X, op.P_block, tol=eig_tol, maxiter=maxiter)
            ev = X[:, band].copy()
            dk = (lam[band] - omega ** 2) / (2.0 * op.HMkH(ev))
            k -= dk
            if abs(dk) < k_tol:
                break
        kmags.append(k)
        evecs.append(canonicalize_phase(ev, k, epsinv, g) if canonicalize else ev)
    return np.array(kmags), evecs


def _epsinv_bar3(d, ld):
    """3D ``ε⁻¹_bar(d, λd)`` → (3, 3, Nx, Ny, Nz), off-diagonals mirrored."""
    out = np.zeros(d.shape[:3] + (3, 3))
    for a in range(3):
        out[..., a, a] = np.real(-ld[..., a] * np.conj(d[..., a]))
    for a, b in ((0, 1), (1, 2), (0, 2)):
        v = np.real(-np.conj(ld[..., b]) * d[..., a] - ld[..., a] * np.conj(d[..., b]))
        out[..., a, b] = v
        out[..., b, a] = v
    return np.transpose(out, (3, 4, 2, 1, 0)).copy()


def _wbar_z(magbar, mbar, nbar, mag, m, n):
    """z-component of w̄ = māg·ŵ − (m̄·ŵ/mag)·m̂ − (n̄·ŵ/mag)·n̂, ŵ = m̂ × n̂ (``period.jl:113-117``)."""
    w = np.cross(m, n)
    mw = np.sum(mbar * w, axis=-1) / mag
    nw = np.sum(nbar * w, axis=-1) / mag
    return magbar * w[..., 2] - mw * m[..., 2] - nw * n[..., 2]


def solve_k_periodic_pullback(omega: float, epsinv, L: float, grid: Grid3, kmags, evecs, kbar=None, evbar=None,
                              rtol: float = 1e-13):
    """(ω̄, ε̄⁻¹, Λ̄) for cotangents (k̄, ē) of ``solve_k_periodic``'s outputs
    (``_solve_k_period_grads``, ``period.jl:136-200``)."""
    g = grid.with_period(L)
    epsinv = np.asarray(epsinv, dtype=np.float64)
    nev = len(kmags)
    kbar = [None] * nev if kbar is None else list(kbar)
    evbar = [None] * nev if evbar is None else list(evbar)
    ei_bar = np.zeros_like(epsinv)
    wbar_tot, Lbar = 0.0, 0.0
    Ninv = 1.0 / g.N
    wt = period_weight(g)
    for j in range(nev):
        k, ev = float(kmags[j]), np.asarray(evecs[j], dtype=np.complex128)
        op = Operator3(k, epsinv, g)
        dw2dk = 2.0 * op.HMkH(ev)
        dw2dL = 2.0 * op.HMkH_weighted(ev, wt)
        evg = _field(ev, g, 2)
        kb = 0.0 if kbar[j] is None else float(kbar[j])
        eb = evbar[j]
        if eb is not None and np.any(eb):
            lam = eig_adjt(op.M, omega ** 2, ev, 0.0, np.asarray(eb, dtype=np.complex128), op.P_diag, rtol)
            lam = lam - np.vdot(ev, lam) * ev
            lg = _field(lam, g, 2)
            d = fft3(kx_tc(evg * Ninv, op.mag, op.m, op.n))
            ld = fft3(kx_tc(lg, op.mag, op.m, op.n))
            ei_bar += _epsinv_bar3(d, ld)
            ld = ld * Ninv
            le = bfft3(op._eid(ld))
            e = bfft3(op._eid(d))
            kxbar_m = np.real(le * np.conj(evg[..., 1:2]) + e * np.conj(lg[..., 1:2]))
            kxbar_n = -np.real(le * np.conj(evg[..., 0:1]) + e * np.conj(lg[..., 0:1]))
            magbar = np.sum(op.n * kxbar_n, axis=-1) + np.sum(op.m * kxbar_m, axis=-1)
            wz = _wbar_z(magbar, kxbar_m * op.mag[..., None], kxbar_n * op.mag[..., None], op.mag, op.m, op.n)
            kbar_h = -float(np.sum(wz))
            Lbar_h = -float(np.sum(wz * wt))
        else:
            kbar_h, Lbar_h = 0.0, 0.0
        ktot = kb + kbar_h
        d = fft3(kx_tc(evg * Ninv, op.mag, op.m, op.n))
        ld = fft3(kx_tc((ktot / dw2dk) * evg, op.mag, op.m, op.n))
        ei_bar += _epsinv_bar3(d, ld)
        wbar_tot += 2.0 * omega * ktot / dw2dk
        Lbar += Lbar_h + ktot * (-dw2dL / dw2dk)
    return wbar_tot, ei_bar, Lbar
