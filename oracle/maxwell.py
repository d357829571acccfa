"""FP64 restatement of the plane-wave Helmholtz operator (oracle; test infrastructure).

Internal layout: a field with C components on an Nx×Ny grid is a numpy array of shape
``(Ny, Nx, C)`` in C order, which has exactly the memory layout of the reference's
column-major Julia array ``(C, Nx, Ny)``.  Public functions take and return flat vectors
in that order.  The inverse permittivity is accepted with the reference's index
semantics ``epsinv[a, b, ix, iy]`` and held internally as ``E[iy, ix, a, b]``.
"""

from __future__ import annotations

import dataclasses

import numpy as np
import scipy.fft as sfft

#: worker threads for scipy.fft (all host cores by default)
FFT_WORKERS = -1


@dataclasses.dataclass(frozen=True)
class Grid:
    """2D periodic cell of size Dx × Dy (μm) sampled on Nx × Ny pixels.

    Mirrors ``Grid(Δx, Δy, Nx, Ny)`` (``lib/DielectricSmoothing/src/grid.jl:46-76``);
    pixel centres are ``x_i = -Δx/2 + (i-1)·Δx/Nx`` (``grid.jl:120-127``).
    """

    Dx: float
    Dy: float
    Nx: int
    Ny: int

    @property
    def N(self) -> int:
        return self.Nx * self.Ny

    def x(self) -> np.ndarray:
        return -self.Dx / 2 + np.arange(self.Nx) * (self.Dx / self.Nx)

    def y(self) -> np.ndarray:
        return -self.Dy / 2 + np.arange(self.Ny) * (self.Dy / self.Ny)


def _fftfreq_index(n: int) -> np.ndarray:
    """Signed FFT-order frequency indices, ``my_fftfreq`` (``grid.jl:241-244``) times n/fs."""
    if n % 2 == 0:
        return np.concatenate([np.arange(0, n // 2), np.arange(-(n // 2), 0)]).astype(np.float64)
    h = (n - 1) // 2
    return np.concatenate([np.arange(0, h + 1), np.arange(-h, 0)]).astype(np.float64)


def g_vectors(grid: Grid):
    """Reciprocal lattice in cycles/μm, no 2π (``g⃗``, ``grid.jl:255-258``).

    ``gx = fftfreq(Nx, Nx/Δx)`` reduces to ``index/Δx``.  Returns ``(gx[Nx], gy[Ny])``.
    """
    return _fftfreq_index(grid.Nx) / grid.Dx, _fftfreq_index(grid.Ny) / grid.Dy


def mag_mn(k: float, grid: Grid):
    """Transverse basis at k ẑ (``mag_mn!``, ``ME/src/maxwell.jl:646-660``).

    kpg = k ẑ − G;  mag = |kpg|;  n̂ = normalize(ẑ × kpg) (ŷ when kpg ∥ ẑ);
    m̂ = normalize(n̂ × kpg).  Returns ``mag (Ny,Nx)``, ``m (Ny,Nx,3)``, ``n (Ny,Nx,3)``.
    """
    gx, gy = g_vectors(grid)
    GX, GY = np.meshgrid(gx, gy, indexing="xy")  # shape (Ny, Nx)
    kpg = np.stack([-GX, -GY, np.full_like(GX, float(k))], axis=-1)
    mag = np.sqrt(np.sum(kpg * kpg, axis=-1))
    zhat = np.array([0.0, 0.0, 1.0])
    perp2 = kpg[..., 0] ** 2 + kpg[..., 1] ** 2
    zxk = np.cross(np.broadcast_to(zhat, kpg.shape), kpg)
    nrm = np.sqrt(np.sum(zxk * zxk, axis=-1))
    with np.errstate(invalid="ignore", divide="ignore"):
        n = np.where((perp2 > 0.0)[..., None], zxk / nrm[..., None], np.array([0.0, 1.0, 0.0]))
    m = np.cross(n, kpg)
    m = m / np.sqrt(np.sum(m * m, axis=-1))[..., None]
    return mag, m, n


def _field(v: np.ndarray, grid: Grid, ncomp: int) -> np.ndarray:
    return np.asarray(v).reshape(grid.Ny, grid.Nx, ncomp)


def _epsinv_internal(epsinv: np.ndarray) -> np.ndarray:
    """(3,3,Nx,Ny) reference-indexed ε⁻¹ → internal ``E[iy, ix, a, b]``."""
    epsinv = np.asarray(epsinv, dtype=np.float64)
    assert epsinv.ndim == 4 and epsinv.shape[:2] == (3, 3)
    return np.ascontiguousarray(np.transpose(epsinv, (3, 2, 0, 1)))


def kx_tc(H: np.ndarray, mag, m, n) -> np.ndarray:
    """d_a = (H₁ n_a − H₂ m_a)·(−mag)   (``kx_tc!``, ``ME/src/maxwell.jl:385-394``)."""
    return (H[..., 0:1] * n - H[..., 1:2] * m) * (-mag)[..., None]


def kx_ct(e: np.ndarray, mag, m, n, scale: float) -> np.ndarray:
    """H₁ = −(e·n)·mag·s, H₂ = (e·m)·mag·s   (``kx_ct!``, ``ME/src/maxwell.jl:404-411``)."""
    s = (mag * scale)
    h1 = -np.sum(e * n, axis=-1) * s
    h2 = np.sum(e * m, axis=-1) * s
    return np.stack([h1, h2], axis=-1)


def zx_tc(H: np.ndarray, m, n) -> np.ndarray:
    """ẑ × (H₁ m̂ + H₂ n̂)   (``zx_tc!``, ``ME/src/maxwell.jl:396-402``)."""
    d1 = -(H[..., 0] * m[..., 1] + H[..., 1] * n[..., 1])
    d2 = H[..., 0] * m[..., 0] + H[..., 1] * n[..., 0]
    return np.stack([d1, d2, np.zeros_like(d1)], axis=-1)


def eid(E: np.ndarray, d: np.ndarray, transpose: bool = True) -> np.ndarray:
    """Per-pixel 3×3 contraction.

    ``transpose=True`` is ``eid!`` (``ME/src/maxwell.jl:413-420``): e_h = Σ_l ε⁻¹[l,h] d_l.
    ``transpose=False`` is ``ε⁻¹_dot`` (``ME/src/maxwell.jl:236-240``): e_a = Σ_b ε⁻¹[a,b] d_b.
    """
    if transpose:
        return np.einsum("yxlh,yxl->yxh", E, d)
    return np.einsum("yxab,yxb->yxa", E, d)


def fft2(a: np.ndarray) -> np.ndarray:
    """Unnormalised forward 2D FFT (sign −1) over the grid axes (``𝓕!``)."""
    return sfft.fft2(a, axes=(0, 1), workers=FFT_WORKERS)


def bfft2(a: np.ndarray) -> np.ndarray:
    """Unnormalised inverse 2D FFT (sign +1) over the grid axes (``𝓕⁻¹!`` = ``bfft``)."""
    return sfft.ifft2(a, axes=(0, 1), norm="forward", workers=FFT_WORKERS)


class Operator:
    """Matrix-free M̂(k) and P̂(k) for one (k, ε⁻¹, grid) (``HelmholtzMap``,
    ``ME/src/maxwell.jl:834-854, 922-949``)."""

    def __init__(self, k: float, epsinv: np.ndarray, grid: Grid):
        self.grid = grid
        self.epsinv = np.asarray(epsinv, dtype=np.float64)
        self.E = _epsinv_internal(self.epsinv)
        # ε_ave = 3 / tr(ε⁻¹) for the preconditioner (maxwell.jl:945)
        self.eps_ave = 3.0 / (self.E[..., 0, 0] + self.E[..., 1, 1] + self.E[..., 2, 2])
        self.set_k(k)

    def set_k(self, k: float) -> None:
        """``update_k!`` (``ME/src/maxwell.jl:1098-1104``)."""
        self.k = float(k)
        self.mag, self.m, self.n = mag_mn(self.k, self.grid)
        self.inv_mag = 1.0 / self.mag

    @property
    def size(self) -> int:
        return 2 * self.grid.N

    def M(self, Hv: np.ndarray) -> np.ndarray:
        """M̂ H = kx_ct(bfft(ε⁻¹ᵀ·fft(kx_tc H)))/N   (``_M!``, ``ME/src/maxwell.jl:471-481``)."""
        g = self.grid
        H = _field(Hv, g, 2)
        d = fft2(kx_tc(H, self.mag, self.m, self.n))
        e = bfft2(eid(self.E, d, transpose=True))
        return kx_ct(e, self.mag, self.m, self.n, 1.0 / g.N).reshape(-1)

    def P(self, Hv: np.ndarray) -> np.ndarray:
        """MPB-style preconditioner (``_P!``, ``ME/src/maxwell.jl:430-469``):
        e = (H₁n − H₂m)/mag → bfft → ε_ave·e → fft → H₁ = (d·n)/(mag N), H₂ = −(d·m)/(mag N)."""
        g = self.grid
        H = _field(Hv, g, 2)
        e = (H[..., 0:1] * self.n - H[..., 1:2] * self.m) * self.inv_mag[..., None]
        e = bfft2(e)
        d = fft2(e * self.eps_ave[..., None])
        s = self.inv_mag / g.N
        h1 = np.sum(d * self.n, axis=-1) * s
        h2 = -np.sum(d * self.m, axis=-1) * s
        return np.stack([h1, h2], axis=-1).reshape(-1)

    def P_diag(self, Hv: np.ndarray) -> np.ndarray:
        """Diagonal (k+G)² preconditioner: H ← H · ⟨ε⟩ / |k+G|² with ⟨ε⟩ the cell mean of
        ``ε_ave``.  The exact inverse of M̂ for a uniform medium; no FFTs."""
        g = self.grid
        H = _field(Hv, g, 2)
        scale = float(np.mean(self.eps_ave)) * self.inv_mag ** 2
        return (H * scale[..., None]).reshape(-1)

    def M_block(self, X: np.ndarray) -> np.ndarray:
        return np.stack([self.M(X[:, j]) for j in range(X.shape[1])], axis=1)

    def P_block(self, X: np.ndarray, kind: str = "mpb") -> np.ndarray:
        f = self.P if kind == "mpb" else self.P_diag
        return np.stack([f(X[:, j]) for j in range(X.shape[1])], axis=1)

    def HMkH(self, Hv: np.ndarray) -> float:
        """⟨H|∂M̂/∂k|H⟩ (``HMₖH``, ``ME/src/maxwell.jl:267-269``): normalised ifft, ε⁻¹·d
        (``ε⁻¹_dot``), ``kx_ct`` without 1/N."""
        g = self.grid
        H = _field(Hv, g, 2)
        d = fft2(zx_tc(H, self.m, self.n))
        e = bfft2(eid(self.E, d, transpose=False)) / g.N
        out = kx_ct(e, self.mag, self.m, self.n, 1.0)
        return float(-np.real(np.vdot(H.reshape(-1), out.reshape(-1))))

    def HMH(self, Hv: np.ndarray) -> float:
        """⟨H|M̂|H⟩ (``HMH``, ``ME/src/maxwell.jl:288-290``)."""
        g = self.grid
        H = _field(Hv, g, 2)
        d = fft2(kx_tc(H, self.mag, self.m, self.n))
        e = bfft2(eid(self.E, d, transpose=False)) / g.N
        out = kx_ct(e, self.mag, self.m, self.n, 1.0)
        return float(np.real(np.vdot(H.reshape(-1), out.reshape(-1))))


def apply_M(k, epsinv, grid, Hv):
    return Operator(k, epsinv, grid).M(Hv)


def apply_P(k, epsinv, grid, Hv):
    return Operator(k, epsinv, grid).P(Hv)


def apply_P_diag(k, epsinv, grid, Hv):
    return Operator(k, epsinv, grid).P_diag(Hv)


def HMkH(k, epsinv, grid, Hv):
    return Operator(k, epsinv, grid).HMkH(Hv)


def HMH(k, epsinv, grid, Hv):
    return Operator(k, epsinv, grid).HMH(Hv)


def k_guess(omega: float, epsinv: np.ndarray) -> float:
    """k₀ = ω·√(1/min diag ε⁻¹)   (``ME/src/MaxwellEigenmodes.jl:121``)."""
    epsinv = np.asarray(epsinv)
    mins = min(float(np.min(epsinv[a, a])) for a in range(3))
    return float(omega) * np.sqrt(1.0 / mins)


def E_field(k: float, Hv: np.ndarray, epsinv: np.ndarray, grid: Grid) -> np.ndarray:
    """Un-normalised, un-canonicalised E = ε⁻¹·fft(kx_tc H) (``E⃗``, ``ME/src/fields.jl:194-210``).
    Returns the flat vector in ``(3, Nx, Ny)`` column-major order."""
    mag, m, n = mag_mn(k, grid)
    H = _field(Hv, grid, 2)
    d = fft2(kx_tc(H, mag, m, n))
    return eid(_epsinv_internal(epsinv), d, transpose=False).reshape(-1)


def canonicalize_phase(Hv: np.ndarray, k: float, epsinv: np.ndarray, grid: Grid) -> np.ndarray:
    """H·exp(−i·arg E[argmax |E|²]) (``canonicalize_phase``, ``ME/src/fields.jl:258-260``).
    ``argmax`` takes the first maximum in column-major ``(3, Nx, Ny)`` order, as Julia does."""
    E = E_field(k, Hv, epsinv, grid)
    idx = int(np.argmax(np.abs(E) ** 2))
    return np.asarray(Hv) * np.exp(-1j * np.angle(E[idx]))
