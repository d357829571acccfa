"""Waveguide cross-sections → sub-pixel-smoothed inverse permittivity (host, FP64).

The input generator of the benchmark and the tests: convex polygons (rectangles, ridge
trapezoids) with constant dielectric tensors are rendered onto a ``Grid`` with the
anisotropic sub-pixel average of Kottke, Farjadpour & Johnson, Phys. Rev. E 77, 036611
(2008), following the reference's per-pixel rule (``lib/DielectricSmoothing/src/smooth.jl:90-121``,
``src/kottke.jl:44-101``):

* a pixel whose four corners lie in one material takes that material's ε;
* a pixel whose corners see exactly two materials takes the τ-average of the two,
  weighted by the exact area fraction of the higher-priority shape inside the pixel, in the
  frame of that shape's nearest edge normal;
* a pixel whose corners see three or more materials takes the mean of the corner ε.

Shapes are listed in priority order (the first shape containing a point wins); the
reference queries GeometryPrimitives (an un-vendored dependency) for the same fill
fraction and normal, so ε maps agree with the reference only up to that library's
geometry routines.
"""

from __future__ import annotations

import dataclasses
from typing import Sequence

import numpy as np

from .grid import Grid


def diag_eps(a, b=None, c=None) -> np.ndarray:
    b = a if b is None else b
    c = a if c is None else c
    return np.diag([float(a), float(b), float(c)])


@dataclasses.dataclass
class Polygon:
    """Convex polygon with counter-clockwise vertices ``(n, 2)`` and a 3×3 ε tensor."""

    vertices: np.ndarray
    eps: np.ndarray

    def __post_init__(self):
        v = np.asarray(self.vertices, dtype=np.float64)
        area2 = np.sum(v[:, 0] * np.roll(v[:, 1], -1) - np.roll(v[:, 0], -1) * v[:, 1])
        if area2 < 0:
            v = v[::-1]
        self.vertices = v
        self.eps = np.asarray(self.eps, dtype=np.float64)

    def contains(self, x: np.ndarray, y: np.ndarray) -> np.ndarray:
        v = self.vertices
        inside = np.ones(np.broadcast(x, y).shape, dtype=bool)
        for i in range(len(v)):
            a, b = v[i], v[(i + 1) % len(v)]
            inside &= (b[0] - a[0]) * (y - a[1]) - (b[1] - a[1]) * (x - a[0]) >= 0
        return inside

    def clip_area(self, x0, x1, y0, y1) -> float:
        """Area of the intersection with the box [x0,x1]×[y0,y1] (Sutherland–Hodgman)."""
        poly = [(x0, y0), (x1, y0), (x1, y1), (x0, y1)]
        v = self.vertices
        for i in range(len(v)):
            a, b = v[i], v[(i + 1) % len(v)]
            side = lambda p: (b[0] - a[0]) * (p[1] - a[1]) - (b[1] - a[1]) * (p[0] - a[0])
            out = []
            for j in range(len(poly)):
                p, q = poly[j], poly[(j + 1) % len(poly)]
                sp, sq = side(p), side(q)
                if sp >= 0:
                    out.append(p)
                if (sp >= 0) != (sq >= 0):
                    t = sp / (sp - sq)
                    out.append((p[0] + t * (q[0] - p[0]), p[1] + t * (q[1] - p[1])))
            poly = out
            if not poly:
                return 0.0
        P = np.array(poly)
        return 0.5 * abs(np.sum(P[:, 0] * np.roll(P[:, 1], -1) - np.roll(P[:, 0], -1) * P[:, 1]))

    def nearest_normal(self, x: float, y: float) -> np.ndarray:
        """Outward unit normal of the edge nearest to (x, y)."""
        v = self.vertices
        best, nrm = np.inf, None
        for i in range(len(v)):
            a, b = v[i], v[(i + 1) % len(v)]
            d = b - a
            t = np.clip(np.dot([x - a[0], y - a[1]], d) / np.dot(d, d), 0.0, 1.0)
            p = a + t * d
            dist = np.hypot(x - p[0], y - p[1])
            if dist < best:
                best = dist
                nrm = np.array([d[1], -d[0]]) / np.hypot(d[0], d[1])
        return nrm


def rectangle(cx, cy, wx, wy, eps) -> Polygon:
    return Polygon(np.array([[cx - wx / 2, cy - wy / 2], [cx + wx / 2, cy - wy / 2],
                             [cx + wx / 2, cy + wy / 2], [cx - wx / 2, cy + wy / 2]]), eps)


def ridge(cx, y0, top_width, height, sidewall_deg, eps) -> Polygon:
    """Trapezoid standing on y = y0 with the given top width and sidewall angle."""
    dx = height / np.tan(np.deg2rad(sidewall_deg))
    wb = top_width + 2 * dx
    return Polygon(np.array([[cx - wb / 2, y0], [cx + wb / 2, y0], [cx + top_width / 2, y0 + height],
                             [cx - top_width / 2, y0 + height]]), eps)


def _tau(e):
    i = 1.0 / e[0, 0]
    return np.array([[-i, e[0, 1] * i, e[0, 2] * i],
                     [e[1, 0] * i, e[1, 1] - e[1, 0] * e[0, 1] * i, e[1, 2] - e[1, 0] * e[0, 2] * i],
                     [e[2, 0] * i, e[2, 1] - e[2, 0] * e[0, 1] * i, e[2, 2] - e[2, 0] * e[0, 2] * i]])


def _tau_inv(t):
    i = 1.0 / t[0, 0]
    return np.array([[-i, -t[0, 1] * i, -t[0, 2] * i],
                     [-t[1, 0] * i, t[1, 1] - t[1, 0] * t[0, 1] * i, t[1, 2] - t[1, 0] * t[0, 2] * i],
                     [-t[2, 0] * i, t[2, 1] - t[2, 0] * t[0, 1] * i, t[2, 2] - t[2, 0] * t[0, 2] * i]])


def kottke_average(e1, e2, normal2d, r1) -> np.ndarray:
    """S τ⁻¹(r τ(Sᵀε₁S) + (1−r) τ(Sᵀε₂S)) Sᵀ with S's first column the interface normal."""
    n = np.array([normal2d[0], normal2d[1], 0.0])
    t = np.array([-normal2d[1], normal2d[0], 0.0])
    S = np.stack([n, t, np.array([0.0, 0.0, 1.0])], axis=1)
    tau = r1 * _tau(S.T @ e1 @ S) + (1 - r1) * _tau(S.T @ e2 @ S)
    return S @ _tau_inv(tau) @ S.T


def smooth_epsinv(shapes: Sequence[Polygon], background_eps, grid: Grid) -> np.ndarray:
    """Smoothed ε⁻¹ with the reference's index semantics ``(3, 3, Nx, Ny)``."""
    bg = np.asarray(background_eps, dtype=np.float64)
    mats = [s.eps for s in shapes] + [bg]
    dx, dy = grid.Dx / grid.Nx, grid.Dy / grid.Ny
    xc, yc = grid.x(), grid.y()
    # shape index at every pixel corner: corners (i ± 1/2, j ± 1/2)
    xk = np.concatenate([xc - dx / 2, [xc[-1] + dx / 2]])
    yk = np.concatenate([yc - dy / 2, [yc[-1] + dy / 2]])
    XK, YK = np.meshgrid(xk, yk, indexing="ij")
    sid = np.full(XK.shape, len(shapes), dtype=np.int32)
    for i in range(len(shapes) - 1, -1, -1):
        sid[shapes[i].contains(XK, YK)] = i
    c4 = np.stack([sid[:-1, :-1], sid[1:, :-1], sid[:-1, 1:], sid[1:, 1:]], axis=-1)  # (Nx, Ny, 4)
    eps = np.empty((grid.Nx, grid.Ny, 3, 3))
    first = c4[..., 0]
    uniform = np.all(c4 == first[..., None], axis=-1)
    M = np.stack(mats)  # (nmat, 3, 3)
    eps[uniform] = M[first[uniform]]
    for ix, iy in zip(*np.nonzero(~uniform)):
        ids = sorted(set(int(v) for v in c4[ix, iy]))
        if len(ids) == 2:
            s1, s2 = ids
            x0, x1 = xc[ix] - dx / 2, xc[ix] + dx / 2
            y0, y1 = yc[iy] - dy / 2, yc[iy] + dy / 2
            r1 = shapes[s1].clip_area(x0, x1, y0, y1) / (dx * dy)
            # remove the parts of higher-priority shapes (none here: s1 has top priority)
            nrm = shapes[s1].nearest_normal(xc[ix], yc[iy])
            eps[ix, iy] = kottke_average(mats[s1], mats[s2], nrm, min(max(r1, 0.0), 1.0))
        else:
            eps[ix, iy] = np.mean([mats[int(v)] for v in c4[ix, iy]], axis=0)
    ei = np.linalg.inv(eps)
    ei = 0.5 * (ei + np.swapaxes(ei, -1, -2))
    return np.ascontiguousarray(np.transpose(ei, (2, 3, 0, 1)))


# ---- the benchmark cross-sections -------------------------------------------------------

EPS_SIO2 = 2.09
EPS_SI3N4 = 3.98
EPS_SI = 12.1
EPS_LN_XCUT = (4.97, 4.61, 4.97)


def si3n4_rect(grid: Grid, w=1.7, h=0.7, eps_core=EPS_SI3N4, eps_clad=EPS_SIO2) -> np.ndarray:
    """Centred rectangular core in uniform cladding (isotropic)."""
    return smooth_epsinv([rectangle(0.0, 0.0, w, h, diag_eps(eps_core))], diag_eps(eps_clad), grid)


def ln_ridge(grid: Grid, top_width=1.5, film=0.6, etch=0.3, sidewall_deg=70.0,
             eps_core=EPS_LN_XCUT, eps_sub=EPS_SIO2, eps_top=1.0) -> np.ndarray:
    """x-cut LiNbO₃ ridge: a slab of thickness film−etch on SiO₂ with a trapezoidal ridge
    of height `etch` on top, air above; the film is centred in the cell."""
    slab = film - etch
    y_sub = -film / 2
    big = 4 * max(grid.Dx, grid.Dy)
    shapes = [
        ridge(0.0, y_sub + slab, top_width, etch, sidewall_deg, diag_eps(*eps_core)),
        rectangle(0.0, y_sub + slab / 2, big, slab, diag_eps(*eps_core)),
        rectangle(0.0, y_sub - big / 2, big, big, diag_eps(eps_sub)),
    ]
    return smooth_epsinv(shapes, diag_eps(eps_top), grid)
