"""Waveguide cross-sections → Kottke sub-pixel-smoothed permittivity on the GPU.

Convex polygons (rectangles, ridge trapezoids, any convex outline) in priority order are
rendered onto a ``Grid`` by the library's smoothing kernels, which follow the reference's
``lib/DielectricSmoothing`` (``smoothing_plan`` / ``smooth_ε`` / ``smooth_ε(plan, mat_vals)``,
``src/smoothing_plan.jl``, ``src/smooth.jl:24-121``, ``src/kottke.jl``) and fuse
``sliceinv_3x3`` so the solver's ε⁻¹ input comes out of the same pass:

* a pixel whose four corners lie in one material takes that material's data;
* a pixel whose corners see exactly two materials takes the dispersive τ-average of the two
  (ε, ∂ωε and ∂²ωε by a second-order Taylor jet), weighted by the fill fraction of the
  higher-priority shape, in the frame of that shape's nearest edge normal;
* a pixel whose corners see three or more materials takes the mean of its corners' data.

Material data are the reference's 27-entry columns vcat(vec(ε), vec(∂ωε), vec(∂²ωε)).
GeometryPrimitives (the reference's un-vendored geometry library) is restated for convex
polygons, so ε maps agree with the reference up to that library's polygon routines.
"""

from __future__ import annotations

import ctypes
import dataclasses
from typing import Sequence

import numpy as np

from . import _lib
from .grid import Grid


def diag_eps(a, b=None, c=None) -> np.ndarray:
    b = a if b is None else b
    c = a if c is None else c
    return np.diag([float(a), float(b), float(c)])


@dataclasses.dataclass
class Polygon:
    """Convex polygon: ``(n, 2)`` vertices (stored counter-clockwise) and, for
    :func:`smooth_epsinv`, a constant 3×3 ε tensor."""

    vertices: np.ndarray
    eps: np.ndarray | None = None

    def __post_init__(self):
        v = np.asarray(self.vertices, dtype=np.float64)
        if v.ndim != 2 or v.shape[1] != 2 or v.shape[0] < 3:
            raise ValueError("a polygon needs an (n ≥ 3, 2) vertex array")
        area2 = np.sum(v[:, 0] * np.roll(v[:, 1], -1) - np.roll(v[:, 0], -1) * v[:, 1])
        if area2 < 0:
            v = v[::-1]
        self.vertices = np.ascontiguousarray(v)
        if self.eps is not None:
            self.eps = np.asarray(self.eps, dtype=np.float64)


def rectangle(cx, cy, wx, wy, eps) -> Polygon:
    return Polygon(np.array([[cx - wx / 2, cy - wy / 2], [cx + wx / 2, cy - wy / 2],
                             [cx + wx / 2, cy + wy / 2], [cx - wx / 2, cy + wy / 2]]), eps)


def ridge(cx, y0, top_width, height, sidewall_deg, eps) -> Polygon:
    """Trapezoid standing on y = y0 with the given top width and sidewall angle."""
    dx = height / np.tan(np.deg2rad(sidewall_deg))
    wb = top_width + 2 * dx
    return Polygon(np.array([[cx - wb / 2, y0], [cx + wb / 2, y0], [cx + top_width / 2, y0 + height],
                             [cx - top_width / 2, y0 + height]]), eps)


def material_column(eps, deps=None, ddeps=None) -> np.ndarray:
    """The reference's 27-entry material column vcat(vec(ε), vec(∂ωε), vec(∂²ωε)) from 3×3
    arrays (None → zeros), the layout of ``MaterialDispersion._f_ε_mats`` columns."""
    parts = []
    for m in (eps, deps, ddeps):
        m = np.zeros((3, 3)) if m is None else np.asarray(m, dtype=np.float64)
        if m.shape != (3, 3):
            raise ValueError("material tensors must be 3×3")
        parts.append(m.reshape(9, order="F"))
    return np.concatenate(parts)


_FILL = {"plane": 0, "exact": 1}
UNIFORM, INTERFACE, MULTI = 1, 2, 3


class SmoothingPlan:
    """Frequency-independent geometry scaffold on the device (the reference's
    ``SmoothingPlan``, ``lib/DielectricSmoothing/src/smoothing_plan.jl:26-100``).

    ``shapes`` are convex polygons in priority order (the first containing a point wins),
    ``minds`` the 0-based material column of every shape and then of the background, and
    ``fill`` the interface fill-fraction rule: ``"plane"`` (the reference's ``volfrac`` of the
    voxel cut by the tangent line at the nearest surface point) or ``"exact"`` (the exact
    polygon ∩ voxel area).  Apply it per frequency with :meth:`smooth_eps`."""

    def __init__(self, shapes: Sequence, minds: Sequence[int], grid: Grid, fill: str = "plane", device: int = 0):
        if fill not in _FILL:
            raise ValueError(f"fill must be 'plane' or 'exact', got {fill!r}")
        if len(minds) != len(shapes) + 1:
            raise ValueError("minds needs one material column per shape plus the background")
        self.grid = grid
        self.fill = fill
        self.nmat_min = int(max(minds)) + 1
        self._ctx = _lib.context(device)
        lib = _lib.load()
        nv = np.array([np.asarray(getattr(s, "vertices", s)).shape[0] for s in shapes] or [0], dtype=np.int32)
        verts = (np.concatenate([np.asarray(getattr(s, "vertices", s), dtype=np.float64).reshape(-1)
                                 for s in shapes]) if shapes else np.zeros(2))
        verts = np.ascontiguousarray(verts)
        md = np.ascontiguousarray(np.asarray(minds, dtype=np.int32))
        h = ctypes.c_void_p()
        _lib.check(lib.omb_smoothing_plan_create(
            self._ctx.handle, ctypes.byref(grid.c()), len(shapes), nv.ctypes.data_as(_lib._ip),
            _lib.dptr(verts), md.ctypes.data_as(_lib._ip), _FILL[fill], ctypes.byref(h)))
        self._h = h
        counts = (ctypes.c_int64 * 3)()
        _lib.check(lib.omb_smoothing_plan_query(self._h, counts, None, None, None, None))
        self.counts = tuple(int(c) for c in counts)

    def close(self):
        if getattr(self, "_h", None):
            _lib.load().omb_smoothing_plan_destroy(self._h)
            self._h = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            if not _lib.finalizing():
                self.close()
        except Exception:
            pass

    def query(self):
        """(kind (N,), mats (N, 4), rvol (N,), normal (N, 2)), pixels in corners(grid) order."""
        N = self.grid.N
        kind = np.empty(N, dtype=np.uint8)
        mats = np.empty((N, 4), dtype=np.int32)
        rvol = np.empty(N)
        normal = np.empty((N, 2))
        _lib.check(_lib.load().omb_smoothing_plan_query(
            self._h, None, kind.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8)), mats.ctypes.data_as(_lib._ip),
            _lib.dptr(rvol), _lib.dptr(normal)))
        return kind, mats, rvol, normal

    def _mats(self, mat_vals):
        M = np.asarray(mat_vals, dtype=np.float64)
        single = M.ndim == 2
        if single:
            M = M[:, :, None]
        if M.ndim != 3 or M.shape[0] != 27:
            raise ValueError("mat_vals must be (27, n_materials) or (27, n_materials, n_sets)")
        return np.asfortranarray(M), single

    def smooth_eps(self, mat_vals, eps: bool = True, epsinv: bool = False):
        """``smooth_ε(plan, mat_vals)`` on the device.  ``mat_vals`` is the reference's
        (27, n_materials) matrix, or (27, n_materials, n_sets) for several frequencies at
        once.  Returns the reference-indexed (3, 3, 3, Nx, Ny[, n_sets]) (ε, ∂ωε, ∂²ωε) and/or
        the (3, 3, Nx, Ny[, n_sets]) ``sliceinv_3x3`` of its ε slice."""
        M, single = self._mats(mat_vals)
        nmat, nsets = M.shape[1], M.shape[2]
        g = self.grid
        e = np.empty((3, 3, 3, g.Nx, g.Ny, nsets), order="F") if eps else None
        ei = np.empty((3, 3, g.Nx, g.Ny, nsets), order="F") if epsinv else None
        if e is None and ei is None:
            raise ValueError("ask for eps, epsinv or both")
        _lib.check(_lib.load().omb_smooth_eps(self._h, _lib.dptr(M), nmat, nsets,
                                             _lib.dptr(e) if e is not None else None,
                                             _lib.dptr(ei) if ei is not None else None))
        if single:
            e = e[..., 0] if e is not None else None
            ei = ei[..., 0] if ei is not None else None
        if eps and epsinv:
            return e, ei
        return e if eps else ei

    def smooth_eps_device(self, mat_vals, eps_out=None, epsinv_out=None, stream=None):
        """As :meth:`smooth_eps` into caller-owned device buffers (torch float64 CUDA tensors
        holding 27·N·n_sets and 9·N·n_sets values), queued on ``stream`` (a torch stream, or
        the library's own stream when None)."""
        M, _ = self._mats(mat_vals)
        nmat, nsets = M.shape[1], M.shape[2]
        N = self.grid.N
        for t, per in ((eps_out, 27), (epsinv_out, 9)):
            if t is not None and (t.dtype.__str__() != "torch.float64" or not t.is_cuda or not t.is_contiguous()
                                  or t.numel() != per * N * nsets):
                raise ValueError(f"device outputs must be contiguous float64 CUDA tensors of {per}·N·n_sets values")
        st = None if stream is None else ctypes.c_void_p(stream.cuda_stream)
        _lib.check(_lib.load().omb_smooth_eps_device(
            self._h, _lib.dptr(M), nmat, nsets,
            ctypes.c_void_p(eps_out.data_ptr()) if eps_out is not None else None,
            ctypes.c_void_p(epsinv_out.data_ptr()) if epsinv_out is not None else None, st))


    def smooth_eps_vjp(self, mat_vals, eps_bar):
        """Material-data VJP of :meth:`smooth_eps` (``_plan_vjp``): the cotangent
        (3, 3, 3, Nx, Ny[, n_sets]) of its output → (27, n_materials[, n_sets])."""
        M, single = self._mats(mat_vals)
        nmat, nsets = M.shape[1], M.shape[2]
        g = self.grid
        Y = np.asarray(eps_bar, dtype=np.float64)
        if single:
            Y = Y[..., None]
        if Y.shape != (3, 3, 3, g.Nx, g.Ny, nsets):
            raise ValueError(f"eps_bar must have shape (3, 3, 3, {g.Nx}, {g.Ny}[, n_sets])")
        Y = np.asfortranarray(Y)
        out = np.empty((27, nmat, nsets), order="F")
        _lib.check(_lib.load().omb_smooth_eps_vjp(self._h, _lib.dptr(M), nmat, nsets, _lib.dptr(Y), _lib.dptr(out)))
        return out[..., 0] if single else out

    def smooth_scalar(self, vals):
        """``smooth_scalar`` on the plan's geometry: a per-material scalar (indexed like the
        material columns) → the (Nx, Ny) map, mixed linearly by fill fraction at interfaces."""
        v = np.ascontiguousarray(np.asarray(vals, dtype=np.float64).reshape(-1))
        g = self.grid
        out = np.empty((g.Nx, g.Ny), order="F")
        _lib.check(_lib.load().omb_smooth_scalar(self._h, _lib.dptr(v), v.size, _lib.dptr(out)))
        return out

    def smooth_eps_rrule(self, mat_vals):
        """(smooth_ε(plan, mat_vals), pullback) like ``rrule(smooth_ε, plan, mat_vals)``
        (``smoothing_plan.jl:206-218``): the pullback maps the output's cotangent to the
        material data's."""
        y = self.smooth_eps(mat_vals)
        return y, (lambda ybar: self.smooth_eps_vjp(mat_vals, ybar))


def smoothing_plan(shapes: Sequence, minds: Sequence[int], grid: Grid, fill: str = "plane",
                   device: int = 0) -> SmoothingPlan:
    """``smoothing_plan(shapes, minds, grid)`` (0-based ``minds``)."""
    return SmoothingPlan(shapes, minds, grid, fill, device)


def smooth_eps(shapes, mat_vals, minds=None, grid: Grid | None = None, fill: str = "plane", device: int = 0):
    """``smooth_ε(shapes, mat_vals, minds, grid)`` or ``smooth_ε(plan, mat_vals)``:
    reference-indexed (3, 3, 3, Nx, Ny) smoothed (ε, ∂ωε, ∂²ωε), computed on the GPU."""
    if isinstance(shapes, SmoothingPlan):
        return shapes.smooth_eps(mat_vals)
    plan = SmoothingPlan(shapes, minds, grid, fill, device)
    try:
        return plan.smooth_eps(mat_vals)
    finally:
        plan.close()


def smooth_epsinv(shapes: Sequence[Polygon], background_eps, grid: Grid, fill: str = "plane",
                  device: int = 0) -> np.ndarray:
    """Smoothed ε⁻¹ (reference index semantics (3, 3, Nx, Ny), Fortran-ordered like the
    reference's arrays) of shapes with constant ε (``shape.eps``) in a constant background,
    computed on the GPU."""
    cols = [material_column(s.eps) for s in shapes] + [material_column(background_eps)]
    M = np.stack(cols, axis=1)
    plan = SmoothingPlan(shapes, list(range(len(cols))), grid, fill, device)
    try:
        # column-major, the memory layout the solver's C ABI reads (no conversion copy there)
        return plan.smooth_eps(M, eps=False, epsinv=True)
    finally:
        plan.close()


# ---- the benchmark cross-sections -------------------------------------------------------

EPS_SIO2 = 2.09
EPS_SI3N4 = 3.98
EPS_SI = 12.1
EPS_LN_XCUT = (4.97, 4.61, 4.97)


def si3n4_rect_shapes(w=1.7, h=0.7, eps_core=EPS_SI3N4, eps_clad=EPS_SIO2):
    """(shapes, background ε) of a centred rectangular core in uniform cladding."""
    return [rectangle(0.0, 0.0, w, h, diag_eps(eps_core))], diag_eps(eps_clad)


def ln_ridge_shapes(grid: Grid, top_width=1.5, film=0.6, etch=0.3, sidewall_deg=70.0,
                    eps_core=EPS_LN_XCUT, eps_sub=EPS_SIO2, eps_top=1.0):
    """(shapes, background ε) of an x-cut LiNbO₃ ridge: a slab of thickness film−etch on SiO₂
    with a trapezoidal ridge of height `etch` on top, air above; the film is centred in the
    cell."""
    slab = film - etch
    y_sub = -film / 2
    big = 4 * max(grid.Dx, grid.Dy)
    shapes = [
        ridge(0.0, y_sub + slab, top_width, etch, sidewall_deg, diag_eps(*eps_core)),
        rectangle(0.0, y_sub + slab / 2, big, slab, diag_eps(*eps_core)),
        rectangle(0.0, y_sub - big / 2, big, big, diag_eps(eps_sub)),
    ]
    return shapes, diag_eps(eps_top)


def si3n4_rect(grid: Grid, device: int = 0, **kw) -> np.ndarray:
    """Smoothed ε⁻¹ of :func:`si3n4_rect_shapes` (GPU)."""
    shapes, bg = si3n4_rect_shapes(**kw)
    return smooth_epsinv(shapes, bg, grid, device=device)


def ln_ridge(grid: Grid, device: int = 0, **kw) -> np.ndarray:
    """Smoothed ε⁻¹ of :func:`ln_ridge_shapes` (GPU)."""
    shapes, bg = ln_ridge_shapes(grid, **kw)
    return smooth_epsinv(shapes, bg, grid, device=device)
