"""CPU restatement of the reference's Kottke sub-pixel smoothing — test infrastructure only.

What it follows (paths relative to the OptiMode.jl project root, ``DS`` =
``lib/DielectricSmoothing``):

* pixel corners ``xc``/``yc`` and ``corners(grid)`` (``DS/src/grid.jl:271-312``, with
  ``myrange``, ``DS/src/grid.jl:107-110``): corner i of the x axis sits at
  ``a + step·i`` with ``a = -(Δx+δx)/2`` and ``step = ((Δx-δx)/2 - a)/Nx``; a pixel's corners
  are listed as (x0,y0), (x0,y1), (x1,y1), (x1,y0);
* ``corner_sinds`` / ``proc_sinds`` (``DS/src/smooth.jl:24-72``): the first shape containing a
  corner wins, the background is slot ``nshapes``; one distinct slot → uniform, two → one
  interface between (min, max), more → the corner average;
* ``smooth_ε_single!`` and ``_interface_geometry`` (``DS/src/smooth.jl:80-121``): the interface
  frame comes from the surface point nearest the pixel centre ``sum(corners)/4`` on the
  higher-priority shape, the fill fraction from ``volfrac`` of the voxel
  ``(vxlmin, vxlmax)`` cut by that tangent plane;
* ``normcart`` (``DS/src/kottke.jl:13-20``), ``τ_trans``/``τ⁻¹_trans`` (``kottke.jl:44-74``),
  ``avg_param_rot`` (``kottke.jl:96-99``), the second-order Taylor jet ``J2`` and its ``*``,
  ``inv`` and ``/`` rules (``kottke.jl:114-137``), and the lab-frame dispersive kernel
  ``εₑ_∂ωεₑ_∂²ωεₑ`` (``kottke.jl:218-268``: ``_rotate(S, ε) = Sᵀ(εS)``, jets through
  ``avg_param_rot``, results rotated back with ``S(X Sᵀ)``);
* ``smoothing_plan`` and the plan apply ``smooth_ε(plan, mat_vals)``
  (``DS/src/smoothing_plan.jl:26-140``): kinds 1 = uniform, 2 = interface, 3 = multi; the
  multi-material pixel sums its four corner columns in corner order and divides by 4;
* ``smooth_scalar`` (``DS/src/smooth.jl:232-263``) on a plan;
* ``sliceinv_3x3`` (``lib/MaxwellEigenmodes/src/linalg.jl:126-147``), here written as the
  adjugate over the determinant.

GeometryPrimitives (the un-vendored dependency behind ``in``, ``surfpt_nearby`` and
``volfrac``) is restated for convex polygons, the shapes of the reference's smoothing tests
(``GeometryPrimitives.Polygon``, axis-aligned ``Cuboid``): a point is inside when it is on the
inner side of, or on, every edge; the nearest surface point is the clamped projection onto
the nearest edge (ties: the first edge in vertex order) with that edge's outward unit normal;
``volfrac`` is the area of the voxel on the inner side of the tangent line through that point
("plane" rule).  The "exact" rule replaces it by the exact area of polygon ∩ voxel.

Every floating-point step is written out scalar by scalar in a fixed order (no fused
multiply-adds, no library reductions), so a device implementation that performs the same
IEEE operations in the same order reproduces this module bit for bit.

Parity status.  The reference is Julia and cannot run here; it is pinned by its own
smoothing tests restated as invariants (``DS/test/runtests.jl:62-128, 266-290``: the τ
limits, harmonic/arithmetic means at an axis-aligned interface, uniform-pixel values, bounds,
symmetry, plan = direct and plan reuse across frequencies).  Absolute parity of ε maps with
GeometryPrimitives' own polygon routines is unpinned.
"""

from __future__ import annotations

import math
from typing import Sequence

import numpy as np

PLAN_UNIFORM = 1
PLAN_INTERFACE = 2
PLAN_MULTI = 3

FILL_PLANE = "plane"
FILL_EXACT = "exact"


# ---- shapes ---------------------------------------------------------------------------

def polygon_vertices(shape) -> np.ndarray:
    """Counter-clockwise ``(n, 2)`` vertices of a convex polygon (a shape object with a
    ``vertices`` attribute, or the array itself); clockwise input is reversed."""
    v = np.asarray(getattr(shape, "vertices", shape), dtype=np.float64)
    if v.ndim != 2 or v.shape[1] != 2 or v.shape[0] < 3:
        raise ValueError("a polygon needs an (n ≥ 3, 2) vertex array")
    n = v.shape[0]
    area2 = 0.0
    for i in range(n):
        j = (i + 1) % n
        area2 += v[i, 0] * v[j, 1] - v[j, 0] * v[i, 1]
    if area2 < 0:
        v = v[::-1]
    return np.ascontiguousarray(v)


def _edge_cross(ax, ay, bx, by, px, py):
    return (bx - ax) * (py - ay) - (by - ay) * (px - ax)


def contains(v: np.ndarray, px, py):
    """Inclusive point-in-convex-polygon test (vectorised over points)."""
    inside = np.ones(np.broadcast(px, py).shape, dtype=bool)
    n = v.shape[0]
    for i in range(n):
        j = (i + 1) % n
        inside &= _edge_cross(v[i, 0], v[i, 1], v[j, 0], v[j, 1], px, py) >= 0
    return inside


# ---- grid corners ---------------------------------------------------------------------

def corner_axis(D: float, N: int) -> np.ndarray:
    d = D / N
    a = -(D + d) / 2
    b = (D - d) / 2
    step = (b - a) / N
    return np.array([a + step * i for i in range(N + 1)])


def corner_slots(polys: Sequence[np.ndarray], grid) -> np.ndarray:
    """Shape slot at every corner point, ``(Nx+1, Ny+1)`` int (background = len(polys))."""
    xk, yk = corner_axis(grid.Dx, grid.Nx), corner_axis(grid.Dy, grid.Ny)
    XK, YK = np.meshgrid(xk, yk, indexing="ij")
    sid = np.full(XK.shape, len(polys), dtype=np.int64)
    for s in range(len(polys) - 1, -1, -1):
        sid[contains(polys[s], XK, YK)] = s
    return sid


# ---- interface geometry ---------------------------------------------------------------

def surfpt_nearby(v: np.ndarray, cx: float, cy: float):
    """(r0x, r0y, nx, ny): nearest boundary point and the outward unit normal there."""
    best = math.inf
    out = None
    n = v.shape[0]
    for i in range(n):
        j = (i + 1) % n
        ax, ay = float(v[i, 0]), float(v[i, 1])
        dx, dy = float(v[j, 0]) - ax, float(v[j, 1]) - ay
        dd = dx * dx + dy * dy
        t = ((cx - ax) * dx + (cy - ay) * dy) / dd
        t = 0.0 if t < 0.0 else (1.0 if t > 1.0 else t)
        px, py = ax + t * dx, ay + t * dy
        ex, ey = cx - px, cy - py
        d2 = ex * ex + ey * ey
        if d2 < best:
            best = d2
            L = math.sqrt(dd)
            out = (px, py, dy / L, -dx / L)
    return out


def _clip(poly, fx):
    """Sutherland–Hodgman step: keep the part of `poly` where fx(p) ≥ 0."""
    out = []
    m = len(poly)
    for j in range(m):
        p, q = poly[j], poly[(j + 1) % m]
        sp, sq = fx(p), fx(q)
        if sp >= 0:
            out.append(p)
        if (sp >= 0) != (sq >= 0):
            t = sp / (sp - sq)
            out.append((p[0] + t * (q[0] - p[0]), p[1] + t * (q[1] - p[1])))
    return out


def _area(poly) -> float:
    m = len(poly)
    if m < 3:
        return 0.0
    s = 0.0
    for j in range(m):
        p, q = poly[j], poly[(j + 1) % m]
        s += p[0] * q[1] - q[0] * p[1]
    return 0.5 * abs(s)


def _box(x0, x1, y0, y1):
    return [(x0, y0), (x1, y0), (x1, y1), (x0, y1)]


def volfrac_plane(x0, x1, y0, y1, r0x, r0y, nx, ny) -> float:
    """Fraction of the voxel on the inner side ((p − r0)·n ≤ 0) of the tangent line."""
    poly = _clip(_box(x0, x1, y0, y1), lambda p: -((p[0] - r0x) * nx + (p[1] - r0y) * ny))
    return _area(poly) / ((x1 - x0) * (y1 - y0))


def volfrac_exact(v: np.ndarray, x0, x1, y0, y1) -> float:
    """Exact area fraction of polygon ∩ voxel."""
    poly = _box(x0, x1, y0, y1)
    n = v.shape[0]
    for i in range(n):
        j = (i + 1) % n
        ax, ay, bx, by = float(v[i, 0]), float(v[i, 1]), float(v[j, 0]), float(v[j, 1])
        poly = _clip(poly, lambda p: _edge_cross(ax, ay, bx, by, p[0], p[1]))
        if not poly:
            return 0.0
    return _area(poly) / ((x1 - x0) * (y1 - y0))


# ---- the plan -------------------------------------------------------------------------

class Plan:
    """Frequency-independent geometry scaffold (``SmoothingPlan``): per pixel, in
    ``corners(grid)`` order (x fastest), the kind, four material columns (uniform: [a];
    interface: [a, b]; multi: the corners' columns; unused entries −1), the fill fraction
    and the interface normal."""

    def __init__(self, grid, kind, mats, rvol, normal):
        self.grid = grid
        self.kind = kind
        self.mats = mats
        self.rvol = rvol
        self.normal = normal

    @property
    def counts(self):
        return tuple(int(np.count_nonzero(self.kind == k)) for k in (PLAN_UNIFORM, PLAN_INTERFACE, PLAN_MULTI))


def smoothing_plan(shapes: Sequence, minds: Sequence[int], grid, fill: str = FILL_PLANE) -> Plan:
    if fill not in (FILL_PLANE, FILL_EXACT):
        raise ValueError(f"fill must be 'plane' or 'exact', got {fill!r}")
    polys = [polygon_vertices(s) for s in shapes]
    if len(minds) != len(polys) + 1:
        raise ValueError("minds needs one material column per shape plus the background")
    Nx, Ny = grid.Nx, grid.Ny
    xk, yk = corner_axis(grid.Dx, Nx), corner_axis(grid.Dy, Ny)
    sid = corner_slots(polys, grid)
    N = Nx * Ny
    kind = np.zeros(N, dtype=np.uint8)
    mats = np.full((N, 4), -1, dtype=np.int32)
    rvol = np.zeros(N)
    normal = np.zeros((N, 2))
    for iy in range(Ny):
        for ix in range(Nx):
            v = ix + Nx * iy
            c = (int(sid[ix, iy]), int(sid[ix, iy + 1]), int(sid[ix + 1, iy + 1]), int(sid[ix + 1, iy]))
            u = sorted(set(c))
            if len(u) == 1:
                kind[v] = PLAN_UNIFORM
                mats[v, 0] = minds[u[0]]
            elif len(u) == 2:
                s1, s2 = u
                x0, x1, y0, y1 = float(xk[ix]), float(xk[ix + 1]), float(yk[iy]), float(yk[iy + 1])
                cx = (((x0 + x0) + x1) + x1) / 4
                cy = (((y0 + y1) + y1) + y0) / 4
                r0x, r0y, nx, ny = surfpt_nearby(polys[s1], cx, cy)
                if fill == FILL_PLANE:
                    r = volfrac_plane(x0, x1, y0, y1, r0x, r0y, nx, ny)
                else:
                    r = volfrac_exact(polys[s1], x0, x1, y0, y1)
                kind[v] = PLAN_INTERFACE
                mats[v, 0], mats[v, 1] = minds[s1], minds[s2]
                rvol[v] = 0.0 if r < 0.0 else (1.0 if r > 1.0 else r)
                normal[v] = (nx, ny)
            else:
                kind[v] = PLAN_MULTI
                mats[v] = [minds[s] for s in c]
    return Plan(grid, kind, mats, rvol, normal)


# ---- the Kottke kernel with a second-order Taylor jet ------------------------------------

class Dual:
    """A value and its forward derivatives along several directions at once (``d`` is an
    array, one entry per direction; every entry follows the scalar rule)."""

    __slots__ = ("v", "d")

    def __init__(self, v, d):
        self.v, self.d = v, d

    def __add__(self, o):
        return Dual(self.v + o.v, self.d + o.d)

    def __sub__(self, o):
        return Dual(self.v - o.v, self.d - o.d)

    def __neg__(self):
        return Dual(-self.v, -self.d)

    def __mul__(self, o):
        if isinstance(o, Dual):
            return Dual(self.v * o.v, self.d * o.v + self.v * o.d)
        return Dual(self.v * o, self.d * o)

    def __rmul__(self, f):
        return Dual(f * self.v, f * self.d)

    def __rtruediv__(self, f):
        i = f / self.v
        return Dual(i, -(i * self.d) / self.v)


class J2:
    """Truncated Taylor number (v, d, dd) = (f, f′, f″), closed under + − × / inv."""

    __slots__ = ("v", "d", "dd")

    def __init__(self, v, d=0.0, dd=0.0):
        self.v, self.d, self.dd = v, d, dd

    def __add__(self, o):
        return J2(self.v + o.v, self.d + o.d, self.dd + o.dd)

    def __sub__(self, o):
        return J2(self.v - o.v, self.d - o.d, self.dd - o.dd)

    def __neg__(self):
        return J2(-self.v, -self.d, -self.dd)

    def __mul__(self, o):
        return J2(self.v * o.v, self.d * o.v + self.v * o.d, (self.dd * o.v + 2.0 * self.d * o.d) + self.v * o.dd)

    def inv(self):
        i = 1.0 / self.v
        return J2(i, -self.d * i * i, -self.dd * i * i + 2.0 * self.d * self.d * i * i * i)


def _tau(e):
    """τ_trans of a jet matrix e[r][c] (0-based)."""
    i = e[0][0].inv()
    return [[-i, e[0][1] * i, e[0][2] * i],
            [e[1][0] * i, e[1][1] - e[1][0] * e[0][1] * i, e[1][2] - e[1][0] * e[0][2] * i],
            [e[2][0] * i, e[2][1] - e[2][0] * e[0][1] * i, e[2][2] - e[2][0] * e[0][2] * i]]


def _tau_inv(t):
    i = t[0][0].inv()
    return [[-i, -t[0][1] * i, -t[0][2] * i],
            [-t[1][0] * i, t[1][1] - t[1][0] * t[0][1] * i, t[1][2] - t[1][0] * t[0][2] * i],
            [-t[2][0] * i, t[2][1] - t[2][0] * t[0][1] * i, t[2][2] - t[2][0] * t[0][2] * i]]


def _matmul(A, B):
    return [[(A[r][0] * B[0][c] + A[r][1] * B[1][c]) + A[r][2] * B[2][c] for c in range(3)] for r in range(3)]


def _T(A):
    return [[A[c][r] for c in range(3)] for r in range(3)]


def normcart(nx: float, ny: float):
    """S = [n h v] for n = (nx, ny, 0): h = ẑ×n normalised, v = n×h."""
    n = (nx, ny, 0.0)
    hx, hy = -ny, nx
    L = math.sqrt(hx * hx + hy * hy)
    h = (hx / L, hy / L, 0.0 / L)
    v = (n[1] * h[2] - n[2] * h[1], n[2] * h[0] - n[0] * h[2], n[0] * h[1] - n[1] * h[0])
    return [[n[0], h[0], v[0]], [n[1], h[1], v[1]], [n[2], h[2], v[2]]]


def _scalar(x):
    return x if isinstance(x, Dual) else float(x)


def _slice(col, s):
    """3×3 matrix of slice s (0 = ε, 1 = ∂ωε, 2 = ∂²ωε) of a 27-entry material column."""
    return [[_scalar(col[9 * s + r + 3 * c]) for c in range(3)] for r in range(3)]


def kottke_jet(r1: float, S, col1, col2, dual: bool = False):
    """εₑ_∂ωεₑ_∂²ωεₑ(r₁, S, col₁, col₂): 27 values vcat(vec(εₑ), vec(∂ωεₑ), vec(∂²ωεₑ))
    (a list of :class:`Dual` when the columns hold Duals and ``dual`` is set)."""
    St = _T(S)
    rot1 = [_matmul(St, _matmul(_slice(col1, s), S)) for s in range(3)]
    rot2 = [_matmul(St, _matmul(_slice(col2, s), S)) for s in range(3)]
    j1 = [[J2(rot1[0][r][c], rot1[1][r][c], rot1[2][r][c]) for c in range(3)] for r in range(3)]
    j2 = [[J2(rot2[0][r][c], rot2[1][r][c], rot2[2][r][c]) for c in range(3)] for r in range(3)]
    t1, t2 = _tau(j1), _tau(j2)
    ra, rb = J2(r1), J2(1.0 - r1)
    tav = [[ra * t1[r][c] + rb * t2[r][c] for c in range(3)] for r in range(3)]
    e = _tau_inv(tav)
    out = [None] * 27 if dual else np.empty(27)
    for s, part in enumerate(("v", "d", "dd")):
        X = [[getattr(e[r][c], part) for c in range(3)] for r in range(3)]
        Y = _matmul(S, _matmul(X, St))
        for c in range(3):
            for r in range(3):
                out[9 * s + r + 3 * c] = Y[r][c]
    return out


def avg_param(e1: np.ndarray, e2: np.ndarray, S, r1: float) -> np.ndarray:
    """Plain (non-dispersive) lab-frame Kottke average S τ⁻¹(r₁τ(Sᵀε₁S) + (1−r₁)τ(Sᵀε₂S)) Sᵀ."""
    c1 = np.concatenate([np.asarray(e1, dtype=np.float64).reshape(9, order="F"), np.zeros(18)])
    c2 = np.concatenate([np.asarray(e2, dtype=np.float64).reshape(9, order="F"), np.zeros(18)])
    return kottke_jet(r1, S, c1, c2)[:9].reshape(3, 3, order="F")


# ---- the apply -----------------------------------------------------------------------

def apply_plan(plan: Plan, mat_vals: np.ndarray) -> np.ndarray:
    """``smooth_ε(plan, mat_vals)``: (27, N) per-pixel (ε, ∂ωε, ∂²ωε), columns in
    ``corners(grid)`` order.  ``mat_vals`` is the reference's (27, n_materials) matrix."""
    M = np.asarray(mat_vals, dtype=np.float64)
    if M.ndim != 2 or M.shape[0] != 27:
        raise ValueError("mat_vals must be (27, n_materials)")
    N = plan.kind.size
    out = np.empty((27, N))
    uni = plan.kind == PLAN_UNIFORM
    out[:, uni] = M[:, plan.mats[uni, 0]]
    for v in np.nonzero(plan.kind == PLAN_INTERFACE)[0]:
        S = normcart(float(plan.normal[v, 0]), float(plan.normal[v, 1]))
        out[:, v] = kottke_jet(float(plan.rvol[v]), S, M[:, plan.mats[v, 0]], M[:, plan.mats[v, 1]])
    for v in np.nonzero(plan.kind == PLAN_MULTI)[0]:
        acc = np.zeros(27)
        for c in plan.mats[v]:
            acc = acc + M[:, c]
        out[:, v] = acc / 4.0
    return out


def plan_vjp(plan: Plan, mat_vals: np.ndarray, ybar: np.ndarray) -> np.ndarray:
    """Material-data VJP of ``smooth_ε(plan, mat_vals)`` (``_plan_vjp``,
    ``DS/src/smoothing_plan.jl:160-203``): ``ybar`` (27, N) → (27, n_materials).  Uniform
    pixels pass their cotangent to their column, multi-material pixels a quarter to each corner
    column, interface pixels Jᵀȳ of the Taylor-jet kernel for both columns, here by forward
    derivatives along all 54 column entries at once.  Contributions are summed in pixel
    order."""
    M = np.asarray(mat_vals, dtype=np.float64)
    Y = np.asarray(ybar, dtype=np.float64)
    out = np.zeros(M.shape)
    eye = np.eye(54)
    for v in range(plan.kind.size):
        kd = plan.kind[v]
        y = Y[:, v]
        if kd == PLAN_UNIFORM:
            out[:, plan.mats[v, 0]] += y
        elif kd == PLAN_MULTI:
            for c in plan.mats[v]:
                out[:, c] += y / 4.0
        else:
            a, b = plan.mats[v, 0], plan.mats[v, 1]
            c1 = [Dual(float(M[q, a]), eye[q]) for q in range(27)]
            c2 = [Dual(float(M[q, b]), eye[27 + q]) for q in range(27)]
            S = normcart(float(plan.normal[v, 0]), float(plan.normal[v, 1]))
            r = kottke_jet(float(plan.rvol[v]), S, c1, c2, dual=True)
            g = np.zeros(54)
            for q in range(27):
                g = g + y[q] * r[q].d
            out[:, a] += g[:27]
            out[:, b] += g[27:]
    return out


def apply_scalar(plan: Plan, vals) -> np.ndarray:
    """``smooth_scalar`` (``DS/src/smooth.jl:232-263``) on a plan: (Nx, Ny) map of a
    per-material scalar, r·v_a + (1 − r)·v_b at interfaces, the corner mean elsewhere."""
    v = [float(x) for x in np.asarray(vals, dtype=np.float64).reshape(-1)]
    N = plan.kind.size
    out = np.empty(N)
    for p in range(N):
        kd, m = plan.kind[p], plan.mats[p]
        if kd == PLAN_UNIFORM:
            out[p] = v[m[0]]
        elif kd == PLAN_INTERFACE:
            r = float(plan.rvol[p])
            out[p] = r * v[m[0]] + (1.0 - r) * v[m[1]]
        else:
            out[p] = (((v[m[0]] + v[m[1]]) + v[m[2]]) + v[m[3]]) / 4.0
    return out.reshape(plan.grid.Nx, plan.grid.Ny, order="F")


def inv3(m) -> list:
    """Inverse of a column-major 3×3 (m[r + 3c]) by the adjugate: 9 values, column-major.
    The entries may be floats or equally shaped arrays (one matrix per element)."""
    a, b, c = m[0], m[3], m[6]
    d, e, f = m[1], m[4], m[7]
    g, h, i = m[2], m[5], m[8]
    A = e * i - f * h
    B = f * g - d * i
    C = d * h - e * g
    det = (a * A + b * B) + c * C
    r = 1.0 / det
    return [A * r, B * r, C * r,
            (c * h - b * i) * r, (a * i - c * g) * r, (b * g - a * h) * r,
            (b * f - c * e) * r, (c * d - a * f) * r, (a * e - b * d) * r]


def smooth_eps(shapes: Sequence, mat_vals: np.ndarray, minds: Sequence[int], grid,
               fill: str = FILL_PLANE) -> np.ndarray:
    """Reference-indexed (3, 3, 3, Nx, Ny) smoothed (ε, ∂ωε, ∂²ωε)."""
    flat = apply_plan(smoothing_plan(shapes, minds, grid, fill), mat_vals)
    return to_reference_layout(flat, grid)


def to_reference_layout(flat: np.ndarray, grid) -> np.ndarray:
    """(27, Nx·Ny) columns → array indexed [i, j, slice, ix, iy]."""
    return np.ascontiguousarray(flat.reshape(3, 3, 3, grid.Nx, grid.Ny, order="F"))


def epsinv_of(flat: np.ndarray, grid) -> np.ndarray:
    """``sliceinv_3x3`` of the ε slice of (27, N) columns → reference-indexed (3, 3, Nx, Ny)."""
    out = np.stack(inv3([flat[k] for k in range(9)]))  # elementwise, same operations per pixel
    return np.ascontiguousarray(out.reshape(3, 3, grid.Nx, grid.Ny, order="F"))


# ---- material columns and the benchmark cross-sections ---------------------------------------

def material_column(eps, deps=None, ddeps=None) -> np.ndarray:
    """27-entry column vcat(vec(ε), vec(∂ωε), vec(∂²ωε)) from 3×3 arrays (None → zeros)."""
    parts = []
    for m in (eps, deps, ddeps):
        m = np.zeros((3, 3)) if m is None else np.asarray(m, dtype=np.float64)
        parts.append(m.reshape(9, order="F"))
    return np.concatenate(parts)


def smooth_epsinv_constant(shapes: Sequence, background_eps, grid, fill: str = FILL_PLANE) -> np.ndarray:
    """ε⁻¹ of constant-ε shapes (``shape.eps``) in a background: one material column per
    shape, the background last."""
    cols = [material_column(s.eps) for s in shapes] + [material_column(background_eps)]
    M = np.stack(cols, axis=1)
    flat = apply_plan(smoothing_plan(shapes, list(range(len(cols))), grid, fill), M)
    return epsinv_of(flat, grid)
