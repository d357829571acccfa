"""The smoothing oracle against the reference's own smoothing tests, restated as invariants
(lib/DielectricSmoothing/test/runtests.jl:62-128, 266-290), and against finite differences
for the dispersive Taylor-jet kernel.  CPU only."""

from __future__ import annotations

import math

import numpy as np
import pytest

import oracle.smoothing as S
from oracle.maxwell import Grid


def ridge_wg(p):
    """The reference test geometry (runtests.jl:25-42): a sidewall-angled core on a slab on a
    substrate, 0-based material columns 0, 1, 2 and vacuum background 3."""
    w_top, t_core, theta, t_slab = p
    edge_gap = 0.5
    Dx, Dy = 6.0, 4.0
    t_subs = (Dy - t_core - edge_gap) / 2.0 - t_slab
    c_subs_y = -Dy / 2.0 + edge_gap / 2.0 + t_subs / 2.0
    c_slab_y = -Dy / 2.0 + edge_gap / 2.0 + t_subs + t_slab / 2.0
    wt, wb, tc = w_top / 2, w_top / 2 + t_core * math.tan(theta), t_core / 2
    core = np.array([[wt, tc], [-wt, tc], [-wb, -tc], [wb, -tc]])

    def box(cx, cy, wx, wy):
        return np.array([[cx - wx / 2, cy - wy / 2], [cx + wx / 2, cy - wy / 2],
                         [cx + wx / 2, cy + wy / 2], [cx - wx / 2, cy + wy / 2]])

    return [core, box(0.0, c_slab_y, Dx - edge_gap, t_slab), box(0.0, c_subs_y, Dx - edge_gap, t_subs)]


def sym(rng, lo, hi, aniso=0.0):
    d = rng.uniform(lo, hi, 3)
    A = np.diag(d)
    if aniso:
        B = rng.standard_normal((3, 3)) * aniso
        A = A + (B + B.T) / 2
    return A


def random_mats(rng, n, aniso=0.2):
    cols = []
    for _ in range(n):
        e = sym(rng, 2.0, 5.0, aniso)
        d = sym(rng, -0.3, 0.3, 0.05)
        dd = sym(rng, -0.2, 0.2, 0.05)
        cols.append(S.material_column(e, d, dd))
    return np.stack(cols, axis=1)


GRID = Grid(6.0, 4.0, 32, 24)
P0 = [1.7, 0.7, math.pi / 14.0, 0.2]


def test_kottke_kernel_limits():
    e1 = 3.0 * np.eye(3)
    Sx = S.normcart(1.0, 0.0)
    assert np.allclose(S.avg_param(e1, e1, Sx, 0.3), e1, rtol=1e-14)
    e2 = np.diag([5.0, 4.0, 4.5])
    assert np.allclose(S.avg_param(e1, e2, Sx, 1.0), e1, rtol=1e-14)
    assert np.allclose(S.avg_param(e1, e2, Sx, 0.0), e2, rtol=1e-14)
    # axis-aligned interface with normal ŷ: harmonic mean across, arithmetic along
    es = S.avg_param(e1, e2, S.normcart(0.0, 1.0), 0.5)
    harm = 2 / (1 / 3.0 + 1 / 4.0)
    assert es[1, 1] == pytest.approx(harm, rel=1e-12)
    assert es[0, 0] == pytest.approx((3.0 + 5.0) / 2, rel=1e-12)
    assert es[2, 2] == pytest.approx((3.0 + 4.5) / 2, rel=1e-12)


def test_kottke_value_slice_is_the_plain_average():
    """The jet kernel's value slice against an independent plain-float τ average."""
    rng = np.random.default_rng(1)
    for _ in range(5):
        e1, e2 = sym(rng, 2, 6, 0.4), sym(rng, 1, 3, 0.3)
        th = rng.uniform(0, 2 * np.pi)
        n = (math.cos(th), math.sin(th))
        r = rng.uniform()
        Sm = np.array(S.normcart(*n))

        def tau(e):
            i = 1 / e[0, 0]
            return np.array([[-i, e[0, 1] * i, e[0, 2] * i],
                             [e[1, 0] * i, e[1, 1] - e[1, 0] * e[0, 1] * i, e[1, 2] - e[1, 0] * e[0, 2] * i],
                             [e[2, 0] * i, e[2, 1] - e[2, 0] * e[0, 1] * i, e[2, 2] - e[2, 0] * e[0, 2] * i]])

        def tau_inv(t):
            i = 1 / t[0, 0]
            return np.array([[-i, -t[0, 1] * i, -t[0, 2] * i],
                             [-t[1, 0] * i, t[1, 1] - t[1, 0] * t[0, 1] * i, t[1, 2] - t[1, 0] * t[0, 2] * i],
                             [-t[2, 0] * i, t[2, 1] - t[2, 0] * t[0, 1] * i, t[2, 2] - t[2, 0] * t[0, 2] * i]])

        ref = Sm @ tau_inv(r * tau(Sm.T @ e1 @ Sm) + (1 - r) * tau(Sm.T @ e2 @ Sm)) @ Sm.T
        got = S.avg_param(e1, e2, S.normcart(*n), r)
        assert np.allclose(got, ref, rtol=1e-12, atol=1e-13)
        assert np.allclose(got, got.T, atol=1e-13)


def test_kottke_jet_derivatives_match_finite_differences():
    """∂ωεₑ and ∂²ωεₑ of the jet kernel against central differences of its value slice with
    ε_m(ω0+δ) = ε_m + ∂ωε_m δ + ∂²ωε_m δ²/2."""
    rng = np.random.default_rng(2)
    M = random_mats(rng, 2, aniso=0.3)
    Sm = S.normcart(0.6, 0.8)
    r = 0.37

    def val(delta):
        cols = []
        for m in range(2):
            c = M[:, m]
            e = c[:9] + c[9:18] * delta + c[18:] * delta ** 2 / 2
            cols.append(np.concatenate([e, np.zeros(18)]))
        return S.kottke_jet(r, Sm, cols[0], cols[1])[:9]

    out = S.kottke_jet(r, Sm, M[:, 0], M[:, 1])
    h = 1e-4
    d1 = (val(h) - val(-h)) / (2 * h)
    d2 = (val(h) - 2 * val(0.0) + val(-h)) / h ** 2
    assert np.allclose(out[9:18], d1, rtol=1e-6, atol=1e-8)
    assert np.allclose(out[18:], d2, rtol=1e-4, atol=1e-6)


def test_smooth_eps_primal_properties():
    """runtests.jl:112-128 with synthetic constant materials."""
    rng = np.random.default_rng(3)
    M = random_mats(rng, 3, aniso=0.0)
    M = np.concatenate([M, S.material_column(np.eye(3))[:, None]], axis=1)
    sm = S.smooth_eps(ridge_wg(P0), M, [0, 1, 2, 3], GRID)
    assert sm.shape == (3, 3, 3, 32, 24)
    eg = sm[:, :, 0]
    assert np.array_equal(eg[:, :, 15, 3], M[:9, 2].reshape(3, 3, order="F"))   # substrate
    assert np.array_equal(eg[:, :, 15, 12], M[:9, 0].reshape(3, 3, order="F"))  # core
    diags = np.stack([eg[i, i] for i in range(3)])
    assert diags.min() >= 1.0 - 1e-9
    assert diags.max() <= max(M[i, j] for i in (0, 4, 8) for j in range(4)) + 1e-9
    assert np.max(np.abs(eg - eg.transpose(1, 0, 2, 3))) < 1e-9


def test_plan_classification_and_reuse():
    """runtests.jl:266-290: every pixel has one kind, the ridge has interfaces, the plan
    applied at two frequencies equals the direct path."""
    rng = np.random.default_rng(4)
    shapes = ridge_wg(P0)
    plan = S.smoothing_plan(shapes, [0, 1, 2, 3], GRID)
    nu, ni, nm = plan.counts
    assert nu + ni + nm == GRID.Nx * GRID.Ny and ni > 0
    for _ in range(2):
        M = random_mats(rng, 4)
        direct = S.smooth_eps(shapes, M, [0, 1, 2, 3], GRID)
        cached = S.to_reference_layout(S.apply_plan(plan, M), GRID)
        assert np.array_equal(cached, direct)


def test_fill_rules_agree_on_straight_edges_and_recover_area():
    """An axis-aligned rectangle: every interface pixel is cut by one straight edge except
    the four corner pixels, where the exact rule still recovers the polygon area."""
    g = Grid(4.0, 3.0, 40, 30)
    rect = np.array([[-1.03, -0.51], [0.97, -0.51], [0.97, 0.77], [-1.03, 0.77]])
    pp = S.smoothing_plan([rect], [0, 1], g, "plane")
    pe = S.smoothing_plan([rect], [0, 1], g, "exact")
    assert np.array_equal(pp.kind, pe.kind)
    dA = (g.Dx / g.Nx) * (g.Dy / g.Ny)
    inside = np.count_nonzero((pe.kind == S.PLAN_UNIFORM) & (pe.mats[:, 0] == 0))
    area = (inside + pe.rvol[pe.kind == S.PLAN_INTERFACE].sum()) * dA
    assert area == pytest.approx(2.0 * 1.28, rel=1e-12)
    xk, yk = S.corner_axis(g.Dx, g.Nx), S.corner_axis(g.Dy, g.Ny)
    for v in np.nonzero(pe.kind == S.PLAN_INTERFACE)[0]:
        ix, iy = v % g.Nx, v // g.Nx
        corner_px = any(xk[ix] < x < xk[ix + 1] and yk[iy] < y < yk[iy + 1] for x, y in rect)
        if not corner_px:
            assert pp.rvol[v] == pytest.approx(pe.rvol[v], rel=1e-12, abs=1e-14)


def test_multi_material_pixels_average_corners():
    g = Grid(2.0, 2.0, 8, 8)
    a = np.array([[-1.0, -1.0], [0.1, -1.0], [0.1, 1.0], [-1.0, 1.0]])
    b = np.array([[0.1, -1.0], [1.0, -1.0], [1.0, 0.12], [0.1, 0.12]])
    plan = S.smoothing_plan([a, b], [0, 1, 2], g)
    assert plan.counts[2] > 0
    M = random_mats(np.random.default_rng(5), 3)
    flat = S.apply_plan(plan, M)
    for v in np.nonzero(plan.kind == S.PLAN_MULTI)[0]:
        ref = sum(M[:, c] for c in plan.mats[v]) / 4.0
        assert np.allclose(flat[:, v], ref, rtol=1e-15)


def test_inverse_matches_numpy():
    rng = np.random.default_rng(6)
    for _ in range(20):
        A = sym(rng, 1, 6, 0.5)
        got = np.array(S.inv3(list(A.reshape(9, order="F")))).reshape(3, 3, order="F")
        assert np.allclose(got, np.linalg.inv(A), rtol=1e-12, atol=1e-14)


def test_plan_vjp_matches_finite_differences():
    """runtests.jl:266-290's material-data gradient through the cached apply, here as a
    directional central difference of ⟨ȳ, smooth_ε(plan, M + hD)⟩ against ⟨VJP(ȳ), D⟩."""
    rng = np.random.default_rng(8)
    g = Grid(6.0, 4.0, 24, 16)
    plan = S.smoothing_plan(ridge_wg(P0), [0, 1, 2, 3], g)
    assert plan.counts[1] > 0
    M = random_mats(rng, 4, aniso=0.2)
    Y = rng.standard_normal((27, g.Nx * g.Ny))
    D = rng.standard_normal(M.shape)
    grad = S.plan_vjp(plan, M, Y)
    h = 1e-6
    f = lambda X: float(np.sum(Y * S.apply_plan(plan, X)))
    fd = (f(M + h * D) - f(M - h * D)) / (2 * h)
    assert float(np.sum(grad * D)) == pytest.approx(fd, rel=1e-7)


def test_smooth_scalar_properties():
    """runtests.jl:130-141: a per-material scalar map (Kerr n₂) takes the material value in
    uniform pixels, stays within the material extremes and mixes at interfaces."""
    vals = np.array([2.5e-19, 2.6e-20, 1.8e-19, 0.0])
    plan = S.smoothing_plan(ridge_wg(P0), [0, 1, 2, 3], GRID)
    n2 = S.apply_scalar(plan, vals)
    assert n2.shape == (GRID.Nx, GRID.Ny)
    assert n2[15, 12] == vals[0]   # core
    assert n2[15, 3] == vals[2]    # substrate
    assert np.all((n2 >= vals.min() - 1e-15) & (n2 <= vals.max() + 1e-15))
    assert np.any((n2 > vals.min() + 1e-12 * vals.max()) & (n2 < vals.max() * (1 - 1e-12)) & ~np.isin(n2, vals))
