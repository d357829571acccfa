"""Device Kottke smoothing (``omb_smoothing_plan_create`` / ``omb_smooth_eps``) against the
CPU oracle (``oracle.smoothing``).

Both sides perform the same IEEE-rounded operations in the same order (the device file is
compiled without contraction), so the bar is bit-exact: pixel kinds, material columns, fill
fractions, normals, the 27 (ε, ∂ωε, ∂²ωε) values and ε⁻¹ must be identical."""

from __future__ import annotations

import math

import numpy as np
import pytest

import oracle.smoothing as S
from oracle.maxwell import Grid as OGrid
from test_smoothing_oracle import P0, random_mats, ridge_wg

pytestmark = pytest.mark.gpu


def _grid(Dx, Dy, Nx, Ny):
    import omb200
    return omb200.Grid(Dx, Dy, Nx, Ny), OGrid(Dx, Dy, Nx, Ny)


def _regular(cx, cy, r, n, phase):
    t = phase + 2 * np.pi * np.arange(n) / n
    return np.stack([cx + r * np.cos(t), cy + r * np.sin(t)], axis=1)


def _cases():
    rng = np.random.default_rng(11)
    many = [_regular(rng.uniform(-1, 1), rng.uniform(-0.8, 0.8), rng.uniform(0.3, 1.2), int(rng.integers(3, 12)),
                     rng.uniform(0, 1)) for _ in range(6)]
    return {
        "ridge_wg_32x24": (ridge_wg(P0), (6.0, 4.0, 32, 24)),
        "ridge_wg_odd_37x23": (ridge_wg([1.3, 0.55, math.pi / 9, 0.3]), (6.0, 4.0, 37, 23)),
        "six_polygons_64x48": (many, (4.0, 3.0, 64, 48)),
        "grid_aligned_box_40x30": ([np.array([[-1.0, -0.5], [1.0, -0.5], [1.0, 0.75], [-1.0, 0.75]])],
                                   (4.0, 3.0, 40, 30)),
        "no_shapes_8x8": ([], (2.0, 2.0, 8, 8)),
    }


@pytest.mark.parametrize("fill", ["plane", "exact"])
@pytest.mark.parametrize("name", list(_cases()))
def test_plan_and_apply_bit_exact(name, fill):
    import omb200
    shapes, (Dx, Dy, Nx, Ny) = _cases()[name]
    g, og = _grid(Dx, Dy, Nx, Ny)
    minds = list(range(len(shapes) + 1))
    ref = S.smoothing_plan(shapes, minds, og, fill)
    plan = omb200.SmoothingPlan(shapes, minds, g, fill)
    kind, mats, rvol, normal = plan.query()
    assert plan.counts == ref.counts
    assert np.array_equal(kind, ref.kind)
    assert np.array_equal(mats, ref.mats)
    assert np.array_equal(rvol, ref.rvol)
    assert np.array_equal(normal, ref.normal)
    M = random_mats(np.random.default_rng(len(name)), len(minds), aniso=0.2)
    e, ei = plan.smooth_eps(M, eps=True, epsinv=True)
    flat = S.apply_plan(ref, M)
    assert np.array_equal(e, S.to_reference_layout(flat, og))
    assert np.array_equal(ei, S.epsinv_of(flat, og))
    plan.close()


def test_material_sets_batch_and_minds_mapping():
    """Several frequencies in one call equal one call each; minds may repeat and skip
    material columns."""
    import omb200
    g, og = _grid(6.0, 4.0, 48, 32)
    shapes = ridge_wg(P0)
    minds = [4, 1, 1, 0]
    plan = omb200.SmoothingPlan(shapes, minds, g)
    rng = np.random.default_rng(3)
    sets = np.stack([random_mats(rng, 5) for _ in range(3)], axis=2)
    both = plan.smooth_eps(sets)
    ref = S.smoothing_plan(shapes, minds, og)
    for s in range(3):
        one = plan.smooth_eps(sets[:, :, s])
        assert np.array_equal(both[..., s], one)
        assert np.array_equal(one, S.to_reference_layout(S.apply_plan(ref, sets[:, :, s]), og))


def test_device_outputs_match_host_outputs():
    import torch

    import omb200
    g, _ = _grid(6.0, 4.0, 64, 48)
    plan = omb200.SmoothingPlan(ridge_wg(P0), [0, 1, 2, 3], g)
    M = np.stack([random_mats(np.random.default_rng(s), 4) for s in range(2)], axis=2)
    e, ei = plan.smooth_eps(M, eps=True, epsinv=True)
    de = torch.empty(27 * g.N * 2, dtype=torch.float64, device="cuda")
    di = torch.empty(9 * g.N * 2, dtype=torch.float64, device="cuda")
    st = torch.cuda.Stream()
    plan.smooth_eps_device(M, de, di, stream=st)
    st.synchronize()
    assert np.array_equal(de.cpu().numpy(), e.reshape(-1, order="F"))
    assert np.array_equal(di.cpu().numpy(), ei.reshape(-1, order="F"))


def test_cross_sections_match_oracle():
    import omb200
    from omb200 import geometry as G
    g, og = _grid(6.0, 4.0, 128, 96)
    shapes, bg = G.ln_ridge_shapes(g, top_width=1.5)
    assert np.array_equal(G.smooth_epsinv(shapes, bg, g), S.smooth_epsinv_constant(shapes, bg, og))
    shapes, bg = G.si3n4_rect_shapes()
    assert np.array_equal(omb200.smooth_epsinv(shapes, bg, g, fill="exact"),
                          S.smooth_epsinv_constant(shapes, bg, og, fill="exact"))


def test_invalid_inputs_raise():
    import omb200
    g, _ = _grid(2.0, 2.0, 8, 8)
    square = np.array([[-0.5, -0.5], [0.5, -0.5], [0.5, 0.5], [-0.5, 0.5]])
    dart = np.array([[0.0, 0.0], [1.0, -1.0], [0.2, 0.0], [1.0, 1.0]])
    with pytest.raises(omb200.OmbError):
        omb200.SmoothingPlan([dart], [0, 1], g)
    with pytest.raises(omb200.OmbError):
        omb200.SmoothingPlan([square], [0, 300], g)
    plan = omb200.SmoothingPlan([square], [0, 2], g)
    with pytest.raises(omb200.OmbError):
        plan.smooth_eps(random_mats(np.random.default_rng(0), 2))  # column 2 missing
    with pytest.raises(ValueError):
        omb200.SmoothingPlan([square], [0, 1], g, fill="area")


def test_smooth_solve_group_index_pipeline():
    """The reference's end-to-end check (test/runtests.jl:21-38): dispersive smoothing →
    ε⁻¹ → solve_k → group_index, with constant-dispersion materials standing in for Si₃N₄
    and SiO₂ (n ≈ 2.0 and 1.444 near 1.55 μm)."""
    import omb200
    g, _ = _grid(4.0, 3.0, 32, 24)
    w = 1 / 1.55
    core = np.array([[-0.8, -0.35], [0.8, -0.35], [0.8, 0.35], [-0.8, 0.35]])
    M = np.stack([S.material_column(np.eye(3) * 3.98, np.eye(3) * 0.12),
                  S.material_column(np.eye(3) * 2.085, np.eye(3) * 0.03)], axis=1)
    plan = omb200.SmoothingPlan([core], [0, 1], g)
    sm, ei = plan.smooth_eps(M, eps=True, epsinv=True)
    assert sm.shape == (3, 3, 3, 32, 24)
    km, kv = omb200.solve_k(w, np.ascontiguousarray(ei), g, nev=1)
    neff = km[0] / w
    assert 1.444 < neff < 2.1
    ng = omb200.group_index(km[0], kv[0], w, np.ascontiguousarray(ei), g, np.ascontiguousarray(sm[:, :, 1]))
    assert neff < ng < 3.0


@pytest.mark.parametrize("case", ["ridge_wg", "multi_material", "repeated_columns"])
def test_material_vjp_matches_oracle(case):
    """Device ``_plan_vjp`` against the oracle's (same per-pixel operations, a different
    summation order over pixels: relative 1e-12)."""
    import omb200
    rng = np.random.default_rng(21)
    if case == "ridge_wg":
        g, og = _grid(6.0, 4.0, 32, 24)
        shapes, minds = ridge_wg(P0), [0, 1, 2, 3]
    elif case == "multi_material":
        g, og = _grid(2.0, 2.0, 16, 16)
        shapes = [np.array([[-1.0, -1.0], [0.1, -1.0], [0.1, 1.0], [-1.0, 1.0]]),
                  np.array([[0.1, -1.0], [1.0, -1.0], [1.0, 0.12], [0.1, 0.12]])]
        minds = [0, 1, 2]
    else:
        g, og = _grid(6.0, 4.0, 40, 24)
        shapes, minds = ridge_wg([1.3, 0.55, math.pi / 9, 0.3]), [2, 2, 0, 2]
    nmat = max(minds) + 1
    plan = omb200.SmoothingPlan(shapes, minds, g)
    ref = S.smoothing_plan(shapes, minds, og)
    sets = np.stack([random_mats(rng, nmat) for _ in range(2)], axis=2)
    ybar = rng.standard_normal((3, 3, 3, g.Nx, g.Ny, 2))
    got = plan.smooth_eps_vjp(sets, ybar)
    for s in range(2):
        yf = ybar[..., s].reshape(27, g.N, order="F")
        exp = S.plan_vjp(ref, sets[:, :, s], yf)
        assert np.allclose(got[:, :, s], exp, rtol=1e-12, atol=1e-12 * np.abs(exp).max())
    # the rrule form on one set
    y, pb = plan.smooth_eps_rrule(sets[:, :, 0])
    assert np.array_equal(pb(ybar[..., 0]), plan.smooth_eps_vjp(sets[:, :, 0], ybar[..., 0]))


@pytest.mark.parametrize("name", ["ridge_wg_odd_37x23", "six_polygons_64x48"])
def test_smooth_scalar_bit_exact(name):
    import omb200
    shapes, (Dx, Dy, Nx, Ny) = _cases()[name]
    g, og = _grid(Dx, Dy, Nx, Ny)
    minds = list(range(len(shapes) + 1))
    vals = np.random.default_rng(5).uniform(0.5, 2.0, len(minds))
    plan = omb200.SmoothingPlan(shapes, minds, g)
    assert np.array_equal(plan.smooth_scalar(vals), S.apply_scalar(S.smoothing_plan(shapes, minds, og), vals))
