"""Parity of the device solver with the FP64 oracle on the benchmark cross-sections, through
the C ABI, against the committed golden fixtures (``tests/golden/solve_k_configs.json``,
made by ``tests/golden/make_golden.py`` with the oracle at k_tol 1e-12, eig_tol 1e-11).

* config 1: 6×4 μm, 128², Si₃N₄ rectangle, ω = 1/1.55, 2 bands, FP64 and mixed precision,
  plus the pull-back of the seeded cotangent;
* config 2: 8×5 μm, 256², x-cut LiNbO₃ ridges, 4 bands, mixed precision: the benchmark's
  12-instance batch (widths 1.0/1.5/2.0 μm × 4 frequencies) with and without the sweep warm
  start; the (1.5 μm, ω = 1/1.55) instance against the fixture, every instance's residual
  under the oracle's FP64 operator.

Tolerances, at the product's default k_tol = eig_tol = 1e-8 (the benchmarked settings):
k relative error ≤ 1e-9 (the target after the FP64 polish); residual ‖M̂h − ω²h‖ of the
returned unit eigenvector under the oracle's FP64 operator ≤ 5e-8 (eig_tol plus the
|Δk|·∂ω²/∂k offset of the last Newton update); group index n_g = 2ω/(∂ω²/∂k) relative
≤ 1e-7; field projections ⟨r, h⟩ onto seeded Gaussian probes within 2e-5·‖r‖ (the
eigenvector error is of order residual/gap)."""

from __future__ import annotations

import json
import os

import numpy as np
import pytest

import oracle as O
from oracle import smoothing as OS

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = json.load(open(os.path.join(HERE, "golden", "solve_k_configs.json")))
OMEGA = 1.0 / 1.55


@pytest.fixture(scope="module")
def omb():
    import omb200
    return omb200


def _inputs(name):
    from golden.make_golden import config_inputs, epsinv_checksum
    g, nev, ei = config_inputs(name)
    assert np.allclose(epsinv_checksum(ei), GOLD[name]["epsinv_checksum"], rtol=1e-12)
    return g, nev, ei


def _probes(n2):
    from golden.make_golden import field_probes
    return field_probes(n2)


def _check_against_gold(name, g, ei, km, kv, dw2dk):
    gold = GOLD[name]
    og = O.Grid(g.Dx, g.Dy, g.Nx, g.Ny)
    probes = _probes(2 * g.N)
    rnorm = np.linalg.norm(probes, axis=1)
    errs = {"k": [], "ng": [], "resid": [], "field": []}
    for b in range(gold["nev"]):
        k, h = km[b], kv[b]
        kr = gold["kmags"][b]
        errs["k"].append(abs(k - kr) / kr)
        ng = 2 * OMEGA / dw2dk[b]
        errs["ng"].append(abs(ng - gold["n_g"][b]) / gold["n_g"][b])
        errs["resid"].append(np.linalg.norm(O.Operator(k, ei, og).M(h) - OMEGA ** 2 * h))
        pr = np.array([complex(*p) for p in gold["field_probes"][b]])
        errs["field"].append(float(np.max(np.abs(probes.conj() @ h - pr) / rnorm)))
    assert max(errs["k"]) <= 1e-9, errs
    assert max(errs["resid"]) <= 5e-8, errs
    assert max(errs["ng"]) <= 1e-7, errs
    assert max(errs["field"]) <= 2e-5, errs
    return errs


@pytest.mark.parametrize("prec", ["fp64", "mixed"])
def test_config1_solve_k(omb, prec):
    g, nev, ei = _inputs("config1")
    km, kv, info = omb.solve_k(OMEGA, ei, g, omb.B200Solver(precision=prec), nev=nev, return_info=True)
    assert np.all(info["status"] == 0), info
    _check_against_gold("config1", g, ei, km, kv, info["dw2dk"])
    # group index through the device HMkH pass, on the device's own modes
    for b in range(nev):
        ng = omb.group_index(km[b], kv[b], OMEGA, ei, g)
        assert abs(ng - GOLD["config1"]["n_g"][b]) / GOLD["config1"]["n_g"][b] <= 1e-7


def test_config1_pullback(omb):
    """Seeded cotangent (k̄ ~ N(0,1)², ē ~ CN(0,1)^{2N×2}) pulled back on the device's own FP64
    modes, against the oracle's pull-back of the oracle's modes: ω̄ and projections of ε̄⁻¹
    and ε̄ within 1e-6 relative (both adjoint solves reach ~1e-11; the modes agree to ~1e-9)."""
    from golden.make_golden import tensor_probes
    g, nev, ei = _inputs("config1")
    km, kv = omb.solve_k(OMEGA, ei, g, omb.B200Solver(precision="fp64"), nev=nev, k_tol=1e-12,
                         eig_tol=1e-11)
    rng = np.random.default_rng(0)
    kbar = rng.standard_normal(nev)
    evbar = [rng.standard_normal(2 * g.N) + 1j * rng.standard_normal(2 * g.N) for _ in range(nev)]
    wb, eib, eb = omb.pullback(OMEGA, ei, g, km, kv, kbar, evbar, want_eps_bar=True)
    gp = GOLD["config1"]["pullback"]
    assert abs(wb - gp["omega_bar"]) <= 1e-6 * abs(gp["omega_bar"])
    tp = tensor_probes(g.Nx, g.Ny)
    scale = gp["epsinv_bar_norm"] * np.linalg.norm(tp[0])
    for t, ref in zip(tp, gp["epsinv_bar_probes"]):
        assert abs(np.sum(t * eib) - ref) <= 1e-6 * scale
    eps_scale = max(abs(x) for x in gp["eps_bar_probes"])
    for t, ref in zip(tp, gp["eps_bar_probes"]):
        assert abs(np.sum(t * eb) - ref) <= 1e-5 * eps_scale


def _bench_batch(omb, warm):
    """The benchmark's batch: widths 1.0/1.5/2.0 μm × ω = 1/λ, λ ∈ {1.50, 1.525, 1.55, 1.575},
    ε⁻¹ from the oracle's smoothing (bit-identical to the device smoothing)."""
    from omb200 import geometry as G
    g = omb.Grid(8.0, 5.0, 256, 256)
    eps = {}
    for w in (1.0, 1.5, 2.0):
        shapes, bg = G.ln_ridge_shapes(g, top_width=w)
        eps[w] = OS.smooth_epsinv_constant(shapes, bg, g)
    lams = [1.50, 1.525, 1.55, 1.575]
    probs = [{"omega": 1 / lam, "eps_inv": eps[w], "grid": g, "nev": 4} for lam in lams for w in (1.0, 1.5, 2.0)]
    res, info = omb.solve_k_batch(probs, omb.B200Solver(precision="mixed", warm_start=warm), return_info=True)
    return g, probs, res, info


@pytest.mark.parametrize("warm", ["sweep", "none"])
def test_config2_bench_batch(omb, warm):
    g, probs, res, info = _bench_batch(omb, warm)
    og = O.Grid(g.Dx, g.Dy, g.Nx, g.Ny)
    hit = 0
    for pr, (km, kv), inf in zip(probs, res, info):
        assert np.all(inf["status"] == 0), inf
        ei = pr["eps_inv"]
        w = pr["omega"]
        # every result: unit norm, FP64 residual under the oracle's operator, guided index
        for b in range(4):
            h = kv[b]
            assert abs(np.linalg.norm(h) - 1) < 1e-10
            r = np.linalg.norm(O.Operator(km[b], ei, og).M(h) - w ** 2 * h)
            assert r <= 5e-8, (pr["omega"], b, r)
            assert 1.0 < km[b] / w < np.sqrt(4.97)
        assert np.all(np.diff(km) < 0)  # bands in order of decreasing k
        if abs(w - OMEGA) < 1e-15 and ei is probs[1]["eps_inv"]:
            _check_against_gold("config2", g, ei, km, kv, inf["dw2dk"])
            hit += 1
    assert hit == 1


def test_config3_subset_uneven_batch(omb):
    """Four problems of the uneven batch (128² and 192×128 grids, 2–3 bands, LiNbO₃ and Si
    cores, ω from 0.54 to 0.90) solved together in one batch with other problems of the same
    sweep groups, against their golden oracle solves."""
    from golden.make_golden import CONFIG3_SUBSET
    from omb200 import workloads as W
    spec = W.sweep_spec()
    # the subset plus the other members of their sweep groups (on the same ε⁻¹ arrays)
    groups = {spec[i]["group"] for i in CONFIG3_SUBSET}
    idx = [i for i, s in enumerate(spec) if s["group"] in groups][:24]
    idx = sorted(set(idx) | set(CONFIG3_SUBSET))
    probs = W.sweep_batch(subset=idx, smoothing="oracle")
    res, info = omb.solve_k_batch(probs, omb.B200Solver(precision="mixed", warm_start="sweep"), return_info=True)
    for i, pr, (km, kv), inf in zip(idx, probs, res, info):
        assert np.all(inf["status"] == 0), (i, inf)
        if i not in CONFIG3_SUBSET:
            continue
        name = f"config3_{i}"
        g = pr["grid"]
        assert np.allclose(epsinv_checksum_of(pr["eps_inv"]), GOLD[name]["epsinv_checksum"], rtol=1e-12)
        gold = GOLD[name]
        og = O.Grid(g.Dx, g.Dy, g.Nx, g.Ny)
        for b in range(gold["nev"]):
            assert abs(km[b] - gold["kmags"][b]) <= 1e-9 * gold["kmags"][b], (i, b, km[b], gold["kmags"][b])
            r = np.linalg.norm(O.Operator(km[b], pr["eps_inv"], og).M(kv[b]) - pr["omega"] ** 2 * kv[b])
            assert r <= 5e-8


def epsinv_checksum_of(ei):
    from golden.make_golden import epsinv_checksum
    return epsinv_checksum(ei)


def test_config5_large_slot_cell(omb):
    """The 512² seed-0 slot row, 2 bands, mixed precision, against its golden oracle solve
    (k relative ≤ 1e-9, residual under the oracle's operator ≤ 5e-8, n_g ≤ 1e-7); then the
    pull-back of k̄ = 1 on band 0 against the oracle's on the device's modes (ω̄ and ε̄⁻¹
    within 1e-6)."""
    g, nev, ei = _inputs("config5")
    km, kv, info = omb.solve_k(OMEGA, ei, g, omb.B200Solver(precision="mixed"), nev=nev, return_info=True)
    assert np.all(info["status"] == 0)
    _check_against_gold("config5", g, ei, km, kv, info["dw2dk"])
    og = O.Grid(g.Dx, g.Dy, g.Nx, g.Ny)
    wb, eib = omb.pullback(OMEGA, ei, g, km[:1], kv[:1], [1.0], None)
    wr, eir = O.solve_k_pullback(OMEGA, ei, og, km[:1], kv[:1], kbar=[1.0], evbar=None)
    assert abs(wb - wr) <= 1e-6 * abs(wr)
    assert np.linalg.norm(eib - eir) <= 1e-6 * np.linalg.norm(eir)
