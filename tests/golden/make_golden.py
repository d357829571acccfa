#!/usr/bin/env python
"""Generate the golden solve_k fixtures of the two benchmark cross-sections with the FP64
oracle (the reference algorithm restated on the CPU).

    python tests/golden/make_golden.py [--only config1|config2]

writes ``tests/golden/solve_k_configs.json``.  The ε⁻¹ inputs come from the oracle's Kottke
smoothing of the shapes in ``omb200.geometry`` (constant-ε materials), the same arrays the
GPU tests feed to the device solver.  Stored per configuration:

* checksums of the ε⁻¹ input (sum and a seeded random projection), so a test can tell that
  it solved the same problem;
* ``kmags`` after the last Newton update (k_tol 1e-12, eig_tol 1e-11), ``dw2dk`` =
  2⟨h|∂M̂/∂k|h⟩ and the group index n_g = 2ω/dw2dk of every band;
* field projections ⟨r_j, h_b⟩ of the phase-canonicalised unit eigenvectors onto three
  seeded complex Gaussian vectors r_j (a 2N-length field is too large for a fixture; the
  projections pin it to the same accuracy);
* config 1 only: the pull-back of a seeded cotangent (k̄ ~ N(0,1)², ē ~ CN(0,1)^{2N×2},
  ``numpy.random.default_rng(0)``) to ω̄, and ε̄⁻¹ and ε̄ (through the per-pixel inverse)
  projected onto three seeded symmetric tensor fields.

Configurations (the benchmark's cross-sections):
  config1  6×4 μm, 128², Si₃N₄ 1.7×0.7 μm core (ε 3.98) in SiO₂ (2.09), ω = 1/1.55, 2 bands
  config2  8×5 μm, 256², x-cut LiNbO₃ ridge (diag 4.97, 4.61, 4.97), top width 1.5 μm,
           film 0.6 μm, etch 0.3 μm, 70° sidewalls, SiO₂ below, air above, ω = 1/1.55, 4 bands
  config3_<i>  problem i of the uneven batch (``omb200.workloads.sweep_spec``, seed 3), for the
           subset on 128² and 192×128 grids with 2–3 bands
  config5  8×5 μm, 512², the seed-0 slot / coupled-waveguide row (``omb200.workloads``),
           ω = 1/1.55, 2 bands (k_tol 1e-11, eig_tol 1e-10)
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "optimode.jl_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

OUT = os.path.join(HERE, "solve_k_configs.json")
OMEGA = 1.0 / 1.55


def field_probes(n2: int, count: int = 3, seed: int = 101) -> np.ndarray:
    rng = np.random.default_rng(seed)
    return rng.standard_normal((count, n2)) + 1j * rng.standard_normal((count, n2))


def tensor_probes(Nx: int, Ny: int, count: int = 3, seed: int = 202) -> np.ndarray:
    """Symmetric (3, 3, Nx, Ny) probe fields."""
    rng = np.random.default_rng(seed)
    out = rng.standard_normal((count, 3, 3, Nx, Ny))
    return 0.5 * (out + out.transpose(0, 2, 1, 3, 4))


def epsinv_checksum(ei: np.ndarray) -> list:
    r = np.random.default_rng(303).standard_normal(ei.shape)
    return [float(np.sum(ei)), float(np.sum(ei * r))]


def project(probes: np.ndarray, h: np.ndarray) -> list:
    v = probes.conj() @ h
    return [[float(x.real), float(x.imag)] for x in v]


CONFIG3_SUBSET = [0, 1, 65, 258]  # uneven-batch problems on 128² / 192×128 grids with 2–3 bands


def config_inputs(name: str):
    """(grid, nev, ε⁻¹) of a configuration, smoothed by the oracle; also the ω for the
    uneven-batch subset ("config3_<index>")."""
    import oracle.smoothing as OS
    from omb200 import geometry as G
    from omb200 import workloads as W
    from omb200.grid import Grid
    if name.startswith("config3_"):
        i = int(name.split("_")[1])
        s = W.sweep_spec()[i]
        g = Grid(W.CELL[0], W.CELL[1], *s["grid"])
        return g, s["nev"], W.ridge_epsinv(s["width"], s["core"], g, smoothing="oracle")
    if name == "config5":
        g, ei = W.slot_cell(0, 512, smoothing="oracle")
        return g, 2, ei
    if name == "config1":
        g = Grid(6.0, 4.0, 128, 128)
        shapes, bg = G.si3n4_rect_shapes()
        nev = 2
    else:
        g = Grid(8.0, 5.0, 256, 256)
        shapes, bg = G.ln_ridge_shapes(g, top_width=1.5)
        nev = 4
    return g, nev, OS.smooth_epsinv_constant(shapes, bg, g)


def config_omega(name: str) -> float:
    if name.startswith("config3_"):
        from omb200 import workloads as W
        return W.sweep_spec()[int(name.split("_")[1])]["omega"]
    return OMEGA


def solve_case(name: str) -> dict:
    import oracle as O
    g, nev, ei = config_inputs(name)
    og = O.Grid(g.Dx, g.Dy, g.Nx, g.Ny)
    omega = config_omega(name)
    tol = (1e-11, 1e-10) if name == "config5" else (1e-12, 1e-11)
    t0 = time.perf_counter()
    km, kv = O.solve_k(omega, ei, og, nev=nev, k_tol=tol[0], eig_tol=tol[1])
    t_solve = time.perf_counter() - t0
    probes = field_probes(2 * g.N)
    out = {
        "grid": [g.Dx, g.Dy, g.Nx, g.Ny], "omega": omega, "nev": nev,
        "epsinv_checksum": epsinv_checksum(ei),
        "kmags": [float(k) for k in km],
        "dw2dk": [], "n_g": [], "residuals": [], "field_probes": [],
        "oracle_seconds": t_solve, "oracle_cores": os.cpu_count(),
    }
    for k, h in zip(km, kv):
        op = O.Operator(k, ei, og)
        d = 2.0 * op.HMkH(h)
        out["dw2dk"].append(float(d))
        out["n_g"].append(float(2.0 * omega / d))
        out["residuals"].append(float(np.linalg.norm(op.M(h) - omega ** 2 * h)))
        out["field_probes"].append(project(probes, h))
    if name == "config1":
        rng = np.random.default_rng(0)
        kbar = rng.standard_normal(nev)
        evbar = [rng.standard_normal(2 * g.N) + 1j * rng.standard_normal(2 * g.N) for _ in range(nev)]
        wb, eib = O.solve_k_pullback(OMEGA, ei, og, km, kv, kbar=kbar, evbar=evbar)
        eb = O.sliceinv_3x3_pullback(ei, eib)
        tp = tensor_probes(g.Nx, g.Ny)
        out["pullback"] = {
            "cotangent_seed": 0, "omega_bar": float(wb),
            "epsinv_bar_probes": [float(np.sum(t * eib)) for t in tp],
            "eps_bar_probes": [float(np.sum(t * eb)) for t in tp],
            "epsinv_bar_norm": float(np.linalg.norm(eib)),
        }
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", help="config1, config2, config3 (the uneven-batch subset) or config5")
    args = ap.parse_args()
    import oracle as O
    O.maxwell.FFT_WORKERS = os.cpu_count() or 1
    data = {}
    if os.path.exists(OUT):
        with open(OUT) as f:
            data = json.load(f)
    names = ["config1", "config2"] + [f"config3_{i}" for i in CONFIG3_SUBSET] + ["config5"]
    for name in names:
        if args.only and not name.startswith(args.only):
            continue
        data[name] = solve_case(name)
        print(name, data[name]["kmags"], f"{data[name]['oracle_seconds']:.1f} s", flush=True)
    data["generator"] = "tests/golden/make_golden.py (FP64 oracle, k_tol 1e-12, eig_tol 1e-11)"
    with open(OUT, "w") as f:
        json.dump(data, f, indent=1)


if __name__ == "__main__":
    main()
