"""Seeded synthetic cross-sections of the benchmark's workloads (no public dataset exists
for this path; every geometry is generated from a seed).

* ``sweep_batch`` — the uneven batch: 64 frequencies uniform in [0.5, 1.0] μm⁻¹ × 8 ridge
  widths uniform in [0.6, 2.4] μm; per width a core of Si₃N₄ (3.98), x-cut LiNbO₃
  diag(4.97, 4.61, 4.97) or Si (12.1); per (width, grid) a grid from {128², 192×128,
  256×192, 256²} and 2–6 bands (seed 3).  Problems sharing a width and a grid share one
  ε⁻¹ array, so ``warm_start="sweep"`` treats them as frequency sweeps.
* ``slot_cell`` — the large instances: 512×512 (8×5 μm), 2–6 seeded rectangles (widths
  0.1–1.5 μm, gaps 0.05–0.5 μm, ε from {2.09, 3.98, 4.2, 12.1}) side by side in a slot /
  coupled-waveguide row on SiO₂, air above.
"""

from __future__ import annotations

import numpy as np

from . import geometry as G
from .grid import Grid

CELL = (8.0, 5.0)
CORES = [("Si3N4", (3.98, 3.98, 3.98)), ("LiNbO3", (4.97, 4.61, 4.97)), ("Si", (12.1, 12.1, 12.1))]
SWEEP_GRIDS = [(128, 128), (192, 128), (256, 192), (256, 256)]


def sweep_spec(n_omega: int = 64, n_width: int = 8, seed: int = 3):
    """The (ω, width, core, grid, nev) of every problem of the uneven batch, without ε."""
    rng = np.random.default_rng(seed)
    omegas = rng.uniform(0.5, 1.0, n_omega)
    widths = rng.uniform(0.6, 2.4, n_width)
    cores = [int(rng.integers(len(CORES))) for _ in range(n_width)]
    spec = []
    group_of = {}
    for wi in range(n_width):
        for om in omegas:
            gi = int(rng.integers(len(SWEEP_GRIDS)))
            key = (wi, gi)
            if key not in group_of:
                group_of[key] = int(rng.integers(2, 7))
            spec.append({"omega": float(om), "width": float(widths[wi]), "core": cores[wi],
                         "grid": SWEEP_GRIDS[gi], "nev": group_of[key], "group": key})
    return spec


def ridge_epsinv(width: float, core: int, grid: Grid, smoothing: str = "gpu", device: int = 0):
    """ε⁻¹ of a ridge of the sweep batch (0.6 μm film, 0.3 μm etch, 70° sidewalls)."""
    shapes, bg = G.ln_ridge_shapes(grid, top_width=width, eps_core=CORES[core][1])
    if smoothing == "gpu":
        return G.smooth_epsinv(shapes, bg, grid, device=device)
    from oracle import smoothing as OS  # the CPU arms only
    return OS.smooth_epsinv_constant(shapes, bg, grid)


def sweep_batch(n_omega: int = 64, n_width: int = 8, seed: int = 3, smoothing: str = "gpu", device: int = 0,
                subset=None):
    """Problems of the uneven batch (optionally only the indices in `subset`)."""
    spec = sweep_spec(n_omega, n_width, seed)
    if subset is not None:
        spec = [spec[i] for i in subset]
    eps = {}
    probs = []
    for s in spec:
        key = s["group"]
        if key not in eps:
            nx, ny = s["grid"]
            g = Grid(CELL[0], CELL[1], nx, ny)
            eps[key] = (g, ridge_epsinv(s["width"], s["core"], g, smoothing, device))
        g, e = eps[key]
        probs.append({"omega": s["omega"], "eps_inv": e, "grid": g, "nev": s["nev"]})
    return probs


def slot_shapes(seed: int, grid: Grid):
    """(shapes, background ε) of a seeded slot / coupled-waveguide row: 2–6 rectangles of
    height 0.3–0.9 μm on the substrate, left to right with the drawn widths and gaps."""
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 7))
    widths = rng.uniform(0.1, 1.5, n)
    gaps = rng.uniform(0.05, 0.5, n - 1)
    eps = [float(rng.choice([2.09, 3.98, 4.2, 12.1])) for _ in range(n)]
    # at least one high-index member so the row guides
    if max(eps) < 3.98:
        eps[int(rng.integers(n))] = 3.98
    h = float(rng.uniform(0.3, 0.9))
    total = widths.sum() + gaps.sum()
    x = -total / 2
    y0 = -0.5
    big = 4 * max(grid.Dx, grid.Dy)
    shapes = []
    for i in range(n):
        shapes.append(G.rectangle(x + widths[i] / 2, y0 + h / 2, widths[i], h, G.diag_eps(eps[i])))
        x += widths[i] + (gaps[i] if i < n - 1 else 0)
    shapes.append(G.rectangle(0.0, y0 - big / 2, big, big, G.diag_eps(2.09)))
    return shapes, G.diag_eps(1.0)


def slot_cell(seed: int, n: int = 512, smoothing: str = "gpu", device: int = 0):
    g = Grid(CELL[0], CELL[1], n, n)
    shapes, bg = slot_shapes(seed, g)
    if smoothing == "gpu":
        return g, G.smooth_epsinv(shapes, bg, g, device=device)
    from oracle import smoothing as OS
    return g, OS.smooth_epsinv_constant(shapes, bg, g)
