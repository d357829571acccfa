"""The batched forms of eigenmode expansion's cell solves and ModeSweeps' solve tasks
against per-problem oracle solves (k rtol 1e-9, n_g rtol 1e-7), on small grids."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from conftest import OMEGA0, gaussian_epsinv

pytestmark = pytest.mark.gpu


def _taper(n):
    # a slowly widening Gaussian guide: the cross-sections of an adiabatic taper
    return [gaussian_epsinv((4.2, 2.1, 0.8 + 0.1 * i, 0.6)) for i in range(n)]


def test_solve_cells_matches_oracle_and_shares_duplicates():
    import omb200
    from omb200.consumers import solve_cells
    g = omb200.Grid(6.0, 4.0, 24, 16)
    og = O.Grid(6.0, 4.0, 24, 16)
    cells = _taper(5)
    cells = cells[:3] + [cells[1].copy()] + cells[3:]  # a repeated section
    for warm in (False, True):
        res, info = solve_cells(cells, OMEGA0, g, nev=2, warmstart=warm, return_info=True)
        assert res[1] is res[3]  # one dedup group, one result
        for e, (km, kv) in zip(cells, res):
            ref, _ = O.solve_k(OMEGA0, e, og, nev=2, k_tol=1e-12, eig_tol=1e-11)
            assert np.allclose(km, ref, rtol=1e-9, atol=0)
        if warm:
            it_warm = sum(int(np.sum(i["iterations"])) for i in info)
        else:
            it_cold = sum(int(np.sum(i["iterations"])) for i in info)
    assert it_warm < it_cold


def test_sweep_tasks_match_oracle():
    import omb200
    from omb200.consumers import solve_sweep_tasks
    g = omb200.Grid(6.0, 4.0, 24, 16)
    og = O.Grid(6.0, 4.0, 24, 16)
    geoms = {w: gaussian_epsinv((4.2, 2.1, w, 0.6)) for w in (0.9, 1.2)}
    params = [{"width": w, "omega": om} for w in (0.9, 1.2) for om in (1 / 1.5, 1 / 1.55, 1 / 1.6)]
    out = solve_sweep_tasks(params, lambda p: {"eps_inv": geoms[p["width"]], "grid": g}, nev=2)
    for t in out:
        assert np.all(t["status"] == 0)
        e = geoms[t["params"]["width"]]
        w = t["params"]["omega"]
        km, kv = O.solve_k(w, e, og, nev=2, k_tol=1e-12, eig_tol=1e-11)
        assert np.allclose(t["kmags"], km, rtol=1e-9, atol=0)
        ng = [2 * w / (2 * O.Operator(k, e, og).HMkH(h)) for k, h in zip(km, kv)]
        assert np.allclose(t["ng"], ng, rtol=1e-7)
        assert np.allclose(t["neff"], km / w, rtol=1e-9)
