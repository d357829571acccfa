"""Batched forms of the reference's two callers that loop over ``solve_k``.

* ``solve_cells`` — eigenmode expansion's per-cell modal bases
  (``lib/EigenmodeExpansion/src/eme.jl:58-79``, ``_solve_cells``): identical cross-sections
  are solved once and share their result (``dedup``), and with ``warmstart`` the unique
  cross-sections start from a solved neighbour.  The reference chains the solves (each cell
  from the previous one); here all unique cells go to the device in one batch with
  ``warm_start="cells"``: the middle cross-section is solved first and every other one starts
  from its eigenvectors and per-band k, all in parallel.
* ``solve_sweep_tasks`` — ModeSweeps' solve tasks (``lib/ModeSweeps/src/worker.jl:64-90,
  112-135``): every parameter set (with its frequency ``omega``) becomes a problem through
  the caller's ``make_problem``; parameter sets that share a cross-section form a frequency
  sweep solved in one batch with ``warm_start="sweep"``, and each task gets the summary the
  worker writes first (``kmags``, ``neff = k/ω``, ``ng`` from ∂ω²/∂k, residuals).
"""

from __future__ import annotations

import dataclasses

import numpy as np

from .solver import B200Solver, solve_k_batch


def dedup_groups(eps_invs):
    """(representatives, group of each cell): cells with identical ε⁻¹ arrays share a group
    (the reference's ``dedup_groups`` compares the cells' geometry; equal arrays are the
    arrays that geometry produces)."""
    reps, gid = [], []
    for i, e in enumerate(eps_invs):
        e = np.asarray(e)
        for g, r in enumerate(reps):
            if np.array_equal(np.asarray(eps_invs[r]), e):
                gid.append(g)
                break
        else:
            gid.append(len(reps))
            reps.append(i)
    return reps, gid


def solve_cells(eps_invs, omega: float, grid, nev: int = 2, solver: B200Solver | None = None,
                dedup: bool = True, warmstart: bool = False, return_info: bool = False, **kwargs):
    """Modal bases ``[(kmags, evecs), ...]`` of every cell's cross-section at frequency ω (one
    batched device run); cells of one dedup group share the same result object."""
    solver = solver or B200Solver()
    reps, gid = dedup_groups(eps_invs) if dedup else (list(range(len(eps_invs))), list(range(len(eps_invs))))
    s = dataclasses.replace(solver, warm_start="cells" if warmstart else "none")
    probs = [{"omega": omega, "eps_inv": eps_invs[r], "grid": grid, "nev": nev} for r in reps]
    out = solve_k_batch(probs, s, return_info=return_info, **kwargs)
    if return_info:
        res, info = out
        return [res[g] for g in gid], [info[g] for g in gid]
    return [out[g] for g in gid]


def solve_sweep_tasks(params, make_problem, nev: int = 2, solver: B200Solver | None = None, **kwargs):
    """Solve ModeSweeps-style tasks in one batch.  ``params`` is a sequence of dicts with at
    least ``omega``; ``make_problem(p)`` returns a dict with ``eps_inv`` and ``grid``.  Tasks
    whose problems return the same ε⁻¹ object form a sweep.  Returns one summary per task."""
    solver = solver or B200Solver()
    s = dataclasses.replace(solver, warm_start="sweep")
    probs = []
    for p in params:
        if "omega" not in p:
            raise ValueError("parameter sets must include the frequency `omega`")
        pr = make_problem(p)
        probs.append({"omega": float(p["omega"]), "eps_inv": pr["eps_inv"], "grid": pr["grid"], "nev": nev})
    res, info = solve_k_batch(probs, s, return_info=True, raise_on_failure=False, **kwargs)
    out = []
    for p, pr, (km, kv), inf in zip(params, probs, res, info):
        w = pr["omega"]
        out.append({"params": dict(p), "kmags": km, "evecs": kv, "neff": km / w, "ng": 2 * w / inf["dw2dk"],
                    "residuals": inf["residuals"], "status": inf["status"], "iterations": inf["iterations"]})
    return out
