"""``solve_k`` / ``solve_omega2`` through the C ABI, mirroring the reference's Python API
(``python/optimode/solvers.py:50-80``: ``solve_k(omega, eps_inv, grid, solver, nev, **kwargs)``
returning ``(kmags, evecs)``) with a ``B200Solver`` factory beside the reference's
``GPUSolver`` (``python/optimode/solvers.py:27-37``), plus a batched form."""

from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import _lib
from .grid import Grid
from .ops import epsinv_host

_PRECOND = {"mpb": 1, "diag": 2}
_NEWTON = {"inner": 0, "outer": 1}
_WARM = {"none": 0, "sweep": 1, "cells": 2, "learned": 3, "sweep_learned": 4}


@dataclasses.dataclass(frozen=True)
class B200Solver:
    """Backend settings for the B200 eigensolver.

    * ``precision``: ``"mixed"`` (FP32 iterations, FP64 polish to the tolerance),
      ``"fp64"`` or ``"fp32"`` (tolerance clamped to the FP32 floor).
    * ``preconditioner``: ``"diag"`` (⟨ε⟩/|k+G|², the default: fewer iterations than the
      MPB-style one on the benchmark ridges and no FFTs) or ``"mpb"`` (``_P!``, two FFT pairs).
    * ``newton``: ``"inner"`` (Newton steps inside the iteration, one track per band) or
      ``"outer"`` (the reference loop: bands in turn, a converged block eigensolve per step).
    * ``warm_start``: ``"none"`` or ``"sweep"``: in a batch, problems that share one
      ``eps_inv`` array (the same object) and grid form a frequency sweep; the one nearest
      the group's mean ω is solved first and the others start from its eigenvectors and a
      first-order k per band (``OMB_WARM_SWEEP``); ``"cells"``: problems with the same ω
      and grid form a stack of cross-sections (eigenmode expansion); the middle one is solved
      first and the others start from its eigenvectors and k (``OMB_WARM_CELLS``);
      ``"learned"``: problems on 128², 256² or 512² grids start from the learned network's fields and
      effective indices (``OMB_WARM_LEARNED``; the trained parameters committed with the
      package, or a ``omb200.warmstart.WarmStartNet`` attached by the caller);
      ``"sweep_learned"``: ``"sweep"`` whose first-solved instances (each sweep's anchor and
      the instances in no sweep) start from the learned network (``OMB_WARM_SWEEP_LEARNED``).
    """

    precision: str = "mixed"
    preconditioner: str = "diag"
    newton: str = "inner"
    device: int = 0
    maxiter: int = 1000
    seed: int = 0
    guard_bands: int = 1
    warm_start: str = "none"

    def options(self, k_tol=1e-8, eig_tol=1e-8, max_eigsolves=60, maxiter=None, canonicalize=True):
        o = _lib.c_options()
        _lib.load().omb_options_default(ctypes.byref(o))
        o.k_tol = float(k_tol)
        o.eig_tol = float(eig_tol)
        o.max_eigsolves = int(max_eigsolves)
        o.maxiter = int(maxiter if maxiter is not None else self.maxiter)
        o.precision = _lib.PREC[self.precision]
        o.preconditioner = _PRECOND[self.preconditioner]
        o.newton = _NEWTON[self.newton]
        o.canonicalize = 1 if canonicalize else 0
        o.seed = int(self.seed)
        o.guard_bands = int(self.guard_bands)
        o.warm_start = _WARM[self.warm_start]
        return o


def _guess_block(Hguess, n2):
    if Hguess is None:
        return None, 0
    if isinstance(Hguess, np.ndarray) and Hguess.ndim == 2:
        cols = [Hguess[:, j] for j in range(Hguess.shape[1])]
    elif isinstance(Hguess, np.ndarray) and Hguess.ndim == 1:
        cols = [Hguess]
    else:
        cols = list(Hguess)
    cols = [np.asarray(c, dtype=np.complex128) for c in cols if np.asarray(c).shape == (n2,)]
    if not cols:
        return None, 0
    return np.asfortranarray(np.stack(cols, axis=1)), len(cols)


class Batch:
    """A staged batched solve: ``Batch(problems, solver)`` uploads the inputs
    (``omb_batch_create``), ``run()`` solves on the device with the inputs resident
    (``omb_batch_run``), ``results()`` copies them back (``omb_batch_results``)."""

    def __init__(self, problems, solver: B200Solver | None = None, k_tol=1e-8, eig_tol=1e-8,
                 max_eigsolves=60, maxiter=None, canonicalize=True):
        self.solver = solver or B200Solver()
        self._lib = _lib.load()
        self._ctx = _lib.context(self.solver.device)
        if self.solver.warm_start in ("learned", "sweep_learned"):
            from .warmstart import ensure_attached
            ensure_attached(self.solver.device)
        insts, results, keep, outs = _marshal(problems)
        self._insts, self._results, self._keep, self._outs = insts, results, keep, outs
        opt = self.solver.options(k_tol, eig_tol, max_eigsolves, maxiter, canonicalize)
        h = ctypes.c_void_p()
        _lib.check(self._lib.omb_batch_create(self._ctx.handle, insts, len(problems), ctypes.byref(opt),
                                              ctypes.byref(h)))
        self.handle = h

    def run(self):
        _lib.check(self._lib.omb_batch_run(self.handle))

    def results(self, return_info=False, raise_on_failure=True):
        rc = self._lib.omb_batch_results(self.handle, self._results)
        if rc != 0 and (raise_on_failure or rc != 3):
            _lib.check(rc)
        return _unmarshal(self._outs, return_info)

    def stats(self) -> dict:
        s = _lib.c_stats()
        _lib.check(self._lib.omb_batch_stats(self.handle, ctypes.byref(s)))
        return {name: getattr(s, name) for name, _ in _lib.c_stats._fields_}

    def close(self):
        if self.handle:
            self._lib.omb_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            if not _lib.finalizing():
                self.close()
        except Exception:
            pass


def _unmarshal(outs, return_info, copy=True):
    # copy=False: the output arrays are fresh and owned by these results (one-shot calls),
    # so the eigenvectors are returned as column views instead of copies
    c = (lambda a: a.copy()) if copy else (lambda a: a)
    ret = [(c(o["kmags"]), [c(o["evecs"][:, j]) for j in range(o["kmags"].size)]) for o in outs]
    if return_info:
        info = [{k: o[k].copy() for k in ("residuals", "dw2dk", "status", "iterations", "newton_steps")}
                for o in outs]
        return ret, info
    return ret


def _marshal(problems):
    n = len(problems)
    insts = (_lib.c_instance * n)()
    results = (_lib.c_result * n)()
    keep = []
    outs = []
    converted = {}  # one host ε⁻¹ buffer per distinct input array, so sweep groups share it
    for i, pr in enumerate(problems):
        g: Grid = pr["grid"]
        nev = int(pr.get("nev", 1))
        key = (id(pr["eps_inv"]), g.Nx, g.Ny, g.Dx, g.Dy)
        if key not in converted:
            converted[key] = epsinv_host(pr["eps_inv"], g)
        e = converted[key]
        n2 = 2 * g.N
        G, ng = _guess_block(pr.get("Hguess"), n2)
        o = {
            # every entry of evecs is written by the library (no need to clear 16·n2·nev bytes)
            "kmags": np.zeros(nev), "evecs": np.empty((n2, nev), dtype=np.complex128, order="F"),
            "residuals": np.zeros(nev), "dw2dk": np.zeros(nev),
            "status": np.zeros(nev, dtype=np.int32), "iterations": np.zeros(nev, dtype=np.int32),
            "newton_steps": np.zeros(nev, dtype=np.int32),
        }
        keep += [e, G]
        outs.append(o)
        insts[i].grid = g.c()
        insts[i].omega = float(pr["omega"])
        insts[i].epsinv = _lib.dptr(e)
        insts[i].nev = nev
        insts[i].kguess = float(pr["kguess"]) if pr.get("kguess") is not None else 0.0
        insts[i].Hguess = _lib.dptr(G) if G is not None else ctypes.cast(None, _lib._dp)
        insts[i].nguess = ng
        kb = pr.get("kguess_bands")
        if kb is not None:
            kb = np.ascontiguousarray(np.broadcast_to(np.asarray(kb, dtype=np.float64), (nev,)))
            keep.append(kb)
            insts[i].kguess_bands = _lib.dptr(kb)
        else:
            insts[i].kguess_bands = ctypes.cast(None, _lib._dp)
        r = results[i]
        for key in ("kmags", "evecs", "residuals", "dw2dk"):
            setattr(r, key, _lib.dptr(o[key]))
        for key in ("status", "iterations", "newton_steps"):
            setattr(r, key, o[key].ctypes.data_as(_lib._ip))
    return insts, results, keep, outs


def solve_k_batch(problems, solver: B200Solver | None = None, k_tol=1e-8, eig_tol=1e-8,
                  max_eigsolves=60, maxiter=None, canonicalize=True, return_info=False,
                  raise_on_failure=True):
    """Solve many independent problems in one device run (``omb_solve_k``).

    ``problems`` is a sequence of dicts with keys ``omega``, ``eps_inv``, ``grid``, ``nev``
    and optionally ``kguess``, ``Hguess``.  Returns a list of ``(kmags, evecs)`` (and a
    list of info dicts when ``return_info``)."""
    solver = solver or B200Solver()
    lib = _lib.load()
    ctx = _lib.context(solver.device)
    if solver.warm_start in ("learned", "sweep_learned"):
        from .warmstart import ensure_attached
        ensure_attached(solver.device)
    insts, results, keep, outs = _marshal(problems)
    opt = solver.options(k_tol, eig_tol, max_eigsolves, maxiter, canonicalize)
    rc = lib.omb_solve_k(ctx.handle, insts, len(problems), ctypes.byref(opt), results)
    if rc != 0 and (raise_on_failure or rc != 3):
        _lib.check(rc)
    return _unmarshal(outs, return_info, copy=False)


def solve_k(omega: float, eps_inv, grid: Grid, solver: B200Solver | None = None, nev: int = 1,
            k_tol=1e-8, eig_tol=1e-8, max_eigsolves=60, maxiter=None, kguess=None, Hguess=None,
            canonicalize=True, return_info=False):
    """Propagation constants and phase-canonicalised unit eigenvectors of the lowest ``nev``
    modes at frequency ``omega`` (``n_eff = kmags/omega``).  Mirrors the reference
    ``solve_k(ω, ε⁻¹, grid, solver; nev, k_tol, eig_tol, max_eigsolves, kguess, Hguess)``
    (``lib/MaxwellEigenmodes/src/solve.jl:182-196``)."""
    res = solve_k_batch([{"omega": omega, "eps_inv": eps_inv, "grid": grid, "nev": nev,
                          "kguess": kguess, "Hguess": Hguess}], solver, k_tol, eig_tol,
                        max_eigsolves, maxiter, canonicalize, return_info)
    if return_info:
        return res[0][0][0], res[0][0][1], res[1][0]
    return res[0]


def solve_omega2(k: float, eps_inv, grid: Grid, solver: B200Solver | None = None, nev: int = 1,
                 tol=1e-8, maxiter=None, Hguess=None, return_info=False):
    """Lowest ``nev`` eigenpairs ``(ω², H)`` of M̂(k) (``solve_ω²``,
    ``lib/MaxwellEigenmodes/src/solve.jl:38-63``)."""
    solver = solver or B200Solver()
    lib = _lib.load()
    ctx = _lib.context(solver.device)
    e = epsinv_host(eps_inv, grid)
    n2 = 2 * grid.N
    G, ng = _guess_block(Hguess, n2)
    evals = np.zeros(nev)
    evecs = np.zeros((n2, nev), dtype=np.complex128, order="F")
    resid = np.zeros(nev)
    status = np.zeros(nev, dtype=np.int32)
    opt = solver.options(eig_tol=tol, maxiter=maxiter)
    _lib.check(lib.omb_solve_omega2(ctx.handle, ctypes.byref(grid.c()), float(k), _lib.dptr(e), int(nev),
                                    _lib.dptr(G) if G is not None else ctypes.cast(None, _lib._dp), ng,
                                    ctypes.byref(opt), _lib.dptr(evals), _lib.dptr(evecs),
                                    _lib.dptr(resid), status.ctypes.data_as(_lib._ip)))
    out = (evals, [evecs[:, j].copy() for j in range(nev)])
    if return_info:
        return out + ({"residuals": resid, "status": status},)
    return out
