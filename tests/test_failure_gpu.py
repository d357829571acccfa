"""Failure detection on the device, tested without faulting a GPU: every device wait is
bounded, and the failing statuses come back through the C ABI with the context still usable.

* a self-test kernel waits on a barrier phase that nothing completes, with a 1 ms limit:
  the call returns OMB_ERR_TIMEOUT and the kernel's error code;
* a 1 µs limit on the Gram and update pipelines leaves a healthy solve unchanged (a copy
  that lands while the barrier is being polled is never a timeout);
* maxiter = 1: OMB_ERR_NOT_CONVERGED with the per-band status, results still written
  (the reference's LOBPCG reports non-convergence the same way, ``ME/src/solvers/dftk.jl:457-462``);
* an all-zero warm-start block: the Rayleigh–Ritz basis has no rank, OMB_ERR_ORTHO_FAIL
  (the reference's ``ortho!`` failure, ``ME/src/solvers/dftk.jl:164-192``);
* a non-finite ε⁻¹ entry: OMB_ERR_NAN before any device work."""

from __future__ import annotations

import ctypes

import numpy as np
import pytest

from conftest import OMEGA0, P_WG, gaussian_epsinv

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def omb():
    import omb200
    return omb200


def test_selftest_wait_runs_out_and_context_survives(omb):
    from omb200 import _lib
    lib = _lib.load()
    ctx = _lib.context(0)
    try:
        _lib.set_wait_limit(1e-3)
        code = ctypes.c_int32(-1)
        rc = lib.omb_selftest_wait(ctx.handle, ctypes.byref(code))
        assert rc == 5 and code.value == 1, (rc, code.value)
        assert "ran out" in lib.omb_last_error().decode()
    finally:
        _lib.set_wait_limit(1.0)
    # the context still works
    g = omb.Grid(6.0, 4.0, 24, 16)
    ei = gaussian_epsinv(P_WG)
    H = np.random.default_rng(0).standard_normal(2 * g.N) + 0j
    out = omb.apply_M(1.2, ei, g, H)
    assert np.all(np.isfinite(out))


def test_short_wait_limit_leaves_healthy_solves_alone(omb):
    """A 1 µs limit on the streaming kernels' waits does not break a healthy solve: a bulk copy
    that lands while mbarrier.try_wait is still polling never counts as a timeout (the
    runaway case is the self-test above)."""
    from omb200 import _lib
    g = omb.Grid(6.0, 4.0, 24, 16)
    ei = gaussian_epsinv(P_WG)
    ref, _ = omb.solve_k(OMEGA0, ei, g, omb.B200Solver(precision="mixed"), nev=2)
    try:
        _lib.set_wait_limit(1e-6)
        km, _, info = omb.solve_k(OMEGA0, ei, g, omb.B200Solver(precision="mixed"), nev=2, return_info=True)
    finally:
        _lib.set_wait_limit(1.0)
    assert np.all(info["status"] == 0) and np.allclose(km, ref, rtol=1e-9)


def test_maxiter_one_is_not_converged(omb):
    g = omb.Grid(6.0, 4.0, 24, 16)
    ei = gaussian_epsinv(P_WG)
    res, info = omb.solve_k_batch([{"omega": OMEGA0, "eps_inv": ei, "grid": g, "nev": 2}],
                                  omb.B200Solver(precision="fp64"), maxiter=1, return_info=True,
                                  raise_on_failure=False)
    st = info[0]["status"]
    assert np.all(st == 3), st
    assert np.all(np.isfinite(res[0][0]))
    with pytest.raises(omb.OmbError) as ex:
        omb.solve_k(OMEGA0, ei, g, omb.B200Solver(precision="fp64"), nev=2, maxiter=1)
    assert ex.value.code == 3


def test_zero_warm_start_block_is_ortho_fail(omb):
    g = omb.Grid(6.0, 4.0, 24, 16)
    ei = gaussian_epsinv(P_WG)
    # solve_ω² with nev = 2 iterates a block of nev + 1 columns: all of them zero
    zeros = np.zeros((2 * g.N, 3), dtype=np.complex128)
    with pytest.raises(omb.OmbError) as ex:
        omb.solve_omega2(1.2, ei, g, omb.B200Solver(precision="fp64"), nev=2, Hguess=zeros)
    assert ex.value.code == 4


def test_non_finite_epsinv_is_rejected(omb):
    g = omb.Grid(6.0, 4.0, 24, 16)
    ei = gaussian_epsinv(P_WG)
    ei[0, 0, 3, 5] = np.nan
    with pytest.raises(omb.OmbError) as ex:
        omb.solve_k(OMEGA0, ei, g, nev=1)
    assert ex.value.code == 7
    with pytest.raises(omb.OmbError) as ex:
        omb.apply_M(1.2, ei, g, np.ones(2 * g.N, dtype=np.complex128))
    assert ex.value.code == 7
