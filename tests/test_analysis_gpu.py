"""Modal group index on the device (``omb200.group_index``) against the FP64 oracle
(``oracle.group_index``, itself checked against finite differences of k(ω)) on the modes
the device solver returns.  Tolerance: relative 1e-10 (both evaluate the same FP64
brackets; the device adds FP64 FFT rounding)."""

from __future__ import annotations

import numpy as np
import pytest

import oracle as O
from test_oracle import _dispersive_case, _epsinv_at

pytestmark = pytest.mark.gpu


def test_group_index_parity():
    import omb200
    g, eps0, deps = _dispersive_case()
    w0 = 1 / 1.55
    ei = _epsinv_at(eps0, deps, w0, w0)
    og = omb200.Grid(6.0, 4.0, 24, 16)
    km, kv = omb200.solve_k(w0, ei, og, nev=2)
    for b in range(2):
        for d in (deps, None):
            ng = omb200.group_index(km[b], kv[b], w0, ei, og, d)
            ref = O.group_index(km[b], kv[b], w0, ei, d, g)
            assert abs(ng - ref) / ref < 1e-10
    # the dispersive index of band 0 agrees with the oracle's own solve to the k tolerance
    kr, vr = O.solve_k(w0, ei, g, nev=1, k_tol=1e-12, eig_tol=1e-11)
    assert np.isclose(omb200.group_index(km[0], kv[0], w0, ei, og, deps),
                      O.group_index(kr[0], vr[0], w0, ei, deps, g), rtol=1e-7)


def test_ng_gvd_parity():
    """Device (n_g, GVD) against the oracle's ng_gvd (itself checked against central
    differences of n_g(ω) from re-solved modes) on the device's own modes: n_g to 1e-10,
    GVD to 1e-7 (two MINRES adjoint solves to 1e-12 and FP64 FFT rounding)."""
    import omb200
    from oracle.analysis import ng_gvd as o_ng_gvd
    from test_oracle import _dispersive2_case, _epsinv_at2
    g, eps0, deps, dd = _dispersive2_case()
    w0 = 1 / 1.55
    ei = _epsinv_at2(eps0, deps, dd, w0, w0)
    og = omb200.Grid(6.0, 4.0, 24, 16)
    km, kv = omb200.solve_k(w0, ei, og, nev=2)
    for b in range(2):
        ng, gvd = omb200.ng_gvd(km[b], kv[b], w0, ei, og, deps, dd)
        rng_, rgvd = o_ng_gvd(w0, km[b], kv[b], ei, deps, dd, g)
        assert abs(ng - rng_) / rng_ < 1e-10
        assert abs(gvd - rgvd) / abs(rgvd) < 1e-7
        assert abs(ng - omb200.group_index(km[b], kv[b], w0, ei, og, deps)) / ng < 1e-12
