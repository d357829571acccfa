"""FP64 CPU oracle for the plane-wave Helmholtz eigensolve hot path.

TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library imports this package:
only ``tests/``, ``__graft_entry__.smoke()`` and the ``cpu_baseline`` /
``--impl reference`` legs of ``bench.py`` use it, and only as the checker or as the
timed CPU baseline, never as the thing measured on the GPU.

What it restates (reference paths are relative to the OptiMode.jl project root,
``ME`` = ``lib/MaxwellEigenmodes``):

* ``maxwell.py``  -- reciprocal lattice ``g⃗`` (``lib/DielectricSmoothing/src/grid.jl:241-258``),
  transverse basis ``mag_mn`` (``ME/src/maxwell.jl:646-660``), the curls
  ``kx_tc!``/``kx_ct!``/``zx_tc!`` (``ME/src/maxwell.jl:385-411``), ``eid!``
  (``ME/src/maxwell.jl:413-420``), the operator ``_M!`` (``ME/src/maxwell.jl:471-481``),
  the MPB-style preconditioner ``_P!`` (``ME/src/maxwell.jl:430-469``), ``HMₖH`` /
  ``HMH`` (``ME/src/maxwell.jl:220-290``), ``k_guess`` (``ME/src/MaxwellEigenmodes.jl:121``),
  ``E⃗`` and ``canonicalize_phase`` (``ME/src/fields.jl:194-260``).
* ``lobpcg.py``   -- block LOBPCG restated from Hetmaniuk & Lehoucq (2006) and Duersch
  et al. (2018), keeping the semantics of ``ME/src/solvers/dftk.jl:304-506``
  (absolute residual tolerance on unit vectors, in-order locking, preconditioned
  residuals, warm start from the incoming block).
* ``solve.py``    -- ``solve_ω²`` and the per-band Newton ``solve_k``
  (``ME/src/solve.jl:38-115, 182-210``; Newton loop as ``ME/src/solvers/gpu.jl:222-237``).
* ``smoothing.py`` -- Kottke sub-pixel smoothing (``lib/DielectricSmoothing``: corners,
  ``corner_sinds``/``proc_sinds``, the dispersive Taylor-jet τ average, ``smoothing_plan`` and
  its apply, ``sliceinv_3x3``), the solver's input generator; its header lists the lines.
* ``adjoint.py``  -- ``eig_adjt`` (``ME/src/grads/solve.jl:96-113``), ``ε⁻¹_bar``
  (``ME/src/grads/solve.jl:490-515``), ``∇ₖmag_m_n`` (``ME/src/maxwell.jl:560-566``),
  the ``solve_k`` pull-back (``ME/src/solve.jl:213-289``) and the ``sliceinv_3x3``
  pull-back ``Ā = −Yᵀ Ȳ Yᵀ`` (``ME/src/grads/linalg.jl:40-47``).

Parity status.  The reference is Julia and cannot run on this machine, and its own
tests hold no golden values for this path.  The oracle is pinned instead by every
invariant the reference's tests assert (``ME/test/runtests.jl``: Hermiticity rtol 1e-9,
``HMH`` consistency, eigen-residual, guided-index bounds, ω² round trip, dk/dω and
diagonal ∂ε⁻¹ against finite differences, the dense eigen-adjoint check) and by
analytic known answers (a uniform medium, where M̂ is diagonal with eigenvalues
|k+G|²/ε).  Absolute-value parity with the Julia reference is therefore *unpinned*.

Array conventions follow the reference's memory layout: a field H is a flat complex
vector of length 2·Nx·Ny ordered as the Julia column-major array ``(2, Nx, Ny)``; the
inverse permittivity is passed with the reference's index semantics
``epsinv[a, b, ix, iy]`` (shape ``(3, 3, Nx, Ny)``).
"""

from .maxwell import (  # noqa: F401
    Grid, g_vectors, mag_mn, kx_tc, kx_ct, zx_tc, eid, apply_M, apply_P, apply_P_diag,
    HMkH, HMH, k_guess, E_field, canonicalize_phase, Operator,
)
from .lobpcg import lobpcg  # noqa: F401
from .solve import solve_omega2, solve_k  # noqa: F401
from .analysis import group_index, tensor_product  # noqa: F401
from .adjoint import (  # noqa: F401
    eig_adjt, epsinv_bar, grad_k_mag_m_n, solve_k_pullback, sliceinv_3x3,
    sliceinv_3x3_pullback,
)
