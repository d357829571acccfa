"""omb200 — host-side Python binding of libomb200, the B200-native plane-wave Helmholtz
eigensolver (the ``solve_ω²`` / ``solve_k`` hot path of OptiMode.jl and its adjoint).

The compute path is the CUDA library ``libomb200.so`` behind the C ABI in
``include/omb200.h``; this package only converts arrays and calls it.  There is no CPU
fallback.
"""

from ._lib import OmbError, load as load_library  # noqa: F401
from .grid import Grid  # noqa: F401
from .ops import apply, apply_M, apply_P, HMkH, E_field, H_field, profile_apply  # noqa: F401
from .solver import B200Solver, Batch, solve_k, solve_k_batch, solve_omega2  # noqa: F401
from .adjoint import pullback, solve_k_rrule  # noqa: F401
from .analysis import group_index, ng_gvd  # noqa: F401
from . import warmstart  # noqa: F401  (declares the warm-start symbols before the library loads)
from .periodic import (  # noqa: F401
    Grid3, apply3, HMkH3, solve_k_periodic, solve_k_periodic_pullback, solve_k_periodic_rrule,
)
from .geometry import (  # noqa: F401
    Polygon, SmoothingPlan, smoothing_plan, smooth_eps, smooth_epsinv, material_column,
)
