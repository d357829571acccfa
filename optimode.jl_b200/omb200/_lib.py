"""ctypes binding of ``libomb200.so`` (the C ABI declared in ``include/omb200.h``).

The shared library is built in place next to this package (``make -C optimode.jl_b200``
or ``__graft_entry__.build()``).  There is no CPU fallback: if the library or a CUDA
device is missing, every entry point raises.
"""

from __future__ import annotations

import atexit
import ctypes
import os
import threading

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "libomb200.so")

OMB_OK = 0
ERROR_NAMES = {
    1: "OMB_ERR_INVALID_ARG", 2: "OMB_ERR_CUDA", 3: "OMB_ERR_NOT_CONVERGED",
    4: "OMB_ERR_ORTHO_FAIL", 5: "OMB_ERR_TIMEOUT", 6: "OMB_ERR_UNSUPPORTED", 7: "OMB_ERR_NAN",
}
PREC = {"fp32": 0, "f32": 0, "fp64": 1, "f64": 1, "mixed": 2}
OPS = {"M": 0, "P": 1, "P_diag": 2}

#: every symbol ``include/omb200.h`` declares (checked by the CPU test suite)
EXPORTS = (
    "omb_version", "omb_fft_size_supported", "omb_last_error", "omb_ctx_create",
    "omb_ctx_destroy", "omb_apply", "omb_HMkH", "omb_efield", "omb_hfield", "omb_gram_blocks",
    "omb_autotune", "omb_ctx_set_autotune", "omb_tune_set", "omb_tune_get", "omb_tune_clear", "omb_tune_save",
    "omb_tune_load",
)


class OmbError(RuntimeError):
    """A non-zero status from libomb200, with the library's message."""

    def __init__(self, code: int, msg: str):
        super().__init__(f"{ERROR_NAMES.get(code, code)}: {msg}")
        self.code = code


class c_grid(ctypes.Structure):
    _fields_ = [("Nx", ctypes.c_int32), ("Ny", ctypes.c_int32),
                ("Dx", ctypes.c_double), ("Dy", ctypes.c_double)]


_lib = None
_lock = threading.Lock()
_dp = ctypes.POINTER(ctypes.c_double)
_exiting = False


def _mark_exiting():
    global _exiting
    _exiting = True


# At interpreter exit the library's handles (contexts, batches, plans, networks) are left to
# the process teardown: Python finalises the objects of reference cycles, module globals
# among them, in no particular order, so a context could be destroyed before a network or
# batch that still uses its stream.  ``finalizing()`` makes every ``__del__`` a no-op then;
# explicit ``close()`` calls before exit free resources in the caller's order.
atexit.register(_mark_exiting)


def finalizing() -> bool:
    """True once the interpreter has begun to exit (``__del__`` must not call the library)."""
    return _exiting


def load():
    """Load the library (once).  Raises ``OSError`` naming the missing file."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        if not os.path.exists(LIB_PATH):
            raise OSError(f"libomb200.so not found at {LIB_PATH}: build it with "
                          "`make -C optimode.jl_b200 -j` (there is no CPU fallback)")
        lib = ctypes.CDLL(LIB_PATH)
        vp = ctypes.c_void_p
        gp = ctypes.POINTER(c_grid)
        sig = {
            "omb_version": (ctypes.c_int, []),
            "omb_fft_size_supported": (ctypes.c_int, [ctypes.c_int]),
            "omb_last_error": (ctypes.c_char_p, []),
            "omb_ctx_create": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(vp)]),
            "omb_ctx_destroy": (ctypes.c_int, [vp]),
            "omb_apply": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, gp, ctypes.c_double, _dp,
                                         ctypes.c_int, _dp, _dp]),
            "omb_HMkH": (ctypes.c_int, [vp, ctypes.c_int, gp, ctypes.c_double, _dp, ctypes.c_int,
                                        _dp, _dp]),
            "omb_efield": (ctypes.c_int, [vp, ctypes.c_int, gp, ctypes.c_double, _dp, _dp, _dp]),
            "omb_hfield": (ctypes.c_int, [vp, gp, ctypes.c_double, ctypes.c_int, _dp, _dp]),
            "omb_gram_blocks": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int64, ctypes.c_int32, _dp, _dp, _dp, _dp]),
            "omb_autotune": (ctypes.c_int, [vp, gp, ctypes.c_int32] + [ctypes.POINTER(ctypes.c_int32)] * 3 + [_dp]),
            "omb_ctx_set_autotune": (ctypes.c_int, [vp, ctypes.c_int32]),
            "omb_tune_set": (ctypes.c_int, [ctypes.c_char_p] + [ctypes.c_int32] * 5),
            "omb_tune_get": (ctypes.c_int, [ctypes.c_char_p, ctypes.c_int32, ctypes.c_int32]
                             + [ctypes.POINTER(ctypes.c_int32)] * 3),
            "omb_tune_clear": (ctypes.c_int, []),
            "omb_tune_save": (ctypes.c_int, [ctypes.c_char_p]),
            "omb_tune_load": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ctypes.c_int32)]),
        }
        for name, (res, args) in sig.items():
            f = getattr(lib, name)
            f.restype = res
            f.argtypes = args
        for declare in _DECLARERS:
            declare(lib)
        _lib = lib
        return lib


def check(rc: int) -> None:
    if rc != OMB_OK:
        msg = load().omb_last_error().decode("utf-8", "replace")
        raise OmbError(rc, msg)


def dptr(a: np.ndarray):
    return a.ctypes.data_as(_dp)


class Context:
    """One libomb200 context (a CUDA stream, twiddle tables, a memory pool) per device."""

    def __init__(self, device: int = 0):
        lib = load()
        h = ctypes.c_void_p()
        check(lib.omb_ctx_create(int(device), ctypes.byref(h)))
        self.handle = h
        self.device = int(device)

    def close(self):
        if self.handle:
            load().omb_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover - interpreter shutdown order
        try:
            if not finalizing():
                self.close()
        except Exception:
            pass


_contexts: dict = {}


def context(device: int = 0) -> Context:
    c = _contexts.get(device)
    if c is None or c.handle is None:
        c = Context(device)
        _contexts[device] = c
    return c


class c_options(ctypes.Structure):
    _fields_ = [("k_tol", ctypes.c_double), ("eig_tol", ctypes.c_double),
                ("max_eigsolves", ctypes.c_int32), ("maxiter", ctypes.c_int32),
                ("precision", ctypes.c_int32), ("preconditioner", ctypes.c_int32),
                ("newton", ctypes.c_int32), ("canonicalize", ctypes.c_int32),
                ("seed", ctypes.c_uint64), ("guard_bands", ctypes.c_int32),
                ("warm_start", ctypes.c_int32)]


class c_instance(ctypes.Structure):
    _fields_ = [("grid", c_grid), ("omega", ctypes.c_double), ("epsinv", _dp),
                ("nev", ctypes.c_int32), ("kguess", ctypes.c_double), ("Hguess", _dp),
                ("nguess", ctypes.c_int32), ("kguess_bands", _dp)]


_ip = ctypes.POINTER(ctypes.c_int32)


class c_result(ctypes.Structure):
    _fields_ = [("kmags", _dp), ("evecs", _dp), ("residuals", _dp), ("dw2dk", _dp),
                ("status", _ip), ("iterations", _ip), ("newton_steps", _ip)]


def _declare_solve(lib):
    vp = ctypes.c_void_p
    sig = {
        "omb_options_default": (ctypes.c_int, [ctypes.POINTER(c_options)]),
        "omb_solve_k": (ctypes.c_int, [vp, ctypes.POINTER(c_instance), ctypes.c_int,
                                       ctypes.POINTER(c_options), ctypes.POINTER(c_result)]),
        "omb_solve_omega2": (ctypes.c_int, [vp, ctypes.POINTER(c_grid), ctypes.c_double, _dp,
                                            ctypes.c_int, _dp, ctypes.c_int,
                                            ctypes.POINTER(c_options), _dp, _dp, _dp, _ip]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


EXPORTS = EXPORTS + ("omb_options_default", "omb_solve_k", "omb_solve_omega2")
_DECLARERS = [_declare_solve]


class c_stats(ctypes.Structure):
    _fields_ = [("graph_launches", ctypes.c_int64), ("kernel_launches", ctypes.c_int64),
                ("h2d_bytes", ctypes.c_int64), ("d2h_bytes", ctypes.c_int64),
                ("tracks", ctypes.c_int32), ("max_iterations", ctypes.c_int32),
                ("run_seconds", ctypes.c_double)]


def _declare_batch(lib):
    vp = ctypes.c_void_p
    sig = {
        "omb_batch_create": (ctypes.c_int, [vp, ctypes.POINTER(c_instance), ctypes.c_int,
                                            ctypes.POINTER(c_options), ctypes.POINTER(vp)]),
        "omb_batch_run": (ctypes.c_int, [vp]),
        "omb_batch_results": (ctypes.c_int, [vp, ctypes.POINTER(c_result)]),
        "omb_batch_stats": (ctypes.c_int, [vp, ctypes.POINTER(c_stats)]),
        "omb_batch_destroy": (ctypes.c_int, [vp]),
        "omb_profile_apply": (ctypes.c_int, [vp, ctypes.c_int, ctypes.c_int, ctypes.POINTER(c_grid),
                                             ctypes.c_double, _dp, ctypes.c_int, ctypes.c_int,
                                             ctypes.c_int, _dp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


EXPORTS = EXPORTS + ("omb_batch_create", "omb_batch_run", "omb_batch_results", "omb_batch_stats",
                     "omb_batch_destroy", "omb_profile_apply")
_DECLARERS.append(_declare_batch)


def _declare_noalloc(lib):
    f = lib.omb_apply_M_noalloc
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_int32, ctypes.c_int32, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                  ctypes.c_void_p, ctypes.c_int32, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]


EXPORTS = EXPORTS + ("omb_apply_M_noalloc",)
_DECLARERS.append(_declare_noalloc)


def _declare_pullback(lib):
    f = lib.omb_pullback
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.POINTER(c_grid), ctypes.c_double, _dp, ctypes.c_int, _dp, _dp,
                  _dp, _dp, ctypes.POINTER(c_options), _dp, _dp, _dp, _ip]


EXPORTS = EXPORTS + ("omb_pullback",)
_DECLARERS.append(_declare_pullback)


def _declare_smoothing(lib):
    vp = ctypes.c_void_p
    i32p = ctypes.POINTER(ctypes.c_int32)
    sig = {
        "omb_smoothing_plan_create": (ctypes.c_int, [vp, ctypes.POINTER(c_grid), ctypes.c_int32, i32p, _dp, i32p,
                                                     ctypes.c_int32, ctypes.POINTER(vp)]),
        "omb_smoothing_plan_query": (ctypes.c_int, [vp, ctypes.POINTER(ctypes.c_int64),
                                                    ctypes.POINTER(ctypes.c_uint8), i32p, _dp, _dp]),
        "omb_smooth_eps": (ctypes.c_int, [vp, _dp, ctypes.c_int32, ctypes.c_int32, _dp, _dp]),
        "omb_smooth_eps_device": (ctypes.c_int, [vp, _dp, ctypes.c_int32, ctypes.c_int32, vp, vp, vp]),
        "omb_smooth_eps_vjp": (ctypes.c_int, [vp, _dp, ctypes.c_int32, ctypes.c_int32, _dp, _dp]),
        "omb_smooth_scalar": (ctypes.c_int, [vp, _dp, ctypes.c_int32, _dp]),
        "omb_smoothing_plan_destroy": (ctypes.c_int, [vp]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


EXPORTS = EXPORTS + ("omb_smoothing_plan_create", "omb_smoothing_plan_query", "omb_smooth_eps",
                     "omb_smooth_eps_device", "omb_smooth_eps_vjp", "omb_smooth_scalar",
                     "omb_smoothing_plan_destroy")
_DECLARERS.append(_declare_smoothing)


def _declare_diag(lib):
    f = lib.omb_ctx_set_wait_limit
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.c_double]
    f = lib.omb_selftest_wait
    f.restype = ctypes.c_int
    f.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_int32)]


EXPORTS = EXPORTS + ("omb_ctx_set_wait_limit", "omb_selftest_wait")
_DECLARERS.append(_declare_diag)


def set_wait_limit(seconds: float, device: int = 0) -> None:
    """Limit (seconds) of the streaming kernels' bounded waits on this device's context."""
    check(load().omb_ctx_set_wait_limit(context(device).handle, float(seconds)))
