"""Learned warm start: binding of the tensor-core network in ``libomb200`` (``omb_warmstart_*``
and ``omb_tc_gemm`` in ``include/omb200.h``).

``WarmStartNet`` owns one device network (six BF16 3×3 convolutions, FP32 accumulation on
the tensor cores) and exposes its forward pass, its training step (forward, loss, backward
and Adam, all in the library's kernels) and its parameters.  Device buffers are torch
tensors (plumbing only: every operation on them runs in the library).  The network maps
the ε⁻¹ map and ω of a 128², 256² or 512² cross-section to initial (Hx, Hy) fields and effective
indices of the four lowest bands; ``omb200.solver`` feeds them to the eigensolver as its
starting block (``warm_start="learned"``).
"""

from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _lib

OUT_SIDE = 64
OUT_LD = 16
IN_SIDE = 128
IN_CH = 8

_vp = ctypes.c_void_p
_fp = ctypes.POINTER(ctypes.c_float)


def _declare(lib):
    sig = {
        "omb_warmstart_create": (ctypes.c_int, [_vp, ctypes.c_int32, ctypes.c_uint64, ctypes.POINTER(_vp)]),
        "omb_warmstart_destroy": (ctypes.c_int, [_vp]),
        "omb_warmstart_num_params": (ctypes.c_int64, []),
        "omb_warmstart_get_params": (ctypes.c_int, [_vp, _fp]),
        "omb_warmstart_set_params": (ctypes.c_int, [_vp, _fp]),
        "omb_warmstart_features": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_double, _vp, _vp]),
        "omb_warmstart_forward": (ctypes.c_int, [_vp, _vp, ctypes.c_int32, _vp]),
        "omb_warmstart_train_step": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int32, ctypes.c_float, ctypes.c_int32,
                                                    _fp, _fp]),
        "omb_ctx_set_warmstart": (ctypes.c_int, [_vp, _vp]),
        "omb_tc_gemm": (ctypes.c_int, [_vp, _vp, _vp, _vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32,
                                       ctypes.c_int64, _vp, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args


_lib.EXPORTS = _lib.EXPORTS + ("omb_warmstart_create", "omb_warmstart_destroy", "omb_warmstart_num_params",
                               "omb_warmstart_get_params", "omb_warmstart_set_params", "omb_warmstart_features",
                               "omb_warmstart_forward", "omb_warmstart_train_step", "omb_tc_gemm",
                               "omb_ctx_set_warmstart")
_lib._DECLARERS.append(_declare)

#: committed trained parameters (FP32, the get_params layout), if present
WEIGHTS_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warmstart_net.npz")


def tc_gemm(A, B, D, M: int, N: int, K: int, ldd: int, bias=None, relu=False, epi=0, splits=1, device: int = 0):
    """D = A·Bᵀ (+bias, ReLU) on the tensor cores; A, B, D, bias are device tensors."""
    import torch
    torch.cuda.synchronize(device)
    lib = _lib.load()
    _lib.check(lib.omb_tc_gemm(_lib.context(device).handle, A.data_ptr(), B.data_ptr(), D.data_ptr(), M, N, K, ldd,
                               bias.data_ptr() if bias is not None else None, int(relu), int(epi), int(splits)))


class WarmStartNet:
    def __init__(self, batch_cap: int = 32, seed: int = 0, device: int = 0):
        self._lib = _lib.load()
        self.device = device
        self.ctx = _lib.context(device)
        h = _vp()
        _lib.check(self._lib.omb_warmstart_create(self.ctx.handle, int(batch_cap), int(seed), ctypes.byref(h)))
        self.handle = h
        self.batch_cap = batch_cap

    @staticmethod
    def num_params() -> int:
        return int(_lib.load().omb_warmstart_num_params())

    def get_params(self) -> np.ndarray:
        p = np.zeros(self.num_params(), dtype=np.float32)
        _lib.check(self._lib.omb_warmstart_get_params(self.handle, p.ctypes.data_as(_fp)))
        return p

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        if p.size != self.num_params():
            raise ValueError(f"expected {self.num_params()} parameters, got {p.size}")
        _lib.check(self._lib.omb_warmstart_set_params(self.handle, p.ctypes.data_as(_fp)))

    def load(self, path: str = WEIGHTS_PATH) -> None:
        self.set_params(np.load(path)["params"])

    def _sync(self):
        import torch
        torch.cuda.synchronize(self.device)

    def features(self, eps_inv_dev, Nx: int, Ny: int, omega: float, out):
        """One input image into the BF16 device tensor `out` (128·128·8 elements) from a device
        FP64 ε⁻¹ tensor in the (3, 3, Nx, Ny) column-major layout."""
        self._sync()
        _lib.check(self._lib.omb_warmstart_features(self.handle, eps_inv_dev.data_ptr(), Nx, Ny, float(omega),
                                                    out.data_ptr(), None))

    def forward(self, feat, batch: int, out):
        self._sync()
        _lib.check(self._lib.omb_warmstart_forward(self.handle, feat.data_ptr(), int(batch), out.data_ptr()))

    def train_step(self, feat, tfield, tneff, batch: int, lr: float, update: bool = True, want_grads: bool = False):
        self._sync()
        loss = ctypes.c_float(0)
        g = np.zeros(self.num_params(), dtype=np.float32) if want_grads else None
        _lib.check(self._lib.omb_warmstart_train_step(self.handle, feat.data_ptr(), tfield.data_ptr(),
                                                      tneff.data_ptr(), int(batch), float(lr), int(update),
                                                      ctypes.byref(loss), g.ctypes.data_as(_fp) if g is not None else None))
        return (float(loss.value), g) if want_grads else float(loss.value)

    def attach(self) -> None:
        """Make this network the one ``warm_start="learned"`` solves use on its device."""
        _lib.check(self._lib.omb_ctx_set_warmstart(self.ctx.handle, self.handle))
        _attached[self.device] = self

    def close(self):
        if self.handle:
            if _attached.get(self.device) is self:
                del _attached[self.device]
            self._lib.omb_warmstart_destroy(self.handle)
            self.handle = None

    def __del__(self):  # pragma: no cover
        try:
            if not _lib.finalizing():
                self.close()
        except Exception:
            pass


_attached: dict = {}


def ensure_attached(device: int = 0) -> WarmStartNet:
    """The network attached on `device`; if none is, one with the committed trained
    parameters (``WEIGHTS_PATH``) is created and attached."""
    net = _attached.get(device)
    if net is None or net.handle is None:
        if not os.path.exists(WEIGHTS_PATH):
            raise FileNotFoundError(f"no trained warm-start parameters at {WEIGHTS_PATH}; train them with "
                                    "`python -m omb200.train_warmstart` or attach a WarmStartNet")
        net = WarmStartNet(batch_cap=32, device=device)
        net.load()
        net.attach()
    return net
