"""FP32 CPU restatement of the learned warm-start network (TEST INFRASTRUCTURE ONLY).

The network has no counterpart in OptiMode.jl (the reference starts LOBPCG from random
blocks or the caller's ``Hguess``, ``ME/src/solve.jl:201-210``); this module restates the
device network of ``optimode.jl_b200/csrc/warmstart.cu`` in NumPy so the device forward
pass, loss and every layer's gradients can be checked against it.  BF16 rounding (round to
nearest even) is applied at the same points as on the device: the input image, the
weights, the im2col operand, every hidden activation after its ReLU, and both GEMM
operands of the backward pass (dZ and its transpose); accumulation is FP32 (NumPy float32
matmul), biases, losses and gradients FP32.

Parameter layout (``omb_warmstart_get_params``): per layer the weights [cout × 9·cin]
(column = tap·cin + c, taps row-major over the 3×3 window), then the cout biases.
"""

from __future__ import annotations

import numpy as np

LAYERS = [  # (cin, cout, stride, relu, upsample after, input side)
    (8, 64, 2, True, False, 128), (64, 128, 1, True, False, 64), (128, 256, 2, True, False, 64),
    (256, 256, 1, True, False, 32), (256, 128, 1, True, True, 32), (128, 12, 1, False, False, 64),
]
LAMBDA_N = 100.0
OUT = 64


def bf16(x: np.ndarray) -> np.ndarray:
    """Round FP32 values to BF16 (nearest even), returned as FP32."""
    a = np.ascontiguousarray(x, dtype=np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).reshape(a.shape)


def num_params() -> int:
    return sum(co * 9 * ci + co for ci, co, *_ in LAYERS)


def split_params(p: np.ndarray):
    out, off = [], 0
    for ci, co, *_ in LAYERS:
        w = p[off:off + co * 9 * ci].reshape(co, 9 * ci)
        off += co * 9 * ci
        b = p[off:off + co]
        off += co
        out.append((w, b))
    return out


def im2col(x: np.ndarray, stride: int) -> np.ndarray:
    """x (B, H, W, C) → (B·Ho·Wo, 9·C), column = tap·C + c, zero padding 1."""
    B, H, W, C = x.shape
    Ho, Wo = H // stride, W // stride
    xp = np.zeros((B, H + 2, W + 2, C), dtype=x.dtype)
    xp[:, 1:-1, 1:-1] = x
    cols = []
    for ky in range(3):
        for kx in range(3):
            cols.append(xp[:, ky:ky + stride * Ho:stride, kx:kx + stride * Wo:stride, :])
    return np.concatenate(cols, axis=-1).reshape(B * Ho * Wo, 9 * C)


def col2im(dA: np.ndarray, B: int, H: int, W: int, C: int, stride: int) -> np.ndarray:
    Ho, Wo = H // stride, W // stride
    dA = dA.reshape(B, Ho, Wo, 9, C)
    dxp = np.zeros((B, H + 2, W + 2, C), dtype=dA.dtype)
    for ky in range(3):
        for kx in range(3):
            dxp[:, ky:ky + stride * Ho:stride, kx:kx + stride * Wo:stride, :] += dA[:, :, :, 3 * ky + kx, :]
    return dxp[:, 1:-1, 1:-1]


def forward(params: np.ndarray, feat: np.ndarray):
    """feat (B, 128, 128, 8) → output (B·4096, 12) FP32 and the saved activations."""
    layers = split_params(params)
    x = bf16(feat)
    saved = []
    for (ci, co, s, relu, up, H), (w, b) in zip(LAYERS, layers):
        B = x.shape[0]
        A = bf16(im2col(x, s))
        z = A @ bf16(w).T + b
        Ho = H // s
        if relu:
            z = np.maximum(z, 0)
        saved.append((A, z, x.shape))
        if co == 12:
            return z, saved
        y = bf16(z).reshape(B, Ho, Ho, co)
        if up:
            y = y.repeat(2, axis=1).repeat(2, axis=2)
        x = y
    raise AssertionError


def loss_and_grad_out(out: np.ndarray, tfield: np.ndarray, tneff: np.ndarray):
    """Loss and ∂loss/∂out; out (B·4096, 12), tfield (B·4096, 8), tneff (B, 4)."""
    B = tneff.shape[0]
    o = out.reshape(B, OUT * OUT, 12).astype(np.float64)
    t = tfield.reshape(B, OUT * OUT, 8).astype(np.float64)
    g = np.zeros_like(o)
    loss = 0.0
    scale = 1.0 / (4 * B)
    for s in range(B):
        for b in range(4):
            p, tt = o[s, :, 2 * b:2 * b + 2], t[s, :, 2 * b:2 * b + 2]
            D, P, T = np.sum(p * tt), np.sum(p * p), np.sum(tt * tt)
            T = T if T > 0 else 1.0
            nbar = o[s, :, 8 + b].mean()
            dn = nbar - tneff[s, b]
            loss += ((P + T - 2 * abs(D)) / T + LAMBDA_N * dn * dn) * scale
            sg = 1.0 if D >= 0 else -1.0
            g[s, :, 2 * b:2 * b + 2] = 2.0 / T * scale * (p - sg * tt)
            g[s, :, 8 + b] = 2.0 * LAMBDA_N * dn / (OUT * OUT) * scale
    return loss, g.reshape(B * OUT * OUT, 12).astype(out.dtype)


def backward(params: np.ndarray, saved, gout: np.ndarray) -> np.ndarray:
    """Parameter gradients in the get_params layout."""
    layers = split_params(params)
    grads = [None] * len(LAYERS)
    dY = gout
    for l in range(len(LAYERS) - 1, -1, -1):
        ci, co, s, relu, up, H = LAYERS[l]
        w, _ = layers[l]
        A, z, xshape = saved[l]
        dZ = dY.copy()
        if relu:
            dZ[bf16(z) <= 0] = 0
        gb = dZ.sum(axis=0)
        gw = bf16(dZ).T @ A
        grads[l] = (gw, gb)
        if l == 0:
            break
        dA = bf16(dZ) @ bf16(w)
        B = xshape[0]
        dx = col2im(dA, B, H, H, ci, s)
        pci, pco, ps, prelu, pup, pH = LAYERS[l - 1]
        if pup:
            dx = dx.reshape(B, H // 2, 2, H // 2, 2, ci).sum(axis=(2, 4))
        dY = dx.reshape(-1, ci)
    return np.concatenate([np.concatenate([gw.ravel(), gb]) for gw, gb in grads])
