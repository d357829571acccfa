"""The CPU restatement of the warm-start network (``oracle.warmstart``), which the device
gradients are checked against, is itself checked here: with the BF16 rounding switched off
its backward pass equals central finite differences of its loss (FP64 arithmetic), for
weights and biases of every layer.""" 

from __future__ import annotations

import numpy as np

from oracle import warmstart as OW


def test_cpu_network_backward_matches_finite_differences(monkeypatch):
    monkeypatch.setattr(OW, "bf16", lambda x: np.asarray(x, dtype=np.float64))
    rng = np.random.default_rng(0)
    B = 1
    n = OW.num_params()
    p = np.zeros(n)
    off = 0
    for ci, co, *_ in OW.LAYERS:
        p[off:off + co * 9 * ci] = rng.standard_normal(co * 9 * ci) * np.sqrt(2.0 / (9 * ci))
        off += co * 9 * ci
        p[off:off + co] = rng.standard_normal(co) * 0.1
        off += co
    feat = np.zeros((B, 128, 128, 8))
    feat[..., :6] = rng.uniform(0.05, 1.0, (B, 128, 128, 6))
    feat[..., 6] = 0.7
    tf = rng.standard_normal((B * 4096, 8))
    tn = rng.uniform(1.5, 2.2, (B, 4))

    def loss_of(q):
        out, _ = OW.forward(q, feat)
        return OW.loss_and_grad_out(out, tf, tn)[0]

    out, saved = OW.forward(p, feat)
    _, gout = OW.loss_and_grad_out(out, tf, tn)
    g = OW.backward(p, saved, gout.astype(np.float64))
    # one weight and the bias of one channel in every layer
    idx, off = [], 0
    for ci, co, *_ in OW.LAYERS:
        idx += [off + int(rng.integers(co * 9 * ci)), off + co * 9 * ci + int(rng.integers(co))]
        off += co * 9 * ci + co
    for i in idx:
        # a ReLU kink crossed by the step spoils a difference quotient; with two steps at
        # least one is kink-free (checked: the kink-free quotients agree to ~1e-8)
        errs = []
        for h in (1e-5, 1e-7):
            e = np.zeros(n)
            e[i] = h
            fd = (loss_of(p + e) - loss_of(p - e)) / (2 * h)
            errs.append(abs(fd - g[i]) / max(abs(g[i]), 1e-3))
        assert min(errs) <= 1e-5, (i, errs, g[i])
