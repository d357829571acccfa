"""The learned warm start's device kernels against their CPU restatement.

* ``omb_tc_gemm`` (tcgen05 + TMA, BF16 operands, FP32 accumulation in tensor memory) against
  a NumPy FP32 product of the same BF16-rounded operands: every tile width (N = 12 … 1152,
  tails in M and N), bias + ReLU, BF16 stores and split-K atomics.  Tolerance: relative
  max-error 1e-5 (FP32 accumulation order only), BF16 stores within one BF16 ulp.
* The network's forward pass, loss and every layer's weight and bias gradients against
  ``oracle.warmstart`` (the same network in NumPy FP32 with BF16 rounding at the same points).
  Tolerances: output and loss 2e-3 relative, gradients 3e-2 relative L2 per layer (a hidden
  activation that rounds to the other BF16 neighbour on one side moves the later layers'
  gradients by about a BF16 ulp)."""

from __future__ import annotations

import numpy as np
import pytest

from oracle import warmstart as OW

pytestmark = pytest.mark.gpu


def _bf16_tensor(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.float32)).to(torch.bfloat16).cuda()


@pytest.mark.parametrize("M,N,K,relu,epi,splits", [
    (256, 64, 128, 0, 0, 1),
    (300, 12, 576, 1, 0, 1),      # M and N tails, N < 16
    (1000, 256, 1152, 1, 1, 1),   # BF16 store
    (130, 1152, 64, 0, 0, 1),     # several N tiles of 256
    (64, 576, 8192, 0, 2, 8),     # split-K with FP32 atomics (weight-gradient shape)
    (128, 128, 2304, 0, 0, 1),
])
def test_tc_gemm(M, N, K, relu, epi, splits):
    import torch
    from omb200.warmstart import tc_gemm
    rng = np.random.default_rng(M + N + K)
    A = OW.bf16(rng.standard_normal((M, K)).astype(np.float32))
    B = OW.bf16(rng.standard_normal((N, K)).astype(np.float32))
    bias = rng.standard_normal(N).astype(np.float32) if epi != 2 else None
    ref = A.astype(np.float64) @ B.T.astype(np.float64)
    if bias is not None:
        ref = ref + bias
    if relu:
        ref = np.maximum(ref, 0)
    dA, dB = _bf16_tensor(A), _bf16_tensor(B)
    db = torch.from_numpy(bias).cuda() if bias is not None else None
    if epi == 1:
        D = torch.zeros((M, N), dtype=torch.bfloat16, device="cuda")
    else:
        D = torch.zeros((M, N), dtype=torch.float32, device="cuda")
    tc_gemm(dA, dB, D, M, N, K, N, bias=db, relu=relu, epi=epi, splits=splits)
    got = D.float().cpu().numpy().astype(np.float64)
    scale = np.max(np.abs(ref)) + 1e-30
    if epi == 1:
        assert np.max(np.abs(got - ref) / (np.abs(ref) + 1e-3 * scale)) <= 2 ** -8 + 1e-6
    else:
        assert np.max(np.abs(got - ref)) / scale < 1e-5


def _batch(seed, B):
    rng = np.random.default_rng(seed)
    feat = np.zeros((B, 128, 128, 8), dtype=np.float32)
    feat[..., :6] = rng.uniform(0.05, 1.0, (B, 128, 128, 6))
    feat[..., 6] = rng.uniform(0.5, 1.0, (B, 1, 1))
    tf = rng.standard_normal((B * 4096, 8)).astype(np.float32)
    tn = rng.uniform(1.5, 2.2, (B, 4)).astype(np.float32)
    return feat, tf, tn


def test_network_forward_and_gradients_match_cpu():
    import torch
    from omb200.warmstart import WarmStartNet
    B = 2
    net = WarmStartNet(batch_cap=4, seed=3)
    p = net.get_params()
    assert p.size == OW.num_params()
    feat, tf, tn = _batch(5, B)
    dfeat = _bf16_tensor(feat.reshape(B, -1))
    dtf = torch.from_numpy(tf).cuda()
    dtn = torch.from_numpy(tn).cuda()
    out = torch.zeros((B * 4096, 16), dtype=torch.float32, device="cuda")
    net.forward(dfeat, B, out)
    ref_out, saved = OW.forward(p, feat)
    got = out.cpu().numpy()[:, :12]
    assert np.linalg.norm(got - ref_out) / np.linalg.norm(ref_out) < 2e-3
    loss, g = net.train_step(dfeat, dtf, dtn, B, 0.0, update=False, want_grads=True)
    ref_loss, gout = OW.loss_and_grad_out(ref_out, tf, tn)
    assert abs(loss - ref_loss) / abs(ref_loss) < 2e-3
    ref_g = OW.backward(p, saved, gout)
    off = 0
    for l, (ci, co, *_rest) in enumerate(OW.LAYERS):
        for part, n in (("W", co * 9 * ci), ("b", co)):
            a, r = g[off:off + n], ref_g[off:off + n]
            err = np.linalg.norm(a - r) / (np.linalg.norm(r) + 1e-30)
            assert err < 3e-2, f"layer {l + 1} {part}: rel err {err:.3e}"
            off += n


def test_training_reduces_the_loss_on_a_fixed_batch():
    import torch
    from omb200.warmstart import WarmStartNet
    B = 4
    net = WarmStartNet(batch_cap=4, seed=11)
    feat, tf, tn = _batch(9, B)
    dfeat = _bf16_tensor(feat.reshape(B, -1))
    dtf, dtn = torch.from_numpy(tf).cuda(), torch.from_numpy(tn).cuda()
    first = net.train_step(dfeat, dtf, dtn, B, 1e-3)
    for _ in range(30):
        last = net.train_step(dfeat, dtf, dtn, B, 1e-3)
    assert np.isfinite(last) and last < 0.5 * first, (first, last)


def test_learned_start_gains_on_heldout_cross_sections():
    """The committed trained network on 16 held-out seeded cross-sections (the training
    distribution, another seed), 128², 4 bands: every band reaches the same tolerance from the
    learned start as from a random start (same k to 1e-7), in fewer iterations and less device
    time (the network only changes the starting block)."""
    from omb200.train_warmstart import evaluate, heldout_problems
    ev = evaluate(heldout_problems(16, 4242, 128))
    none, learned = ev["none"], ev["learned"]
    assert learned["converged"] >= none["converged"] >= 60
    assert learned["max_rel_k_diff_vs_none"] < 1e-7
    assert learned["iterations_total"] < 0.97 * none["iterations_total"], ev


def test_sweep_with_learned_anchors():
    """``sweep_learned``: each sweep's anchor starts from the network, the other members from
    the anchor; the results equal the cold solves' (k to 1e-7) with every band converged, in
    fewer iterations than random starts."""
    import omb200
    from omb200.train_warmstart import heldout_problems
    base = heldout_problems(3, 777, 128)
    probs = [{**p, "omega": p["omega"] + d} for p in base for d in (-0.01, 0.0, 0.01)]
    out = {}
    for warm in ("none", "sweep", "sweep_learned"):
        res, info = omb200.solve_k_batch(probs, omb200.B200Solver(warm_start=warm), return_info=True,
                                         raise_on_failure=False)
        out[warm] = (np.array([r[0] for r in res]), sum(int(np.sum(i["iterations"])) for i in info),
                     all(np.all(i["status"] == 0) for i in info))
    for warm in ("sweep", "sweep_learned"):
        assert out[warm][2]
        assert np.max(np.abs(out[warm][0] - out["none"][0]) / out["none"][0]) < 1e-7
        assert out[warm][1] < out["none"][1]
