#!/usr/bin/env python
"""Benchmark: converged modes/s at residual 1e-8 on 256² LiNbO₃ ridge cross-sections.

One *step* is one batched ``solve_k`` over a fixed batch of synthetic cross-sections of the
x-cut LiNbO₃ ridge family (8×5 μm cell, 256×256 grid, 4 bands, film 0.6 μm, etch 0.3 μm,
70° sidewalls, top widths {1.0, 1.5, 2.0} μm, ω = 1/λ with λ stepping by 0.025 μm around
1.55 μm: {1.50, 1.525, 1.55, 1.575} on one GPU, ω = 1/1.55 always included), solved
with the batched, mixed-precision, inner-Newton B200 solver.  ``value`` counts converged
modes (Newton |Δk| < 1e-8 and FP64 residual < 1e-8) per device second with the inputs
resident (``omb_batch_run``); ``e2e`` is the same metric through ``omb_solve_k`` with host
buffers (upload, solve, download, phase canonicalisation).  The plain arm (one instance,
FP64, the reference's band-by-band Newton loop) runs on the same GPU for comparison.

``--impl reference`` times the reference algorithm's CPU restatement (the FP64 oracle,
NumPy/SciPy with every host thread) on the same workload: each step solves one mode.

Launch: ``python bench.py [--gpus 1] [--steps K] [--warmup W]``; for N>1 through
``torch.distributed.run`` (one rank per GPU, every rank solves its own batch: weak scaling,
no data-path collective).
"""

from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "optimode.jl_b200"))

METRIC = "converged modes/s at residual 1e-8, 256² grid: batched+warm-start vs plain"
UNIT = "modes/s"
NX = NY = 256
DX, DY = 8.0, 5.0
NEV = 4
WIDTHS = (1.0, 1.5, 2.0)
FALLBACK_HBM_GBS = 6650.0


def rank_omegas(n_om: int, rank: int = 0, world: int = 1):
    """The ω values of one rank: the whole job sweeps n_om·world wavelengths
    λ_j = 1.55 + 0.025·(j − ⌊n_om·world/2⌋) μm (so ω = 1/1.55, the oracle's comparison point,
    is always in the job, on rank ⌊world/2⌋) and rank r takes the r-th contiguous block of
    n_om (weak scaling: every rank gets the same amount of work, no two ranks solve the same
    instance)."""
    n = n_om * world
    lam = 1.55 + 0.025 * (np.arange(n) - n // 2)
    return (1.0 / lam)[rank * n_om:(rank + 1) * n_om]


def ridge_epsinv(g, width: float, smoothing: str = "gpu"):
    """Smoothed ε⁻¹ of the LiNbO₃ ridge of top width `width`: the library's device smoothing,
    or (for the CPU arms, which must not run this library) the oracle's CPU restatement,
    which the GPU tests hold bit-identical to it."""
    from omb200 import geometry as G
    shapes, bg = G.ln_ridge_shapes(g, top_width=width)
    if smoothing == "gpu":
        return G.smooth_epsinv(shapes, bg, g)
    sys.path.insert(0, ROOT)
    import oracle.smoothing as OS
    return OS.smooth_epsinv_constant(shapes, bg, g)


def workload(n_inst: int, rank: int = 0, world: int = 1, smoothing: str = "gpu"):
    from omb200 import Grid
    g = Grid(DX, DY, NX, NY)
    n_w = len(WIDTHS)
    n_om = max(1, (n_inst + n_w - 1) // n_w)
    omegas = rank_omegas(n_om, rank, world)
    eps = {w: ridge_epsinv(g, w, smoothing) for w in WIDTHS}
    probs = []
    for i in range(n_inst):
        w = WIDTHS[i % n_w]
        om = omegas[(i // n_w) % n_om]
        probs.append({"omega": float(om), "eps_inv": eps[w], "grid": g, "nev": NEV})
    return g, probs


def combine_ranks(times, counts, dist=None, device="cpu"):
    """Whole-job numbers from each rank's own: every entry of `times` maxed over ranks (the
    slowest rank's device and end-to-end seconds) and every entry of `counts` summed over
    ranks (converged modes).  Every rank calls this once, at the same point, so the
    collectives line up."""
    times = [float(x) for x in times]
    counts = [int(x) for x in counts]
    if dist is None:
        return times, counts
    import torch
    t = torch.tensor(times, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    c = torch.tensor(counts, dtype=torch.int64, device=device)
    dist.all_reduce(c, op=dist.ReduceOp.SUM)
    return [float(x) for x in t.tolist()], [int(x) for x in c.tolist()]


def sample_clocks(stop: threading.Event, out: list, index: int):
    q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    while not stop.is_set():
        try:
            r = subprocess.run(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                "-i", str(index)], capture_output=True, text=True, timeout=5)
            if r.returncode == 0 and r.stdout.strip():
                out.append([x.strip() for x in r.stdout.strip().split(",")])
        except Exception:
            pass
        stop.wait(0.2)


def clock_summary(samples):
    if not samples:
        return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
    sm = [float(s[1]) for s in samples if s[1].replace(".", "").isdigit()]
    mx = [float(s[2]) for s in samples if s[2].replace(".", "").isdigit()]
    reasons = set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    for s in samples:
        for name, v in zip(names, s[5:9]):
            if v.strip().lower() == "active":
                reasons.add(name)
    return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
            "reasons": sorted(reasons), "samples": len(samples)}


def measured_peak_hbm():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one roofline launch of the
# operator apply (4 columns x 64 cells of 256x256, FP32) with the tiles the autotuner picks on
# B200 (row variant 4, column variant 1), from an ncu capture of
#   python bench.py --case apply --steps 3 --apply-cells 16 --tiles 4,1,0
# (the three passes k_row_in_sp / k_col2 / k_row_out_sp, 416.7 MB per 16-cell apply) scaled
# by the cells processed (x4).  A fixed per-apply constant of the current kernels: bench runs
# are never profiled, and the figure changes only when the apply kernels change.
APPLY_TRAFFIC_BYTES = 1.6669e9


def smoothing_materials(n_shapes: int, nsets: int) -> np.ndarray:
    """(27, n_shapes + 1, nsets) material columns for the ridge's shapes and air: the
    cross-section's ε with a seeded synthetic dispersion, one set per frequency."""
    from omb200 import geometry as G
    rng = np.random.default_rng(7)
    base = [np.diag(G.EPS_LN_XCUT), np.diag(G.EPS_LN_XCUT), G.EPS_SIO2 * np.eye(3), np.eye(3)][:n_shapes + 1]
    d1 = [np.diag(rng.uniform(0.05, 0.2, 3)) for _ in base]
    d2 = [np.diag(rng.uniform(-0.1, 0.1, 3)) for _ in base]
    sets = []
    for s in range(nsets):
        dw = (s - nsets / 2) * 1e-3
        sets.append(np.stack([G.material_column(e + d * dw + dd * dw * dw / 2, d + dd * dw, dd)
                              for e, d, dd in zip(base, d1, d2)], axis=1))
    return np.stack(sets, axis=2)


def smoothing_measure(device: int, nsets: int = 64, reps: int = 10):
    """Device Kottke smoothing of the bench cross-section (the 1.5 um LiNbO3 ridge, 256x256):
    the geometry plan once, then the material pass for `nsets` frequencies (27 values
    (eps, d eps/d omega, d2 eps/d omega2) and the fused inverse per pixel, 1.2 GB written per
    launch, above L2) timed with CUDA events on its stream; beside it the same pass through
    the host-buffer C ABI call and the oracle's CPU restatement on one frequency."""
    import torch
    import omb200
    from omb200 import geometry as G
    g = omb200.Grid(DX, DY, NX, NY)
    shapes, _ = G.ln_ridge_shapes(g, top_width=1.5)
    minds = list(range(len(shapes) + 1))
    M = smoothing_materials(len(shapes), nsets)
    G.SmoothingPlan(shapes, minds, g, device=device).close()  # library and context set-up
    torch.cuda.synchronize(device)
    t0 = time.perf_counter()
    plan = G.SmoothingPlan(shapes, minds, g, device=device)
    plan_s = time.perf_counter() - t0
    N = g.N
    de = torch.empty(27 * N * nsets, dtype=torch.float64, device=f"cuda:{device}")
    di = torch.empty(9 * N * nsets, dtype=torch.float64, device=f"cuda:{device}")
    st = torch.cuda.Stream(device)
    for _ in range(3):
        plan.smooth_eps_device(M, de, di, stream=st)
    st.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(reps):
        plan.smooth_eps_device(M, de, di, stream=st)
    e1.record(st)
    e1.synchronize()
    t = e0.elapsed_time(e1) / 1e3 / reps
    nu, ni, nm = plan.counts
    alg = nsets * (296 * N + 24 * ni)  # writes 27+9 doubles, reads the 8 B code (+24 B geometry)
    peak, peak_kind = measured_peak_hbm()
    t0 = time.perf_counter()
    plan.smooth_eps(M, eps=True, epsinv=True)
    e2e = time.perf_counter() - t0
    plan.close()
    del de, di
    sys.path.insert(0, ROOT)
    import oracle.smoothing as OS
    t0 = time.perf_counter()
    oplan = OS.smoothing_plan(shapes, minds, g)
    t1 = time.perf_counter()
    OS.epsinv_of(OS.apply_plan(oplan, M[:, :, 0]), g)
    t2 = time.perf_counter()
    return {"what": f"Kottke smoothing of the 1.5 um ridge, {NX}x{NY}, {nsets} frequency sets per launch",
            "pixels": {"uniform": nu, "interface": ni, "multi": nm},
            "plan_seconds": plan_s, "apply_seconds_per_launch": t, "pixel_sets_per_s": N * nsets / t,
            "roofline": {"bound": "hbm", "achieved": alg / t / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": alg / t / 1e9 / peak, "algorithmic_bytes_per_launch": alg,
                         "peak_source": peak_kind},
            "e2e_seconds_host_buffers": e2e,
            "cpu_oracle": {"plan_seconds": t1 - t0, "apply_seconds_per_set": t2 - t1, "cores": 1,
                           "kind": "port"}}


def cpu_baseline_and_errors(probs, results, infos):
    """The FP64 oracle (the reference algorithm restated in NumPy/SciPy, all host threads for
    the FFTs) as the timed CPU baseline and as the checker of the device results.

    Timed: one mode of the workload, band 0 of the 1.5 μm ridge at ω = 1/1.55.  Checked:
    that mode's k, group index n_g = 2ω/(∂ω²/∂k) and field against the device's result for
    the same instance, and for every device result (all instances and bands of the step) the
    residual ‖M̂h − ω²h‖ of the returned unit eigenvector under the oracle's FP64 operator,
    with the a-posteriori bounds it gives for a Hermitian operator: eigenvalue error
    ≤ r²/gap and so |δk| ≤ r²/(gap·∂ω²/∂k), field angle ≤ r/gap, the gap to the instance's
    other computed bands estimated to first order in k."""
    sys.path.insert(0, ROOT)
    import oracle as O
    og = O.Grid(DX, DY, NX, NY)
    cores = os.cpu_count() or 1
    O.maxwell.FFT_WORKERS = cores
    from omb200 import Grid
    ei = ridge_epsinv(Grid(DX, DY, NX, NY), 1.5, "oracle")
    t0 = time.perf_counter()
    kr, vr = O.solve_k(1 / 1.55, ei, og, nev=1)
    dt = time.perf_counter() - t0
    base = {"value": 1.0 / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "sample": f"1 converged mode (band 0, 1.5 um ridge, omega=1/1.55, 256^2) in {dt:.1f} s"}
    # the device's result for the same instance (same ε⁻¹: the device smoothing is held
    # bit-identical to the oracle's by the GPU tests; compared here by value)
    errs = {"vs_oracle_solve": None}
    for pr, (km, kv), inf in zip(probs, results, infos):
        if abs(pr["omega"] - 1 / 1.55) < 1e-15 and np.array_equal(np.asarray(pr["eps_inv"]), ei):
            d_ref = 2 * O.Operator(kr[0], ei, og).HMkH(vr[0])
            ng_ref = 2 * pr["omega"] / d_ref
            ng = 2 * pr["omega"] / inf["dw2dk"][0]
            errs["vs_oracle_solve"] = {
                "instance": "1.5 um ridge, omega=1/1.55, band 0",
                "rel_err_k": abs(km[0] - kr[0]) / kr[0], "rel_err_neff": abs(km[0] - kr[0]) / kr[0],
                "rel_err_ng": abs(ng - ng_ref) / ng_ref,
                "field_err": float(np.sqrt(max(0.0, 1 - abs(np.vdot(vr[0], kv[0])) ** 2)))}
            break
    worst = {"resid": 0.0, "k_bound": 0.0, "field_bound": 0.0}
    per = []
    for pr, (km, kv), inf in zip(probs, results, infos):
        w2 = pr["omega"] ** 2
        e = np.asarray(pr["eps_inv"])
        for b in range(len(km)):
            r = float(np.linalg.norm(O.Operator(km[b], e, og).M(kv[b]) - w2 * kv[b]))
            # gap at k_b to the instance's other computed bands, to first order in k:
            # ω_j²(k_b) − ω² ≈ (k_b − k_j)·(∂ω²/∂k)_j
            gaps = [abs(km[b] - km[j]) * inf["dw2dk"][j] for j in range(len(km)) if j != b]
            gap = min(gaps) if gaps else w2
            kb = r * r / gap / inf["dw2dk"][b]
            per.append({"omega": pr["omega"], "band": b, "resid": r,
                        "k_err_bound": kb / km[b], "field_angle_bound": r / gap})
            worst["resid"] = max(worst["resid"], r)
            worst["k_bound"] = max(worst["k_bound"], kb / km[b])
            worst["field_bound"] = max(worst["field_bound"], r / gap)
    errs.update({"results_checked": len(per), "max_resid_oracle_fp64": worst["resid"],
                 "max_rel_err_k_bound": worst["k_bound"], "max_field_angle_bound": worst["field_bound"],
                 "note": "residuals of the device's unit eigenvectors under the oracle's FP64 operator "
                         "at the device's k; bounds r^2/gap (eigenvalue, then k via d omega^2/dk) "
                         "and r/gap (field angle)"})
    return base, errs


def _solve_bytes(p) -> float:
    """Device bytes of one problem's tracks (FP64 + FP32 blocks [X W P] and A·[X W P], two
    parities), to cut large batches into chunks that fit in HBM."""
    g = p["grid"]
    n2 = 2 * g.Nx * g.Ny
    cols = sum(b + 2 for b in range(p["nev"]))
    return 288.0 * n2 * cols


def _chunks(probs, budget: float):
    """Consecutive chunks under `budget` bytes that keep each shared ε⁻¹ array (a sweep group)
    in one chunk."""
    groups, order = {}, []
    for p in probs:
        key = id(p["eps_inv"])
        if key not in groups:
            groups[key] = []
            order.append(key)
        groups[key].append(p)
    chunks, cur, cur_b = [], [], 0.0
    for key in order:
        gb = sum(_solve_bytes(p) for p in groups[key])
        if cur and cur_b + gb > budget:
            chunks.append(cur)
            cur, cur_b = [], 0.0
        cur += groups[key]
        cur_b += gb
    if cur:
        chunks.append(cur)
    return chunks


def _solve_chunks(chunks, solver):
    """Device seconds (CUDA events of each omb_batch_run), wall seconds of the whole
    create/run/results path with host buffers, converged modes, modes and iterations."""
    import omb200
    dev, conv, modes, iters = 0.0, 0, 0, []
    t0 = time.perf_counter()
    for ch in chunks:
        b = omb200.Batch(ch, solver)
        b.run()
        dev += b.stats()["run_seconds"]
        _, info = b.results(return_info=True, raise_on_failure=False)
        b.close()
        conv += int(sum(int(np.sum(i["status"] == 0)) for i in info))
        modes += int(sum(len(i["status"]) for i in info))
        iters += [int(x) for i in info for x in i["iterations"]]
    wall = time.perf_counter() - t0
    return {"device_seconds": dev, "e2e_seconds": wall, "converged": conv, "modes": modes,
            "modes_per_s": conv / dev, "e2e_modes_per_s": conv / wall,
            "iterations_mean": float(np.mean(iters)), "iterations_max": int(max(iters))}


def config3_measure(device: int):
    """The uneven batch: 512 problems (64 ω in [0.5, 1.0] μm⁻¹ × 8 ridge widths in [0.6, 2.4]
    μm, grids {128², 192×128, 256×192, 256²}, 2–6 bands, Si₃N₄ / LiNbO₃ / Si cores, seed 3),
    solved in HBM-sized chunks of whole sweep groups, from random starts and with the sweep
    warm start, mixed precision, residual 1e-8."""
    import omb200
    from omb200 import workloads as W
    probs = W.sweep_batch(device=device)
    chunks = _chunks(probs, 40e9)
    out = {"case": "config3", "problems": len(probs), "modes": sum(p["nev"] for p in probs), "chunks": len(chunks),
           "grids": sorted({(p["grid"].Nx, p["grid"].Ny) for p in probs})}
    for warm in ("sweep", "none"):
        solver = omb200.B200Solver(precision="mixed", warm_start=warm, device=device)
        _solve_chunks(chunks[:1], solver)  # warm-up (tuning, allocation caches)
        out[warm] = _solve_chunks(chunks, solver)
    return out


def config5_measure(device: int, n_inst: int = 16, per_chunk: int = 4):
    """Large instances: 512², 8 bands, seeded slot / coupled-waveguide rows (seeds 0..15),
    solved in chunks of `per_chunk` with the learned warm start (when trained parameters are
    present) and the FP32 + FP64 polish, then each instance's pull-back of a seeded cotangent
    to ∂ε⁻¹ and ∂ω: k̄ on all 8 bands (the n_eff sensitivities) and ē on the fundamental band
    (a mode-overlap objective).  A random ē on every band is not used: these rows hold
    near-degenerate supermode pairs, for which (M̂ − ω²) is ill-conditioned on the
    complement of the band's own mode and the adjoint solve does not reach 1e-8 in thousands
    of iterations (nor does the reference's GMRES, which returns its iterate after 1000)."""
    import omb200
    from omb200 import workloads as W
    from omb200.warmstart import WEIGHTS_PATH
    cells = [W.slot_cell(s, 512, device=device) for s in range(n_inst)]
    probs = [{"omega": 1 / 1.55, "eps_inv": e, "grid": g, "nev": 8} for g, e in cells]
    warm = "learned" if os.path.exists(WEIGHTS_PATH) else "none"
    solver = omb200.B200Solver(precision="mixed", warm_start=warm, device=device)
    chunks = [probs[i:i + per_chunk] for i in range(0, len(probs), per_chunk)]
    _solve_chunks(chunks[:1], solver)
    res = _solve_chunks(chunks, solver)
    # pull-back of every instance (one chunk's results at a time)
    t_adj, n_adj, n_ok, its, fails = 0.0, 0, 0, [], []
    rng = np.random.default_rng(5)
    for ch in chunks:
        sols = omb200.solve_k_batch(ch, solver, raise_on_failure=False)
        for p, (km, kv) in zip(ch, sols):
            kbar = rng.standard_normal(8)
            evbar = [rng.standard_normal(kv[0].size) + 1j * rng.standard_normal(kv[0].size)] + [None] * 7
            t0 = time.perf_counter()
            try:
                _, _, info = omb200.pullback(p["omega"], p["eps_inv"], p["grid"], km, kv, kbar, evbar,
                                             solver=solver, return_info=True)
                n_ok += 1
                its.append(int(info["iterations"][0]))
            except omb200.OmbError as exc:
                fails.append(str(exc)[:160])
            t_adj += time.perf_counter() - t0
            n_adj += 1
    return {"case": "config5", "instances": n_inst, "nev": 8, "grid": [512, 512], "warm_start": warm,
            "solve": res, "pullback_seconds_per_instance": t_adj / max(n_adj, 1),
            "pullback_converged": n_ok, "pullback_minres_iterations_band0": its, "pullback_failures": fails,
            "pullback_what": "seeded k-bar on all 8 bands and e-bar on band 0, host buffers, FP64 MINRES"}


def tc_gemm_measure(device: int, reps: int = 20):
    """The learned warm start's widest GEMM on the tensor cores (32 images: M = 32·32·32
    output pixels, N = 256 channels, K = 9·128, BF16 in, FP32 accumulation in TMEM, bias +
    ReLU, BF16 out), timed with CUDA events over `reps` launches, against measured BF16 peak."""
    import torch
    from omb200.warmstart import tc_gemm
    M, N, K = 32768, 256, 1152
    gen = torch.Generator(device=f"cuda:{device}").manual_seed(0)
    A = torch.randn(M, K, device=f"cuda:{device}", generator=gen).to(torch.bfloat16)
    B = torch.randn(N, K, device=f"cuda:{device}", generator=gen).to(torch.bfloat16)
    bias = torch.randn(N, device=f"cuda:{device}", generator=gen)
    D = torch.empty(M, N, device=f"cuda:{device}", dtype=torch.bfloat16)
    for _ in range(3):
        tc_gemm(A, B, D, M, N, K, N, bias=bias, relu=True, epi=1, device=device)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(device)
    e0.record()
    for _ in range(reps):
        tc_gemm(A, B, D, M, N, K, N, bias=bias, relu=True, epi=1, device=device)
    e1.record()
    torch.cuda.synchronize(device)
    s = e0.elapsed_time(e1) / reps * 1e-3
    ref = (A.float() @ B.float().T + bias).relu()
    err = float((D.float() - ref).abs().max() / ref.abs().max())
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = json.load(f).get("bf16_tflops")
    except OSError:
        pass
    tf = 2.0 * M * N * K / s / 1e12
    return {"case": "tc_gemm", "M": M, "N": N, "K": K, "seconds_per_gemm": s, "tflops": tf,
            "peak_bf16_tflops": peak, "frac": tf / peak if peak else None, "max_rel_err_vs_fp32": err,
            "note": "each call synchronises the device before its launch (the Python wrapper), so this is a lower bound"}


def run_reference(args, rank):
    if rank != 0:
        return
    sys.path.insert(0, ROOT)
    import oracle as O
    from omb200 import Grid
    g, probs = workload(max(args.instances, 1), smoothing="oracle")
    cores = os.cpu_count() or 1
    O.maxwell.FFT_WORKERS = cores
    og = O.Grid(DX, DY, NX, NY)

    def step(i):
        pr = probs[i % len(probs)]
        O.solve_k(pr["omega"], pr["eps_inv"], og, nev=1)

    for i in range(args.warmup):
        step(i)
    t0 = time.perf_counter()
    for i in range(args.steps):
        step(args.warmup + i)
    dt = time.perf_counter() - t0
    v = args.steps / dt
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * dt / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded LiNbO3 ridge cross-sections, Kottke-smoothed)",
        "config": {"workload": "LiNbO3 ridge 8x5um 256x256, band 0 per step (one converged mode)",
                   "grid": [NX, NY], "nev": 1},
        "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "port",
                         "sample": f"{args.steps} modes, one per step, scipy.fft workers={cores}"},
        "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--instances", type=int, default=12)
    ap.add_argument("--e2e-steps", type=int, default=None, help="end-to-end steps (default: --steps)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-smoothing", action="store_true")
    ap.add_argument("--case", default="full",
                    choices=["full", "apply", "solve1", "batch", "smoothing", "tc_gemm", "config3", "config5"],
                    help="apply / solve1 / batch / smoothing: one operator-apply timing, one "
                         "single-instance solve, one batched solve of --instances cells, or the "
                         "smoothing measurement with --smoothing-sets frequency sets (small, "
                         "self-contained runs for profiling); tc_gemm: the warm-start network's "
                         "widest tensor-core GEMM; config3: the 512-problem uneven "
                         "batch; config5: sixteen 512x512 8-band slot cells with their pull-backs")
    ap.add_argument("--apply-cells", type=int, default=64)
    ap.add_argument("--tiles", default=None,
                    help="apply case: row,col,wave tile variants to time (default: the tuned or default tiles)")
    ap.add_argument("--smoothing-sets", type=int, default=64)
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return run_reference(args, rank)
    if args.case == "config3":
        print(json.dumps(config3_measure(local)), flush=True)
        return
    if args.case == "config5":
        print(json.dumps(config5_measure(local)), flush=True)
        return
    if args.case == "smoothing":
        print(json.dumps({"case": "smoothing", **smoothing_measure(local, nsets=args.smoothing_sets,
                                                                    reps=args.steps)}))
        return
    if args.case == "tc_gemm":
        print(json.dumps(tc_gemm_measure(local, reps=max(args.steps, 10))))
        return
    if args.case != "full":
        import omb200
        g, probs = workload(args.instances if args.case == "batch" else 1)
        if args.case == "apply":
            tiles = None
            if args.tiles:
                import torch
                from omb200 import ops
                tiles = [int(x) for x in args.tiles.split(",")]
                ops.tune_set(torch.cuda.get_device_name(local), NX, NY, *tiles)
            t = omb200.profile_apply("M", 1.3, probs[0]["eps_inv"], g, NEV, args.apply_cells, reps=args.steps)
            print(json.dumps({"case": "apply", "seconds_per_apply": t, "cells": args.apply_cells, "ncol": NEV,
                              "tiles": tiles}))
        else:
            b = omb200.Batch(probs, omb200.B200Solver(device=local, warm_start="sweep"))
            b.run()
            _, info = b.results(return_info=True, raise_on_failure=False)
            print(json.dumps({"case": args.case, **{k: v for k, v in b.stats().items()},
                              "iterations": [i["iterations"].tolist() for i in info]}))
            b.close()
        return

    import torch
    dist = None
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    import omb200
    # batched + warm start: each ridge's ω values form a sweep whose anchor starts from the
    # learned network (OMB_WARM_SWEEP_LEARNED; OMB_WARM_SWEEP without trained parameters)
    from omb200.warmstart import WEIGHTS_PATH
    headline_warm = "sweep_learned" if os.path.exists(WEIGHTS_PATH) else "sweep"
    solver = omb200.B200Solver(precision="mixed", preconditioner="diag", newton="inner", device=local,
                               warm_start=headline_warm)
    g, probs = workload(args.instances, rank, world)
    batch = omb200.Batch(probs, solver)

    def barrier():
        torch.cuda.synchronize(local)
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        batch.run()
    barrier()
    stop = threading.Event()
    samples: list = []
    th = threading.Thread(target=sample_clocks, args=(stop, samples, local), daemon=True)
    th.start()
    dev_s = 0.0
    kernels = 0
    converged = 0
    for _ in range(args.steps):
        batch.run()
        st = batch.stats()
        dev_s += st["run_seconds"]  # CUDA events around the device run on the library stream
        kernels += st["kernel_launches"]
        # this step's converged modes (the download is outside the device-timed region)
        _, info = batch.results(return_info=True, raise_on_failure=False)
        converged += int(sum(int(np.sum(i["status"] == 0)) for i in info))
    barrier()
    stop.set()
    th.join(timeout=5)
    batch.close()

    # end to end through the public C ABI call with host buffers, every step's converged
    # modes counted from its own results
    e2e_steps = args.e2e_steps if args.e2e_steps is not None else args.steps
    e2e_s = 0.0
    e2e_conv = 0
    res = info = None
    for _ in range(e2e_steps):
        barrier()
        t0 = time.perf_counter()
        res, info = omb200.solve_k_batch(probs, solver, raise_on_failure=False, return_info=True)
        torch.cuda.synchronize(local)
        e2e_s += time.perf_counter() - t0
        e2e_conv += int(sum(int(np.sum(i["status"] == 0)) for i in info))
    # byte counts of one end-to-end step from a staged run of the same batch, and where its
    # host-side time goes (validation + uploads, device run, canonicalisation + downloads)
    t0 = time.perf_counter()
    b4 = omb200.Batch(probs, solver)
    torch.cuda.synchronize(local)
    t1 = time.perf_counter()
    b4.run()
    torch.cuda.synchronize(local)
    t2 = time.perf_counter()
    b4.results(raise_on_failure=False)
    t3 = time.perf_counter()
    st4 = b4.stats()
    h2d, d2h = st4["h2d_bytes"], st4["d2h_bytes"]
    b4.close()
    e2e_parts = {"create_s": t1 - t0, "run_s": t2 - t1, "run_device_s": st4["run_seconds"], "results_s": t3 - t2}
    (max_dev_s, max_e2e_s), (converged_all, e2e_conv_all) = combine_ranks(
        [dev_s, e2e_s], [converged, e2e_conv], dist, f"cuda:{local}")
    value = converged_all / max_dev_s
    e2e_val = e2e_conv_all / max_e2e_s

    out = None
    if rank == 0:
        # roofline of the fused operator apply (3 passes) on the bench grid, 4 columns per
        # cell, 64 cells (≈1.3 GB resident, far above L2)
        N = NX * NY
        ncol, nbatch = NEV, 64
        t_apply = omb200.profile_apply("M", 1.3, probs[0]["eps_inv"], g, ncol, nbatch, reps=20,
                                       precision="fp32", device=local)
        alg = (32 * N * ncol + 24 * N) * nbatch
        peak, peak_kind = measured_peak_hbm()
        achieved = alg / t_apply / 1e9
        traffic = APPLY_TRAFFIC_BYTES
        # the same launch against FP32 issue: nominal flops 5·N·log2(N) per complex 2D transform
        # (six per column: three components, forward and inverse) + ≈60·N for the basis, curls
        # and the ε⁻¹ contraction; FP32 peak from the SM count and the maximum SM clock
        flops = (30.0 * N * np.log2(N) + 60.0 * N) * ncol * nbatch
        fp32_peak = 148 * 128 * 2 * 1.965e9 / 1e12
        roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                    "frac": achieved / peak, "traffic": traffic,
                    "kernel": "operator apply M(k) (row_in + col + row_out, FP32), 4 columns x 64 cells",
                    "algorithmic_bytes_per_launch": alg, "seconds_per_launch": t_apply,
                    "peak_source": peak_kind,
                    "fp32": {"flops_per_launch": flops, "achieved_tflops": flops / t_apply / 1e12,
                             "peak_tflops": fp32_peak, "frac": flops / t_apply / 1e12 / fp32_peak,
                             "peak_source": "nominal: 148 SMs x 128 FP32 lanes x 2 x 1965 MHz"}}
        plain = None
        if not args.no_plain:
            # the reference loop's per-eigensolve budget is raised so that it converges
            # every band from its random start
            ps = omb200.B200Solver(precision="fp64", preconditioner="diag", newton="outer", device=local)
            pb = omb200.Batch(probs[:1], ps, maxiter=3000)
            pb.run()
            pst = pb.stats()
            _, pinfo = pb.results(return_info=True, raise_on_failure=False)
            pconv = int(np.sum(pinfo[0]["status"] == 0))
            plain = {"value": pconv / pst["run_seconds"], "unit": UNIT,
                     "what": "one instance, FP64, reference band-by-band Newton loop, same kernels",
                     "seconds": pst["run_seconds"], "converged": pconv}
            pb.close()
        # the same batch from the other starts: random (none) and the learned network
        arms = {}
        for warm in [w for w in ("none", "learned", "sweep", "sweep_learned") if w != headline_warm]:
            try:
                ab = omb200.Batch(probs, omb200.B200Solver(precision="mixed", preconditioner="diag", newton="inner",
                                                           device=local, warm_start=warm))
                ab.run()
                ast = ab.stats()
                _, ainfo = ab.results(return_info=True, raise_on_failure=False)
                ab.close()
                aconv = int(sum(int(np.sum(i["status"] == 0)) for i in ainfo))
                arms[warm] = {"modes_per_s": aconv / ast["run_seconds"], "device_seconds": ast["run_seconds"],
                              "converged": aconv,
                              "iterations_mean": float(np.mean([x for i in ainfo for x in i["iterations"]]))}
            except Exception as exc:  # e.g. no trained parameters in this checkout
                arms[warm] = {"unavailable": str(exc)[:200]}
        arms[headline_warm] = {"modes_per_s": value, "device_seconds": max_dev_s / args.steps,
                         "converged": converged_all / args.steps,
                         "iterations_mean": float(np.mean([x for i in info for x in i["iterations"]]))}
        from omb200 import ops as _ops
        try:
            tuned = dict(zip(("row", "col", "wave"), _ops.tune_get(torch.cuda.get_device_name(local), NX, NY)))
        except Exception:
            tuned = None
        roofline["tuned_tiles"] = tuned
        cpu, errors = (None, None) if args.no_cpu_baseline or world > 1 else cpu_baseline_and_errors(probs, res, info)
        smoothing = None if args.no_smoothing else smoothing_measure(local, nsets=args.smoothing_sets)
        out = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * max_dev_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "fp32+fp64",
            "data": "synthetic (seeded LiNbO3 ridge cross-sections, Kottke-smoothed eps)",
            "config": {"workload": f"x-cut LiNbO3 ridge, 8x5 um cell, {NX}x{NY}, {NEV} bands, "
                                   f"{len(probs)} instances per GPU (widths {list(WIDTHS)} x omega)",
                       "instances_per_gpu": len(probs), "nev": NEV, "grid": [NX, NY],
                       "precision": "mixed (FP32 iterations, FP64 polish)", "tol": 1e-8, "k_tol": 1e-8,
                       "warm_start": ("per-ridge omega sweep: the instance nearest the mean omega is solved first"
                                      + (" from the learned network's fields and n_eff" if headline_warm == "sweep_learned"
                                         else "") +
                                      ", the others start from its device-resident eigenvectors and a first-order k"),
                       "l2": "working set per step is GBs (inputs larger than L2)",
                       "parallelism": f"instances sharded, {world} rank(s)"},
            "converged_modes_per_step": converged_all / args.steps, "modes_per_step": len(probs) * NEV * world,
            "e2e": {"value": e2e_val, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "steps": e2e_steps, "staged_step_breakdown": e2e_parts},
            "gpu_launches": int(kernels),
            "roofline": roofline,
            "plain_fp64_single": plain,
            "warm_start_arms": arms,
            "smoothing": smoothing,
            "cpu_baseline": cpu,
            "errors_vs_oracle": errors,
            "clocks": clock_summary(samples),
        }
        print(json.dumps(out), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
