"""Train the learned warm start on solves the method itself generates.

    python -m omb200.train_warmstart [--samples 4096] [--epochs 12] [--out PATH]

1. Seeded random rib/ridge cross-sections (``random_ridge``): top width 0.4–3 μm, film
   0.2–1 μm, etch fraction 0.3–1, sidewall 60–90°, core ε from {3.98, x-cut LiNbO₃
   diag(4.97, 4.61, 4.97), 12.1}, SiO₂ substrate (2.09) and an upper cladding of 2.09 or 1.0,
   in an 8×5 μm cell on a 128×128 grid, ω uniform in [0.5, 1.0] μm⁻¹.
2. ε⁻¹ from the device Kottke smoothing; the four lowest bands from the device solver
   (mixed precision, random start, residual 1e-8).
3. Targets: each band's real-space transverse (Hx, Hy) from ``omb_hfield`` (rotated to its
   most real phase, averaged 2×2 to 64×64, scaled to unit RMS) and its n_eff = k/ω.
4. Training with the library's tensor-core forward/backward kernels and Adam
   (``omb_warmstart_train_step``), cosine learning-rate decay; the last 10 % of the samples
   are held out for the validation loss.
5. The FP32 parameters are written with the run's record (sizes, seeds, losses, timings).
"""

from __future__ import annotations

import argparse
import json
import os
import time

import numpy as np

from . import geometry as G
from .grid import Grid
from .warmstart import WEIGHTS_PATH, WarmStartNet

CELL = (8.0, 5.0)
NGRID = 128
EPS_CORES = [("Si3N4", G.diag_eps(3.98)), ("LiNbO3", G.diag_eps(4.97, 4.61, 4.97)), ("Si", G.diag_eps(12.1))]


def random_ridge(rng: np.random.Generator, grid: Grid):
    """(shapes, background ε, description) of one seeded rib/ridge cross-section."""
    width = rng.uniform(0.4, 3.0)
    film = rng.uniform(0.2, 1.0)
    etch = film * rng.uniform(0.3, 1.0)
    side = rng.uniform(60.0, 90.0)
    core_name, core = EPS_CORES[int(rng.integers(len(EPS_CORES)))]
    top = 2.09 if rng.random() < 0.5 else 1.0
    slab = film - etch
    y_sub = -film / 2
    big = 4 * max(grid.Dx, grid.Dy)
    shapes = [G.ridge(0.0, y_sub + slab, width, etch, min(side, 89.9), core)]
    if slab > 0.02:
        shapes.append(G.rectangle(0.0, y_sub + slab / 2, big, slab, core))
    shapes.append(G.rectangle(0.0, y_sub - big / 2, big, big, G.diag_eps(2.09)))
    desc = {"width": width, "film": film, "etch": etch, "sidewall": side, "core": core_name, "top": top}
    return shapes, G.diag_eps(top), desc


def transverse_targets(H_cart: np.ndarray, grid: Grid) -> np.ndarray:
    """(Hx, Hy) real parts at 64×64 with unit RMS from one band's real-space Cartesian field
    (flat (3, Nx, Ny) column-major complex), after rotating it to its most real phase."""
    f = H_cart.reshape(grid.Ny, grid.Nx, 3)  # [iy, ix, component]
    ht = f[..., :2]
    alpha = 0.5 * np.angle(np.sum(ht * ht))
    ht = (ht * np.exp(-1j * alpha)).real
    s = grid.Nx // 64
    ht = ht.reshape(64, s, 64, s, 2).mean(axis=(1, 3))  # [y, x, c]
    rms = np.sqrt(np.mean(np.sum(ht * ht, axis=-1)))
    return (ht / (rms if rms > 0 else 1.0)).astype(np.float32)


def generate(n: int, seed: int, batch: int = 64, device: int = 0, log=print):
    """Features (n, 128·128·8) BF16 on the device, field targets (n·4096, 8) and n_eff targets
    (n, 4) FP32 on the device, and the per-sample records (only fully converged samples)."""
    import torch

    import omb200
    net = WarmStartNet(batch_cap=1, device=device)  # for the feature kernel only
    grid = Grid(CELL[0], CELL[1], NGRID, NGRID)
    rng = np.random.default_rng(seed)
    feats, tfs, tns, recs = [], [], [], []
    solver = omb200.B200Solver(precision="mixed", warm_start="none", device=device, seed=seed)
    t0 = time.perf_counter()
    made = 0
    while made < n:
        probs, descs = [], []
        for _ in range(min(batch, n - made)):
            shapes, bg, desc = random_ridge(rng, grid)
            desc["omega"] = float(rng.uniform(0.5, 1.0))
            ei = G.smooth_epsinv(shapes, bg, grid, device=device)
            probs.append({"omega": desc["omega"], "eps_inv": ei, "grid": grid, "nev": 4})
            descs.append(desc)
        res, info = omb200.solve_k_batch(probs, solver, return_info=True, raise_on_failure=False)
        for pr, (km, kv), inf, desc in zip(probs, res, info, descs):
            if not np.all(inf["status"] == 0):
                continue
            tf = np.zeros((64, 64, 8), dtype=np.float32)
            for b in range(4):
                Hc = omb200.H_field(km[b], grid, kv[b], device=device)
                tf[..., 2 * b:2 * b + 2] = transverse_targets(Hc, grid)
            ei_dev = torch.from_numpy(np.asfortranarray(pr["eps_inv"]).ravel(order="F")).to(f"cuda:{device}")
            f = torch.empty(128 * 128 * 8, dtype=torch.bfloat16, device=f"cuda:{device}")
            net.features(ei_dev, NGRID, NGRID, pr["omega"], f)
            feats.append(f)
            tfs.append(tf.reshape(4096, 8))
            tns.append((km / pr["omega"]).astype(np.float32))
            recs.append({**desc, "kmags": km.tolist(), "iterations": inf["iterations"].tolist()})
        made += len(probs)
        log(f"  generated {made}/{n} ({len(recs)} converged) in {time.perf_counter() - t0:.0f} s")
    net.close()
    F = torch.stack(feats)
    TF = torch.from_numpy(np.concatenate(tfs)).to(f"cuda:{device}")
    TN = torch.from_numpy(np.stack(tns)).to(f"cuda:{device}")
    return F, TF, TN, recs, time.perf_counter() - t0


def train(F, TF, TN, epochs: int, batch: int = 32, lr: float = 1e-3, seed: int = 0, device: int = 0, log=print):
    import torch
    n = F.shape[0]
    nval = max(batch, n // 10)
    ntr = n - nval
    net = WarmStartNet(batch_cap=batch, seed=seed, device=device)
    rng = np.random.default_rng(seed)
    steps = epochs * (ntr // batch)
    hist = []
    t0 = time.perf_counter()
    step = 0
    for ep in range(epochs):
        perm = rng.permutation(ntr)
        tot = 0.0
        for i in range(ntr // batch):
            idx = torch.from_numpy(perm[i * batch:(i + 1) * batch]).to(F.device)
            fb = F.index_select(0, idx).contiguous()
            tfb = TF.view(n, 4096, 8).index_select(0, idx).contiguous()
            tnb = TN.index_select(0, idx).contiguous()
            cur = lr * 0.5 * (1 + np.cos(np.pi * step / max(steps, 1)))
            tot += net.train_step(fb, tfb, tnb, batch, cur)
            step += 1
        vl = 0.0
        nb = nval // batch
        for i in range(nb):
            sl = slice(ntr + i * batch, ntr + (i + 1) * batch)
            vl += net.train_step(F[sl].contiguous(), TF.view(n, 4096, 8)[sl].contiguous(), TN[sl].contiguous(),
                                 batch, 0.0, update=False)
        hist.append({"epoch": ep + 1, "train_loss": tot / max(1, ntr // batch), "val_loss": vl / max(nb, 1)})
        log(f"  epoch {ep + 1}: train {hist[-1]['train_loss']:.4f}  val {hist[-1]['val_loss']:.4f}  "
            f"({time.perf_counter() - t0:.0f} s)")
    return net, hist, time.perf_counter() - t0


def heldout_problems(n: int, seed: int, ngrid: int = NGRID, device: int = 0):
    """n seeded held-out cross-sections (the training distribution, another seed)."""
    grid = Grid(CELL[0], CELL[1], ngrid, ngrid)
    rng = np.random.default_rng(seed)
    probs = []
    for _ in range(n):
        shapes, bg, desc = random_ridge(rng, grid)
        om = float(rng.uniform(0.5, 1.0))
        probs.append({"omega": om, "eps_inv": G.smooth_epsinv(shapes, bg, grid, device=device), "grid": grid,
                      "nev": 4})
    return probs


def evaluate(probs, device: int = 0, d_omega: float = 0.01, chunk: int = 64):
    """Iterations to the 1e-8 tolerance and device seconds of batched solves of `probs` (in
    batches of `chunk` instances) from three starts: random (``none``), the learned network
    (``learned``), and the previous frequency's converged modes (``previous_omega``: each
    problem solved first at ω − d_omega, untimed, then at ω from those eigenvectors and
    k·ω/ω_prev).  Every arm is checked to converge every band, and the arms' k to agree."""
    import omb200
    out = {}
    ks = {}

    def run(arm, problems, solver):
        secs, conv, its, kk = 0.0, 0, [], []
        for i in range(0, len(problems), chunk):
            b = omb200.Batch(problems[i:i + chunk], solver)
            b.run()
            secs += b.stats()["run_seconds"]
            res, info = b.results(return_info=True, raise_on_failure=False)
            b.close()
            conv += int(sum(int(np.sum(x["status"] == 0)) for x in info))
            its += [int(x) for r in info for x in r["iterations"]]
            kk += [r[0] for r in res]
        out[arm] = {"device_seconds": secs, "converged": conv, "modes": 4 * len(problems),
                    "iterations_total": int(sum(its)), "iterations_mean": float(np.mean(its)),
                    "iterations_max": int(max(its))}
        ks[arm] = np.array(kk)

    run("none", probs, omb200.B200Solver(precision="mixed", warm_start="none", device=device))
    run("learned", probs, omb200.B200Solver(precision="mixed", warm_start="learned", device=device))
    prev = [{**p, "omega": p["omega"] - d_omega} for p in probs]
    pres = []
    for i in range(0, len(prev), chunk):
        pres += omb200.solve_k_batch(prev[i:i + chunk], omb200.B200Solver(precision="mixed", device=device),
                                     raise_on_failure=False)
    warm = [{**p, "Hguess": np.stack(kv, axis=1), "kguess_bands": km * p["omega"] / q["omega"]}
            for p, q, (km, kv) in zip(probs, prev, pres)]
    run("previous_omega", warm, omb200.B200Solver(precision="mixed", warm_start="none", device=device))
    for arm in ("learned", "previous_omega"):
        out[arm]["max_rel_k_diff_vs_none"] = float(np.max(np.abs(ks[arm] - ks["none"]) / ks["none"]))
    out["instances"] = len(probs)
    out["grid"] = [probs[0]["grid"].Nx, probs[0]["grid"].Ny]
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=4096)
    ap.add_argument("--epochs", type=int, default=12)
    ap.add_argument("--batch", type=int, default=32)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=20)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=WEIGHTS_PATH)
    ap.add_argument("--heldout", type=int, default=64, help="held-out cross-sections evaluated after training")
    ap.add_argument("--heldout-256", type=int, default=None,
                    help="held-out cross-sections on 256² grids (default: as --heldout)")
    args = ap.parse_args()
    print(f"generating {args.samples} samples (seed {args.seed})", flush=True)
    F, TF, TN, recs, t_gen = generate(args.samples, args.seed, device=args.device,
                                      log=lambda s: print(s, flush=True))
    print(f"training on {F.shape[0]} converged samples", flush=True)
    net, hist, t_train = train(F, TF, TN, args.epochs, args.batch, args.lr, args.seed, args.device,
                               log=lambda s: print(s, flush=True))
    os.makedirs(os.path.dirname(os.path.abspath(args.out)), exist_ok=True)
    record = {"samples_requested": args.samples, "samples_converged": int(F.shape[0]), "seed": args.seed,
              "epochs": args.epochs, "batch": args.batch, "lr": args.lr, "grid": [NGRID, NGRID], "cell_um": CELL,
              "generate_seconds": t_gen, "train_seconds": t_train, "history": hist}
    np.savez_compressed(args.out, params=net.get_params(), record=json.dumps(record))
    print(json.dumps({k: v for k, v in record.items() if k != "history"}), flush=True)
    print(f"final val loss {hist[-1]['val_loss']:.4f}; wrote {args.out}", flush=True)
    if args.heldout > 0:
        net.attach()
        for ngrid, n in ((128, args.heldout), (256, args.heldout if args.heldout_256 is None else args.heldout_256)):
            if n > 0:
                ev = evaluate(heldout_problems(n, args.seed + 1000, ngrid, args.device), args.device)
                print("heldout", json.dumps(ev), flush=True)


if __name__ == "__main__":
    main()
