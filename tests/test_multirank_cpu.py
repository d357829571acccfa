"""The N>1 path of bench.py on CPU: two ``gloo`` ranks (world size 2), no GPU.

``bench.py --gpus N`` shards the job by instances: every rank solves its own block of the
frequency sweep (weak scaling, no data-path collective) and the only collectives are the
final reductions — the slowest rank's device and end-to-end times (max) and the converged
modes of all ranks (sum).  These tests run that sharding and that reduction with real
process groups on the host."""

from __future__ import annotations

import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

import bench


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, q):
    import datetime

    import torch.distributed as dist

    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        # every rank builds its own shard of the job exactly as bench.py does (ε⁻¹ from the
        # oracle's smoothing here, the device smoothing on a GPU box: bit-identical)
        g, probs = bench.workload(12, rank, world, smoothing="oracle")
        shard = sorted((round(1 / p["omega"], 6), float(np.sum(p["eps_inv"]))) for p in probs)
        # per-rank timings and counts; the reduction must give the max / sum over ranks
        times, counts = [1.0 + rank, 2.0 + 3 * rank], [10 * (rank + 1), 7 + rank]
        out = bench.combine_ranks(times, counts, dist, "cpu")
        om = bench.rank_omegas(4, rank, world)
        q.put((rank, out, om.tolist(), shard))
    finally:
        dist.barrier()
        dist.destroy_process_group()


def test_two_rank_reduction_and_sharding():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    got = [q.get(timeout=120) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    got.sort(key=lambda x: x[0])
    for rank, out, _, _ in got:
        # max of device and e2e times over ranks, sum of converged modes
        assert out == ([2.0, 5.0], [30, 15])
    oms = [np.array(o) for _, _, o, _ in got]
    assert len(set(oms[0]) & set(oms[1])) == 0                       # disjoint shards
    assert np.allclose(np.sort(np.concatenate(oms)), np.sort(bench.rank_omegas(8, 0, 1)))  # cover the job
    shards = [set(s) for _, _, _, s in got]
    assert all(len(s) == 12 for s in shards) and not (shards[0] & shards[1])
    # 3 ridge widths × 8 wavelengths over the job; ω = 1/1.55 (the oracle's check) on one rank
    assert len(shards[0] | shards[1]) == 24
    assert sum(any(abs(lam - 1.55) < 1e-9 for lam, _ in s) for s in shards) == 1


def test_single_rank_is_identity_and_one_shard():
    assert bench.combine_ranks([1.5, 2.5], [7, 3]) == ([1.5, 2.5], [7, 3])
    assert np.allclose(1 / bench.rank_omegas(4, 0, 1), [1.50, 1.525, 1.55, 1.575])
