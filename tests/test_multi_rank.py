"""Sharding of a stage across ranks (gloo, world size 2, CPU): the union of the
shards is the series, and the all-reduced average equals the single-process
average of the oracle."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, frames, phis, level, out_q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    sys.path.insert(0, os.path.join(root, "match-series_b200"))
    sys.path.insert(0, os.path.join(root, "oracle"))
    import torch
    import torch.distributed as dist
    import msor
    from msgpu import dist as mdist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = mdist.shard(frames.shape[0], rank, world)
    warped = np.stack([msor.deform_image(level, frames[f], phis[f, 0], phis[f, 1]) for f in mine])
    s, c = mdist.warped_sum_count(warped)

    def ar(a):
        t = torch.from_numpy(np.ascontiguousarray(a))
        dist.all_reduce(t)
        return t.numpy()

    mean, count = mdist.reduce_mean(s, c, float(frames[-1].mean()), all_reduce=ar)
    out_q.put((rank, list(mine), mean, count))
    dist.barrier()
    dist.destroy_process_group()


def test_shards_cover_series():
    from msgpu import dist as mdist
    for F in (1, 5, 20):
        for W in (1, 2, 3, 8):
            got = [f for r in range(W) for f in mdist.shard(F, r, W)]
            assert got == list(range(F))


def test_two_rank_average_matches_single_process(oracle):
    import multiprocessing as mp
    level = 5
    n = (1 << level) + 1
    rng = np.random.default_rng(0)
    frames = rng.uniform(0, 50, size=(5, n * n))
    phis = rng.normal(0, 2.0 / (n - 1), size=(5, 2, n * n))
    ref_mean, ref_count = oracle.warp_mean(level, frames, phis)
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, frames, phis, level, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = [q.get(timeout=120) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    res.sort()
    assert res[0][1] + res[1][1] == list(range(5))
    for _, _, mean, count in res:
        assert np.array_equal(count, ref_count)
        assert np.abs(mean - ref_mean).max() <= 1e-12 * np.abs(ref_mean).max()
