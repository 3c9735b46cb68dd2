"""The sharded average on the GPU: two ranks (processes on one GPU, gloo for
the exchange) each warp their shard of the frames with the CUDA kernel
(msgpu_warp_sum_device), the per-pixel sums and counts are all-reduced, and
msgpu_mean_from_sums_device divides.  The result is the single-process
average (msgpu_warp_mean over all frames): counts equal, means equal up to
the order of the per-pixel sums.  No kernel of one rank waits for the other
(the exchange is on the host), so the two processes can share the GPU."""
import os
import socket

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, frames, phis, level, out_q):
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.join(os.path.dirname(here), "match-series_b200"))
    import torch
    import torch.distributed as dist
    import msgpu
    from msgpu import dist as mdist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = list(mdist.shard(frames.shape[0], rank, world))
    n = (1 << level) + 1
    N = n * n
    dev = torch.device("cuda", 0)
    ctx = msgpu.Context(0)
    d_fr = torch.from_numpy(np.ascontiguousarray(frames[mine])).to(dev)
    d_ph = torch.from_numpy(np.ascontiguousarray(phis[mine])).to(dev)
    d_sum = torch.empty(N, dtype=torch.float64, device=dev)
    d_cnt = torch.zeros(N + 1, dtype=torch.float64, device=dev)
    last = rank == world - 1
    ctx.warp_sum_device(level, d_fr.data_ptr(), d_ph.data_ptr(), len(mine), d_sum.data_ptr(), d_cnt.data_ptr(),
                        d_cnt[N:].data_ptr() if last else 0)
    torch.cuda.synchronize(dev)
    s, c = d_sum.cpu(), d_cnt.cpu()
    dist.all_reduce(s)
    dist.all_reduce(c)
    d_sum.copy_(s)
    d_cnt.copy_(c)
    d_mean = torch.empty(N, dtype=torch.float64, device=dev)
    ctx.mean_from_sums_device(level, d_sum.data_ptr(), d_cnt.data_ptr(), d_cnt[N:].data_ptr(), d_mean.data_ptr())
    torch.cuda.synchronize(dev)
    out_q.put((rank, mine, d_mean.cpu().numpy(), c[:N].numpy()))
    ctx.close()
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_sharded_average_matches_single_process_average(gpu):
    import multiprocessing as mp
    level = 7
    n = (1 << level) + 1
    rng = np.random.default_rng(3)
    F = 5
    frames = rng.uniform(0, 50, size=(F, n * n))
    phis = rng.normal(0, 4.0 / (n - 1), size=(F, 2, n * n))   # some samples leave the domain
    ref_mean, ref_count = gpu.warp_mean(level, frames, phis)
    assert (ref_count < F).any()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, frames, phis, level, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=300) for _ in range(2))
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert res[0][1] + res[1][1] == list(range(F))
    for _, _, mean, count in res:
        assert np.array_equal(count, ref_count)
        assert np.abs(mean - ref_mean).max() <= 1e-12 * np.abs(ref_mean).max()
