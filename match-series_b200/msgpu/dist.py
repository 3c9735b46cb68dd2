"""Multi-GPU layout of one stage of series matching.

The registrations of a stage are independent (every frame against the fixed
reference, matchSeries.h:141-155, 223-245), so the frames are sharded across
ranks without any exchange.  The only collective is the reconstruction: each
rank warps its own frames and the per-pixel sums of finite samples and their
counts are summed over ranks with one all-reduce (averageSeries,
matchSeries.h:410-425); pixels without any sample take the mean of the
series' last frame.  On the GPU the per-rank part is msgpu_warp_sum_device
and the division msgpu_mean_from_sums_device (Context.warp_sum_device,
Context.mean_from_sums_device); the helpers below are the same steps on host
arrays.
"""
from __future__ import annotations

import numpy as np


def shard(num_frames: int, rank: int, world: int) -> range:
    """Contiguous block of frames owned by `rank` (sizes differ by at most one)."""
    base, extra = divmod(num_frames, world)
    start = rank * base + min(rank, extra)
    return range(start, start + base + (1 if rank < extra else 0))


def warped_sum_count(warped: np.ndarray):
    """Per-pixel sum over the finite (non-Inf) samples and their count."""
    finite = warped != np.inf
    return np.where(finite, warped, 0.0).sum(axis=0), finite.sum(axis=0).astype(np.float64)


def reduce_mean(local_sum, local_count, last_frame_mean: float, all_reduce=None):
    """Combines the ranks' partial sums/counts (all_reduce sums tensors in place)."""
    s, c = local_sum, local_count
    if all_reduce is not None:
        s, c = all_reduce(s), all_reduce(c)
    mean = np.where(c > 0, s / np.maximum(c, 1), last_frame_mean)
    return mean, c
