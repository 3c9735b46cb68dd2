"""The learned warm start end to end: training pairs generated and registered
by the plain GPU method, training of the network (msgpu_net_train_step), and
registration started from its prediction against the plain start.

Training pair = (prepared reference and template at the network's input
level l0, the plain method's displacement at the warm level l0-1).  The
target is the plain method's own solution of the coarse levels startLevel ..
l0-1 (a batch with stopLevel = precisionLevel = l0-1 on the full-size
images): exactly the displacement the plain multilevel run carries into level
l0-1, which the warm start replaces.  Device memory holds the whole set;
tensors are torch (device memory and streams only).
"""
from __future__ import annotations

import time

import numpy as np

from . import Context, Net, default_params, n_of
from . import synthetic as syn


def pair_params(level: int, warm_level: int, start_level: int, max_iter: int, fp64: bool, lam: float = 0.1):
    """Parameters of the plain method on images of `level` solved up to warm_level (the targets)."""
    return default_params(precision_level=warm_level, input_level=level, start_level=start_level,
                          stop_level=warm_level, max_gd_iterations=max_iter, use_fp64=int(fp64), lambda_=lam)


def training_set(ctx: Context, *, level: int, net_level: int, num_series: int, frames_per_series: int, seed: int,
                 start_level: int = 4, max_iter: int = 30, fp64: bool = True, device=None):
    """Synthetic lattice series (random spec per series, msgpu.synthetic),
    each registered to its first frame by the plain method up to level
    net_level-1.  Returns (R, T, target) device tensors: prepared images at
    net_level, pairs x N0 each, and displacements pairs x 2 x N1 (domain
    units), plus the seconds spent."""
    import torch
    dev = device or torch.device("cuda", torch.cuda.current_device())
    warm = net_level - 1
    n, n0, n1 = n_of(level), n_of(net_level), n_of(warm)
    F = frames_per_series
    P = num_series * F
    R = torch.empty((P, n0 * n0), dtype=torch.float64, device=dev)
    T = torch.empty((P, n0 * n0), dtype=torch.float64, device=dev)
    tgt = torch.empty((P, 2, n1 * n1), dtype=torch.float64, device=dev)
    prep = torch.empty((F + 1, n0 * n0), dtype=torch.float64, device=dev)
    p = pair_params(level, warm, start_level, max_iter, fp64)
    rng = np.random.default_rng(seed)
    stream = torch.cuda.current_stream(dev).cuda_stream
    t0 = time.perf_counter()
    for s in range(num_series):
        spec = syn.random_spec(rng)
        fr = syn.make_series_torch(n, F + 1, spec, seed=int(rng.integers(1 << 31)), device=dev).reshape(F + 1, -1)
        fr = fr.contiguous()
        ctx.register_batch_device(p, fr[0].data_ptr(), fr[1].data_ptr(), F, tgt[s * F].data_ptr(), stream=stream)
        ctx.prepare_images_device(p, fr.data_ptr(), F + 1, net_level, prep.data_ptr(), stream)
        R[s * F:(s + 1) * F] = prep[0]
        T[s * F:(s + 1) * F] = prep[1:]
    torch.cuda.synchronize(dev)
    return R, T, tgt, time.perf_counter() - t0


def train(net: Net, R, T, tgt, *, steps: int, batch: int, lr: float = 2e-3, seed: int = 0, log_every: int = 0):
    """Adam steps on random minibatches with a cosine learning-rate decay;
    returns (losses per step, seconds)."""
    import torch
    dev = R.device
    P = R.shape[0]
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    bR = torch.empty((batch, R.shape[1]), dtype=R.dtype, device=dev)
    bT = torch.empty_like(bR)
    bt = torch.empty((batch,) + tuple(tgt.shape[1:]), dtype=tgt.dtype, device=dev)
    stream = torch.cuda.current_stream(dev).cuda_stream
    losses = []
    torch.cuda.synchronize(dev)
    t0 = time.perf_counter()
    for k in range(steps):
        idx = torch.randint(0, P, (batch,), generator=g, device=dev)
        torch.index_select(R, 0, idx, out=bR)
        torch.index_select(T, 0, idx, out=bT)
        torch.index_select(tgt, 0, idx, out=bt)
        a = lr * 0.5 * (1 + np.cos(np.pi * k / steps))
        want = bool(log_every) and (k % log_every == 0 or k == steps - 1)
        loss = net.train_step_device(bR.data_ptr(), bR.shape[1], bT.data_ptr(), bt.data_ptr(), batch, a, stream,
                                     want_loss=want)
        if want:
            losses.append((k, loss))
    torch.cuda.synchronize(dev)
    return losses, time.perf_counter() - t0


def prediction_error(net: Net, R, T, tgt, batch: int = 32):
    """Mean squared error (pixels of the warm level) of the prediction and of the zero start."""
    import torch
    P = R.shape[0]
    n1 = n_of(net.level - 1)
    out = torch.empty_like(tgt)
    stream = torch.cuda.current_stream(R.device).cuda_stream
    for b in range(0, P, batch):
        m = min(batch, P - b)
        net.predict_device(R[b].data_ptr(), R.shape[1], T[b].data_ptr(), m, out[b].data_ptr(), stream)
    torch.cuda.synchronize(R.device)
    s = (n1 - 1) ** 2
    return float(((out - tgt) ** 2).mean()) * s, float((tgt ** 2).mean()) * s
