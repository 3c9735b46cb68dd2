"""Oracle (test infrastructure only): FP64 CPU restatement of the warm-start
network, forward and backward.  The registration method has no learned part
in the reference; this network is the project's own, so the oracle restates
the project's definition below.  It is the checker of the CUDA kernels
(forward values and every parameter gradient), never a product path.

Network: a U-Net on 2^l+1 node grids.  Input: the normalised reference and
template images of a frame pair on the input grid (n0 = 2^l0+1 nodes per
side).  Stride-2 3x3 convolutions map node 2i of a grid to node i of the
next coarser one (n -> (n+1)/2); the decoder upsamples by the bilinear
prolongation of the node grids (coarse node i -> fine node 2i, midpoints
averaged) and concatenates [skip | upsampled] channels.  3x3 convolutions
with zero padding, ReLU after every convolution but the head.  Output: two
channels on the grid n1 = (n0+1)/2, the displacement in pixels of that
grid; loss = mean squared difference to the target over batch, nodes and
both channels.

Parameter layout (flat float vector, layer after layer): W[cout][3][3][cin]
(tap (ky, kx) reads the input node at offset (ky-1, kx-1)), then b[cout].

`rnd` (optional) is applied wherever the CUDA path stores a tensor in bf16:
every activation, the loss gradient, every data gradient and the
upsampling's adjoint; with the identity (default) everything is FP64.
"""
from __future__ import annotations

import numpy as np

# name, input channels, output channels, stride, ReLU
LAYERS = [
    ("e0a", 2, 16, 1, True), ("e0b", 16, 16, 1, True),
    ("e1a", 16, 32, 2, True), ("e1b", 32, 32, 1, True),
    ("e2a", 32, 64, 2, True), ("e2b", 64, 64, 1, True),
    ("e3a", 64, 128, 2, True), ("e3b", 128, 128, 1, True),
    ("d2a", 192, 64, 1, True), ("d2b", 64, 64, 1, True),
    ("d1a", 96, 32, 1, True), ("d1b", 32, 32, 1, True),
    ("head", 32, 2, 1, False),
]
STRIDE = {l[0]: l[3] for l in LAYERS}


def _ident(a):
    return a


def num_params() -> int:
    return sum(co * 9 * ci + co for _, ci, co, _, _ in LAYERS)


def unpack(theta: np.ndarray):
    out, o = {}, 0
    for name, ci, co, _, _ in LAYERS:
        w = theta[o:o + co * 9 * ci].reshape(co, 3, 3, ci)
        o += co * 9 * ci
        b = theta[o:o + co]
        o += co
        out[name] = (w, b)
    return out


def conv(x, w, b, stride):
    """x [B, n, n, ci] -> [B, m, m, co], m = (n-1)/stride + 1, zero padding."""
    B, n, _, ci = x.shape
    m = (n - 1) // stride + 1
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    y = np.zeros((B, m, m, w.shape[0]))
    for ky in range(3):
        for kx in range(3):
            patch = xp[:, ky:ky + stride * (m - 1) + 1:stride, kx:kx + stride * (m - 1) + 1:stride, :]
            y += patch @ w[:, ky, kx, :].T
    return y + b


def conv_backward(x, w, dy, stride):
    """Gradients of conv: (dx, dw, db)."""
    m = dy.shape[1]
    xp = np.pad(x, ((0, 0), (1, 1), (1, 1), (0, 0)))
    dxp = np.zeros_like(xp)
    dw = np.zeros_like(w)
    for ky in range(3):
        for kx in range(3):
            sl = (slice(None), slice(ky, ky + stride * (m - 1) + 1, stride),
                  slice(kx, kx + stride * (m - 1) + 1, stride), slice(None))
            dw[:, ky, kx, :] = np.einsum("bijo,bijc->oc", dy, xp[sl])
            dxp[sl] += dy @ w[:, ky, kx, :]
    return dxp[:, 1:-1, 1:-1, :], dw, dy.sum(axis=(0, 1, 2))


def up(c):
    """Bilinear prolongation of node grids: [B, m, m, C] -> [B, 2m-1, 2m-1, C]."""
    B, m, _, C = c.shape
    f = np.zeros((B, 2 * m - 1, 2 * m - 1, C))
    f[:, ::2, ::2] = c
    f[:, 1::2, ::2] = 0.5 * (c[:, :-1] + c[:, 1:])
    f[:, ::2, 1::2] = 0.5 * (c[:, :, :-1] + c[:, :, 1:])
    f[:, 1::2, 1::2] = 0.25 * (c[:, :-1, :-1] + c[:, 1:, :-1] + c[:, :-1, 1:] + c[:, 1:, 1:])
    return f


def up_backward(df):
    """Adjoint of up."""
    B, nf, _, C = df.shape
    m = (nf + 1) // 2
    dc = np.zeros((B, m, m, C))
    dc += df[:, ::2, ::2]
    dc[:, :-1] += 0.5 * df[:, 1::2, ::2]
    dc[:, 1:] += 0.5 * df[:, 1::2, ::2]
    dc[:, :, :-1] += 0.5 * df[:, ::2, 1::2]
    dc[:, :, 1:] += 0.5 * df[:, ::2, 1::2]
    q = 0.25 * df[:, 1::2, 1::2]
    dc[:, :-1, :-1] += q
    dc[:, 1:, :-1] += q
    dc[:, :-1, 1:] += q
    dc[:, 1:, 1:] += q
    return dc


def forward(theta, R, T, rnd=_ident):
    """R, T [B, n0, n0] -> (out [B, n1, n1, 2], cache)."""
    P = unpack(theta)
    relu = lambda v: np.maximum(v, 0.0)
    c = {}
    x = np.stack([R, T], axis=-1)
    c["x"] = x
    a = x
    for name, key in [("e0a", "a0"), ("e0b", "a1"), ("e1a", "b0"), ("e1b", "s1"), ("e2a", "c0"), ("e2b", "s2"),
                      ("e3a", "d0"), ("e3b", "d1")]:
        a = rnd(relu(conv(a, *P[name], STRIDE[name])))
        c[key] = a
    c["cat2"] = np.concatenate([c["s2"], rnd(up(c["d1"]))], axis=-1)
    c["g0"] = rnd(relu(conv(c["cat2"], *P["d2a"], 1)))
    c["g1"] = rnd(relu(conv(c["g0"], *P["d2b"], 1)))
    c["cat1"] = np.concatenate([c["s1"], rnd(up(c["g1"]))], axis=-1)
    c["h0"] = rnd(relu(conv(c["cat1"], *P["d1a"], 1)))
    c["h1"] = rnd(relu(conv(c["h0"], *P["d1b"], 1)))
    out = conv(c["h1"], *P["head"], 1)
    return out, c


def loss_and_grad(theta, R, T, target, rnd=_ident):
    """Mean squared error to target [B, n1, n1, 2] and its gradient (flat)."""
    P = unpack(theta)
    out, c = forward(theta, R, T, rnd)
    diff = out - target
    loss = float(np.mean(diff * diff))
    g = {}
    dy = rnd(2.0 * diff / diff.size)

    def back(name, xin, dy_pre):
        dx, dw, db = conv_backward(xin, P[name][0], dy_pre, STRIDE[name])
        g[name] = (dw, db)
        return dx

    mask = lambda a: (a > 0).astype(np.float64)
    d = rnd(back("head", c["h1"], dy) * mask(c["h1"]))
    d = rnd(back("d1b", c["h0"], d) * mask(c["h0"]))
    dcat1 = rnd(back("d1a", c["cat1"], d))
    cs1 = c["s1"].shape[-1]
    d = rnd(up_backward(dcat1[..., cs1:]) * mask(c["g1"]))
    d = rnd(back("d2b", c["g0"], d) * mask(c["g0"]))
    dcat2 = rnd(back("d2a", c["cat2"], d))
    cs2 = c["s2"].shape[-1]
    d = rnd(up_backward(dcat2[..., cs2:]) * mask(c["d1"]))
    d = rnd(back("e3b", c["d0"], d) * mask(c["d0"]))
    d = rnd((back("e3a", c["s2"], d) + dcat2[..., :cs2]) * mask(c["s2"]))
    d = rnd(back("e2b", c["c0"], d) * mask(c["c0"]))
    d = rnd((back("e2a", c["s1"], d) + dcat1[..., :cs1]) * mask(c["s1"]))
    d = rnd(back("e1b", c["b0"], d) * mask(c["b0"]))
    d = rnd(back("e1a", c["a1"], d) * mask(c["a1"]))
    d = rnd(back("e0b", c["a0"], d) * mask(c["a0"]))
    back("e0a", c["x"], d)
    flat = np.concatenate([np.concatenate([g[name][0].ravel(), g[name][1]]) for name, *_ in LAYERS])
    return loss, flat, out
