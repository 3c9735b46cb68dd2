"""The warm-start network's oracle (oracle/unet_oracle.py) pinned on the CPU:
its gradient against central differences, and the adjoint pairs its
backward pass uses (convolution / its data gradient at strides 1 and 2,
prolongation / its adjoint).  No GPU."""
import numpy as np
import pytest

import unet_oracle as U


def he_params(rng):
    th = []
    for name, ci, co, _, _ in U.LAYERS:
        sd = np.sqrt(2.0 / (9 * ci)) * (0.1 if name == "head" else 1.0)
        th.append(rng.normal(0, sd, co * 9 * ci))
        th.append(rng.normal(0, 0.05, co))
    return np.concatenate(th)


def test_param_count():
    assert U.num_params() == 478466


@pytest.mark.parametrize("stride", [1, 2])
def test_conv_adjoint(stride):
    rng = np.random.default_rng(stride)
    x = rng.normal(size=(2, 9, 9, 3))
    w = rng.normal(size=(4, 3, 3, 3))
    y = U.conv(x, w, np.zeros(4), stride)
    dy = rng.normal(size=y.shape)
    dx, dw, db = U.conv_backward(x, w, dy, stride)
    assert abs(np.sum(y * dy) - np.sum(x * dx)) < 1e-10 * abs(np.sum(y * dy))
    assert abs(np.sum(y * dy) - np.sum(w * dw)) < 1e-10 * abs(np.sum(y * dy))
    assert np.allclose(db, dy.sum(axis=(0, 1, 2)))


def test_up_adjoint():
    rng = np.random.default_rng(3)
    c = rng.normal(size=(2, 5, 5, 3))
    f = U.up(c)
    assert f.shape == (2, 9, 9, 3)
    assert np.allclose(f[:, ::2, ::2], c)
    df = rng.normal(size=f.shape)
    assert abs(np.sum(f * df) - np.sum(c * U.up_backward(df))) < 1e-12 * np.abs(f * df).sum()


def test_gradient_against_central_differences():
    rng = np.random.default_rng(0)
    th = he_params(rng)
    B, n = 2, 17
    R, T = rng.random((B, n, n)), rng.random((B, n, n))
    t = rng.normal(0, 0.5, (B, 9, 9, 2))
    loss, g, out = U.loss_and_grad(th, R, T, t)
    assert out.shape == (B, 9, 9, 2)
    offs, o = {}, 0
    for name, ci, co, _, _ in U.LAYERS:
        offs[name] = o
        o += co * 9 * ci + co
    # a few weights and the first bias of every layer
    idx = []
    for name, ci, co, _, _ in U.LAYERS:
        idx += list(offs[name] + rng.choice(co * 9 * ci, 3, replace=False)) + [offs[name] + co * 9 * ci]
    h = 1e-6
    for i in idx:
        e = np.zeros_like(th)
        e[i] = h
        fd = (U.loss_and_grad(th + e, R, T, t)[0] - U.loss_and_grad(th - e, R, T, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 * max(abs(g[i]), 1e-3 * np.abs(g).max()), (i, fd, g[i])
