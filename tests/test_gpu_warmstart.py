"""What the trained warm-start network gains over the method without it, on a
small case: series of 513^2 lattice frames, the network (input level 9)
trained on the GPU for a few hundred steps on pairs the plain method
registered, then used to start held-out registrations at level 8.

Checked: the learned start is much closer to the plain method's level-8
solution than the zero start; the warm-started registration skips the
coarse levels (less work); its final energies stay near the plain ones; and
with the plain energies as judge, the fallback leaves no frame worse than the
tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

LEVEL, NET_LEVEL, START = 9, 9, 4


@pytest.fixture(scope="module")
def trained(gpu):
    import msgpu
    from msgpu import warmstart as ws
    R, T, tgt, _ = ws.training_set(gpu, level=LEVEL, net_level=NET_LEVEL, num_series=16, frames_per_series=8,
                                   seed=21)
    net = msgpu.Net(gpu, NET_LEVEL, seed=4)
    ws.train(net, R, T, tgt, steps=250, batch=8, lr=2e-3, seed=1)
    yield net
    net.close()


def test_learned_start_beats_the_zero_start(gpu, trained):
    from msgpu import warmstart as ws
    R, T, tgt, _ = ws.training_set(gpu, level=LEVEL, net_level=NET_LEVEL, num_series=2, frames_per_series=8,
                                   seed=999)
    pred, zero = ws.prediction_error(trained, R, T, tgt)
    assert pred < 0.25 * zero, (pred, zero)


def test_warm_started_registration(gpu, trained):
    import msgpu
    import torch
    from msgpu import synthetic as syn
    dev = torch.device("cuda", 0)
    n = msgpu.n_of(LEVEL)
    F = 8
    frames = syn.make_series_torch(n, F + 1, syn.random_spec(np.random.default_rng(5)), 55, dev)
    frames = frames.reshape(F + 1, -1).cpu().numpy()
    p = msgpu.default_params(precision_level=LEVEL, input_level=LEVEL, start_level=START, stop_level=LEVEL,
                             max_gd_iterations=30, use_fp64=1)
    ph, pe, ps = gpu.register_batch(p, frames[0], frames[1:])
    wh, we, wsteps, used = gpu.register_batch_warm(p, trained, frames[0], frames[1:])
    assert used.tolist() == [1] * F
    # the levels below the warm level are not run; work in node-steps
    warm_level = NET_LEVEL - 1
    k = warm_level - START
    assert np.all(wsteps[:, :k] == 0) and np.all(wsteps[:, k:] > 0)
    nodes = np.array([msgpu.n_of(l) ** 2 for l in range(START, LEVEL + 1)])
    assert (wsteps * nodes).sum() < (ps * nodes).sum()
    r = (we - pe) / np.abs(pe)
    assert np.all(np.isfinite(wh)) and abs(np.median(r)) < 1e-3 and r.max() < 1e-2, r
    # judged by the plain energies: every frame ends within the tolerance --
    # a warm-started frame's stop level ends as soon as its energy is within
    # it (at most twice the plain steps), a frame that does not get there is
    # registered again from the plain start, bit for bit the plain result
    tol = 1e-6
    fh, fe, fs, fused = gpu.register_batch_warm(p, trained, frames[0], frames[1:], plain_energies=pe, rel_tol=tol)
    assert np.all(fe <= pe + tol * np.abs(pe))
    for f in range(F):
        if fused[f]:
            assert np.array_equal(fs[f, :-1], wsteps[f, :-1]) and 0 <= fs[f, -1] <= 2 * 30
        else:
            assert np.array_equal(fh[f], ph[f]) and fe[f] == pe[f]
