"""The warm-start network on the GPU through the C ABI (msgpu_net_*): forward
values and every parameter gradient against the oracle
(oracle/unet_oracle.py) on the same bf16-rounded weights and inputs, the
oracle rounding to bf16 where the kernels store bf16; deterministic
training steps; the file round trip; the image preparation it reads; and the
warm-started batch with its fallback to the plain start."""
import numpy as np
import pytest

import unet_oracle as U

pytestmark = pytest.mark.gpu

# Against the oracle with the kernels' bf16 rounding points (level 4, where
# fp32 versus fp64 accumulation moves almost no value across a bf16 rounding
# boundary -- the tensor-core forward adds a wide layer's channels in groups,
# an order in which a few outputs round to the neighbouring bf16): agreement
# to fp32 accumulation, the error growing toward the first layers through
# the backward pass.  On larger grids a few such
# rounding flips occur and cascade through the layers, so there the check is
# against the all-FP64 oracle: bf16 activations and gradients compound over
# the 13 layers to a few 1e-3 in the output and up to ~0.1 per layer's
# gradient, with the gradient direction kept.
TOL_OUT_BF16, TOL_GRAD_BF16 = 1e-4, 1e-2
TOL_OUT_FP64, TOL_GRAD_FP64, COS_FP64 = 1e-2, 0.2, 0.999


def bf16(a):
    """Round to the nearest bf16 (ties to even), returned as float64."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32).astype(np.float64)


def oracle_params(theta):
    """The kernels' view of the parameters: bf16 weights, fp32 biases."""
    out, o = [], 0
    for _, ci, co, _, _ in U.LAYERS:
        out.append(bf16(theta[o:o + co * 9 * ci]))
        o += co * 9 * ci
        out.append(theta[o:o + co].astype(np.float64))
        o += co
    return np.concatenate(out)


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))


def case(level, B, seed):
    rng = np.random.default_rng(seed)
    n0, n1 = (1 << level) + 1, (1 << (level - 1)) + 1
    R = bf16(rng.random((B, n0, n0)))
    T = bf16(rng.random((B, n0, n0)))
    tgt = rng.normal(0, 1.0, (B, 2, n1 * n1)) / (n1 - 1)   # about one pixel of the output grid
    return R, T, tgt, n1


def against_oracle(net, level, B, seed, rnd):
    theta = net.get_params()
    R, T, tgt, n1 = case(level, B, seed)
    loss, phi, grad = net.loss_grad(R, T, tgt)
    t_px = tgt.reshape(B, 2, n1, n1).transpose(0, 2, 3, 1) * (n1 - 1)
    rloss, rgrad, rout = U.loss_and_grad(oracle_params(theta), R, T, t_px, rnd)
    rphi = rout.transpose(0, 3, 1, 2).reshape(B, 2, -1) / (n1 - 1)
    layers, o = {}, 0
    for name, ci, co, _, _ in U.LAYERS:
        nw = co * 9 * ci + co
        layers[name] = rel(grad[o:o + nw].astype(np.float64), rgrad[o:o + nw])
        o += nw
    cos = float(grad @ rgrad / (np.linalg.norm(grad) * np.linalg.norm(rgrad)))
    return rel(phi, rphi), abs(loss - rloss) / rloss, layers, cos


def test_forward_and_gradients_match_the_bf16_oracle(gpu):
    import msgpu
    net = msgpu.Net(gpu, 4, seed=11)
    assert net.get_params().size == U.num_params() == msgpu.Net.num_params()
    e_phi, e_loss, layers, cos = against_oracle(net, 4, 2, 104, bf16)
    assert e_phi < TOL_OUT_BF16 and e_loss < TOL_OUT_BF16
    for name, e in layers.items():
        assert e < TOL_GRAD_BF16, (name, e)
    assert cos > 1 - 1e-6
    net.close()


@pytest.mark.parametrize("level,B", [(4, 2), (5, 3), (6, 2)])
def test_forward_and_gradients_match_the_fp64_oracle(gpu, level, B):
    import msgpu
    net = msgpu.Net(gpu, level, seed=11)
    e_phi, e_loss, layers, cos = against_oracle(net, level, B, 100 + level, lambda a: a)
    assert e_phi < TOL_OUT_FP64 and e_loss < TOL_OUT_FP64
    for name, e in layers.items():
        assert e < TOL_GRAD_FP64, (name, e)
    assert cos > COS_FP64
    net.close()


@pytest.mark.parametrize("level,B", [(4, 2), (7, 3)])
def test_tensor_core_forward_matches_the_mma_sync_forward(gpu, level, B):
    """The forward convolutions on tcgen05 (TMEM accumulators, the default)
    against the same network on mma.sync: the fp32 sums differ only in their
    order, so outputs, loss and gradients agree to the bf16 rounding of the
    activations they pass through."""
    import msgpu
    net = msgpu.Net(gpu, level, seed=17)
    R, T, tgt, _ = case(level, B, 900 + level)
    loss_tc, phi_tc, grad_tc = net.loss_grad(R, T, tgt)
    net.set_tensor_cores(False)
    try:
        loss_ms, phi_ms, grad_ms = net.loss_grad(R, T, tgt)
    finally:
        net.set_tensor_cores(True)
    assert np.isfinite(phi_tc).all() and np.abs(phi_tc).max() > 0
    assert rel(phi_tc, phi_ms) < 1e-2, rel(phi_tc, phi_ms)
    assert abs(loss_tc - loss_ms) / loss_ms < 1e-2
    g1, g2 = grad_tc.astype(np.float64), grad_ms.astype(np.float64)
    assert float(g1 @ g2 / (np.linalg.norm(g1) * np.linalg.norm(g2))) > 0.999
    net.close()


def test_training_steps_are_deterministic_and_reduce_the_loss(gpu):
    import msgpu
    import torch
    level, B = 5, 4
    R, T, _, n1 = case(level, B, 7)
    # a learnable target: a shift of about a pixel per frame and component
    shift = np.random.default_rng(8).uniform(-1.5, 1.5, (B, 2, 1)) / (n1 - 1)
    tgt = np.repeat(shift, n1 * n1, axis=2)
    dev = torch.device("cuda", 0)
    dR, dT = torch.from_numpy(R.reshape(B, -1)).to(dev), torch.from_numpy(T.reshape(B, -1)).to(dev)
    dt = torch.from_numpy(tgt).to(dev)
    runs = []
    for _ in range(2):
        net = msgpu.Net(gpu, level, seed=3)
        losses = [net.train_step_device(dR.data_ptr(), dR.shape[1], dT.data_ptr(), dt.data_ptr(), B, 2e-3)
                  for _ in range(60)]
        runs.append((losses, net.get_params()))
        net.close()
    assert runs[0][0] == runs[1][0]
    assert np.array_equal(runs[0][1], runs[1][1])
    assert runs[0][0][-1] < 0.25 * runs[0][0][0]


def test_save_load_round_trip(gpu, tmp_path):
    import msgpu
    a = msgpu.Net(gpu, 4, seed=5)
    b = msgpu.Net(gpu, 4, seed=6)
    assert not np.array_equal(a.get_params(), b.get_params())
    p = str(tmp_path / "w.msgpunet")
    a.save(p)
    b.load(p)
    assert np.array_equal(a.get_params(), b.get_params())
    with pytest.raises(msgpu.MsgpuError, match="not a network file"):
        b.load(__file__)
    with pytest.raises(msgpu.MsgpuError, match="Could not open"):
        b.load(str(tmp_path / "missing"))
    a.close()
    b.close()


def test_prepare_images_matches_the_pipeline_operators(gpu):
    import msgpu
    import torch
    rng = np.random.default_rng(9)
    lvl = 6
    n = (1 << lvl) + 1
    imgs = rng.poisson(30 * rng.random((3, n, n))).astype(np.float64)
    p = msgpu.default_params(precision_level=lvl, input_level=lvl, start_level=2, stop_level=lvl)
    dev = torch.device("cuda", 0)
    d_in = torch.from_numpy(imgs.reshape(3, -1)).to(dev)
    d_out = torch.zeros((3, ((1 << 4) + 1) ** 2), dtype=torch.float64, device=dev)
    gpu.prepare_images_device(p, d_in.data_ptr(), 3, 4, d_out.data_ptr())
    torch.cuda.synchronize()
    for i in range(3):
        x = gpu.normalize(imgs[i], p.saturation_percent, p.normalize_min_to_zero)
        for l in (6, 5):
            x = gpu.restrict(l, x)
        assert np.array_equal(d_out[i].cpu().numpy(), x)


def test_warm_batch_and_fallback(gpu):
    import msgpu
    from msgpu import synthetic as syn
    lvl = 7
    n = (1 << lvl) + 1
    frames, _, _ = syn.make_series(n, 4, syn.SQUARE_257, seed=321)
    p = msgpu.default_params(precision_level=lvl, input_level=lvl, start_level=3, stop_level=lvl,
                             max_gd_iterations=10, use_fp64=1)
    ref, tm = frames[0], frames[1:]
    plain, pe, ps = gpu.register_batch(p, ref, tm)
    net = msgpu.Net(gpu, 6, seed=2)   # predicts level 5
    ph, e, s, used = gpu.register_batch_warm(p, net, ref, tm)
    assert used.tolist() == [1, 1, 1]
    assert s.shape == ps.shape and np.all(s[:, :2] == 0) and np.all(s[:, 2:] > 0)
    assert np.all(np.isfinite(ph)) and np.all(e > 0)
    # every warm start judged worse than the plain result: the plain start, bit for bit
    ph2, e2, s2, used2 = gpu.register_batch_warm(p, net, ref, tm, plain_energies=pe, rel_tol=-1.0)
    assert used2.tolist() == [0, 0, 0]
    assert np.array_equal(ph2, plain) and np.array_equal(e2, pe) and np.array_equal(s2, ps)
    # kept when within the tolerance: with an unbounded tolerance every frame
    # is within it at its first stop-level energy, so the stop level ends
    # there (registration to the stated energy tolerance); the coarser levels
    # are those of the run without targets
    ph3, e3, s3, used3 = gpu.register_batch_warm(p, net, ref, tm, plain_energies=pe, rel_tol=np.inf)
    assert used3.tolist() == [1, 1, 1] and np.all(np.isfinite(e3)) and np.all(np.isfinite(ph3))
    assert np.all(s3[:, -1] == 0) and np.array_equal(s3[:, :-1], s[:, :-1])
    bad = msgpu.default_params(precision_level=lvl, input_level=lvl, start_level=6, stop_level=lvl)
    with pytest.raises(msgpu.MsgpuError, match="network input level"):
        gpu.register_batch_warm(bad, net, ref, tm)
    net.close()


def test_warm_batch_larger_than_one_network_pass(gpu):
    """70 frames: the prediction runs in passes of 64; every frame's result
    equals the one it gets in a batch of 5 (neither the network nor the
    registration depends on the batch a frame is in)."""
    import msgpu
    from msgpu import synthetic as syn
    lvl = 5
    n = (1 << lvl) + 1
    frames, _, _ = syn.make_series(n, 71, syn.SQUARE_257, seed=77)
    p = msgpu.default_params(precision_level=lvl, input_level=lvl, start_level=2, stop_level=lvl,
                             max_gd_iterations=5, use_fp64=1)
    net = msgpu.Net(gpu, 5, seed=9)   # predicts level 4
    ph, e, _, _ = gpu.register_batch_warm(p, net, frames[0], frames[1:])
    for f0 in (0, 63, 65):
        ph5, e5, _, _ = gpu.register_batch_warm(p, net, frames[0], frames[1 + f0:6 + f0])
        assert np.array_equal(ph5, ph[f0:f0 + 5]) and np.array_equal(e5, e[f0:f0 + 5])
    net.close()
