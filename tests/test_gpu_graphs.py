"""CUDA-graph capture and replay of the device batch call: the second call
with the same parameters and buffers captures the batch's launches, later
calls replay the graph as one launch, and every call gives the same bits as
a direct run (graphs off).  A change of parameters or of a buffer runs
directly again, and a buffer that the context reallocates in between makes
the next call capture anew instead of replaying stale addresses."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _setup(level, F, seed):
    import torch
    import msgpu
    from msgpu import synthetic as syn
    n = (1 << level) + 1
    fr, _, _ = syn.make_series(n, F + 1, syn.HEX_513, seed=seed)
    dev = torch.device("cuda", 0)
    d_ref = torch.from_numpy(fr[0].ravel().copy()).to(dev)
    d_tmpl = torch.from_numpy(fr[1:].reshape(F, -1).copy()).to(dev)
    d_phis = torch.empty((F, 2, n * n), dtype=torch.float64, device=dev)
    d_e = torch.empty(F, dtype=torch.float64, device=dev)
    p = msgpu.default_params(precision_level=level, input_level=level, start_level=4, stop_level=level,
                             max_gd_iterations=10, use_fp64=1)
    return p, d_ref, d_tmpl, d_phis, d_e


def _call(ctx, p, d_ref, d_tmpl, d_phis, d_e):
    import torch
    ctx.register_batch_device(p, d_ref.data_ptr(), d_tmpl.data_ptr(), d_tmpl.shape[0], d_phis.data_ptr(),
                              d_e.data_ptr())
    torch.cuda.synchronize()
    return d_phis.cpu().numpy().copy(), d_e.cpu().numpy().copy(), ctx.stats()


def test_replayed_graph_gives_the_direct_run_bits():
    import msgpu
    ctx = msgpu.Context(0)
    try:
        p, d_ref, d_tmpl, d_phis, d_e = _setup(7, 3, 7301)
        ctx.set_graphs(False)
        want_phi, want_e, st = _call(ctx, p, d_ref, d_tmpl, d_phis, d_e)
        assert not st["graph_replayed"] and st["kernel_launches"] > 10
        ctx.set_graphs(True)
        replayed = []
        for _ in range(4):
            d_phis.fill_(np.nan)
            phi, e, st = _call(ctx, p, d_ref, d_tmpl, d_phis, d_e)
            assert np.array_equal(phi, want_phi) and np.array_equal(e, want_e)
            replayed.append(st["graph_replayed"])
        # first call direct, second captures and launches the graph, then replays
        assert replayed == [False, True, True, True]
        # other parameters: a direct run, right results
        p2 = msgpu.default_params(precision_level=7, input_level=7, start_level=4, stop_level=7,
                                  max_gd_iterations=6, use_fp64=1)
        ctx.set_graphs(False)
        ref6, e6, _ = _call(ctx, p2, d_ref, d_tmpl, d_phis, d_e)
        ctx.set_graphs(True)
        phi, e, st = _call(ctx, p2, d_ref, d_tmpl, d_phis, d_e)
        assert not st["graph_replayed"] and np.array_equal(phi, ref6) and np.array_equal(e, e6)
    finally:
        ctx.close()


def test_reallocated_buffers_invalidate_the_graph():
    import msgpu
    ctx = msgpu.Context(0)
    try:
        p, d_ref, d_tmpl, d_phis, d_e = _setup(6, 2, 7302)
        want_phi, want_e, _ = _call(ctx, p, d_ref, d_tmpl, d_phis, d_e)
        _call(ctx, p, d_ref, d_tmpl, d_phis, d_e)           # captured
        # a larger single-level solve grows the context's buffers
        from msgpu import synthetic as syn
        fr, _, _ = syn.make_series(257, 2, syn.HEX_513, seed=7303)
        z = np.zeros(257 * 257)
        ctx.gd_level(8, ctx.normalize(fr[0].ravel()), ctx.normalize(fr[1].ravel()), z, z, 0.1, 3, fp64=True)
        phi, e, st = _call(ctx, p, d_ref, d_tmpl, d_phis, d_e)
        assert not st["graph_replayed"]
        assert np.array_equal(phi, want_phi) and np.array_equal(e, want_e)
        phi, e, st = _call(ctx, p, d_ref, d_tmpl, d_phis, d_e)
        assert np.array_equal(phi, want_phi) and np.array_equal(e, want_e)
    finally:
        ctx.close()


def test_autotuner_fills_the_table_and_keeps_the_results():
    """msgpu_autotune_device times every level under each candidate setting
    and keeps the fastest; a batch under the tuned settings gives the same
    bits as under the defaults (the scheduling never changes a result)."""
    import torch
    import msgpu
    ctx = msgpu.Context(0)
    try:
        p, d_ref, d_tmpl, d_phis, d_e = _setup(7, 3, 7304)
        ctx.set_graphs(False)
        want_phi, want_e, _ = _call(ctx, p, d_ref, d_tmpl, d_phis, d_e)
        scratch = torch.empty_like(d_phis)
        table = ctx.autotune_device(p, d_ref.data_ptr(), d_tmpl.data_ptr(), d_tmpl.shape[0], scratch.data_ptr())
        assert sorted(table) == list(range(p.start_level, p.stop_level + 1))
        for lv, t in table.items():
            assert t["chunk_div"] in (12, 24, 48) and t["chunk_max"] in (8, 16, 32)
            assert t["ctas_per_sm"] in (1, 2) and 0 < t["ms"] < 1e4
        phi, e, _ = _call(ctx, p, d_ref, d_tmpl, d_phis, d_e)
        assert np.array_equal(phi, want_phi) and np.array_equal(e, want_e)
    finally:
        ctx.close()
