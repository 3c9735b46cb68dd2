"""Ragged batches (msgpu_register_ragged): series of different sizes, each
registered to its own reference, one launch per level for all of them.  A
frame's result does not depend on the batch it is in (per-tile partial sums
added in tile order), so every series of a ragged batch must equal, bit for
bit, the same series registered alone by msgpu_register_batch -- with the SSD
and NCC data terms, FP64 and FP32, and a lambdaFactor that makes the level
weights count from each series' own stop level."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _series(level, F, seed):
    from msgpu import synthetic as syn
    n = (1 << level) + 1
    fr, _, _ = syn.make_series(n, F + 1, syn.SQUARE_257, seed=seed)
    return fr[0].ravel(), fr[1:].reshape(F, -1)


@pytest.mark.parametrize("fp64,data_term,lam_factor", [(1, 0, 1.0), (0, 0, 1.0), (1, 1, 1.0), (1, 0, 0.7)])
def test_ragged_equals_separate_batches(gpu, fp64, data_term, lam_factor):
    import msgpu
    spec = [(6, 2, 11), (5, 3, 12), (7, 2, 13), (6, 1, 14)]
    series = [_series(l, F, s) for l, F, s in spec]
    p = msgpu.default_params(start_level=4, max_gd_iterations=8, use_fp64=fp64, data_term=data_term,
                             lambda_factor=lam_factor)
    got = gpu.register_ragged(p, series)
    for (level, F, _), (ref, tm), (phis, en) in zip(spec, series, got):
        q = msgpu.default_params(precision_level=level, input_level=level, start_level=4, stop_level=level,
                                 max_gd_iterations=8, use_fp64=fp64, data_term=data_term, lambda_factor=lam_factor)
        ph2, e2, _ = gpu.register_batch(q, ref, tm)
        assert np.array_equal(phis, ph2), (level, fp64, data_term)
        assert np.array_equal(en, e2), (level, fp64, data_term)


def test_ragged_rejects_bad_series(gpu):
    import msgpu
    p = msgpu.default_params(start_level=5)
    ref, tm = _series(4, 1, 3)
    with pytest.raises(msgpu.MsgpuError):
        gpu.register_ragged(p, [(ref, tm)])   # level 4 below startLevel 5
