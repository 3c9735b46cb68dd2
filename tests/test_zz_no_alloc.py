"""msgpu_gd_level_noalloc, the level solve for callers that cannot allocate
device memory, against msgpu_gd_level (the allocating entry point).

Both run the same level kernel with the global sums in the fixed parallel
order (the allocating entry point set to sum order 1 for the comparison; the
exact-sum scratch of the reference order does not fit the static array), so
the results are held to the parity tolerances of the FP64 path: displacements
within 1e-6 px, energies within 1e-9 relative, identical step counts.  Several
calls in a row share the one static scratch array; a smaller level after a
larger one checks that leftovers of the previous call do not leak into the
next."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MSGPU_ERR_SIZE = 2


def _entry():
    import msgpu
    f = ctypes.CDLL(msgpu.LIB_PATH).msgpu_gd_level_noalloc
    f.argtypes = [ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
                  ctypes.c_double, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return f


@pytest.fixture
def gpu_parallel_sums(gpu):
    gpu.set_sum_order(1)
    yield gpu
    gpu.set_sum_order(0)


def _images(gpu, level, seed):
    from msgpu import synthetic as syn
    n = (1 << level) + 1
    fr, _, _ = syn.make_series(n, 2, syn.HEX_513, seed=seed)
    return gpu.normalize(fr[0].ravel()), gpu.normalize(fr[1].ravel())


def _noalloc(f, level, R, T, phix, phiy, lam, max_iter, fp64):
    import torch
    dev = torch.device("cuda", 0)
    dR = torch.from_numpy(np.ascontiguousarray(R)).to(dev)
    dT = torch.from_numpy(np.ascontiguousarray(T)).to(dev)
    dphi = torch.from_numpy(np.concatenate([phix, phiy])).to(dev)
    de = torch.full((1,), -1.0, dtype=torch.float64, device=dev)
    ds = torch.full((1,), -1, dtype=torch.int32, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = f(level, dR.data_ptr(), dT.data_ptr(), dphi.data_ptr(), lam, max_iter, 0.0, fp64, de.data_ptr(),
           ds.data_ptr(), stream.cuda_stream)
    torch.cuda.synchronize(dev)
    assert rc == 0
    N = R.size
    out = dphi.cpu().numpy()
    return out[:N], out[N:], float(de.item()), int(ds.item())


@pytest.mark.parametrize("order", ["large_then_small", "small_then_large"])
def test_noalloc_matches_gd_level_on_calls_in_a_row(gpu_parallel_sums, order):
    gpu = gpu_parallel_sums
    f = _entry()
    # level 8 in FP64 is the largest solve the scratch array holds
    cases = [(8, 24, 1, 6), (7, 21, 1, 12), (6, 22, 1, 10), (8, 25, 0, 6), (6, 23, 0, 10)]
    if order == "small_then_large":
        cases = cases[::-1]
    for level, seed, fp64, iters in cases:
        n = (1 << level) + 1
        R, T = _images(gpu, level, seed)
        rng = np.random.default_rng(seed)
        px0 = rng.normal(0, 0.3 / (n - 1), n * n)
        py0 = rng.normal(0, 0.3 / (n - 1), n * n)
        qx, qy, e0, s0, _ = gpu.gd_level(level, R, T, px0, py0, 0.1, iters, fp64=fp64)
        px, py, e, s = _noalloc(f, level, R, T, px0, py0, 0.1, iters, fp64)
        assert s == s0, (level, fp64)
        assert abs(e - e0) / e0 <= 1e-9, (level, fp64)
        assert max(np.abs(px - qx).max(), np.abs(py - qy).max()) * (n - 1) <= 1e-6, (level, fp64)


def test_noalloc_rejects_levels_beyond_its_scratch(gpu_parallel_sums):
    gpu = gpu_parallel_sums
    f = _entry()
    # level 9 needs more than the 12 MiB scratch: refused before any device work
    assert f(9, 16, 16, 16, 0.1, 1, 0.0, 1, None, None, None) == MSGPU_ERR_SIZE
    # and the entry point keeps working afterwards
    level = 5
    n = (1 << level) + 1
    R, T = _images(gpu, level, 5)
    z = np.zeros(n * n)
    qx, qy, e0, s0, _ = gpu.gd_level(level, R, T, z, z, 0.1, 6, fp64=1)
    px, py, e, s = _noalloc(f, level, R, T, z, z, 0.1, 6, 1)
    assert s == s0 and abs(e - e0) / e0 <= 1e-9
    assert max(np.abs(px - qx).max(), np.abs(py - qy).max()) * (n - 1) <= 1e-6


def test_noalloc_reports_a_stalled_solve_in_its_outputs(gpu_parallel_sums):
    gpu = gpu_parallel_sums
    """The call returns before the GPU runs, so a scheduler that gave up
    waiting (its wait bound shortened on purpose) is reported in the outputs:
    steps -1 and energy NaN.  With the default bound the next call is whole."""
    import msgpu
    f = _entry()
    level = 6
    n = (1 << level) + 1
    R, T = _images(gpu, level, 27)
    z = np.zeros(n * n)
    msgpu.set_wait_limits(1e-9, 0.0)
    try:
        _, _, e, s = _noalloc(f, level, R, T, z, z, 0.1, 6, 1)
    finally:
        msgpu.set_wait_limits(0.0, 0.0)
    assert s == -1 and np.isnan(e)
    qx, qy, e0, s0, _ = gpu.gd_level(level, R, T, z, z, 0.1, 6, fp64=1)
    px, py, e, s = _noalloc(f, level, R, T, z, z, 0.1, 6, 1)
    assert s == s0 and abs(e - e0) / e0 <= 1e-9
    assert max(np.abs(px - qx).max(), np.abs(py - qy).max()) * (n - 1) <= 1e-6
