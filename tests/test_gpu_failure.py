"""Failure detection without a GPU fault.

The device-side waits (a level-kernel worker waiting for work, a grid barrier
of the composition kernel) are bounded; here the bounds are shortened so that
the waits run out on purpose, and the tests check that the synchronous entry
points report the error and that the context stays usable afterwards.  Inputs
the reference cannot handle either (non-finite pixels) are refused with an
error status; degenerate inputs the reference does handle (constant frames
under NCC) follow its trace.  Nothing here traps, faults or hangs a GPU: a
run-out wait only makes the kernel return early."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

MSGPU_ERR_INVALID_ARG = 1
MSGPU_ERR_CUDA = 3


def _pair(level, seed):
    from msgpu import synthetic as syn
    n = (1 << level) + 1
    fr, _, _ = syn.make_series(n, 2, syn.HEX_513, seed=seed)
    return fr


@pytest.fixture
def short_waits():
    import msgpu
    yield msgpu.set_wait_limits
    msgpu.set_wait_limits(0.0, 0.0)


def test_level_wait_runs_out_and_context_stays_usable(gpu, short_waits):
    import msgpu
    level = 7
    fr = _pair(level, 31)
    R, T = gpu.normalize(fr[0].ravel()), gpu.normalize(fr[1].ravel())
    z = np.zeros(R.size)
    ref = gpu.gd_level(level, R, T, z, z, 0.1, 8, fp64=True)
    # a 1 ns bound: the first worker that finds no work gives up at once
    short_waits(1e-9, 0.0)
    with pytest.raises(msgpu.MsgpuError) as ei:
        gpu.gd_level(level, R, T, z, z, 0.1, 8, fp64=True)
    assert ei.value.status == MSGPU_ERR_CUDA and "stalled" in str(ei.value)
    # default bounds again: the same context solves the level as before
    short_waits(0.0, 0.0)
    px, py, e, steps, _ = gpu.gd_level(level, R, T, z, z, 0.1, 8, fp64=True)
    assert steps == ref[3] and e == ref[2]
    assert np.array_equal(px, ref[0]) and np.array_equal(py, ref[1])


def test_composition_barrier_wait_runs_out_and_context_stays_usable(gpu, short_waits):
    import msgpu
    level = 6
    n = (1 << level) + 1
    rng = np.random.default_rng(5)
    d1 = rng.normal(0, 1.0 / (n - 1), (2, n * n))
    d2 = rng.normal(0, 1.0 / (n - 1), (2, n * n))
    ref, it = gpu.compose(level, d1, d2)
    short_waits(0.0, 1e-9)
    with pytest.raises(msgpu.MsgpuError) as ei:
        gpu.compose(level, d1, d2)
    assert ei.value.status == MSGPU_ERR_CUDA and "barrier" in str(ei.value)
    short_waits(0.0, 0.0)
    out, it2 = gpu.compose(level, d1, d2)
    assert np.array_equal(out, ref) and np.array_equal(it, it2)


@pytest.mark.parametrize("bad", [np.nan, np.inf, -np.inf])
def test_non_finite_input_is_refused(gpu, bad):
    import msgpu
    level = 6
    fr = _pair(level, 41)
    p = msgpu.default_params(precision_level=level, input_level=level, start_level=4, stop_level=level,
                             max_gd_iterations=5, use_fp64=1)
    T = fr[1].copy()
    T.ravel()[1234] = bad
    with pytest.raises(msgpu.MsgpuError) as ei:
        gpu.register_batch(p, fr[0], T[None])
    assert ei.value.status == MSGPU_ERR_INVALID_ARG and "non-finite" in str(ei.value)
    # in the reference image too
    R = fr[0].copy()
    R.ravel()[7] = bad
    with pytest.raises(msgpu.MsgpuError):
        gpu.register_batch(p, R, fr[1:2])
    # the context is usable afterwards
    phis, e, steps = gpu.register_batch(p, fr[0], fr[1:2])
    assert np.isfinite(e).all() and np.isfinite(phis).all()


@pytest.mark.parametrize("which", ["template", "reference"])
def test_constant_frame_under_ncc_follows_the_reference_trace(gpu, oracle, which):
    """A zero-variance frame under NCC: the normalisation skips its division
    (registration.h:1932-1944), the energy is 0 at every step, the line
    search returns tau = 0 (ArmijoSearch.h:146-151) and sigma halves every
    step, as in the oracle (which matches the reference bit for bit)."""
    level = 6
    n = (1 << level) + 1
    fr = _pair(level, 7)
    R = oracle.normalize(fr[0].ravel())
    C = np.full(n * n, 0.5)
    R, T = (R, C) if which == "template" else (C, R)
    z = np.zeros(n * n)
    gpu.set_data_term(1)
    try:
        px, py, e, steps, tr = gpu.gd_level(level, R, T, z, z, 0.1, 10, fp64=True)
    finally:
        gpu.set_data_term(0)
    rx, ry, re, rsteps, rtr = oracle.gd_level(level, R, T, z, z, 0.1, 10, ncc=True)
    assert steps == rsteps and e == re == 0.0
    assert np.array_equal(px, rx) and np.array_equal(py, ry) and not px.any()
    # accepted tau (0) and the filter width of every step as in the reference
    assert [(row[1], row[2]) for row in tr] == [(t[2], t[3]) for t in rtr]
    if which == "template":
        # and the number of line-search evaluations
        assert [int(row[3]) for row in tr] == [t[4] for t in rtr]
    # (a constant reference is normalised to rounding noise: its mean differs
    # from the constant in the last bits, so the descent direction is noise
    # of the order of the unit roundoff and the length of each futile line
    # search depends on the order of the normalisation's sums)
