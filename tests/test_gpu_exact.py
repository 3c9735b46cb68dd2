"""The FP64 path with the reference's sum order (sum_order 0, the default):
every global sum of a level solve is the reference's double bit for bit, so
the CUDA path takes the reference's gradient-flow steps and returns the
reference's displacements and energies exactly.

The pins are the fixtures written by the reference itself (tests/golden,
make_golden.py) and the oracle, which matches them bit for bit; at the
benchmark configuration (513^2, levels 5-9, 30 steps) the fixture holds the
SHA-256 of the reference's displacements."""
import hashlib

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def _digest(px, py):
    return hashlib.sha256(np.concatenate([px, py]).astype("<f8").tobytes()).hexdigest()


@pytest.mark.parametrize("name", ["ops_L5.npz", "ops_L6.npz"])
def test_energy_is_the_reference_double(gpu, name):
    d = golden(name)
    level = int(d["level"])
    for tag in ("", "_clip"):
        px = d["px" + tag] if tag else d["px"]
        e, dex, dey = gpu.energy(level, d["R"], d["T"], px, d["py"], float(d["lam"]), fp64=True)
        assert e == d["E" + tag][2], (tag, e - d["E" + tag][2])


@pytest.mark.parametrize("name", ["gd_L5.npz", "gd_L6.npz"])
def test_level_solve_is_the_reference_solve(gpu, name):
    d = golden(name)
    level = int(d["level"])
    n = (1 << level) + 1
    z = np.zeros(n * n)
    px, py, e, steps, tr = gpu.gd_level(level, d["R"], d["T"], z, z, float(d["lam"]), int(d["max_iter"]), fp64=True)
    ref = d["trace"][1:]   # row 0 of the reference's trace is the initial state
    assert steps == int(d["steps"]) and e == float(d["energy"])
    assert np.array_equal(px, d["px"]) and np.array_equal(py, d["py"])
    # every step: energy, tau, sigma and energy evaluations as in the reference
    assert np.array_equal(tr[:, 0], ref[:, 1]) and np.array_equal(tr[:, 1], ref[:, 2])
    assert np.array_equal(tr[:, 2], ref[:, 3]) and np.array_equal(tr[:, 3], ref[:, 4])


@pytest.mark.parametrize("level,seed", [(7, 71), (8, 81)])
def test_level_solve_from_a_displacement_matches_the_oracle_bit_for_bit(gpu, oracle, level, seed):
    from msgpu import synthetic as syn
    n = (1 << level) + 1
    fr, _, _ = syn.make_series(n, 2, syn.HEX_513, seed=seed)
    R, T = oracle.normalize(fr[0].ravel()), oracle.normalize(fr[1].ravel())
    rng = np.random.default_rng(seed)
    px0, py0 = rng.normal(0, 0.4 / (n - 1), n * n), rng.normal(0, 0.4 / (n - 1), n * n)
    px, py, e, steps, tr = gpu.gd_level(level, R, T, px0, py0, 0.1, 25, fp64=True)
    rx, ry, re, rsteps, rtr = oracle.gd_level(level, R, T, px0, py0, 0.1, 25)
    assert steps == rsteps and e == re
    assert np.array_equal(px, rx) and np.array_equal(py, ry)
    assert [tuple(r[1:]) for r in rtr] == [(row[0], row[1], row[2], int(row[3])) for row in tr]


@pytest.mark.parametrize("case", [0, 1, 2])
def test_multilevel_registration_matches_the_reference_fixture(gpu, case):
    """The three level-7 registrations written by the reference (one with
    resampleInsteadOfProlongateDeformation), bit for bit."""
    import msgpu
    d = golden("register_L7.npz")
    start, stop, lam, lf, mi, se, rs = d[f"case{case}"]
    p = msgpu.default_params(precision_level=7, input_level=7, start_level=int(start), stop_level=int(stop),
                             lambda_=lam, lambda_factor=lf, max_gd_iterations=int(mi), stop_epsilon=se,
                             resample_deformation=int(rs), use_fp64=1, dont_normalize_input=1)
    phis, e, _ = gpu.register_batch(p, d["R"], d["T"][None])
    assert e[0] == d[f"E{case}"][0]
    assert np.array_equal(phis[0], d[f"phi{case}"])


def test_batch_of_frames_matches_the_oracle_bit_for_bit(gpu, oracle):
    """A batch of 257^2 frames, levels 4..8: every frame's displacement and
    energy is the oracle's (the reference's) bit for bit, and a frame's
    result does not depend on the batch it is in."""
    import msgpu
    from msgpu import synthetic as syn
    level = 8
    n = (1 << level) + 1
    fr, _, _ = syn.make_series(n, 4, syn.SQUARE_257, seed=8808)
    p = msgpu.default_params(precision_level=level, input_level=level, start_level=4, stop_level=level,
                             max_gd_iterations=20, use_fp64=1)
    phis, e, steps = gpu.register_batch(p, fr[0], fr[1:])
    R = oracle.normalize(fr[0].ravel())
    for f in range(1, 4):
        T = oracle.normalize(fr[f].ravel())
        px, py, re, rsteps = oracle.register(level, 4, level, R, T, lam=0.1, max_iter=20)
        assert e[f - 1] == re and list(steps[f - 1]) == list(rsteps)
        assert np.array_equal(phis[f - 1, 0], px) and np.array_equal(phis[f - 1, 1], py)
    one, e1, _ = gpu.register_batch(p, fr[0], fr[2:3])
    assert np.array_equal(one[0], phis[1]) and e1[0] == e[1]


def test_benchmark_configuration_is_the_reference_bit_for_bit(gpu):
    """513^2 hexagonal-lattice frames, levels 5..9, 30 steps per level,
    lambda 0.1 (the benchmark's registration): the displacements are the
    reference's byte for byte (SHA-256) and the energies its doubles."""
    import msgpu
    d = golden("exact_L9.npz")
    raw = d["raw"].astype(np.float64)
    p = msgpu.default_params(precision_level=9, input_level=9, start_level=int(d["start"]),
                             stop_level=int(d["stop"]), lambda_=float(d["lam"]),
                             max_gd_iterations=int(d["max_iter"]), use_fp64=1)
    phis, e, _ = gpu.register_batch(p, raw[0], raw[1:])
    n = 513
    for f in range(raw.shape[0] - 1):
        sub = np.stack([phis[f, 0].reshape(n, n)[::16, ::16], phis[f, 1].reshape(n, n)[::16, ::16]])
        dpx = np.abs(sub - d["phi_sub"][f]).max() * (n - 1)
        assert e[f] == d["energies"][f], (f, e[f], d["energies"][f], dpx)
        assert _digest(phis[f, 0], phis[f, 1]) == str(d["digests"][f]), (f, dpx)


def test_certified_steps_give_the_ordered_sums_results(gpu):
    """Control steps taken on bounded sums (the default) against every pass's
    sums added in the reference's order first: the same displacements,
    energies and step counts, bit for bit, while most steps of the energy
    passes are settled by the bounds alone."""
    import msgpu
    from msgpu import synthetic as syn
    level = 8
    n = (1 << level) + 1
    fr, _, _ = syn.make_series(n, 5, syn.SQUARE_257, seed=8812)
    p = msgpu.default_params(precision_level=level, input_level=level, start_level=4, stop_level=level,
                             max_gd_iterations=25, use_fp64=1)
    gpu.set_profiling(True)
    try:
        phis_c, e_c, s_c = gpu.register_batch(p, fr[0], fr[1:])
        st_c = gpu.stats()
        gpu.set_certified_steps(False)
        phis_o, e_o, s_o = gpu.register_batch(p, fr[0], fr[1:])
        st_o = gpu.stats()
    finally:
        gpu.set_certified_steps(True)
        gpu.set_profiling(False)
    assert np.array_equal(phis_c, phis_o)
    assert np.array_equal(e_c, e_o) and np.array_equal(s_c, s_o)
    cert = sum(x["certified_steps"] for x in st_c["level_exact_sums"])
    walked_c = sum(x["passes"] for x in st_c["level_exact_sums"])
    walked_o = sum(x["passes"] for x in st_o["level_exact_sums"])
    assert sum(x["certified_steps"] for x in st_o["level_exact_sums"]) == 0
    assert cert > 0 and walked_c < walked_o, (cert, walked_c, walked_o)


def test_ragged_batch_matches_the_oracle_bit_for_bit(gpu, oracle):
    import msgpu
    from msgpu import synthetic as syn
    p = msgpu.default_params(start_level=4, max_gd_iterations=12, use_fp64=1)
    series = []
    for level, F, seed in ((7, 2, 9701), (6, 3, 9702)):
        n = (1 << level) + 1
        fr, _, _ = syn.make_series(n, F + 1, syn.SQUARE_257, seed=seed)
        series.append((level, fr[0], fr[1:]))
    out = gpu.register_ragged(p, [(ref, tmpl) for _, ref, tmpl in series])
    for (level, ref, tmpl), (phis, energies) in zip(series, out):
        R = oracle.normalize(ref.ravel())
        for f in range(tmpl.shape[0]):
            T = oracle.normalize(tmpl[f].ravel())
            px, py, re, _ = oracle.register(level, 4, level, R, T, lam=0.1, max_iter=12)
            assert energies[f] == re
            assert np.array_equal(phis[f, 0], px) and np.array_equal(phis[f, 1], py)


def test_parallel_sum_order_stays_within_rounding(gpu, oracle):
    """sum_order 1 (the parallel order) gives the same energy to rounding."""
    d = golden("ops_L6.npz")
    gpu.set_sum_order(1)
    try:
        e, _, _ = gpu.energy(6, d["R"], d["T"], d["px"], d["py"], float(d["lam"]), fp64=True)
    finally:
        gpu.set_sum_order(0)
    assert abs(e - d["E"][2]) <= 1e-13 * abs(d["E"][2])


def _sequential(t):
    s = 0.0
    for v in t.tolist():
        s += v
    return s


@pytest.mark.parametrize("level", [6, 9])
def test_exact_sum_is_the_sequential_sum_on_hard_data(level):
    """The reference-order sum on its own (msgpu_exact_sum_device) against a
    plain left-to-right loop, on data made to defeat it: mixed signs, a huge
    dynamic range, dyadic terms that make round-half-even ties frequent,
    cancellations back to zero, signed zeros and subnormals, terms that keep
    the sum crossing binades, and non-finite terms."""
    import torch
    import msgpu
    n = (1 << level) + 1
    N = n * n
    rng = np.random.default_rng(level)
    cases = {
        "normal": rng.normal(size=N),
        "range": np.exp(rng.uniform(-40, 40, N)) * rng.choice([-1.0, 1.0], N),
        "dyadic_ties": rng.integers(-1000, 1000, N) * np.ldexp(1.0, rng.integers(-60, 0, N)),
        "positive_dyadic": rng.integers(1, 8, N) * np.ldexp(1.0, rng.integers(-53, -40, N)),
        "cancel": np.repeat(rng.normal(size=N // 2 + 1), 2)[:N] * np.resize([1.0, -1.0], N),
        "zeros": np.where(rng.random(N) < 0.5, rng.choice([0.0, -0.0, 5e-324, -5e-324], N), rng.normal(size=N)),
        "binades": np.where(np.arange(N) % 3 == 0, 1.0, -np.ldexp(1.0, -rng.integers(1, 60, N))),
    }
    nan = rng.normal(size=N)
    nan[N // 2] = np.nan
    inf = rng.normal(size=N)
    inf[N // 3] = np.inf
    cases["nan"], cases["inf"] = nan, inf
    ctx = msgpu.Context(0)
    try:
        dev = torch.device("cuda", 0)
        out = torch.empty(1, dtype=torch.float64, device=dev)
        for name, t in cases.items():
            d = torch.from_numpy(np.ascontiguousarray(t, dtype=np.float64)).to(dev)
            ctx.exact_sum_device(level, d.data_ptr(), out.data_ptr())
            torch.cuda.synchronize(dev)
            got, want = float(out.item()), _sequential(t)
            if np.isnan(want):
                assert np.isnan(got), name
            else:
                assert got == want and np.signbit(got) == np.signbit(want), (name, got, want)
    finally:
        ctx.close()


def test_pass_timeline_records_every_pass_and_leaves_results_unchanged(gpu):
    """The level kernel's pass timeline (msgpu_set_trace): every published
    pass completes once, every instance finishes once, the waits for work
    it records are at least 500 ns, and tracing does not change a bit of
    the results."""
    import msgpu
    from msgpu import synthetic as syn
    level, F = 7, 4
    n = (1 << level) + 1
    fr, _, _ = syn.make_series(n, F + 1, syn.SQUARE_257, seed=8813)
    p = msgpu.default_params(precision_level=level, input_level=level, start_level=5, stop_level=level,
                             max_gd_iterations=12, use_fp64=1)
    plain = gpu.register_batch(p, fr[0], fr[1:])
    gpu.set_profiling(True)
    gpu.set_trace(level, 1 << 18)
    try:
        traced = gpu.register_batch(p, fr[0], fr[1:])
        tr = gpu.trace()
    finally:
        gpu.set_trace(-1, 0)
        gpu.set_profiling(False)
    for a, b in zip(plain, traced):
        assert np.array_equal(a, b)
    ev, val = tr["event"], tr["value"]
    assert tr["t"].size > 0 and np.all(np.diff(tr["t"]) >= 0)
    kind = val & 255
    done = (ev == 1) & (kind == 13)
    assert sorted((val[done] >> 8).tolist()) == list(range(F))
    for i in range(F):
        pub = (ev == 1) & ((val >> 8) == i) & (kind != 13)
        com = (ev == 2) & ((val >> 8) == i)
        assert pub.sum() == com.sum() > 0, i
        # the passes complete in the order they were published
        assert np.array_equal(kind[pub], kind[com]), i
    assert np.all(val[ev == 3] >= 500)


def test_pass_timeline_of_a_ragged_batch(gpu):
    """The ragged entry point records the timeline too: at a level that two
    series of different sizes both pass, every instance of both finishes
    once and every pass it published completes."""
    import msgpu
    from msgpu import synthetic as syn
    p = msgpu.default_params(start_level=4, max_gd_iterations=8, use_fp64=1)
    series = []
    for level, F, seed in ((7, 2, 9801), (6, 3, 9802)):
        n = (1 << level) + 1
        fr, _, _ = syn.make_series(n, F + 1, syn.SQUARE_257, seed=seed)
        series.append((fr[0], fr[1:]))
    plain = gpu.register_ragged(p, series)
    gpu.set_profiling(True)
    gpu.set_trace(6, 1 << 18)
    try:
        traced = gpu.register_ragged(p, series)
        tr = gpu.trace()
    finally:
        gpu.set_trace(-1, 0)
        gpu.set_profiling(False)
    for (pa, ea), (pb, eb) in zip(plain, traced):
        assert np.array_equal(pa, pb) and np.array_equal(ea, eb)
    ev, val = tr["event"], tr["value"]
    kind = val & 255
    done = (ev == 1) & (kind == 13)
    assert sorted((val[done] >> 8).tolist()) == list(range(5))
    for i in range(5):
        pub = (ev == 1) & ((val >> 8) == i) & (kind != 13)
        com = (ev == 2) & ((val >> 8) == i)
        assert pub.sum() == com.sum() > 0, i
