"""The CPU oracle against the golden fixtures produced by the reference itself.

All comparisons are exact: the restatement follows the reference's operation
order, so equality is bit for bit."""
import numpy as np
import pytest

from conftest import golden


@pytest.mark.parametrize("level", [5, 6])
def test_operators_bit_exact(oracle, level):
    g = golden(f"ops_L{level}.npz")
    R, T, px, py, lam = g["R"], g["T"], g["px"], g["py"], float(g["lam"])
    for tag, qx in (("", px), ("_clip", g["px_clip"])):
        e, ereg = oracle.energy(level, R, T, qx, py, lam)
        essd = oracle.ssd_energy(level, R, T, qx, py)
        assert np.array_equal([essd, ereg, e], g["E" + tag])
        gx, gy = oracle.denergy(level, R, T, qx, py, lam)
        assert np.array_equal(np.stack([gx, gy]), g["DE" + tag])
        fx, fy = oracle.ssd_force(level, R, T, qx, py)
        assert np.array_equal(np.stack([fx, fy]), g["F" + tag])
    for s, out in zip(g["smooth_sigmas"], g["smooth_out"]):
        assert np.array_equal(oracle.smooth(level, s, g["smooth_in"]), out)
    assert np.array_equal(oracle.restrict(level, g["smooth_in"]), g["restrict_out"])
    assert np.array_equal(oracle.prolong(level - 1, g["prolong_in"]), g["prolong_out"])
    assert np.array_equal(oracle.resample(level - 1, g["prolong_in"], level), g["resample_out"])
    assert np.array_equal(oracle.deform_image(level, g["raw_t"], g["deform_px"], g["deform_py"]), g["deform_out"])
    assert np.array_equal(oracle.normalize(g["raw_t"]), g["normalize_out"])
    assert np.array_equal(oracle.normalize(g["raw_t"], sat=-1, min_to_zero=1), g["normalize_nosat_out"])


@pytest.mark.parametrize("level", [5, 6])
def test_gradient_flow_trace_bit_exact(oracle, level):
    g = golden(f"gd_L{level}.npz")
    n = (1 << level) + 1
    z = np.zeros(n * n)
    px, py, e, steps, trace = oracle.gd_level(level, g["R"], g["T"], z, z, float(g["lam"]), int(g["max_iter"]))
    assert steps == int(g["steps"])
    assert e == float(g["energy"])
    assert np.array_equal(px, g["px"]) and np.array_equal(py, g["py"])
    ref_trace = g["trace"][1:]  # row 0 is the initial energy
    got = np.array([[t[0], t[1], t[2], t[3], t[4]] for t in trace])
    assert np.array_equal(got, ref_trace)


def test_multilevel_register_bit_exact(oracle):
    g = golden("register_L7.npz")
    for i in range(3):
        start, stop, lam, lf, mi, se, rs = g[f"case{i}"]
        px, py, e, _ = oracle.register(7, int(start), int(stop), g["R"], g["T"], lam=lam, lam_factor=lf,
                                       max_iter=int(mi), stop_eps=se, resample_phi=bool(rs))
        assert np.array_equal(np.stack([px, py]), g[f"phi{i}"]), i
        assert e == float(g[f"E{i}"][0]), i


def test_series_stage_bit_exact(oracle):
    g = golden("series_L6.npz")
    level, frames = int(g["level"]), g["frames"]
    F = frames.shape[0]
    R = oracle.normalize(frames[0])
    phis = np.zeros((F, 2, frames.shape[1]))
    for f in range(1, F):
        T = oracle.normalize(frames[f])
        px, py, e, _ = oracle.register(level, int(g["start"]), level, R, T, lam=float(g["lam"]),
                                       max_iter=int(g["max_iter"]))
        phis[f] = [px, py]
        assert e == g["energies"][f]
    assert np.array_equal(phis, g["phis"])
    mean, count = oracle.warp_mean(level, frames, phis)
    assert np.array_equal(mean, g["mean"])


def test_live_reference_random_seeds(oracle):
    """When the reference driver is built here, compare on fresh seeds too."""
    import msor
    if not msor.have_ref():
        pytest.skip("oracle/_ref/ms_ref not built")
    from msgpu import synthetic as syn
    ref = msor.RefRunner()
    for seed in (5, 6):
        level = 5
        n = (1 << level) + 1
        fr, _, _ = syn.make_series(n, 2, syn.HEX_513, seed=seed)
        R, T = oracle.normalize(fr[0].ravel()), oracle.normalize(fr[1].ravel())
        a = ref.register(level, 3, level, R, T, lam=0.07, max_iter=25)
        b = oracle.register(level, 3, level, R, T, lam=0.07, max_iter=25)
        assert np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) and a[2] == b[2]
