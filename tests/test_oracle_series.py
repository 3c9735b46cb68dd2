"""The CPU oracle's series pipeline against golden fixtures produced by the
reference itself: ConcatAndSmoothlyExtendDeformations (deformations.h:
364-410, 498-520), the median of warped frames (matchSeries.h:442,
multiVector.cpp:99-117) and the stage loop of matchSeries<>() with
accumulated deformations, refinement and an extra stage against the median
(matchSeries.h:87-265, 353-445, 1250-1320).  All comparisons are bit for bit."""
import numpy as np

from conftest import golden


def test_compose_with_extension_bit_exact(oracle):
    g = golden("compose_L6.npz")
    assert np.array_equal(oracle.compose(6, g["d1"], g["d2"]), g["out"])
    assert np.array_equal(oracle.compose(6, g["d1"], g["d2_in"]), g["out_in"])


def test_warp_median_odd_and_even_counts_bit_exact(oracle):
    g = golden("compose_L6.npz")
    assert np.array_equal(oracle.warp_median(6, g["frames"], g["phis"], 0.5), g["med5"])
    assert np.array_equal(oracle.warp_median(6, g["frames"][:4], g["phis"][:4], 0.25), g["med4"])


def test_compose_identities(oracle):
    """d2 = 0: no node leaves the domain, the result is d1; d1 = 0: the
    result is d2 where x + d2(x) stays inside, and the discrete harmonic
    extension (rows of the stiffness matrix vanish) where it leaves."""
    g = golden("compose_L6.npz")
    n = 65
    z = np.zeros_like(g["d1"])
    assert np.array_equal(oracle.compose(6, g["d1"], z), g["d1"])
    d2 = g["d2"]
    out = oracle.compose(6, z, d2)
    y, x = np.mgrid[0:n, 0:n]
    X = x.ravel() + d2[0] * (n - 1)
    Y = y.ravel() + d2[1] * (n - 1)
    undef = (X < 0) | (X > n - 1) | (Y < 0) | (Y > n - 1)
    assert undef.sum() > 100
    assert np.array_equal(out[:, ~undef], d2[:, ~undef])
    for c in range(2):
        Lu = oracle.stiff_apply(6, out[c])
        assert np.abs(Lu[undef]).max() < 1e-7


def test_match_series_stages_bit_exact(oracle):
    g = golden("match_series_L6.npz")
    kw = dict(start=int(g["start"]), stop=int(g["stop"]), max_iter=int(g["max_iter"]),
              refine_start=int(g["refine_start"]), extra_stages=int(g["extra_stages"]),
              extra_lam_factor=float(g["extra_lam_factor"]), use_median=bool(g["use_median"]))
    phis, avg, med, cnt, energies = oracle.match_series(6, frames=g["frames"], **kw)
    assert np.array_equal(phis, g["phis"])
    assert np.array_equal(avg, g["avg"]) and np.array_equal(med, g["median"]) and np.array_equal(cnt, g["count"])
    assert np.array_equal(energies[0], g["energies1"]) and np.array_equal(energies[1], g["energies2"])


def test_match_series_conditioned_fixture_bit_exact(oracle):
    g = golden("match_series_wc_L6.npz")
    kw = dict(start=int(g["start"]), stop=int(g["stop"]), max_iter=int(g["max_iter"]),
              refine_start=int(g["refine_start"]), extra_stages=int(g["extra_stages"]),
              extra_lam_factor=float(g["extra_lam_factor"]), use_median=bool(g["use_median"]))
    phis, avg, med, cnt, energies = oracle.match_series(6, frames=g["frames"], **kw)
    assert np.array_equal(phis, g["phis"]) and np.array_equal(med, g["median"])
    assert np.array_equal(energies[1], g["energies2"])
    assert float(g["spread_px"]) < 1e-7
