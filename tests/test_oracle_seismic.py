"""The CPU oracle's seismic energy pieces against golden fixtures produced by
the reference itself: FELineShiftRegisEnergy (registration.h:2137-2193, the
1-D NCC per line of matchSeismicSeries) with its derivative, and the
anisotropic regulariser of findXShift (matchSeries.h:819-845).  Bit for bit."""
import numpy as np
import pytest

from conftest import golden


@pytest.mark.parametrize("tag", ["a", "b"])
def test_line_shift_energy_and_derivative_bit_exact(oracle, tag):
    g = golden("seismic.npz")
    e, de = oracle.lineshift(g[f"R_{tag}"], g[f"T_{tag}"], g[f"phi_{tag}"])
    assert e == float(g[f"E_{tag}"])
    assert np.array_equal(de, g[f"DE_{tag}"])


def test_nan_lines_are_skipped(oracle):
    g = golden("seismic.npz")
    _, de = oracle.lineshift(g["R_a"], g["T_a"], g["phi_a"])
    assert np.all(de[4] == 0) and np.all(np.isfinite(de))


@pytest.mark.parametrize("tag", ["a", "b"])
def test_xshift_regulariser_bit_exact(oracle, tag):
    g = golden("seismic.npz")
    e, k = oracle.xshift_reg(g[f"phi_{tag}"], float(g[f"yreg_{tag}"]))
    assert e == float(g[f"Ereg_{tag}"])
    assert np.array_equal(k, g[f"Kphi_{tag}"])
