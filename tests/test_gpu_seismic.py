"""CUDA energy of the seismic line-shift model against the reference (golden
fixtures from FELineShiftRegisEnergy and findXShift's regulariser) and the
oracle.  The line kernel reduces each line's three global sums (mean, norm,
correlation) in a fixed parallel order instead of the reference's sequential
loops: energies within 1e-13 relative, derivatives within 1e-12 of their
largest entry.  K phi is a nine-point stencil with the reference's assembled
coefficients and summation order: bit for bit."""
import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["a", "b"])
def test_line_shift_energy_matches_reference(gpu, tag):
    g = golden("seismic.npz")
    e, de = gpu.lineshift_energy(g[f"R_{tag}"], g[f"T_{tag}"], g[f"phi_{tag}"])
    ref_e, ref_de = float(g[f"E_{tag}"]), g[f"DE_{tag}"]
    assert abs(e - ref_e) <= 1e-13 * abs(ref_e)
    assert np.abs(de - ref_de).max() <= 1e-12 * np.abs(ref_de).max()
    if tag == "a":
        assert np.all(de[4] == 0)


def test_line_shift_energy_long_lines_against_oracle(gpu, oracle):
    rng = np.random.default_rng(9)
    nx, ny = 2049, 33
    x = np.arange(nx)
    R = np.stack([np.sin(x / 7.0 + k) + 0.2 * rng.normal(size=nx) for k in range(ny)])
    T = np.stack([np.sin((x - 2.5) / 7.0 + k) + 0.2 * rng.normal(size=nx) for k in range(ny)])
    phi = rng.normal(0, 2.0 / (nx - 1), (ny, nx))
    e, de = gpu.lineshift_energy(R, T, phi)
    re, rde = oracle.lineshift(R, T, phi)
    assert abs(e - re) <= 1e-12 * abs(re)
    assert np.abs(de - rde).max() <= 1e-11 * np.abs(rde).max()


@pytest.mark.parametrize("tag", ["a", "b"])
def test_xshift_regulariser_matches_reference(gpu, tag):
    g = golden("seismic.npz")
    e, k = gpu.xshift_reg(g[f"phi_{tag}"], float(g[f"yreg_{tag}"]))
    assert np.array_equal(k, g[f"Kphi_{tag}"])
    assert abs(e - float(g[f"Ereg_{tag}"])) <= 1e-13 * abs(float(g[f"Ereg_{tag}"]))
