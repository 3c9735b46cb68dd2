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


@pytest.mark.parametrize("tag", ["a", "b"])
def test_h1_metric_system_matrix_bit_exact_and_inverse(oracle, tag):
    """InverseH1MetricBase's system matrix M + 0.5 sigma^2 L is the
    reference's bit for bit; the oracle's band Cholesky inverts it to
    rounding (the reference inverts it with SuiteSparse's CHOLMOD, which it
    does not vendor)."""
    g = golden("seismic.npz")
    x, sg = g[f"h1x_{tag}"], float(g[f"h1sigma_{tag}"])
    assert np.array_equal(oracle.h1sys_apply(x, sg), g[f"h1y_{tag}"])
    z = oracle.h1_metric(x, sg)
    assert np.abs(oracle.h1sys_apply(z, sg) - x).max() <= 1e-13 * np.abs(x).max()


def test_xshift_recovers_a_line_shift(oracle):
    """findXShift on lines shifted by 1.5 px: the energy decreases step by
    step, the filter width halves on the way, and the mean shift found is
    the planted one."""
    rng = np.random.default_rng(6)
    nx, ny = 65, 17
    x = np.arange(nx)
    R = np.stack([np.sin(x / 4.0 + 0.3 * k) + 0.05 * rng.normal(size=nx) for k in range(ny)])
    T = np.stack([np.sin((x - 1.5) / 4.0 + 0.3 * k) + 0.05 * rng.normal(size=nx) for k in range(ny)])
    ph, e, steps, rows = oracle.xshift(R, T, 0.01, 1.0, 60)
    energies = [r[1] for r in rows]
    assert all(b <= a for a, b in zip(energies, energies[1:]))
    assert rows[-1][3] < rows[0][3]
    assert abs(ph[:, 8:-8].mean() * (nx - 1) - 1.5) < 0.05


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_laplace_regulariser_bit_exact(oracle, tag):
    """findXShift's regulariser with laplaceWeight > 0 (matchSeries.h:828-838):
    laplaceWeight L M^-1 L (qc::assembleLaplaceSquareRegMatrix) + stiffX +
    yRegFactor stiffY applied as the reference's CSR matrix, bit for bit."""
    g = golden("seismic.npz")
    e, k = oracle.xshift_reg_laplace(g[f"phi_{tag}"], float(g[f"yreg_{tag}"]), float(g[f"lapw_{tag}"]))
    assert e == float(g[f"Elap_{tag}"])
    assert np.array_equal(k, g[f"Kphilap_{tag}"])


def test_laplace_regulariser_against_the_reference_driver(oracle):
    if not oracle.have_ref():
        pytest.skip("the reference driver is not built here")
    rng = np.random.default_rng(12)
    phi = rng.normal(0, 0.1, (11, 23))
    e, k = oracle.xshift_reg_laplace(phi, 0.7, 2.5)
    re, rk = oracle.RefRunner().xshift_reg_laplace(phi, 0.7, 2.5)
    assert e == re and np.array_equal(k, rk)


def test_xshift_with_laplace_weight_recovers_a_line_shift(oracle):
    rng = np.random.default_rng(6)
    nx, ny = 65, 17
    x = np.arange(nx)
    R = np.stack([np.sin(x / 4.0 + 0.3 * k) + 0.05 * rng.normal(size=nx) for k in range(ny)])
    T = np.stack([np.sin((x - 1.5) / 4.0 + 0.3 * k) + 0.05 * rng.normal(size=nx) for k in range(ny)])
    ph, e, steps, rows = oracle.xshift(R, T, 0.01, 1.0, 60, laplace_weight=0.01)
    energies = [r[1] for r in rows]
    assert all(b <= a for a, b in zip(energies, energies[1:]))
    assert abs(ph[:, 8:-8].mean() * (nx - 1) - 1.5) < 0.1


@pytest.mark.parametrize("tag", ["a", "b"])
def test_xshift_yconst_bit_exact(oracle, tag):
    """findXShiftYConst (forceNonDyadicXShiftYConst, matchSeries.h:873-920):
    one shift per line, four gridless NCG descents against the template
    smoothed along x; the reference's own run, bit for bit (tag b has a NaN
    line, whose NaN also reaches the neighbouring lines of the smoothed
    template through the filter's zero rows)."""
    g = golden("seismic.npz")
    ph, e, _ = oracle.xshift_yconst(g[f"ycR_{tag}"], g[f"ycT_{tag}"], 60, g[f"ycphi0_{tag}"])
    assert e == float(g[f"ycE_{tag}"])
    assert np.array_equal(ph, g[f"ycphi_{tag}"])


def test_box_filter_keeps_lines_and_spreads_nan(oracle):
    T = np.arange(5 * 11, dtype=float).reshape(5, 11)
    T[2, 4] = np.nan
    B = oracle.box_x(T, 1)   # 5-wide box, 5 x 5 window
    assert np.isnan(B[0:5, 2:7]).all() and np.isfinite(B[:, 8:]).all()
    ok = T.copy()
    ok[2, 4] = 0.0
    B2 = oracle.box_x(ok, 1)
    x = 6
    assert B2[1, x] == sum(0.2 * ok[1, (x + k) % 11] for k in range(-2, 3))


def test_empty_lines_to_nan_matches_the_reference(oracle):
    """replaceEmptyLinesWithNaN (matchSeismicSeries.h:141-157): the reference's own run, NaN for NaN."""
    g = golden("seismic.npz")
    out, n = oracle.empty_lines_to_nan(g["enR"])
    assert np.array_equal(out, g["enOut"], equal_nan=True)
    assert n == 5


@pytest.mark.parametrize("keep", [0, 1])
def test_remove_empty_lines_matches_the_reference(oracle, keep):
    """removeEmptyLinesFromImage (matchSeismicSeries.h:101-136): the reference's own run, bit for bit."""
    g = golden("seismic.npz")
    out = oracle.remove_empty_lines(g["rmR"], bool(keep))
    ref = g[f"rmOut{keep}"]
    assert out.shape == ref.shape and np.array_equal(out.view(np.uint64), ref.view(np.uint64))


def test_remove_empty_lines_error_codes(oracle):
    assert oracle.remove_empty_lines(np.zeros((4, 5))) == -1
    one = np.zeros((4, 5))
    one[2] = 1.0
    assert oracle.remove_empty_lines(one, True) == -2
    assert oracle.remove_empty_lines(one, False).shape == (1, 5)
