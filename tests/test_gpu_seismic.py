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


def _shifted_lines(nx, ny, shift, seed):
    rng = np.random.default_rng(seed)
    x = np.arange(nx)
    R = np.stack([np.sin(x / 4.0 + 0.3 * k) + 0.05 * rng.normal(size=nx) for k in range(ny)])
    T = np.stack([np.sin((x - shift) / 4.0 + 0.3 * k) + 0.05 * rng.normal(size=nx) for k in range(ny)])
    return R, T


def test_find_xshift_matches_oracle(gpu, oracle):
    """findXShift on the GPU (spectral H1 metric) against the oracle (band
    Cholesky): the same steps and filter widths, energies within 1e-9
    relative, shifts within 1e-6 px, and the planted shift recovered."""
    nx, ny = 65, 17
    R, T = _shifted_lines(nx, ny, 1.5, 6)
    ph, e, steps = gpu.find_xshift(R, T, 0.01, 1.0, 60)
    rph, re, rsteps, _ = oracle.xshift(R, T, 0.01, 1.0, 60)
    assert steps == rsteps
    assert abs(e - re) <= 1e-9 * abs(re)
    assert np.abs(ph - rph).max() * (nx - 1) <= 1e-6
    assert abs(ph[:, 8:-8].mean() * (nx - 1) - 1.5) < 0.05


def test_find_xshift_non_square_larger_grid(gpu, oracle):
    nx, ny = 129, 41
    R, T = _shifted_lines(nx, ny, -2.0, 7)
    ph, e, steps = gpu.find_xshift(R, T, 0.05, 0.5, 40)
    rph, re, rsteps, _ = oracle.xshift(R, T, 0.05, 0.5, 40)
    assert steps == rsteps
    assert abs(e - re) <= 1e-8 * abs(re)
    assert np.abs(ph - rph).max() * (nx - 1) <= 1e-4


@pytest.mark.parametrize("lapw", [0.0, 0.01])
def test_find_xshift_device_control_equals_host_control(gpu, lapw):
    """The descent as one device-controlled graph (conditional while/if
    nodes) against the same descent driven from the host (the default): the
    same steps and bit-identical shifts and energy."""
    nx, ny = 129, 33
    R, T = _shifted_lines(nx, ny, 1.25, 31)
    hph, he, hsteps = gpu.find_xshift(R, T, 0.01, 1.0, 80, laplace_weight=lapw)
    gpu.set_seismic_device_control(True)
    try:
        ph, e, steps = gpu.find_xshift(R, T, 0.01, 1.0, 80, laplace_weight=lapw)
        launches = gpu.stats()["kernel_launches"]
    finally:
        gpu.set_seismic_device_control(False)
    assert steps == hsteps and steps > 5
    assert e == he and np.array_equal(ph, hph)
    assert launches <= 2


def test_find_xshift_batch_equals_single_calls(gpu):
    """Images spread over worker threads with their own streams: every image's
    result equals, bit for bit, its own single call."""
    nx, ny = 65, 17
    Rs, Ts = zip(*[_shifted_lines(nx, ny, s, 20 + i) for i, s in enumerate((1.0, -0.5, 2.0, 0.0, 1.5))])
    R = np.stack(Rs)
    T = np.stack(Ts)
    ph, en, st = gpu.find_xshift_batch(R, T, 0.01, 1.0, 30, workers=3)
    for i in range(len(T)):
        p1, e1, s1 = gpu.find_xshift(R[i], T[i], 0.01, 1.0, 30)
        assert np.array_equal(ph[i], p1) and en[i] == e1 and st[i] == s1
    # one reference for all images
    ph2, en2, _ = gpu.find_xshift_batch(R[0], T, 0.01, 1.0, 30, workers=2)
    p1, e1, _ = gpu.find_xshift(R[0], T[3], 0.01, 1.0, 30)
    assert np.array_equal(ph2[3], p1) and en2[3] == e1


@pytest.mark.parametrize("tag", ["a", "b", "c"])
def test_laplace_regulariser_matches_reference(gpu, tag):
    """laplaceWeight > 0: laplaceWeight L M^-1 L + stiffX + yRegFactor stiffY;
    K phi bit for bit against the reference's CSR matrix, the energy (a
    block-parallel sum) within 1e-13."""
    g = golden("seismic.npz")
    e, k = gpu.xshift_reg(g[f"phi_{tag}"], float(g[f"yreg_{tag}"]), float(g[f"lapw_{tag}"]))
    assert np.array_equal(k, g[f"Kphilap_{tag}"])
    assert abs(e - float(g[f"Elap_{tag}"])) <= 1e-13 * abs(float(g[f"Elap_{tag}"]))


def test_find_xshift_with_laplace_weight_matches_oracle(gpu, oracle):
    nx, ny = 65, 17
    R, T = _shifted_lines(nx, ny, 1.5, 6)
    ph, e, steps = gpu.find_xshift(R, T, 0.01, 1.0, 60, laplace_weight=0.01)
    rph, re, rsteps, _ = oracle.xshift(R, T, 0.01, 1.0, 60, laplace_weight=0.01)
    assert steps == rsteps
    assert abs(e - re) <= 1e-9 * abs(re)
    assert np.abs(ph - rph).max() * (nx - 1) <= 1e-6
    assert abs(ph[:, 8:-8].mean() * (nx - 1) - 1.5) < 0.1


def test_laplace_weight_needs_five_nodes(gpu):
    import msgpu
    with pytest.raises(msgpu.MsgpuError, match="5 x 5"):
        gpu.xshift_reg(np.zeros((4, 9)), 1.0, 0.5)


@pytest.mark.parametrize("tag", ["a", "b"])
def test_find_xshift_yconst_matches_reference(gpu, tag):
    """findXShiftYConst on the GPU (line-shift kernel in row mode, control
    on the host) against the reference's own run: the same iterates, so the
    shifts and the energy agree to rounding of the device sums."""
    g = golden("seismic.npz")
    R, T = g[f"ycR_{tag}"], g[f"ycT_{tag}"]
    nx = R.shape[1]
    ph, e, steps = gpu.find_xshift_yconst(R, T, 60, g[f"ycphi0_{tag}"])
    ref = g[f"ycphi_{tag}"]
    assert np.all(ph == ph[:, :1])
    assert np.abs(ph - ref).max() * (nx - 1) <= 1e-9
    assert abs(e - float(g[f"ycE_{tag}"])) <= 1e-12 * abs(float(g[f"ycE_{tag}"]))


def test_empty_lines_to_nan_matches_reference(gpu):
    """replaceEmptyLinesWithNaN on the GPU against the reference's own run
    (zero and -0.0 lines, squares that underflow to 0, a NaN line, a
    subnormal square), NaN for NaN, bit for bit."""
    g = golden("seismic.npz")
    out, n = gpu.empty_lines_to_nan(g["enR"])
    assert n == 5
    assert np.array_equal(out.view(np.uint64), g["enOut"].view(np.uint64))


def test_empty_lines_to_nan_batched_on_device_then_skipped_by_the_energy(gpu, oracle):
    """Three images in one launch on device memory; the lines it turns into
    NaN then contribute nothing to the line-shift energy, as in the
    reference (registration.h:2150-2151)."""
    import torch
    rng = np.random.default_rng(31)
    imgs = rng.normal(size=(3, 9, 40))
    imgs[0, 2] = 0.0
    imgs[2, [0, 8]] = 0.0
    d = torch.from_numpy(imgs).cuda()
    n = gpu.empty_lines_to_nan_device(d.data_ptr(), 40, 9, 3, torch.cuda.current_stream().cuda_stream)
    torch.cuda.synchronize()
    out = d.cpu().numpy()
    ref = np.stack([oracle.empty_lines_to_nan(im)[0] for im in imgs])
    assert n == 3 and np.array_equal(out.view(np.uint64), ref.view(np.uint64))
    phi = rng.normal(0, 0.02, (9, 40))
    e, _ = gpu.lineshift_energy(out[1], out[0], phi)
    eo, _ = oracle.lineshift(out[1], out[0], phi)
    assert np.isfinite(e) and abs(e - eo) <= 1e-12 * abs(eo)


def test_non_dyadic_update_with_empty_lines_matches_oracle(gpu, oracle):
    """updateNonDyadicDeformation of the seismic descent: empty lines (here a
    gap at the top and one inside) become NaN and drop out of the data term;
    findXShift then matches the oracle run on the same NaN-lined images."""
    nx, ny = 65, 17
    R, T = _shifted_lines(nx, ny, 1.0, 41)
    R[0] = 0.0
    T[9] = 0.0
    ph0 = np.zeros((ny, nx))
    ph, e, steps = gpu.update_non_dyadic_xshift(R, T, 0.01, 1.0, ph0, max_iter=40)
    Rn, n_r = oracle.empty_lines_to_nan(R)
    Tn, n_t = oracle.empty_lines_to_nan(T)
    assert (n_r, n_t) == (1, 1)
    rph, re, rsteps, _ = oracle.xshift(Rn, Tn, 0.01, 1.0, 40)
    assert steps == rsteps and np.isfinite(e)
    assert abs(e - re) <= 1e-9 * abs(re)
    assert np.abs(ph - rph).max() * (nx - 1) <= 1e-6
    # forceNonDyadicXShiftYConst takes the one-shift-per-line solve instead
    phy, ey, _ = gpu.update_non_dyadic_xshift(R, T, 0.01, 1.0, ph0, max_iter=40, force_yconst=True)
    assert np.all(phy == phy[:, :1]) and np.isfinite(ey)
    # nothing to register: every sample of R + T is NaN
    Z = np.zeros((ny, nx))
    phz, ez, sz = gpu.update_non_dyadic_xshift(Z, T, 0.01, 1.0, ph0 + 0.25, max_iter=40)
    assert np.all(phz == 0.25) and np.isnan(ez) and sz == 0
    # the reference then keeps its previous energy of the last solution
    phz, ez, sz = gpu.update_non_dyadic_xshift(Z, T, 0.01, 1.0, ph0 + 0.25, max_iter=40, prev_energy=e)
    assert np.all(phz == 0.25) and ez == e and sz == 0


@pytest.mark.parametrize("keep", [0, 1])
def test_remove_empty_lines_matches_reference(gpu, keep):
    """removeEmptyLinesFromImage on the GPU against the reference's own run
    (an all-NaN line dropped, a line with one number kept), bit for bit."""
    g = golden("seismic.npz")
    out = gpu.remove_empty_lines(g["rmR"], bool(keep))
    ref = g[f"rmOut{keep}"]
    assert out.shape == ref.shape and np.array_equal(out.view(np.uint64), ref.view(np.uint64))


def test_remove_empty_lines_errors_and_larger_image(gpu, oracle):
    import msgpu
    with pytest.raises(msgpu.MsgpuError, match="only empty lines"):
        gpu.remove_empty_lines(np.zeros((6, 300)))
    one = np.zeros((6, 300))
    one[3] = 2.0
    with pytest.raises(msgpu.MsgpuError):
        gpu.remove_empty_lines(one, True)
    rng = np.random.default_rng(33)
    img = np.zeros((513, 1000))
    img[7:500:4] = rng.normal(size=(124, 1000))
    for keep in (False, True):
        assert np.array_equal(gpu.remove_empty_lines(img, keep), oracle.remove_empty_lines(img, keep))
