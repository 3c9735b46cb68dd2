"""CUDA path with the normalized cross-correlation data term against the
reference (golden fixtures from NCCRegistrationConfigurator) and the oracle.

Tolerances as for the SSD path: FP64 energies and variations within 1e-13
relative (the global sums are reordered), level solves with identical Armijo
and filter-width decisions, displacements within 1e-6 px and energies within
1e-9 relative of the reference."""
import contextlib

import numpy as np
import pytest

from conftest import golden

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.abs(np.asarray(a) - np.asarray(b)).max() / max(1e-300, np.abs(b).max()))


@contextlib.contextmanager
def ncc_operators(gpu):
    gpu.set_data_term(1)
    try:
        yield
    finally:
        gpu.set_data_term(0)


def _params(level, **kw):
    import msgpu
    p = msgpu.default_params(precision_level=level, input_level=level, data_term=1)
    for k, v in kw.items():
        setattr(p, "lambda_" if k == "lam" else k, v)
    return p


@pytest.mark.parametrize("level", [5, 6])
def test_ncc_energy_and_variation(gpu, level):
    g = golden(f"ncc_L{level}.npz")
    with ncc_operators(gpu):
        for tag, qx in (("", g["px"]), ("_out", g["px_out"])):
            e, gx, gy = gpu.energy(level, g["R"], g["T"], qx, g["py"], float(g["lam"]), fp64=1)
            assert abs(e - g["E" + tag][2]) / abs(g["E" + tag][2]) <= 1e-13
            assert rel(np.stack([gx, gy]), g["DE" + tag]) <= 1e-13
            e32, gx32, _ = gpu.energy(level, g["R"], g["T"], qx, g["py"], float(g["lam"]), fp64=0)
            assert abs(e32 - g["E" + tag][2]) / abs(g["E" + tag][2]) <= 1e-5
            assert rel(gx32, g["DE" + tag][0]) <= 1e-4


@pytest.mark.parametrize("level", [5, 6])
def test_ncc_level_gradient_flow_matches_reference_trace(gpu, level):
    g = golden(f"ncc_L{level}.npz")
    n = (1 << level) + 1
    z = np.zeros(n * n)
    with ncc_operators(gpu):
        px, py, e, steps, trace = gpu.gd_level(level, g["R"], g["T"], z, z, float(g["lam"]), int(g["max_iter"]),
                                               fp64=1)
    ref = g["gd_trace"][1:]
    assert steps == int(g["gd_steps"])
    assert np.array_equal(trace[:, 1], ref[:, 2])   # accepted tau
    assert np.array_equal(trace[:, 2], ref[:, 3])   # filter width
    assert np.array_equal(trace[:, 3], ref[:, 4])   # energy evaluations
    assert np.abs(trace[:, 0] - ref[:, 1]).max() / np.abs(ref[:, 1]).max() <= 1e-9
    assert abs(e - float(g["gd_energy"])) / abs(float(g["gd_energy"])) <= 1e-9
    assert max(np.abs(px - g["gd_px"]).max(), np.abs(py - g["gd_py"]).max()) * (n - 1) <= 1e-6


def test_ncc_multilevel_registration_matches_reference(gpu):
    g = golden("ncc_register_L7.npz")
    n = (1 << 7) + 1
    p = _params(7, start_level=int(g["start"]), stop_level=7, lam=float(g["lam"]),
                max_gd_iterations=int(g["max_iter"]), use_fp64=1, dont_normalize_input=1)
    phis, en, steps = gpu.register_batch(p, g["R"], g["T"][None])
    assert np.abs(phis[0] - g["phi"]).max() * (n - 1) <= 1e-6
    assert abs(en[0] - g["E"][0]) / abs(g["E"][0]) <= 1e-9


def test_ncc_batch_of_frames_matches_oracle(gpu, oracle):
    from msgpu import synthetic as syn
    level, F = 8, 3
    n = (1 << level) + 1
    fr, _, _ = syn.make_series(n, F + 1, syn.HEX_513, seed=88)
    frames = fr.reshape(F + 1, -1)
    p = _params(level, start_level=5, stop_level=level, max_gd_iterations=10, use_fp64=1)
    phis, en, _ = gpu.register_batch(p, frames[0], frames[1:])
    R = oracle.normalize(frames[0])
    for f in range(F):
        T = oracle.normalize(frames[f + 1])
        qx, qy, e, _ = oracle.register(level, 5, level, R, T, lam=0.1, max_iter=10, ncc=True)
        assert max(np.abs(phis[f, 0] - qx).max(), np.abs(phis[f, 1] - qy).max()) * (n - 1) <= 1e-6
        assert abs(en[f] - e) / abs(e) <= 1e-9


def test_ncc_fp32_within_conditioning(gpu):
    from msgpu import synthetic as syn
    level = 6
    n = (1 << level) + 1
    fr, _, _ = syn.make_series(n, 2, syn.HEX_513, seed=19)
    frames = fr.reshape(2, -1)
    a = gpu.register_batch(_params(level, start_level=4, stop_level=level, max_gd_iterations=15, use_fp64=1),
                           frames[0], frames[1:])
    b = gpu.register_batch(_params(level, start_level=4, stop_level=level, max_gd_iterations=15, use_fp64=0),
                           frames[0], frames[1:])
    assert abs(b[1][0] - a[1][0]) / abs(a[1][0]) <= 2e-2
    assert np.abs(b[0] - a[0]).max() * (n - 1) <= 1.0
