"""The CPU oracle's normalized cross-correlation data term against the
golden fixtures produced by the reference itself (NCCRegistrationConfigurator,
registration.h:1766-1780, 1909-2018).  All comparisons are bit for bit."""
import numpy as np
import pytest

from conftest import golden


@pytest.mark.parametrize("level", [5, 6])
def test_ncc_energy_and_variation_bit_exact(oracle, level):
    g = golden(f"ncc_L{level}.npz")
    R, T, py, lam = g["R"], g["T"], g["py"], float(g["lam"])
    for tag, qx in (("", g["px"]), ("_out", g["px_out"])):
        e, ereg = oracle.energy(level, R, T, qx, py, lam, ncc=True)
        encc = oracle.ncc_energy(level, R, T, qx, py)
        assert np.array_equal([encc, ereg, e], g["E" + tag])
        gx, gy = oracle.denergy(level, R, T, qx, py, lam, ncc=True)
        assert np.array_equal(np.stack([gx, gy]), g["DE" + tag])
        fx, fy = oracle.denergy(level, R, T, qx, py, 0.0, ncc=True)
        assert np.array_equal(np.stack([fx, fy]), g["F" + tag])


@pytest.mark.parametrize("level", [5, 6])
def test_ncc_gradient_flow_trace_bit_exact(oracle, level):
    g = golden(f"ncc_L{level}.npz")
    n = (1 << level) + 1
    z = np.zeros(n * n)
    px, py, e, steps, trace = oracle.gd_level(level, g["R"], g["T"], z, z, float(g["lam"]), int(g["max_iter"]),
                                              ncc=True)
    assert steps == int(g["gd_steps"]) and e == float(g["gd_energy"])
    assert np.array_equal(px, g["gd_px"]) and np.array_equal(py, g["gd_py"])
    ref = g["gd_trace"][1:]
    got = np.array([[t[0], t[1], t[2], t[3], t[4]] for t in trace])
    assert np.array_equal(got, ref)


def test_ncc_multilevel_registration_bit_exact(oracle):
    g = golden("ncc_register_L7.npz")
    px, py, e, _ = oracle.register(7, int(g["start"]), 7, g["R"], g["T"], lam=float(g["lam"]),
                                   max_iter=int(g["max_iter"]), ncc=True)
    assert e == float(g["E"][0])
    assert np.array_equal(np.stack([px, py]), g["phi"])


def test_mass_matrix_integrates_constants(oracle):
    # sum_i (M 1)_i is the area of the unit square; M is symmetric positive
    for level in (3, 5):
        n = (1 << level) + 1
        assert abs(oracle.mass_apply(level, np.ones(n * n)).sum() - 1.0) < 1e-13
        rng = np.random.default_rng(level)
        u, v = rng.normal(size=n * n), rng.normal(size=n * n)
        assert abs(u @ oracle.mass_apply(level, v) - v @ oracle.mass_apply(level, u)) < 1e-12
        assert u @ oracle.mass_apply(level, u) > 0
