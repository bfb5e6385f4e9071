"""Distributed series wire loading through the device fill (mw_add_loading):
mixed precision, batched sweeps, the first-order perturbation identity and
the physics windows of the reference's own loading tests."""

import numpy as np
import pytest

from cases import CASES, LOADED
from conftest import golden, rel_err

import momwire_b200
from momwire_b200 import loading as wl

pytestmark = pytest.mark.gpu

SIGMA_CU = 5.8e7
A_28 = 0.16e-3
L_DIP = 10.15
WL = 21.264
DIPOLE = [np.array([[0.0, 0.0, -L_DIP / 2], [0.0, 0.0, L_DIP / 2]])]
LOSSY = dict(wire_conductivity=SIGMA_CU, insulation_radius=0.4e-3, insulation_eps_r=3.0)


def _solver(**kw):
    base = dict(wires=DIPOLE, nsegs=81, wavelength=WL, wire_radius=A_28)
    base.update(kw)
    return momwire_b200.BSplineSolver(**base)


def _zin(y):
    return 1.0 / np.diag(y)


@pytest.mark.parametrize("name", sorted(LOADED))
def test_loaded_mixed_matches_reference(name, cuda_device):
    g = golden(name)
    sol = momwire_b200.BSplineSolver(**CASES[name](), precision="mixed").compute_port_solution()
    assert np.max(np.abs(_zin(sol.y) - _zin(g["y"])) / np.abs(_zin(g["y"]))) <= 1e-6
    assert rel_err(sol.y, g["y"]) < 1e-6


@pytest.mark.parametrize("name", sorted(LOADED))
def test_loaded_batched_fill_mirror(name, cuda_device):
    """The batched fill adds each frequency's own Z'(omega) and keeps the
    complex64 copy the rounded complex128 matrix."""
    import torch

    s = momwire_b200.BSplineSolver(**CASES[name]())
    ks = np.array([0.9, 1.0, 1.1]) * s.k
    Z, Z32 = s._fill_batched(ks, torch.cuda.current_stream().cuda_stream)
    Zh, Z32h = Z.cpu().numpy(), Z32.cpu().numpy()
    for i, kk in enumerate(ks):
        with s._k_restored():
            s._set_k(kk)
            want = s._compute_Z_operator()
        assert rel_err(Zh[i].T, want) < 1e-13
        assert np.array_equal(Z32h[i], Zh[i].astype(np.complex64))
    g = golden(name)
    assert rel_err(Zh[1].T, g["Z"]) < 1e-10


def test_loading_matches_first_order_perturbation(cuda_device):
    """dZin = c0^T L c0 / I0^2 for a small loading, with c0 the unloaded
    coefficients (Galerkin Z is complex symmetric)."""
    z0, c0 = _solver().compute_impedance()
    s1 = _solver(wire_conductivity=5.8e10)
    z1, _ = s1.compute_impedance()
    n = c0.shape[0]
    L = s1._apply_loading(np.zeros((n, n), dtype=np.complex128))
    dz_pred = (c0 @ L @ c0) * z0**2
    assert z1 - z0 == pytest.approx(dz_pred, rel=1e-3)


def test_copper_dipole_loss_physics_window(cuda_device):
    z0, _ = _solver().compute_impedance()
    s = _solver(wire_conductivity=SIGMA_CU)
    z1, c1 = s.compute_impedance()
    rp = np.real(wl.wire_internal_impedance(s.omega, A_28, SIGMA_CU))
    assert z1.real - z0.real == pytest.approx(rp * L_DIP / 2, rel=0.15)
    assert z1.imag - z0.imag == pytest.approx(z1.real - z0.real, rel=0.20)
    p_wire, per_wire = s.wire_loss_power(c1)
    eff = 1.0 - p_wire / (0.5 * np.real(1.0 / np.conj(z1)))
    assert 0.91 < eff < 0.95
    assert per_wire.shape == (1,) and per_wire[0] == pytest.approx(p_wire)


def test_insulation_reactance_shift(cuda_device):
    z0, _ = _solver().compute_impedance()
    s = _solver(insulation_radius=0.4e-3, insulation_eps_r=3.0)
    z1, c1 = s.compute_impedance()
    lp = wl.insulation_inductance(A_28, 0.4e-3, 3.0)
    assert z1.imag - z0.imag == pytest.approx(s.omega * lp * L_DIP / 2, rel=0.15)
    assert z1.imag > z0.imag
    assert s.wire_loss_power(c1)[0] == 0.0
    assert z1.real == pytest.approx(z0.real, rel=0.1)


def test_lossless_default_bit_identical(cuda_device):
    z_default, c_default = _solver().compute_impedance()
    z_nan, c_nan = _solver(wire_conductivity=np.nan).compute_impedance()
    assert z_nan == z_default
    np.testing.assert_array_equal(c_nan, c_default)
    z_scalar, _ = _solver(wire_conductivity=SIGMA_CU).compute_impedance()
    z_seq, _ = _solver(wire_conductivity=[SIGMA_CU]).compute_impedance()
    assert z_seq == z_scalar


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_loaded_swept_matches_per_k(precision, cuda_device):
    ks = 2 * np.pi / np.array([WL * 0.98, WL, WL * 1.02])
    ys = _solver(**LOSSY, precision=precision).compute_y_matrix_swept(ks)
    for i, kk in enumerate(ks):
        z_i, _ = _solver(wavelength=2 * np.pi / kk, **LOSSY).compute_impedance()
        assert 1.0 / ys[i, 0, 0] == pytest.approx(z_i, rel=1e-9 if precision == "fp64" else 1e-6)
    zs = _solver(**LOSSY).compute_impedance_swept(ks)
    for i, kk in enumerate(ks):
        z_i, _ = _solver(wavelength=2 * np.pi / kk, **LOSSY).compute_impedance()
        assert zs[i] == pytest.approx(z_i, rel=1e-9)


def test_loaded_y_matches_impedance(cuda_device):
    z, _ = _solver(**LOSSY).compute_impedance()
    Y = _solver(**LOSSY).compute_y_matrix()
    assert 1.0 / Y[0, 0] == pytest.approx(z, rel=1e-9)
