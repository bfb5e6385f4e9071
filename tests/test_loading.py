"""Distributed series wire loading on the host: per-unit-length impedances,
the same-wire overlap Gram, keyword validation -- against the reference's
own values (fixtures written by running it) and the oracle's restatement."""

import numpy as np
import pytest

from cases import CASES, LOADED
from conftest import golden, rel_err
from oracle import bspline_oracle as O

import momwire_b200
from momwire_b200 import loading as wl

MU0 = wl.MU0
SIGMA_CU = 5.8e7
A_28 = 0.16e-3
DIPOLE = [np.array([[0.0, 0.0, -10.15 / 2], [0.0, 0.0, 10.15 / 2]])]


def _solver(**kw):
    base = dict(wires=DIPOLE, nsegs=81, wavelength=21.264, wire_radius=A_28)
    base.update(kw)
    return momwire_b200.BSplineSolver(**base)


def test_internal_impedance_matches_reference_table():
    g = golden("wire_impedance")
    for i, om in enumerate(g["omega"]):
        for j, a in enumerate(g["radius"]):
            for k, sig in enumerate(g["sigma"]):
                want = g["z_int"][i, j, k]
                got = wl.wire_internal_impedance(om, a, sig)
                assert abs(got - want) <= 1e-13 * abs(want)
                # the oracle's unscaled-Bessel form, where it does not overflow
                if abs(np.sqrt(om * MU0 * sig / 2.0) * a) < 300:
                    assert abs(O.internal_impedance(om, a, sig) - want) <= 1e-10 * abs(want)
    for i, b in enumerate(g["ins_b"]):
        for j, e in enumerate(g["ins_eps"]):
            assert wl.insulation_inductance(1e-3, b, e) == pytest.approx(g["ins_L"][i, j], rel=1e-14, abs=0)


def test_internal_impedance_limits():
    """DC: R = 1/(sigma pi a^2), X = omega mu0 / (8 pi); strong skin:
    R = X = 1/(2 pi a sigma delta)."""
    a = 1e-3
    om = 2 * np.pi * 10.0
    z = wl.wire_internal_impedance(om, a, SIGMA_CU)
    assert z.real == pytest.approx(1.0 / (SIGMA_CU * np.pi * a**2), rel=1e-4)
    assert z.imag == pytest.approx(om * MU0 / (8 * np.pi), rel=1e-2)
    om = 2 * np.pi * 100e6
    z = wl.wire_internal_impedance(om, a, SIGMA_CU)
    r_hf = 1.0 / (2 * np.pi * a * SIGMA_CU * np.sqrt(2.0 / (om * MU0 * SIGMA_CU)))
    assert z.real == pytest.approx(r_hf, rel=2e-2) and z.imag == pytest.approx(r_hf, rel=2e-2)
    z = wl.wire_internal_impedance(2 * np.pi * 1e13, 1e-2, SIGMA_CU)
    assert np.isfinite(z.real) and np.isfinite(z.imag) and z.real > 0


def _dense(rows, cols, vals, n):
    S = np.zeros((n, n))
    np.add.at(S, (rows, cols), vals)
    return S


@pytest.mark.parametrize("name", sorted(LOADED))
def test_gram_and_wire_impedance_match_reference(name):
    g = golden(name)
    s = momwire_b200.BSplineSolver(**CASES[name]())
    n = s._basis().n
    lg = s._loading_tables()
    want = _dense(g["load_rows"], g["load_cols"], g["load_vals"], n)
    assert rel_err(_dense(lg.rows, lg.cols, lg.vals, n), want) < 1e-13
    assert rel_err(_dense(lg.u_rows, lg.u_cols, lg.u_vals, n), want) < 1e-13
    # coalesced entries are unique and carry the wire both bases lie on
    assert np.unique(lg.u_rows * n + lg.u_cols).size == lg.u_rows.size
    wires = np.zeros((n, n), dtype=np.int64) - 1
    wires[g["load_rows"], g["load_cols"]] = g["load_wire"]
    assert np.array_equal(wires[lg.u_rows, lg.u_cols], lg.u_wire)
    zw = s._loading.z_wire(s.omega)
    np.testing.assert_allclose(zw, g["load_zw"], rtol=1e-13, atol=0)
    # the oracle's quadrature Gram, per wire
    sp = O.make_spec(**CASES[name]())
    og = O.build_geometry(sp)
    S_w = O.loading_gram(og, O.build_basis(sp, og))
    assert rel_err(S_w.sum(axis=0), want) < 1e-12
    assert rel_err(O.z_per_wire(sp, sp.omega), g["load_zw"]) < 1e-12


@pytest.mark.parametrize("name", sorted(LOADED))
def test_host_apply_loading_matches_oracle(name):
    s = momwire_b200.BSplineSolver(**CASES[name]())
    n = s._basis().n
    L = s._apply_loading(np.zeros((n, n), dtype=np.complex128))
    sp = O.make_spec(**CASES[name]())
    og = O.build_geometry(sp)
    want = O.loading_matrix(sp, og, O.build_basis(sp, og), sp.omega)
    assert rel_err(L, want) < 1e-12
    # the swept form: one matrix per omega
    oms = s.omega * np.array([0.9, 1.0, 1.1])
    Ls = s._apply_loading(np.zeros((3, n, n), dtype=np.complex128), omega=oms)
    for i, om in enumerate(oms):
        assert rel_err(Ls[i], O.loading_matrix(sp, og, O.build_basis(sp, og), om)) < 1e-12


def test_validation_errors():
    """Messages and order as the reference's constructor
    (``_wire_loading.py`` ``configure_loading``)."""
    with pytest.raises(ValueError, match="must exceed"):
        _solver(insulation_radius=A_28 / 2, insulation_eps_r=2.0)
    with pytest.raises(ValueError, match="eps_r must be >= 1"):
        _solver(insulation_radius=1e-3, insulation_eps_r=0.5)
    with pytest.raises(ValueError, match="given together"):
        _solver(insulation_radius=1e-3)
    with pytest.raises(ValueError, match="given together"):
        _solver(insulation_eps_r=2.0)
    with pytest.raises(ValueError, match="length-1"):
        _solver(wire_conductivity=[SIGMA_CU, SIGMA_CU])
    with pytest.raises(ValueError, match="> 0 S/m"):
        _solver(wire_conductivity=-1.0)
    with pytest.raises(ValueError, match="finite on the same wires"):
        momwire_b200.BSplineSolver(**dict(CASES["d1_yagi"](), insulation_radius=[1e-3, np.nan],
                                          insulation_eps_r=[2.0, 2.0]))
    with pytest.raises(NotImplementedError, match="enrichment"):
        _solver(wire_conductivity=SIGMA_CU, use_singular_enrichment=True)


def test_loading_off_states():
    """No keywords, or NaN on every wire: no loading term, no Gram."""
    assert _solver()._loading is None
    s = _solver(wire_conductivity=np.nan)
    n = s._basis().n
    L = s._apply_loading(np.zeros((n, n), dtype=np.complex128))
    assert not L.any()
    assert s.wire_loss_power(np.ones(n))[0] == 0.0
    s = _solver(insulation_radius=0.4e-3, insulation_eps_r=3.0)
    assert s.wire_loss_power(np.ones(s._basis().n))[0] == 0.0  # a jacket is lossless


@pytest.mark.parametrize("name", sorted(LOADED))
def test_wire_loss_power_matches_reference(name):
    """The reference's dissipated power for its own first port column."""
    g = golden(name)
    s = momwire_b200.BSplineSolver(**CASES[name]())
    total, per_wire = s.wire_loss_power(g["coeffs"][:, 0])
    np.testing.assert_allclose(per_wire, g["loss_power"], rtol=1e-12, atol=1e-14 * np.abs(g["loss_power"]).max())
    assert total == pytest.approx(per_wire.sum())
