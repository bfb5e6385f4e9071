"""The Sommerfeld oracle pinned against the reference, and the host-side
grid layout of the product checked against the reference's grids.

Golden fixtures (tests/golden/*somm*.npz) come from running the reference
(``make_golden.py``): Z, Y and the wavelength-normalised grid master each
solve interpolated."""

import numpy as np
import pytest

from cases import CASES, LAM_SOMM, SOMMERFELD
from conftest import golden, rel_err
from oracle import bspline_oracle as O
from oracle import sommerfeld_oracle as S

from momwire_b200 import sommerfeld as P

SOMM_CASES = sorted(SOMMERFELD)


def _master_tables(g):
    return [g[f"somm_vals_{i}"] for i in range(int(g["somm_n_region"]))]


@pytest.mark.parametrize("name", SOMM_CASES)
def test_oracle_matches_reference_with_its_grid(name):
    """Z and Y of the oracle (C2 image + remainder block Q over the
    reference's own grid tables) against the reference's solve."""
    g = golden(name)
    Y, _X, Z, _geom, _basis = O.port_solution(O.make_spec(**CASES[name]()), somm_master_values=_master_tables(g))
    assert rel_err(Z, g["Z"]) < 1e-10
    assert rel_err(Y, g["y"]) < 1e-11


def test_oracle_grid_fill_matches_reference():
    """The oracle's own six-integral fill of a whole master (343 nodes)
    against the reference's C++ fill."""
    g = golden("d2_somm_contact")
    m = S.Grid(complex(g["somm_eps_b"]), S.K2_REF, float(g["somm_r1b_wl"]), omega=S.K2_REF * S.C_LIGHT,
               mu=S.MU0_GRID)
    for reg, want in zip(m.regions, _master_tables(g)):
        assert reg["vals"].shape == want.shape
        assert rel_err(reg["vals"], want) < 1e-9


@pytest.mark.parametrize("name", SOMM_CASES)
def test_master_key_and_layout_match_reference(name):
    """The product's bucketing and grid layout give the reference's master:
    same (eps, r1) key and the same region shapes."""
    g = golden(name)
    spec = O.make_spec(**CASES[name]())
    geom = O.build_geometry(spec)
    r1 = S.max_image_distance(geom["seg_l"], geom["seg_r"], spec.ground_z)
    et = O.eps_tilde(spec.ground_eps, spec.omega)
    eb, r1b = P.master_key(et, spec.k, r1)
    assert eb == complex(g["somm_eps_b"])
    assert r1b == float(g["somm_r1b_wl"])
    r1_max, _rb, _rn, _r0f, regions = P.layout(eb, P.K2_REF, r1b)
    tables = _master_tables(g)
    assert len(regions) == len(tables)
    for (r0, r1_, dr, th0, th1, dth), t in zip(regions, tables):
        n_r = max(int(np.ceil((r1_ - r0) / dr)) + 1, 4)
        n_th = int(round((th1 - th0) / dth)) + 1
        assert t.shape == (4, n_r, n_th)
    assert S.grid_layout(eb, S.K2_REF, r1b)[4] == regions


def test_integrand_laplacian_identity():
    """Integrands 0 + 3 + lambda^2 * 4 = 0 pointwise (the J0 Laplacian;
    reference test_sommerfeld_engine)."""
    k2 = 2 * np.pi
    k1 = k2 * np.sqrt(10 - 1.26j)
    k1 = np.conj(k1) if k1.imag > 0 else k1
    lam = np.array([0.3 + 0.1j, 2.0 - 0.5j, 7.0 + 0.2j, 15.0 - 3.0j])
    for form in ("J", "H"):
        f = S.integrands(lam, 0.37, 0.21, k1, k2, form)
        resid = f[0] + f[3] + lam * lam * f[4]
        assert np.max(np.abs(resid)) < 1e-12 * np.max(np.abs(f))


def test_free_space_limit_is_zero():
    assert np.all(S.six_integrals(1.0 + 0.0j, 2 * np.pi, 0.3, 0.2) == 0)


def _nec_dipole(frac, ground, degree):
    """The reference's gn2 test dipole: 0.48-wavelength-class horizontal
    wire in three edges (21, 3, 21 segments) fed at the centre
    (fixtures_refl_coef_geoms.py:11-24), at frac wavelengths height."""
    lam = 10.53011794871795
    y0, y1, z = 2.545656014102564, 0.05, frac * lam
    return dict(wires=[np.array([[0.0, y0, z], [0.0, y1, z], [0.0, -y1, z], [0.0, -y0, z]])],
                n_per_edge_per_wire=[[21, 3, 21]], feeds=[(0, y0, 1.0)], wire_radius=5e-4, wavelength=lam,
                degree=degree, ground_z=0.0, ground_eps=ground, ground_model="sommerfeld")


# nec2c gn 2 feed impedances (golden_refl_coef_ground.py:24-41), gate 3 ohm
# (test_sommerfeld_ground.py:224-244)
GN2 = [(0.02, (10.0, 0.002), 95.08 + 32.413j), (0.05, (10.0, 0.002), 68.002 + 1.5507j)]


@pytest.mark.parametrize("frac,ground,zgn2", GN2)
def test_oracle_tracks_nec2c_gn2(frac, ground, zgn2):
    Y, *_ = O.port_solution(O.make_spec(**_nec_dipole(frac, ground, 2)))
    assert abs(1.0 / Y[0, 0] - zgn2) < 3.0


def test_somm_wavelength_constant():
    assert abs(LAM_SOMM - 299_792_458.0 / 28.47e6) < 1e-12
