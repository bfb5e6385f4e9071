"""End-to-end parity on the GPU through the drop-in solver: Z, Y, coeffs
and currents against golden vectors from the reference, plus the port
algebra invariants the reference's own tests check."""

import numpy as np
import pytest

from cases import BIG_CASES, CASES
from conftest import golden, rel_err

import momwire_b200

pytestmark = pytest.mark.gpu

FULL = [n for n in CASES if n != "array4x4"]


@pytest.mark.parametrize("name", FULL)
def test_z_matches_reference(name, cuda_device):
    s = momwire_b200.BSplineSolver(**CASES[name]())
    Z = s._compute_Z_operator()
    assert rel_err(Z, golden(name)["Z"]) < 1e-10


@pytest.mark.parametrize("name", FULL)
def test_port_solution_matches_reference(name, cuda_device):
    g = golden(name)
    s = momwire_b200.BSplineSolver(**CASES[name]())
    sol = s.compute_port_solution()
    assert sol.port_currents is sol.y
    assert rel_err(sol.y, g["y"]) < 1e-10
    assert rel_err(sol.coeffs, g["coeffs"]) < 1e-9
    cur = np.concatenate(s.currents_at_knots(sol.coeffs[:, 0]))
    assert rel_err(cur, g["currents0"]) < 1e-9
    slopes = np.concatenate(s.current_slopes(sol.coeffs[:, 0]))
    assert rel_err(slopes, g["slopes0"]) < 1e-8


def _sampled_check(name, s):
    g = golden(name)
    Z = s._compute_Z_operator()
    assert rel_err(Z[g["z_i"], g["z_j"]], g["z_v"]) < 1e-10
    sol = s.compute_port_solution()
    assert rel_err(sol.y, g["y"]) < 1e-10
    assert rel_err(sol.coeffs.sum(axis=0), g["coeff_colsum"]) < 1e-9
    assert rel_err(sol.coeffs[:64], g["coeffs_first_rows"]) < 1e-9
    return sol


def test_array4x4_matches_reference(cuda_device):
    _sampled_check("array4x4", momwire_b200.BSplineSolver(**CASES["array4x4"]()))


def test_array16x16_matches_reference(cuda_device):
    """The 16x16 dipole array: 10,496 unknowns, 256 ports."""
    sol = _sampled_check("array16x16", momwire_b200.BSplineSolver(**BIG_CASES["array16x16"]()))
    y = sol.y
    assert rel_err(y, y.T) < 1e-9  # Galerkin reciprocity


def test_port_invariants_junction_port(cuda_device):
    """Reference test_port_solution.py: columns satisfy the KCL rows, Y is
    symmetric, superposition equals the configured drive."""
    s = momwire_b200.BSplineSolver(**CASES["d2_junction"]())
    sol = s.compute_port_solution()
    kcl, _pa, _pv = s._split_kcl_ports(s._basis().kcl_A)
    assert kcl.shape[0] == 1
    assert np.abs(kcl.toarray() @ sol.coeffs).max() < 1e-10 * np.abs(sol.coeffs).max()
    s = momwire_b200.BSplineSolver(**CASES["d2_junction_port"]())
    sol = s.compute_port_solution()
    assert sol.y.shape == (2, 2)
    assert rel_err(sol.y, sol.y.T) < 1e-9
    z, coeffs = s.compute_impedance()
    assert np.allclose(coeffs, sol.coeffs @ np.array([1.0, 0.0]))


def test_config1_known_answer(cuda_device):
    s = momwire_b200.BSplineSolver(**CASES["config1"]())
    z = 1.0 / s.compute_y_matrix()[0, 0]
    assert abs(z - (67.5789431392556 - 30.968698608555457j)) <= 1e-9 * abs(z)


def test_swept_equals_stacked(cuda_device):
    s = momwire_b200.BSplineSolver(**CASES["d1_dipole20"]())
    k0 = s.k
    ks = np.linspace(0.9 * k0, 1.1 * k0, 3)
    ys = s.compute_y_matrix_swept(ks)
    for i, kk in enumerate(ks):
        t = momwire_b200.BSplineSolver(**CASES["d1_dipole20"]())
        t._set_k(kk)
        assert rel_err(ys[i], t.compute_y_matrix()) < 1e-12
    assert s.k == k0


def test_element_currents_shapes(cuda_device):
    s = momwire_b200.BSplineSolver(**CASES["d2_mixed_radius_kink"]())
    sol = s.compute_port_solution()
    mid, mom, nodes, delta = s.element_currents(sol.coeffs[:, 0], subdiv=2)
    assert mid.shape == mom.shape
    assert nodes.shape[0] == mid.shape[0] + len(s.wires_polylines)
    assert abs(delta.sum()) < 1e-9 * np.abs(delta).max()


def test_plate64_sommerfeld_matches_reference(cuda_device):
    """The 64x64-cell wire-grid plate over a Sommerfeld ground with a centre
    monopole: 33,290 unknowns, 4,218 KCL rows, 8 ports.  Z sampled on the
    device (17.7 GB), Y and coefficient checksums against the reference
    (its own quadrature grid; 1e-8 covers the grid's rounding)."""
    import torch

    g = golden("plate64_somm")
    s = momwire_b200.BSplineSolver(**BIG_CASES["plate64_somm"]())
    buf = s._alloc()
    s._fill_device(buf, torch.cuda.current_stream().cuda_stream)
    ii = torch.from_numpy(g["z_i"]).to(cuda_device)
    jj = torch.from_numpy(g["z_j"]).to(cuda_device)
    zs = buf["Z"][jj, ii].cpu().numpy()  # column-major: Z[i, j] is tensor[j, i]
    assert rel_err(zs, g["z_v"]) < 1e-8
    del buf
    sol = s.compute_port_solution()
    assert rel_err(sol.y, g["y"]) < 1e-8
    assert rel_err(sol.coeffs.sum(axis=0), g["coeff_colsum"]) < 1e-7


def test_plate64_sommerfeld_mixed(cuda_device):
    g = golden("plate64_somm")
    s = momwire_b200.BSplineSolver(**BIG_CASES["plate64_somm"](), precision="mixed")
    y = s.compute_port_solution().y
    zin, zref = 1.0 / np.diag(y), 1.0 / np.diag(g["y"])
    assert np.max(np.abs(zin - zref) / np.abs(zref)) <= 1e-6


def test_impedance_swept_all_ports(cuda_device):
    """Multi-port sweeps return every port's impedance per k, (n_k, n_ports),
    each row the per-k compute_impedance (``bspline.py:4496-4513``)."""
    kw = CASES["d2_junction_port"]()
    s = momwire_b200.BSplineSolver(**kw)
    ks = s.k * np.array([0.97, 1.03])
    zs = s.compute_impedance_swept(ks)
    assert zs.shape == (2, 2)
    for i, kk in enumerate(ks):
        t = momwire_b200.BSplineSolver(**dict(kw, wavelength=2 * np.pi / kk))
        z, _ = t.compute_impedance()
        np.testing.assert_allclose(zs[i], z, rtol=1e-12)
