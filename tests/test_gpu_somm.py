"""Sommerfeld ground on the GPU: grid fill, projected field, remainder
block Q and whole solves against the reference's goldens and the oracle."""

import numpy as np
import pytest

from cases import CASES, SOMMERFELD
from conftest import golden, rel_err
from oracle import bspline_oracle as O
from oracle import sommerfeld_oracle as S
from test_oracle_somm import GN2, _master_tables, _nec_dipole

import momwire_b200
from momwire_b200 import _lib
from momwire_b200 import sommerfeld as P

pytestmark = pytest.mark.gpu
SOMM_CASES = sorted(SOMMERFELD)


def _stream():
    import torch

    return torch.cuda.current_stream().cuda_stream


@pytest.mark.parametrize("name", SOMM_CASES)
def test_master_fill_matches_reference(name, cuda_device):
    """Device six-integral fill of each master against the reference's C++
    fill: per surface and region, within 1e-8 of that table's scale."""
    g = golden(name)
    m = P.MasterGrid(complex(g["somm_eps_b"]), float(g["somm_r1b_wl"]), cuda_device, _stream())
    for mine, want in zip(m.tables(), _master_tables(g)):
        assert mine.shape == want.shape
        for s in range(4):
            scale = np.max(np.abs(want[s]))
            assert np.max(np.abs(mine[s] - want[s])) <= 1e-8 * scale, (name, s)


def test_free_space_master_is_zero(cuda_device):
    m = P.MasterGrid(1.0 + 0.0j, 1.0, cuda_device, _stream())
    assert all(np.all(t == 0) for t in m.tables())


def test_field_proj_matches_oracle(cuda_device):
    """mw_somm_field_proj with the reference's master against the oracle's
    interpolation + eqs 143-147 on the same tables."""
    import torch

    g = golden("d2_somm_far_pair")
    tables = _master_tables(g)
    eb, r1b = complex(g["somm_eps_b"]), float(g["somm_r1b_wl"])
    lam = 10.53
    k2 = 2 * np.pi / lam
    omega, mu = k2 * 2.99792458e8 * 1.0000001, 1.25663706127e-6
    m = P.MasterGrid(eb, r1b, cuda_device, _stream(), tables=tables)
    view = m.view(k2, omega, mu)
    og = S.get_grid(eb, k2, r1b * lam, omega, mu, master_values=tables)
    rng = np.random.default_rng(3)
    n_o, n_s = 37, 53
    obs = np.c_[rng.uniform(-3, 3, (n_o, 2)) * lam, rng.uniform(0.0, 0.3, n_o) * lam]
    src = np.c_[rng.uniform(-3, 3, (n_s, 2)) * lam, rng.uniform(0.0, 0.3, n_s) * lam]
    src[0, :2] = obs[0, :2]  # a vertical (rho = 0) pair
    t_o = rng.standard_normal((n_o, 3))
    t_o /= np.linalg.norm(t_o, axis=1)[:, None]
    t_s = rng.standard_normal((n_s, 3))
    t_s /= np.linalg.norm(t_s, axis=1)[:, None]
    t_s[1] = [0.0, 0.0, 1.0]
    d = {k: torch.from_numpy(np.ascontiguousarray(v)).to(cuda_device)
         for k, v in dict(obs=obs, t_o=t_o, src=src, t_s=t_s).items()}
    out = torch.empty((n_o, n_s), dtype=torch.complex128, device=cuda_device)
    _lib.call("mw_somm_field_proj", n_o, d["obs"].data_ptr(), d["t_o"].data_ptr(), n_s, d["src"].data_ptr(),
              d["t_s"].data_ptr(), 0.0, k2, view, out.data_ptr(), _stream())
    want = S.field_proj(obs, t_o, src, t_s, 0.0, k2, og)
    assert rel_err(out.cpu().numpy(), want) < 1e-12


@pytest.mark.parametrize("name", SOMM_CASES)
def test_remainder_Z_matches_oracle_on_device_grid(name, cuda_device):
    """Whole Sommerfeld Z (free space - C2 image - Q) against the oracle fed
    the device's own master tables: isolates the fill kernels from the
    grid quadrature."""
    s = momwire_b200.BSplineSolver(**CASES[name]())
    Z = s._compute_Z_operator()
    tables = s._somm_master.tables()
    want = O.compute_Z(O.make_spec(**CASES[name]()), somm_master_values=tables)
    assert rel_err(Z, want) < 1e-12


@pytest.mark.parametrize("name", SOMM_CASES)
def test_sommerfeld_solve_matches_reference(name, cuda_device):
    g = golden(name)
    sol = momwire_b200.BSplineSolver(**CASES[name]()).compute_port_solution()
    assert rel_err(sol.y, g["y"]) < 1e-9


def test_free_space_limit(cuda_device):
    """eps~ = 1: C2 = 0 and the remainder vanishes; equals the free-space
    solve (reference test_sommerfeld_ground.py:121-128)."""
    kw = CASES["d2_somm_dipole"]()
    z_g = momwire_b200.BSplineSolver(**dict(kw, ground_eps=1.0 + 0.0j)).compute_impedance()[0]
    free = {k: v for k, v in kw.items() if k not in ("ground_z", "ground_eps", "ground_model")}
    z_free = momwire_b200.BSplineSolver(**free).compute_impedance()[0]
    assert abs(z_g - z_free) / abs(z_free) < 1e-9


def test_pec_limit(cuda_device):
    """eps~ -> 1e16: C2 -> 1 and the remainder scales away, reproducing the
    PEC image (reference test_sommerfeld_ground.py:131-137)."""
    kw = CASES["d2_somm_dipole"]()
    z_g = momwire_b200.BSplineSolver(**dict(kw, ground_eps=1e16 + 0.0j)).compute_impedance()[0]
    pec = {k: v for k, v in kw.items() if k not in ("ground_eps", "ground_model")}
    z_pec = momwire_b200.BSplineSolver(**pec).compute_impedance()[0]
    assert abs(z_g - z_pec) / abs(z_pec) < 1e-5


@pytest.mark.parametrize("degree", [1, 2])
@pytest.mark.parametrize("frac,ground,zgn2", GN2)
def test_tracks_nec2c_gn2(frac, ground, zgn2, degree, cuda_device):
    z = momwire_b200.BSplineSolver(**_nec_dipole(frac, ground, degree)).compute_impedance()[0]
    assert abs(z - zgn2) < 3.0


@pytest.mark.parametrize("name", ["d2_somm_dipole", "d2_somm_radials"])
def test_sommerfeld_mixed_precision(name, cuda_device):
    g = golden(name)
    s = momwire_b200.BSplineSolver(**CASES[name](), precision="mixed")
    y = s.compute_port_solution().y
    zin, zref = 1.0 / np.diag(y), 1.0 / np.diag(g["y"])
    assert np.max(np.abs(zin - zref) / np.abs(zref)) <= 1e-6


def test_sommerfeld_sweep_reuses_master(cuda_device):
    """A 1% sweep interpolates one master (the eps/r1 buckets), as the
    reference's two-level cache does, and each k matches its single solve."""
    P.clear_cache()
    s = momwire_b200.BSplineSolver(**CASES["d2_somm_dipole"]())
    ks = s.k * np.array([0.995, 1.0, 1.005])
    ys = s.compute_y_matrix_swept(ks)
    assert len(P._MASTERS) <= 2
    for kk, y in zip(ks, ys):
        t = momwire_b200.BSplineSolver(**CASES["d2_somm_dipole"]())
        t._set_k(kk)
        assert rel_err(y, t.compute_port_solution().y) < 1e-13
