"""Singular basis enrichment on the GPU against the reference.

Twelve junction structures (``tests/golden/make_enrich.py``): the device
enrichment blocks (``mw_enrich_blocks``, ground reactions included) against
the reference's Z_pe, Z_ep, Z_ee; the augmented FP64 solve's Y,
coefficients (enrichment block included) and knot / midpoint currents; the
mixed path's port impedances; the "auto" variant's junction selection."""

import numpy as np
import pytest

from cases import ENRICH_CASES
from conftest import golden, rel_err

import momwire_b200

pytestmark = pytest.mark.gpu

SOLVED = sorted(ENRICH_CASES)


@pytest.mark.parametrize("name", [n for n in SOLVED if n != "enr_fan_auto"])
def test_device_blocks_match_reference(name, cuda_device):
    import torch

    g = golden(name)
    s = momwire_b200.BSplineSolver(**ENRICH_CASES[name]())
    act = g["auto_active"].tolist()
    s._auto_active_junctions = None if act == [-1] else act
    sp = s._enrichment_specs_now()
    buf = s._alloc(sp)
    st = torch.cuda.current_stream(buf["Z"].device).cuda_stream
    s._fill_device(buf, st)
    n, n_p = buf["n"], buf["n_poly"]
    Z = buf["Z"].cpu().numpy().T  # column-major storage
    assert rel_err(Z[:n_p, :n_p], g["Z"]) < 1e-10
    blocks = {"Z_pe": Z[:n_p, n_p:], "Z_ep": Z[n_p:, :n_p], "Z_ee": Z[n_p:, n_p:]}
    if ENRICH_CASES[name]().get("enrichment_variant") == "tikhonov":
        # the solve-time regularisation sits on the diagonal of Z_ee
        d = np.diag(g["Z_ee"])
        blocks["Z_ee"] = blocks["Z_ee"] - np.eye(len(d)) * 0.05 * np.mean(np.abs(d))
    for key, got in blocks.items():
        assert rel_err(got, g[key]) < 1e-11, key


@pytest.mark.parametrize("name", SOLVED)
def test_enriched_solve_matches_reference(name, cuda_device):
    g = golden(name)
    s = momwire_b200.BSplineSolver(**ENRICH_CASES[name]())
    sol = s.compute_port_solution()
    act = g["auto_active"].tolist()
    assert (s._auto_active_junctions is None) == (act == [-1])
    if act != [-1]:
        assert s._auto_active_junctions == act
    assert sol.coeffs.shape == g["coeffs"].shape
    assert rel_err(sol.y, g["y"]) < 1e-10
    assert rel_err(sol.coeffs, g["coeffs"]) < 1e-9
    assert rel_err(np.concatenate(s.currents_at_knots(sol.coeffs[:, 0])), g["currents0"]) < 1e-9
    mids = [0.5 * (a[1:] + a[:-1]) for a in s._geometry().wire_arc]
    assert rel_err(np.concatenate(s.currents_at_knots(sol.coeffs[:, 0], mids)), g["currents_mid"]) < 1e-9
    z, _c = s.compute_impedance()
    # (an undriven junction port reads 0 / its current: zero in both)
    assert rel_err(np.atleast_1d(z), g["zin"]) < 1e-9


@pytest.mark.parametrize("name", ["enr_star_raw", "enr_fan_raw", "enr_radials_pec", "enr_radials_somm"])
def test_enriched_mixed_precision(name, cuda_device):
    g = golden(name)
    y = momwire_b200.BSplineSolver(**ENRICH_CASES[name](), precision="mixed").compute_port_solution().y
    zin, want = 1.0 / np.diag(y), 1.0 / np.diag(g["y"])
    assert np.max(np.abs(zin - want) / np.abs(want)) <= 1e-6


def test_enriched_sweep_is_per_frequency(cuda_device):
    """A sweep of an enriched structure solves each frequency through the
    augmented system (the reference's per-k route)."""
    s = momwire_b200.BSplineSolver(**ENRICH_CASES["enr_star_raw"]())
    ks = np.array([0.95, 1.05]) * s.k
    ys = s.compute_y_matrix_swept(ks)
    for i, kk in enumerate(ks):
        t = momwire_b200.BSplineSolver(**dict(ENRICH_CASES["enr_star_raw"](), wavelength=2 * np.pi / kk))
        assert rel_err(ys[i], t.compute_port_solution().y) < 1e-12
