"""Swept solves of structures with junction constraint (KCL) rows.

The reference batches the fill over frequency and closes every frequency's
KCL constraints with a Schur step (``bspline.py:3017-3038``,
``_solve_with_kcl_swept_ports``).  Here the KCL rows ride along as extra
right-hand sides of the batched solve and the Schur step runs per
frequency: in the FP64 batched-fill route (complex128 LU per matrix), the
batched mixed route, and the grouped many-structure sweep.  Each is checked
against per-frequency complex128 single solves: Y within 1e-10 (FP64) and
every drive-point impedance within 1e-6 (mixed)."""

import numpy as np
import pytest

from cases import CASES
from conftest import rel_err

import momwire_b200
from momwire_b200 import sweep
from momwire_b200.workloads import C_LIGHT, yagi_sweep

pytestmark = pytest.mark.gpu


def _per_k(kw, ks):
    s = momwire_b200.BSplineSolver(**kw)
    return np.stack([sol.y for sol in s.compute_port_solution_swept(ks)])


def _zin(y):
    return 1.0 / np.einsum("...ii->...i", y)


def _radial_monopole_pec(n_rad=6, f=14e6):
    """A quarter-wave monopole over a PEC ground at 0.05 lambda with
    n_rad horizontal radials joined at its base (one KCL row)."""
    lam = C_LIGHT / f
    base = np.array([0.0, 0.0, 0.05 * lam])
    wires = [np.array([base, base + [0.0, 0.0, 0.25 * lam]])]
    for i in range(n_rad):
        a = 2.0 * np.pi * i / n_rad
        wires.append(np.array([base, base + 0.25 * lam * np.array([np.cos(a), np.sin(a), 0.0])]))
    return dict(wires=wires, nsegs=9, degree=2, wire_radius=1e-3, wavelength=lam, ground_z=0.0,
                junctions=[[(w, "start") for w in range(n_rad + 1)]], feeds=[(0, 0.25 * lam / 18, 1.0)])


def _junctioned_yagi(kw):
    """The Yagi with its driven element cut at the centre into two wires
    joined by a junction and fed by a series node gap there."""
    out = dict(kw)
    wires = list(kw["wires"])
    npe = list(kw["n_per_edge_per_wire"])
    d = wires[1]
    mid = 0.5 * (d[0] + d[1])
    half = max(npe[1] // 2, 3)
    wires[1:2] = [np.array([d[0], mid]), np.array([mid, d[1]])]
    npe[1:2] = [half, half]
    out.update(wires=wires, n_per_edge_per_wire=npe, junctions=[[(1, "end"), (2, "start")]],
               feeds=[], node_gaps=[(2, "start", 1.0)])
    return out


@pytest.mark.parametrize("name", ["d2_junction", "d2_node_gap", "d2_loaded_junction_pec"])
def test_fp64_batched_fill_sweep_with_kcl(name, cuda_device):
    kw = CASES[name]()
    s = momwire_b200.BSplineSolver(**kw)
    assert s._kcl_rows_left() > 0 and s._swept_fp64_batched_available()
    ks = np.linspace(0.9, 1.1, 5) * s.k
    want = _per_k(kw, ks)
    got = s.compute_y_matrix_swept(ks)
    for i in range(len(ks)):
        assert rel_err(got[i], want[i]) < 1e-10


@pytest.mark.parametrize("name", ["d2_junction", "d2_node_gap", "d2_loaded_junction_pec"])
def test_mixed_batched_sweep_with_kcl(name, cuda_device):
    kw = CASES[name]()
    s = momwire_b200.BSplineSolver(**kw, precision="mixed")
    assert s._kcl_rows_left() > 0 and s._swept_batched_available()
    ks = np.linspace(0.9, 1.1, 5) * s.k
    want = _per_k(kw, ks)
    got = s.compute_y_matrix_swept(ks)
    assert np.max(np.abs(_zin(got) - _zin(want)) / np.abs(_zin(want))) <= 1e-6


def test_grouped_sweep_with_junctioned_structures(cuda_device):
    """Plain Yagis, Yagis with a junctioned driven element and node-gap
    feed, and radial monopoles over PEC in one grouped sweep."""
    structs, ks = yagi_sweep(n_structures=6, n_freq=6, seed=5)
    structs = structs[:3] + [_junctioned_yagi(k) for k in structs[3:]]
    structs += [_radial_monopole_pec(4), _radial_monopole_pec(7)]
    ks_m = 2 * np.pi * np.linspace(13e6, 15e6, 6) / C_LIGHT
    out = sweep.grouped_mixed_sweep(structs[:6], ks)
    out_m = sweep.grouped_mixed_sweep(structs[6:], ks_m)
    for i, kw in enumerate(structs[:6]):
        want = _per_k(kw, ks)
        assert np.max(np.abs(_zin(out[i]) - _zin(want)) / np.abs(_zin(want))) <= 1e-6, i
    for j, kw in enumerate(structs[6:]):
        assert momwire_b200.BSplineSolver(**kw, precision="mixed")._kcl_rows_left() == 1
        want = _per_k(kw, ks_m)
        assert np.max(np.abs(_zin(out_m[j]) - _zin(want)) / np.abs(_zin(want))) <= 1e-6, j
