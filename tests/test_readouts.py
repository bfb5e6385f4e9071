"""Host readouts from a solve's coefficients: the current's arc-length
derivative (current_slopes) against the reference's own values for the
golden cases, and at arbitrary arc positions against scipy's B-spline
derivative (the routine the reference evaluates it with); the currents at
knots and the field evaluator's element terms (element_currents) against
the reference's, all from the reference's own coefficients."""

from pathlib import Path

import numpy as np
import pytest
from scipy.interpolate import BSpline

from cases import CASES, SAMPLED
from conftest import golden, rel_err

import momwire_b200

FULL = sorted(n for n in CASES if n not in SAMPLED)


@pytest.mark.parametrize("name", FULL)
def test_current_slopes_match_reference(name):
    g = golden(name)
    s = momwire_b200.BSplineSolver(**CASES[name]())
    got = np.concatenate(s.current_slopes(g["coeffs"][:, 0]))
    assert got.shape == g["slopes0"].shape
    assert rel_err(got, g["slopes0"]) < 1e-12


@pytest.mark.parametrize("name", ["config1", "d1_dipole20", "d2_junction", "d2_mixed_radius_kink"])
def test_current_slopes_at_arc_positions(name):
    g = golden(name)
    s = momwire_b200.BSplineSolver(**CASES[name]())
    c = g["coeffs"][:, 0]
    geo, b = s._geometry(), s._basis()
    rng = np.random.default_rng(11)
    pts = []
    for w in range(len(b.knots)):
        arc = geo.wire_arc[w]
        mids = 0.5 * (arc[1:] + arc[:-1])
        pts.append(np.concatenate([mids, rng.uniform(-0.1, 1.1, 5) * arc[-1]]))  # some outside: clipped
    got = s.current_slopes(c, pts)
    for w, x in enumerate(pts):
        kn = b.knots[w]
        cc = np.zeros(len(kn) - s.degree - 1, dtype=np.complex128)
        for j, _k, _jn, _e, mg in b.kept[w]:
            cc[j] = c[mg]
        want = BSpline(kn, cc, s.degree, extrapolate=False).derivative(1)(np.clip(x, kn[0], kn[-1]))
        np.testing.assert_allclose(got[w], want, rtol=1e-12, atol=1e-12 * np.abs(want).max())
    empty = s.current_slopes(c, [np.zeros(0)] * len(b.knots))
    assert all(e.size == 0 for e in empty)


_READOUT_CASES = sorted(n for n in CASES if (Path(__file__).resolve().parent / "golden" / f"readouts_{n}.npz").exists())


@pytest.mark.parametrize("name", _READOUT_CASES)
def test_currents_at_knots_match_reference(name):
    """Host readout of the reference's own first port column."""
    g = golden(name)
    s = momwire_b200.BSplineSolver(**CASES[name]())
    cur = np.concatenate(s.currents_at_knots(g["coeffs"][:, 0]))
    assert rel_err(cur, g["currents0"]) < 1e-12


@pytest.mark.parametrize("name", _READOUT_CASES)
@pytest.mark.parametrize("subdiv", [1, 3])
def test_element_currents_match_reference(name, subdiv):
    """(mid, moment, nodes, delta) of the reference's own first port column
    against its ``element_currents`` (``_element_currents.py:33-120``)."""
    g = golden(name)
    want = golden(f"readouts_{name}")
    s = momwire_b200.BSplineSolver(**CASES[name]())
    mid, mom, nodes, delta = s.element_currents(g["coeffs"][:, 0], subdiv=subdiv)
    np.testing.assert_allclose(mid, want[f"mid{subdiv}"], rtol=0, atol=1e-12 * np.abs(want[f"mid{subdiv}"]).max())
    np.testing.assert_allclose(nodes, want[f"nodes{subdiv}"], rtol=0,
                               atol=1e-12 * np.abs(want[f"nodes{subdiv}"]).max())
    assert rel_err(mom, want[f"mom{subdiv}"]) < 1e-12
    assert rel_err(delta, want[f"delta{subdiv}"]) < 1e-11
