"""Host readouts from a solve's coefficients: the current's arc-length
derivative (current_slopes) against the reference's own values for the
golden cases, and at arbitrary arc positions against scipy's B-spline
derivative (the routine the reference evaluates it with)."""

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
