"""Host side of singular enrichment, against the reference (CPU).

The enrichment specs (which segment each basis sits on and which end faces
the junction), the stable shape's polynomial, the "auto" variant's tap
ratios and the currents the enrichment shapes add between knots, checked
on the reference's own solutions (``tests/golden/make_enrich.py``)."""

import numpy as np
import pytest

from cases import ENRICH_CASES
from conftest import golden
from oracle import enrich_oracle as EO

import momwire_b200
from momwire_b200 import enrichment as EN


def _solver(name):
    s = momwire_b200.BSplineSolver(**ENRICH_CASES[name]())
    g = golden(name)
    act = g["auto_active"].tolist()
    s._auto_active_junctions = None if act == [-1] else act
    return s, g


@pytest.mark.parametrize("name", sorted(ENRICH_CASES))
def test_specs_match_reference(name):
    s, g = _solver(name)
    sp = s._enrichment_specs_now()
    assert [x.seg for x in sp] == g["spec_seg"].tolist()
    assert [x.origin for x in sp] == g["spec_origin"].tolist()
    assert [x.wire for x in sp] == g["spec_wire"].tolist()
    assert [x.junction for x in sp] == g["spec_junction"].tolist()


@pytest.mark.parametrize("name", sorted(ENRICH_CASES))
def test_currents_with_enrichment_match_reference(name):
    """At the knots the enrichment shapes vanish; at segment midpoints the
    reference adds coefficient x shape on the enriched segments."""
    s, g = _solver(name)
    c = g["coeffs"][:, 0]
    knots = np.concatenate(s.currents_at_knots(c))
    np.testing.assert_allclose(knots, g["currents0"], rtol=1e-12, atol=1e-14 * np.abs(g["currents0"]).max())
    geom = s._geometry()
    mids = [0.5 * (a[1:] + a[:-1]) for a in geom.wire_arc]
    mid = np.concatenate(s.currents_at_knots(c, mids))
    np.testing.assert_allclose(mid, g["currents_mid"], rtol=1e-12, atol=1e-14 * np.abs(g["currents_mid"]).max())


def test_stable_shape_polynomial():
    for d in (1, 2, 3):
        np.testing.assert_allclose(EN.bubble_projection(d), EO.projection_coeffs(d), rtol=1e-13, atol=1e-15)
    assert not np.any(EN.shape_polynomial("raw", 2)) and not np.any(EN.shape_polynomial("tikhonov", 2))
    assert np.any(EN.shape_polynomial("stable", 2))


def test_tap_ratios_select_like_the_reference():
    """The star's balanced split activates its junction, the fan dipole's
    dominant-pair junctions stay off (threshold 0.3)."""
    for name in ("enr_star_auto", "enr_fan_auto"):
        s, g = _solver(name)
        cur = s.currents_at_knots(g["coeffs"][:s._basis().n, 0]) if name == "enr_fan_auto" else None
        if cur is not None:
            r = EN.tap_ratios(s.junctions, cur, s.enrichment_min_k)
            assert all(x is not None and x <= s.auto_tap_ratio_threshold for x in r)
    assert golden("enr_star_auto")["auto_active"].tolist() == [0]
    assert golden("enr_fan_auto")["auto_active"].tolist() == []


def test_current_slopes_refused_under_enrichment():
    s, _g = _solver("enr_star_raw")
    with pytest.raises(NotImplementedError, match="current_slopes does not serve use_singular_enrichment"):
        s.current_slopes(np.zeros(s._basis().n + 3))
