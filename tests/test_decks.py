"""The reference's deck front end drives this solver: the keywords its
``deck.build_solver`` passes to ``BSplineSolver`` for NEC-2 decks (recorded
by ``tests/golden/make_decks.py``: a dipole, a Yagi bare and with copper
conductors, an inverted V over a perfect ground, a monopole with radials
over a Sommerfeld ground, and the dipole again through the degree-1 basis
entry) construct ``momwire_b200.BSplineSolver`` as they
are, with the reference's port count and host tables equal to the oracle's."""

import numpy as np
import pytest

from decks import DECKS, deck_kwargs
from oracle import bspline_oracle as O

import momwire_b200


@pytest.mark.parametrize("name", sorted(DECKS))
def test_deck_keywords_construct_the_solver(name):
    kw = deck_kwargs(name)
    s = momwire_b200.BSplineSolver(**kw)
    B, _kcl = s._port_columns()
    assert B.shape[1] == DECKS[name]["n_ports"]
    sp = O.make_spec(**kw)
    og = O.build_geometry(sp)
    ob = O.build_basis(sp, og)
    g, b = s._geometry(), s._basis()
    assert np.array_equal(g.seg_l, og["seg_l"]) and np.array_equal(g.seg_r, og["seg_r"])
    np.testing.assert_allclose(b.polys, ob.polys, rtol=1e-12, atol=1e-12 * np.abs(ob.polys).max())
    Bo, _ = O.port_columns(sp, og, ob)
    np.testing.assert_allclose(B, Bo, rtol=1e-13, atol=1e-14)


def test_deck_fixtures_cover_the_front_end_paths():
    """The decks exercise the mapping's branches: a merged multi-card
    polyline, a junction, per-wire conductivity and both ground kinds."""
    kinds = {n: DECKS[n]["kwargs"] for n in DECKS}
    assert len(kinds["inverted_v_pec"]["wires"]) == 1  # two GW cards, one polyline
    assert kinds["monopole_finite"]["junctions"] and kinds["monopole_finite"]["ground_model"] == "sommerfeld"
    assert "wire_conductivity" in kinds["yagi3_copper"]
    assert kinds["inverted_v_pec"]["ground_z"] == 0.0 and "ground_eps" not in kinds["inverted_v_pec"]
    assert kinds["dipole_free"]["ground_z"] is None
    assert DECKS["dipole_free_d1"]["basis"] == "bspline-d1" and kinds["dipole_free_d1"]["degree"] == 1
