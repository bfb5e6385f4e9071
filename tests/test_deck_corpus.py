"""The reference's own NEC-2 deck corpus through its deck front end.

``tests/golden/make_deck_corpus.py`` ran every deck of the reference's
corpus (``tests/fixtures/nec_portal``, the decks of its
``test_deck_nec2_corpus.py`` and portal tests) through the reference's
``deck.parse`` and ``deck.build_solver`` and recorded the keywords handed to
``BSplineSolver``.  Replayed here, each constructs this solver with the
reference's unknown and port counts and the oracle's host tables (CPU);
``test_gpu_deck_corpus.py`` checks the solves."""

import numpy as np
import pytest

from decks import CORPUS, corpus_kwargs
from oracle import bspline_oracle as O

import momwire_b200

SERVED = sorted(n for n, r in CORPUS.items() if "refused" not in r and "solve_refused" not in r)


def test_corpus_is_the_whole_reference_set():
    # every deck of the reference's corpus was built and solved there
    assert len(CORPUS) == 60 and len(SERVED) == len(CORPUS)


@pytest.mark.parametrize("name", SERVED)
def test_corpus_keywords_construct_the_solver(name):
    kw = corpus_kwargs(name)
    s = momwire_b200.BSplineSolver(**kw)
    B, _kcl = s._port_columns()
    assert B.shape[1] == CORPUS[name]["n_ports"]
    assert s._basis_count() == CORPUS[name]["n_unknowns"]
    sp = O.make_spec(**kw)
    og = O.build_geometry(sp)
    ob = O.build_basis(sp, og)
    g, b = s._geometry(), s._basis()
    assert np.array_equal(g.seg_l, og["seg_l"]) and np.array_equal(g.seg_r, og["seg_r"])
    np.testing.assert_allclose(b.polys, ob.polys, rtol=1e-12, atol=1e-12 * np.abs(ob.polys).max())
    Bo, _ = O.port_columns(sp, og, ob)
    np.testing.assert_allclose(B, Bo, rtol=1e-13, atol=1e-14)


def test_corpus_covers_the_front_end_paths():
    kinds = [CORPUS[n]["kwargs"] for n in SERVED]
    assert any(k.get("junctions") for k in kinds)
    assert any(k.get("ground_model") == "sommerfeld" for k in kinds)
    assert any(k.get("extended_kernel") for k in kinds)
    assert any("wire_conductivity" in k for k in kinds)
    assert any(k.get("ground_z") is not None and k.get("ground_eps") is None for k in kinds)


_REF = np.load(__import__("pathlib").Path(__file__).resolve().parent / "golden" / "deck_corpus.npz")


@pytest.mark.parametrize("name", SERVED)
def test_oracle_solves_corpus_like_reference(name):
    """The oracle (the checker of the GPU tests) pinned on every corpus deck."""
    Y, *_ = O.port_solution(O.make_spec(**corpus_kwargs(name)))
    want = _REF[f"y_{name}"]
    assert np.max(np.abs(Y - want)) / np.max(np.abs(want)) < 1e-11
