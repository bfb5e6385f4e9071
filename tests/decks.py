"""Decks of the deck front-end fixtures (``tests/golden/make_decks.py`` for
decks written for these tests, ``tests/golden/make_deck_corpus.py`` for the
reference's own deck corpus): the constructor keywords the reference's
``deck.build_solver`` passed to ``BSplineSolver`` for each NEC-2 deck,
decoded back into Python values."""

import json
from pathlib import Path

import numpy as np

_GOLDEN = Path(__file__).resolve().parent / "golden"
DECKS = json.loads((_GOLDEN / "decks.json").read_text())
CORPUS = json.loads((_GOLDEN / "deck_corpus.json").read_text())


def _complex(v):
    return complex(v["re"], v["im"]) if isinstance(v, dict) else v


def deck_kwargs(name, table=None):
    kw = dict((DECKS if table is None else table)[name]["kwargs"])
    kw["wires"] = [np.asarray(w, dtype=np.float64) for w in kw["wires"]]
    kw["feeds"] = [(int(w), float(s), _complex(v)) for w, s, v in kw["feeds"]]
    if kw.get("junctions") is not None:
        kw["junctions"] = [[(int(w), str(e)) for w, e in j] for j in kw["junctions"]]
    if kw.get("ground_eps") is not None and isinstance(kw["ground_eps"], list):
        kw["ground_eps"] = tuple(kw["ground_eps"])
    for key in ("wire_conductivity", "insulation_radius", "insulation_eps_r"):
        if key in kw:
            kw[key] = np.asarray(kw[key], dtype=np.float64)
    return kw


def corpus_kwargs(name):
    return deck_kwargs(name, CORPUS)
