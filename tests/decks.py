"""Decks of the deck front-end fixtures (``tests/golden/make_decks.py``):
the constructor keywords the reference's ``deck.build_solver`` passed to
``BSplineSolver`` for each NEC-2 deck, decoded back into Python values."""

import json
from pathlib import Path

import numpy as np

DECKS = json.loads((Path(__file__).resolve().parent / "golden" / "decks.json").read_text())


def _complex(v):
    return complex(v["re"], v["im"]) if isinstance(v, dict) else v


def deck_kwargs(name):
    kw = dict(DECKS[name]["kwargs"])
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
