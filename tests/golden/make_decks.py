"""Golden fixtures for the deck front end: NEC-2 decks written for this test
suite, parsed and mapped onto a solver by the reference's OWN deck front end
(``momwire.deck.parse`` and ``momwire.deck.build_solver``), with the
constructor keywords that front end passes to ``BSplineSolver`` recorded and
the reference's multi-port solve of each deck stored beside them.

Run where the reference source tree is checked out (its root given by
``--ref`` or ``$MOMWIRE_REF``) and its native kernels are built by
``make -C oracle REF=<root>/src/momwire``:

    python tests/golden/make_decks.py --ref <reference checkout>

Writes ``decks.json`` (deck text, recorded keywords, port plan) and
``deck_<name>.npz`` (the reference's Y and port impedances) next to this
script.  The reference's deck front end drives ``momwire_b200.BSplineSolver``
unchanged when its ``BASES["bspline"]`` entry names that class; the tests
replay the recorded keywords into it.
"""

from __future__ import annotations

import argparse
import os
import json
import sys
from pathlib import Path
from types import MappingProxyType

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from make_golden import import_reference  # noqa: E402

DECKS = {
    "dipole_free": """CM centre-fed dipole, free space
CE
GW 1 21 0 0 -5.05 0 0 5.05 0.001
GE 0
EX 0 1 11 0 1 0
FR 0 1 0 0 14.1 0
XQ
EN
""",
    "yagi3_free": """CM three-element yagi, driven element centre-fed
CE
GW 1 21 -1.6 0 -2.75 -1.6 0 2.75 0.005
GW 2 21 0 0 -2.55 0 0 2.55 0.005
GW 3 21 1.7 0 -2.4 1.7 0 2.4 0.005
GE 0
EX 0 2 11 0 1 0
FR 0 1 0 0 28.0 0
XQ
EN
""",
    "yagi3_copper": """CM the same yagi with copper conductors
CE
GW 1 21 -1.6 0 -2.75 -1.6 0 2.75 0.005
GW 2 21 0 0 -2.55 0 0 2.55 0.005
GW 3 21 1.7 0 -2.4 1.7 0 2.4 0.005
GE 0
LD 5 1 1 21 5.8E7
LD 5 2 1 21 5.8E7
LD 5 3 1 21 5.8E7
EX 0 2 11 0 1 0
FR 0 1 0 0 28.0 0
XQ
EN
""",
    "inverted_v_pec": """CM inverted V over a perfect ground, fed at the apex
CE
GW 1 15 -3.5 0 4.0 0 0 7.0 0.001
GW 2 15 0 0 7.0 3.5 0 4.0 0.001
GE 1
GN 1
EX 0 1 15 0 1 0
FR 0 1 0 0 14.1 0
XQ
EN
""",
    "monopole_finite": """CM quarter-wave monopole with four radials above finite ground
CE
GW 1 11 0 0 1.0 0 0 6.3 0.002
GW 2 9 0 0 1.0 4.5 0 1.0 0.002
GW 3 9 0 0 1.0 -4.5 0 1.0 0.002
GW 4 9 0 0 1.0 0 4.5 1.0 0.002
GW 5 9 0 0 1.0 0 -4.5 1.0 0.002
GE 1
GN 2 0 0 0 13 0.005
EX 0 1 1 0 1 0
FR 0 1 0 0 11.9 0
XQ
EN
""",
}
DECKS["dipole_free_d1"] = DECKS["dipole_free"]

# the reference's basis name per deck (its BASES table): degree 2 unless named
BASIS_OF = {"dipole_free_d1": "bspline-d1"}


def _jsonable(v):
    if isinstance(v, dict):
        return {k: _jsonable(x) for k, x in v.items()}
    if isinstance(v, np.ndarray):
        return _jsonable(v.tolist())
    if isinstance(v, (list, tuple)):
        return [_jsonable(x) for x in v]
    if isinstance(v, complex):
        return {"re": v.real, "im": v.imag}
    if isinstance(v, (np.floating,)):
        return float(v)
    if isinstance(v, (np.integer,)):
        return int(v)
    return v


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MOMWIRE_REF"),
                    help="root of the reference checkout (default: $MOMWIRE_REF)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("--ref (or $MOMWIRE_REF) is required")
    momwire = import_reference(Path(args.ref))
    from momwire import deck
    from momwire.deck import _solver as deck_solver

    recorded = {}

    class Recording(momwire.BSplineSolver):
        def __init__(self, **kw):
            recorded.clear()
            recorded.update(kw)
            super().__init__(**kw)

    stock = deck_solver.BASES
    deck_solver.BASES = MappingProxyType({
        **stock,
        "bspline": (Recording, stock["bspline"][1]),
        "bspline-d1": (Recording, stock["bspline-d1"][1]),
    })
    out = {}
    try:
        for name, text in DECKS.items():
            model = deck.parse(text)
            basis = BASIS_OF.get(name, "bspline")
            built = deck.build_solver(model, basis=basis)
            kw = {k: v for k, v in recorded.items() if k != "cancel"}
            sol = built.solver.compute_port_solution()
            y = np.asarray(sol.y)
            zin = 1.0 / np.diag(y)
            np.savez(HERE / f"deck_{name}.npz", y=y, zin=zin)
            out[name] = {
                "deck": text,
                "basis": basis,
                "kwargs": _jsonable(kw),
                "frequency_mhz": built.frequency_mhz,
                "n_ports": int(y.shape[0]),
                "feed_ports": list(built.ports.feed_ports),
            }
            print(f"{name}: {y.shape[0]} ports, Zin[0] = {zin[0]:.6f}")
    finally:
        deck_solver.BASES = stock
    (HERE / "decks.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
