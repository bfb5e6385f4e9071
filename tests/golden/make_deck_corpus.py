"""Golden fixtures for the reference's own NEC-2 deck corpus.

The reference keeps a corpus of NEC-2 decks as test fixtures
(``tests/fixtures/nec_portal/*.deck``, used by ``tests/test_deck_nec2_corpus.py``
and the portal tests).  For every deck this script runs the reference's own
front end -- ``momwire.deck.parse`` and ``momwire.deck.build_solver`` with
the B-spline basis -- and records what it hands the solver: the keyword
arguments of the ``BSplineSolver`` it constructs (or the exception the front
end or the constructor raised), then the reference's multi-port solve.  The
deck texts themselves are not copied; only the keywords, the port plan and
the solve are stored.

Run where the reference source tree is checked out (its root given by
``--ref`` or ``$MOMWIRE_REF``) and its native kernels are built by
``make -C oracle REF=<root>/src/momwire``:

    python tests/golden/make_deck_corpus.py --ref <reference checkout>

Writes ``deck_corpus.json`` (per deck: keywords, frequency, port plan, or
the refusal) and ``deck_corpus.npz`` (``y_<deck>``, ``zin_<deck>``) next to
this script.
"""

from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path
from types import MappingProxyType

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from make_decks import _jsonable  # noqa: E402
from make_golden import import_reference  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MOMWIRE_REF"),
                    help="root of the reference checkout (default: $MOMWIRE_REF)")
    ap.add_argument("--max-unknowns", type=int, default=4000,
                    help="decks whose solver has more unknowns are recorded without a solve")
    args = ap.parse_args()
    if not args.ref:
        ap.error("--ref (or $MOMWIRE_REF) is required")
    ref = Path(args.ref)
    momwire = import_reference(ref)
    from momwire import deck
    from momwire.deck import _solver as deck_solver

    recorded = {}

    class Recording(momwire.BSplineSolver):
        def __init__(self, **kw):
            recorded.clear()
            recorded.update(kw)
            super().__init__(**kw)

    stock = deck_solver.BASES
    deck_solver.BASES = MappingProxyType({**stock, "bspline": (Recording, stock["bspline"][1])})
    out, arrays = {}, {}
    try:
        for path in sorted((ref / "tests" / "fixtures" / "nec_portal").glob("*.deck")):
            name = path.stem
            rec = {"deck_file": path.name}
            recorded.clear()
            t0 = time.perf_counter()
            try:
                model = deck.parse(path.read_text())
                built = deck.build_solver(model, basis="bspline")
            except Exception as e:  # the front end's or the constructor's refusal
                rec["refused"] = {"type": type(e).__name__, "message": str(e),
                                  "at_constructor": bool(recorded)}
                if recorded:
                    rec["kwargs"] = _jsonable({k: v for k, v in recorded.items() if k != "cancel"})
                out[name] = rec
                print(f"{name}: refused ({type(e).__name__})")
                continue
            rec["kwargs"] = _jsonable({k: v for k, v in recorded.items() if k != "cancel"})
            rec["frequency_mhz"] = float(built.frequency_mhz)
            rec["feed_ports"] = _jsonable(list(built.ports.feed_ports))
            s = built.solver
            n = int(s._basis_count()) if hasattr(s, "_basis_count") else None
            try:
                sol = s.compute_port_solution()
            except Exception as e:
                rec["solve_refused"] = {"type": type(e).__name__, "message": str(e)}
                out[name] = rec
                print(f"{name}: solve refused ({type(e).__name__}: {e})")
                continue
            y = np.asarray(sol.y)
            rec["n_unknowns"] = int(np.asarray(sol.coeffs).shape[0]) if n is None else n
            rec["n_ports"] = int(y.shape[0])
            arrays[f"y_{name}"] = y
            arrays[f"zin_{name}"] = 1.0 / np.diag(y) if y.size else np.zeros(0, np.complex128)
            rec["seconds"] = round(time.perf_counter() - t0, 3)
            out[name] = rec
            print(f"{name}: {y.shape[0]} ports, {rec['n_unknowns']} unknowns, {rec['seconds']} s")
    finally:
        deck_solver.BASES = stock
    np.savez_compressed(HERE / "deck_corpus.npz", **arrays)
    (HERE / "deck_corpus.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
