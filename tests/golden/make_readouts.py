"""Golden readouts: the reference's ``element_currents`` of its own first
port column, for every full golden case.

Run where the reference source tree is checked out (its root given by
``--ref`` or ``$MOMWIRE_REF``) and its native kernels are built by
``make -C oracle REF=<root>/src/momwire``, after
``make_golden.py`` (it reads the ``coeffs`` stored there):

    python tests/golden/make_readouts.py --ref <reference checkout>

The readout is host-side arithmetic on a coefficient vector (no solve), so
each case only constructs the reference's ``BSplineSolver``.  Writes
``readouts_<name>.npz`` next to this script: (mid, moment, nodes, delta) for
subdiv 1 and 3.
"""

from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from cases import CASES  # noqa: E402
from make_golden import import_reference  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MOMWIRE_REF"),
                    help="root of the reference checkout (default: $MOMWIRE_REF)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("--ref (or $MOMWIRE_REF) is required")
    momwire = import_reference(Path(args.ref))
    n = 0
    for name in sorted(CASES):
        path = HERE / f"{name}.npz"
        if not path.exists():
            continue
        g = np.load(path)
        if "coeffs" not in g.files:
            continue
        s = momwire.BSplineSolver(**CASES[name]())
        out = {}
        for sub in (1, 3):
            mid, mom, nodes, delta = s.element_currents(g["coeffs"][:, 0], subdiv=sub)
            out[f"mid{sub}"], out[f"mom{sub}"] = np.asarray(mid), np.asarray(mom)
            out[f"nodes{sub}"], out[f"delta{sub}"] = np.asarray(nodes), np.asarray(delta)
        np.savez(HERE / f"readouts_{name}.npz", **out)
        n += 1
    print(f"{n} cases")


if __name__ == "__main__":
    main()
