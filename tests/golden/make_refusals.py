"""The reference's refusals of invalid inputs: for every case of
``refusal_cases.py``, the exception type and text the reference's
``BSplineSolver`` raises (at construction, or at the solve for the cases it
only refuses there).  Run where the reference and its native kernels (``make
-C oracle REF=...``) are available:

    python tests/golden/make_refusals.py --ref <reference checkout>

Writes ``refusals.json`` next to this script.
"""

from __future__ import annotations

import argparse
import os
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from make_golden import import_reference  # noqa: E402
from refusal_cases import AT_SOLVE, REFUSALS  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MOMWIRE_REF"),
                    help="root of the reference checkout (default: $MOMWIRE_REF)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("--ref (or $MOMWIRE_REF) is required")
    momwire = import_reference(Path(args.ref))
    out = {}
    for name, make in REFUSALS.items():
        try:
            s = momwire.BSplineSolver(**make())
            if name in AT_SOLVE:
                s.compute_impedance()
            out[name] = None
        except Exception as e:  # noqa: BLE001 -- recording what the reference raises
            out[name] = {"type": type(e).__name__, "message": str(e)}
        print(name, out[name])
    (HERE / "refusals.json").write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
