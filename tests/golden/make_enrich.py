"""Golden fixtures for singular basis enrichment, from the reference itself.

For each case of ``ENRICH_CASES`` (``tests/golden/cases.py``) the reference's
``BSplineSolver(use_singular_enrichment=True, ...)`` is solved and its
augmented-system pieces are recorded: the enrichment specs (junction, wire,
end, segment, origin), the three enrichment blocks Z_pe, Z_ep, Z_ee the solve
added to Z (``_enrichment_Z_assemble``, bspline.py:3523-3693, ground
reaction included), the polynomial Z, the port solution (Y, all
coefficients, the enrichment block among them), the junctions the "auto"
variant activated, the drive-point impedance of ``compute_impedance`` and
the first port column's currents at the knots and at the segment
midpoints (and, over a Sommerfeld
ground, the grid master the solve interpolated).

Run where the reference source tree is checked out (its root given by
``--ref`` or ``$MOMWIRE_REF``) and its native kernels are built by
``make -C oracle REF=<root>/src/momwire``:

    python tests/golden/make_enrich.py --ref <reference checkout>

Writes ``enr_<case>.npz`` next to this script.

The blocks come from the reference's numpy assembly
(``_assemble_Z_enrich_numpy``, its documented twin of the C++
``assemble_Z_enrich``): the C++ binding as built here stops on pybind11's
GIL assertion when it is called.
"""

from __future__ import annotations

import argparse
import os
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))
from cases import ENRICH_CASES  # noqa: E402
from make_golden import import_reference, somm_master  # noqa: E402


def record(momwire, kw):
    s = momwire.BSplineSolver(**kw)
    sol = s.compute_port_solution()
    active = s._auto_active_junctions
    geom = s._build_geometry()
    supp, polys, _kcl, _wk, _wbg = s._build_basis_polynomials(geom)
    Z = s._compute_Z_operator(geom, supp, polys)
    out = {"y": np.asarray(sol.y), "coeffs": np.asarray(sol.coeffs), "Z": Z,
           "n_poly": np.int64(supp.shape[0])}
    specs = s._enrichment_specs(geom, active_junction_indices=active)
    out["spec_junction"] = np.array([sp[0] for sp in specs], dtype=np.int64)
    out["spec_wire"] = np.array([sp[1] for sp in specs], dtype=np.int64)
    out["spec_end"] = np.array([0 if sp[2] == "start" else 1 for sp in specs], dtype=np.int64)
    out["spec_seg"] = np.array([sp[3] for sp in specs], dtype=np.int64)
    out["spec_origin"] = np.array([0 if sp[4] == "left" else 1 for sp in specs], dtype=np.int64)
    # "auto": None = every qualifying junction; a list = the activated ones
    out["auto_active"] = np.array([-1] if active is None else list(active), dtype=np.int64)
    if kw.get("enrichment_variant") == "auto" and active is not None and not active:
        out["Z_pe"] = out["Z_ep"] = out["Z_ee"] = np.zeros((0, 0), np.complex128)
    else:
        blocks = s._enrichment_Z_assemble(geom, supp, polys, active_junction_indices=active)
        for key in ("Z_pe", "Z_ep", "Z_ee"):
            out[key] = np.asarray(blocks[key]) if blocks is not None else np.zeros((0, 0), np.complex128)
    out["currents0"] = np.concatenate(s.currents_at_knots(np.asarray(sol.coeffs)[:, 0]))
    # between the knots the enrichment shapes add to the current
    mids = [0.5 * (pw["arc_at_knot"][1:] + pw["arc_at_knot"][:-1]) for pw in geom["per_wire"]]
    out["currents_mid"] = np.concatenate(s.currents_at_knots(np.asarray(sol.coeffs)[:, 0], mids))
    if kw.get("ground_model") == "sommerfeld":
        out.update(somm_master(momwire, s, geom))
    zin = s.compute_impedance()
    out["zin"] = np.atleast_1d(np.asarray(zin[0] if isinstance(zin, tuple) else zin))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MOMWIRE_REF"),
                    help="root of the reference checkout (default: $MOMWIRE_REF)")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    if not args.ref:
        ap.error("--ref (or $MOMWIRE_REF) is required")
    momwire = import_reference(Path(args.ref))
    import momwire.bspline as ref_bspline

    ref_bspline._HAVE_ENRICH_ACCEL = False
    for name, kw in ENRICH_CASES.items():
        if args.only and name != args.only:
            continue
        out = record(momwire, kw())
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(f"{name}: n_poly={int(out['n_poly'])} n_enrich={out['spec_seg'].size} "
              f"active={out['auto_active'].tolist()} y[0,0]={out['y'][0, 0]:.12g}", flush=True)


if __name__ == "__main__":
    main()
