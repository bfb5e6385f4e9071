"""Generate golden vectors by running the reference momwire itself.

Run where the reference source tree is checked out (its root given by
``--ref`` or ``$MOMWIRE_REF``) and its native kernels are built by
``make -C oracle REF=<root>/src/momwire``:

    python tests/golden/make_golden.py --ref <reference checkout> [--big]

The reference package is copied to a temporary directory together with the
compiled ``_accelerators`` module, imported from there, and every case in
``tests/golden/cases.py`` is solved with ``BSplineSolver``.  Outputs are
small ``.npz`` files next to this script.  ``--big`` adds the 16x16 dipole
array (10,496 unknowns, 256 ports; ~30 s on 8 cores), stored as Y plus a
seeded sample of Z entries and per-column checksums of the coefficients.
"""

from __future__ import annotations

import argparse
import glob
import os
import shutil
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parent.parent
sys.path.insert(0, str(HERE))

from cases import BIG_CASES, CASES, SAMPLED, SOMMERFELD  # noqa: E402


def import_reference(ref_root: Path):
    tmp = Path(tempfile.mkdtemp(prefix="momwire_ref_"))
    shutil.copytree(ref_root / "src" / "momwire", tmp / "momwire")
    so = glob.glob(str(REPO / "oracle" / "_ref" / "_accelerators*.so"))
    if not so:
        raise SystemExit("build the reference kernels first: make -C oracle")
    shutil.copy(so[0], tmp / "momwire")
    sys.path.insert(0, str(tmp))
    import momwire  # noqa: E402

    if not momwire.accelerated:
        raise SystemExit("reference accelerator failed to load")
    return momwire


def somm_master(momwire, s, geom):
    """The wavelength-normalised grid master the reference's solve used,
    as region tables vals_<i> (4, n_r, n_th) plus its key."""
    from momwire import _ground_refl, _sommerfeld

    eps_t = _ground_refl.eps_tilde(s.ground_eps, s.omega, s.eps)
    r1 = _sommerfeld.max_image_distance(geom["seg_l"], geom["seg_r"], s.ground_z)
    lam = 2.0 * np.pi / s.k
    r1b = _sommerfeld._somm_r1_bucket_wl(min(r1 / lam, _sommerfeld._SOMM_R1_CAP_LAMBDA))
    eb = _sommerfeld._somm_eps_bucket(complex(eps_t))
    master = _sommerfeld._NORM_CACHE[(eb, r1b)]
    out = {"somm_eps_b": np.complex128(eb), "somm_r1b_wl": np.float64(r1b), "somm_n_region": len(master._regions)}
    for i, reg in enumerate(master._regions):
        out[f"somm_vals_{i}"] = reg["vals"]
    return out


def solve_case(momwire, kw, sample_seed=None, somm=False):
    s = momwire.BSplineSolver(**kw)
    geom = s._build_geometry()
    supp, polys, kcl, wk, wbg = s._build_basis_polynomials(geom)
    t0 = time.perf_counter()
    Z = s._compute_Z_operator(geom, supp, polys)
    t_fill = time.perf_counter() - t0
    n = Z.shape[0]
    samples = None
    if sample_seed is not None:
        # big cases: keep a seeded sample of Z and free it before the solve
        rng = np.random.default_rng(sample_seed)
        ii = rng.integers(0, n, 4096)
        jj = rng.integers(0, n, 4096)
        d = np.arange(min(n, 512))
        ii = np.concatenate([ii, d, d[1:], d[:-1]])
        jj = np.concatenate([jj, d, d[:-1], d[1:]])
        samples = (ii, jj, Z[ii, jj].copy())
        del Z
    t0 = time.perf_counter()
    sol = s.compute_port_solution()
    t_all = time.perf_counter() - t0
    out = {"y": sol.y, "t_fill": t_fill, "t_solve_total": t_all}
    if somm:
        out.update(somm_master(momwire, s, geom))
    if getattr(s, "_loading_active", False):
        from momwire import _wire_loading

        r, c, v, w = s._loading_gram()
        p_tot, p_wire = s.wire_loss_power(sol.coeffs[:, 0])
        out.update(load_rows=r, load_cols=c, load_vals=v, load_wire=w,
                   load_zw=_wire_loading.loading_for(s, s.omega).z_wire, loss_power=p_wire)
    if sample_seed is None:
        out["Z"] = Z
        out["coeffs"] = sol.coeffs
        cur = s.currents_at_knots(sol.coeffs[:, 0])
        out["currents0"] = np.concatenate(cur)
        out["slopes0"] = np.concatenate(s.current_slopes(sol.coeffs[:, 0]))
    else:
        out["z_i"], out["z_j"], out["z_v"] = samples
        out["coeff_colsum"] = sol.coeffs.sum(axis=0)
        out["coeff_colnorm"] = np.linalg.norm(sol.coeffs, axis=0)
        out["coeffs_first_rows"] = sol.coeffs[:64]
    return out


def wire_impedance_table(momwire):
    """The reference's per-unit-length conductor and jacket impedances on a
    grid from DC to extreme skin effect (a / skin depth ~ 1e-3 .. 5e4)."""
    from momwire import _wire_loading

    om = 2 * np.pi * np.array([10.0, 1e3, 1e5, 1e6, 14.1e6, 1e8, 1e10, 1e13])
    rad = np.array([1e-4, 1e-3, 1e-2])
    sig = np.array([1e6, 3.5e7, 5.8e7])
    zi = np.array([[[_wire_loading.wire_internal_impedance(o, a, g) for g in sig] for a in rad] for o in om])
    ins = np.array([[_wire_loading.insulation_inductance(1e-3, b, e) for e in (1.0, 2.3, 3.0, 10.0)]
                    for b in (1.5e-3, 2.5e-3, 1e-2)])
    return {"omega": om, "radius": rad, "sigma": sig, "z_int": zi, "ins_b": np.array([1.5e-3, 2.5e-3, 1e-2]),
            "ins_eps": np.array([1.0, 2.3, 3.0, 10.0]), "ins_L": ins}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MOMWIRE_REF"),
                    help="root of the reference checkout (default: $MOMWIRE_REF)")
    ap.add_argument("--big", action="store_true")
    ap.add_argument("--only", default=None)
    args = ap.parse_args()
    if not args.ref:
        ap.error("--ref (or $MOMWIRE_REF) is required")
    momwire = import_reference(Path(args.ref))
    if args.only in (None, "wire_impedance"):
        np.savez_compressed(HERE / "wire_impedance.npz", **wire_impedance_table(momwire))
        print("wire_impedance: table written", flush=True)
    todo = dict(CASES)
    if args.big:
        todo.update(BIG_CASES)
    for name, kw in todo.items():
        if args.only and name != args.only:
            continue
        out = solve_case(momwire, kw(), sample_seed=1234 if name in SAMPLED else None, somm=name in SOMMERFELD)
        np.savez_compressed(HERE / f"{name}.npz", **out)
        print(f"{name}: y[0,0]={out['y'][0, 0]:.12g} fill={out['t_fill']:.3f}s", flush=True)


if __name__ == "__main__":
    main()
