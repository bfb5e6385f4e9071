"""Golden fixtures for the off-edge block sampler, from the reference itself.

The reference's H-matrix and array-block solvers sample blocks Z[I, J]
through ``bspline_assemble_offedge_block`` and its ``_refl``, ``_ek`` and
``_refl_ek`` twins (``_accelerators.cpp:1977-2680``).  For seven blocks of
golden structures (free space at degrees 1 and 2, a PEC image with the J
side mirrored, a reflection-coefficient image, the extended kernel in free
space and over a reflection-coefficient ground) this script builds the
arguments from the reference's own geometry and basis tables the way
``hmatrix.py`` does (global segment tables, the J side mirrored for an
image, the extended kernel's joint labels), calls the reference's C++
function and stores arguments and result.

Run where the reference source tree is checked out (its root given by
``--ref`` or ``$MOMWIRE_REF``) and its native kernels are built by
``make -C oracle REF=<root>/src/momwire``:

    python tests/golden/make_offedge_blocks.py --ref <reference checkout>

Writes ``offedge_blocks.npz`` next to this script (keys ``<case>/<arg>``).
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

# case -> (structure, I basis range, J basis range, image, refl, ek)
BLOCKS = {
    "free_d2": ("d2_junction", (0, 21), (0, 21), False, False, False),
    "free_d2_far": ("array4x4", (0, 40), (200, 262), False, False, False),
    "free_d1": ("d1_yagi", (0, 19), (19, 38), False, False, False),
    "pec_d2": ("d2_pec", (0, 20), (0, 20), True, False, False),
    "refl_d2": ("d2_refl_normal", (0, 20), (0, 20), True, True, False),
    "ek_d2": ("d2_ek", (0, 10), (8, 20), False, False, True),
    "refl_ek_d2": ("ek_refl", (0, 12), (0, 12), True, True, True),
}
EXTRA = {
    "ek_refl": lambda: dict(wires=[np.array([[0, 0, 1.0], [0, 0, 9.0]])], nsegs=14, degree=2, extended_kernel=True,
                            wire_radius=0.04, ground_z=0.0, ground_eps=(13.0, 0.005), feeds=[(0, 4.0, 1.0)]),
}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("MOMWIRE_REF"),
                    help="root of the reference checkout (default: $MOMWIRE_REF)")
    args = ap.parse_args()
    if not args.ref:
        ap.error("--ref (or $MOMWIRE_REF) is required")
    momwire = import_reference(Path(args.ref))
    from momwire import _accelerators as acc
    from momwire import _bspline_kernels, _ground_mirror, _ground_refl

    out = {}
    for case, (struct, (i0, i1), (j0, j1), image, refl, ek) in BLOCKS.items():
        kw = (EXTRA.get(struct) or CASES[struct])()
        s = momwire.BSplineSolver(**kw)
        geom = s._build_geometry()
        supp, polys, *_ = s._build_basis_polynomials(geom)
        I, J = np.arange(i0, i1), np.arange(j0, j1)
        segl, segr, tan = geom["seg_l"], geom["seg_r"], geom["tangents"]
        segl_J, segr_J, tan_J = segl, segr, tan
        if image:
            segl_J = _ground_mirror.mirror_positions(segl, s.ground_z)
            segr_J = _ground_mirror.mirror_positions(segr, s.ground_z)
            tan_J = _ground_mirror.mirror_tangents(tan)
        a2 = float(s._uniform_radius) ** 2
        xg, wg = np.polynomial.legendre.leggauss(s.n_qp_pair)
        t01, w01 = 0.5 * (xg + 1.0), 0.5 * wg
        base = [np.ascontiguousarray(supp[I], dtype=np.int64), np.ascontiguousarray(polys[I]), segl, segr, tan,
                np.ascontiguousarray(supp[J], dtype=np.int64), np.ascontiguousarray(polys[J]), segl_J, segr_J, tan_J,
                a2, float(s.k), float(s.omega), float(s.eps), float(s.mu), int(s.degree), t01, w01]
        rec = {"supp_I": base[0], "polys_I": base[1], "segl_I": segl, "segr_I": segr, "tan_I": tan,
               "supp_J": base[5], "polys_J": base[6], "segl_J": segl_J, "segr_J": segr_J, "tan_J": tan_J,
               "params": np.array([a2, s.k, s.omega, s.eps, s.mu, s.degree]), "gl_t": t01, "gl_w": w01}
        extra_ek, extra_refl = [], []
        if ek:
            spec = s._ek_spec(geom, mirror=image)
            g_i = np.ascontiguousarray(spec.group_i, dtype=np.int64)
            g_j = np.ascontiguousarray(spec.group_j, dtype=np.int64)
            a_ek = float(_bspline_kernels._ek_radius(spec, np.sqrt(a2)))
            extra_ek = [g_i, g_j, a_ek]
            rec.update(group_I=g_i, group_J=g_j, a_ek=np.float64(a_ek))
        if refl:
            eps_t = _ground_refl.eps_tilde(s.ground_eps, s.omega, s.eps)
            c0, c1 = _ground_refl.phi_mode_coeffs(s.ground_phi_mode, eps_t)
            extra_refl = [complex(eps_t), complex(c0), complex(c1)]
            rec.update(refl=np.array([eps_t, c0, c1], dtype=np.complex128))
        if ek and refl:
            Z = acc.bspline_assemble_offedge_block_refl_ek(*base, *extra_ek, *extra_refl)
        elif ek:
            Z = acc.bspline_assemble_offedge_block_ek(*base, *extra_ek)
        elif refl:
            Z = acc.bspline_assemble_offedge_block_refl(*base, *extra_refl)
        else:
            Z = acc.bspline_assemble_offedge_block(*base)
        rec["Z"] = np.asarray(Z)
        for key, v in rec.items():
            out[f"{case}/{key}"] = v
        print(f"{case}: {rec['Z'].shape} |Z|max {np.abs(rec['Z']).max():.6e}", flush=True)
    np.savez_compressed(HERE / "offedge_blocks.npz", **out)


if __name__ == "__main__":
    main()
