"""Timed CPU baseline: the reference's own native kernels on a bounded sample.

TEST / BASELINE INFRASTRUCTURE ONLY (used by bench.py's CPU-baseline leg and
its ``--impl reference`` arm).  The reference's pybind11 kernels are built
from the reference sources by ``oracle/Makefile`` into ``oracle/_ref/``;
this module drives them the way the reference's chunked dense route does
(``bspline.py:2386-2550``: observer-row windows of
``seg_seg_full_moments_bspline`` accumulated by
``assemble_Z_bspline_windowed``, then the same-edge correction windows), and
times LAPACK ``zgesv`` through ``scipy.linalg.solve`` as
``_solve_with_kcl_ports`` does (``bspline.py:2971``).  The orchestration is
the oracle's restatement; every flop-carrying call is the reference's.

The sample is a band of observer rows (the fill is linear in rows) and a
leading principal block of the filled rows for the factorisation (LU cost
scales as n^3); both are extrapolated to the full workload.
"""

from __future__ import annotations

import glob
import os
import sys
import time
from pathlib import Path

import numpy as np
import scipy.linalg

from . import bspline_oracle as O

HERE = Path(__file__).resolve().parent


def load_reference_kernels():
    """Import the reference's compiled ``_accelerators`` from oracle/_ref."""
    so = glob.glob(str(HERE / "_ref" / "_accelerators*.so"))
    if not so:
        raise ImportError("reference kernels not built: run `make -C oracle` where the reference tree exists")
    sys.path.insert(0, str(HERE / "_ref"))
    try:
        import _accelerators  # noqa: E402
    finally:
        sys.path.pop(0)
    return _accelerators


def _same_edge_correction(acc, spec, geom, k, d, nq, first, n, h, a, t01, w01, Z, supp, polys, tan):
    """Replace the edge's full-kernel block by static + reg (the reference's
    correction window, bspline.py:2502-2548)."""
    st = acc.seg_seg_static_moments_bspline_uniform(float(h), float(a), int(n), int(d))
    s_flat = (np.arange(n)[:, None] * h + t01[None, :] * h).ravel()
    diff = s_flat[:, None] - s_flat[None, :]
    R = np.sqrt(diff * diff + a * a)
    u = t01 * h
    wu = np.stack([np.tile(w01 * h * u**p, (n, 1)) for p in range(d + 1)])
    reg = acc.seg_seg_reg_moments_bspline_swept(np.ascontiguousarray(R), np.ascontiguousarray(wu),
                                                np.asarray([k], dtype=np.float64))[0]
    sl, sr = geom["seg_l"][first : first + n], geom["seg_r"][first : first + n]
    J_edge = acc.seg_seg_full_moments_bspline(sl, sr, sl, sr, float(a * a), float(k), int(d), t01, w01)
    corr = np.ascontiguousarray((st + reg) - J_edge)
    mask = ((supp >= first) & (supp < first + n)).any(axis=1)
    idx = np.nonzero(mask)[0].astype(np.int64)
    acc.assemble_Z_bspline_windowed(corr, supp, polys, tan, idx, idx, int(first), int(first + n), int(first),
                                    int(first + n), float(spec.omega), O.EPS0, O.MU0, Z, 0)


def time_sample(kw, row_fraction=0.25, swept_mem_mb=256):
    """Time the reference path on a band of the workload; returns a dict
    with extrapolated fill and factor+solve seconds for the full problem.
    Observer-row windows are sized as the reference sizes them from its
    ``swept_mem_mb`` budget (bspline.py:2476-2479)."""
    acc = load_reference_kernels()
    spec = O.make_spec(**kw)
    geom = O.build_geometry(spec)
    basis = O.build_basis(spec, geom)
    B, kcl = O.port_columns(spec, geom, basis)
    d, nq, k = spec.degree, spec.n_qp_pair, spec.k
    n_seg, n_b = geom["n"], basis.supp_seg.shape[0]
    chunk_rows = max(1, int(swept_mem_mb * 1024 * 1024 // ((d + 1) ** 2 * n_seg * 16)))
    t01, w01 = O.gl01(nq)
    supp = np.ascontiguousarray(basis.supp_seg, dtype=np.int64)
    polys = np.ascontiguousarray(basis.polys)
    tan = np.ascontiguousarray(geom["tangents"])
    a2 = float(geom["radius"][0]) ** 2
    assert np.all(geom["radius"] == geom["radius"][0]), "sample timer assumes one radius"
    rows = max(chunk_rows, int(round(n_seg * row_fraction)))
    Z = np.zeros((n_b, n_b), dtype=np.complex128, order="F")
    all_n = np.arange(n_b, dtype=np.int64)
    t0 = time.perf_counter()
    for i0 in range(0, rows, chunk_rows):
        i1 = min(i0 + chunk_rows, rows)
        J = acc.seg_seg_full_moments_bspline(geom["seg_l"][i0:i1], geom["seg_r"][i0:i1], geom["seg_l"],
                                             geom["seg_r"], a2, float(k), int(d), t01, w01)
        m_idx = np.nonzero(((supp >= i0) & (supp < i1)).any(axis=1))[0].astype(np.int64)
        acc.assemble_Z_bspline_windowed(J, supp, polys, tan, m_idx, all_n, int(i0), int(i1), 0, int(n_seg),
                                        float(spec.omega), O.EPS0, O.MU0, Z, 0)
    for first, n, h, a, _w in geom["edges"]:
        if first + n <= rows:
            _same_edge_correction(acc, spec, geom, k, d, nq, first, n, h, a, t01, w01, Z, supp, polys, tan)
    t_fill = time.perf_counter() - t0
    # factor + solve on the filled leading block, all port columns
    nb_s = max(1, min(n_b, rows - 2 * d))
    Zs = np.asfortranarray(Z[:nb_s, :nb_s])
    Bs = np.asfortranarray(B[:nb_s, :])
    # zgesv = zgetrf (n^3) + zgetrs (n^2 * nrhs): timed apart so each part
    # is extrapolated by its own exponent
    t0 = time.perf_counter()
    lu = scipy.linalg.lu_factor(Zs, overwrite_a=True, check_finite=False)
    t_lu = time.perf_counter() - t0
    t0 = time.perf_counter()
    scipy.linalg.lu_solve(lu, Bs, overwrite_b=True, check_finite=False)
    t_rs = time.perf_counter() - t0
    scale_fill = n_seg / rows
    scale_lu = (n_b / nb_s) ** 3
    scale_rs = (n_b / nb_s) ** 2
    return {
        "fill_s": t_fill * scale_fill,
        "solve_s": t_lu * scale_lu + t_rs * scale_rs,
        "sample_fill_s": t_fill,
        "sample_solve_s": t_lu + t_rs,
        "rows": rows,
        "n_seg": n_seg,
        "n_basis": n_b,
        "lu_block": nb_s,
        "n_ports": B.shape[1],
        "threads": int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1)),
    }
