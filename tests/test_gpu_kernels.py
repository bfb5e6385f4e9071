"""Kernel-level parity on the GPU: same-edge tables and off-edge moments
against the oracle, through the C ABI."""

import ctypes as C

import numpy as np
import pytest

from cases import CASES
from conftest import rel_err
from oracle import bspline_oracle as O

import momwire_b200
from momwire_b200 import _lib

pytestmark = pytest.mark.gpu


def _solver(name, **extra):
    kw = CASES[name]()
    kw.update(extra)
    return momwire_b200.BSplineSolver(**kw), O.make_spec(**kw)


@pytest.mark.parametrize("name", ["config1", "d1_dipole20", "d2_ek", "d2_mixed_radius_kink", "array4x4"])
def test_same_edge_table_matches_oracle(name, cuda_device):
    import torch

    s, sp = _solver(name)
    dt = s._dev_tables()
    d = s.degree
    table = torch.empty((dt.table_rows, d + 1, d + 1), dtype=torch.complex128, device=cuda_device)
    _lib.call("mw_same_edge_table", C.byref(dt.edges), d, s.n_qp_pair, int(s.extended_kernel), float(s.k),
              table.data_ptr(), None)
    got = table.cpu().numpy()
    g = s._geometry()
    off = 0
    for e in range(len(g.edge_n)):
        n, h, a = int(g.edge_n[e]), float(g.edge_h[e]), float(g.edge_radius[e])
        want = O.same_edge_static_table(h, a, n, d, ek=s.extended_kernel) + O.same_edge_reg_table(
            h, a, n, s.k, d, s.n_qp_pair, ek=s.extended_kernel)
        assert rel_err(got[off : off + 2 * n - 1], want) < 1e-13
        off += 2 * n - 1


@pytest.mark.parametrize("name,mirror", [("config1", 0), ("d2_mixed_radius_kink", 0), ("d2_pec", 1),
                                         ("d2_ek", 0), ("d2_ek_monopole_pec", 1)])
def test_offedge_moments_match_oracle(name, mirror, cuda_device):
    import torch

    s, sp = _solver(name)
    dt = s._dev_tables()
    d = s.degree
    n = s._geometry().n
    out = torch.empty((d + 1, d + 1, n, n), dtype=torch.complex128, device=cuda_device)
    gi = gj = None
    groups = None
    if s.extended_kernel:
        lab, lab_img = s._ek()
        gi = dt.seg.ek_group
        gj = dt.seg.ek_group_img if mirror else dt.seg.ek_group
        groups = (lab, lab_img if mirror else lab)
    gz = float(s.ground_z or 0.0)
    _lib.call("mw_offedge_moments", C.byref(dt.seg), C.byref(dt.seg), d, s.n_qp_pair, float(s.k), mirror, gz,
              gi, gj, out.data_ptr(), None)
    og = O.build_geometry(sp)
    sl, sr = og["seg_l"], og["seg_r"]
    if mirror:
        want = O.offedge_moments(sl, sr, O.mirror_pts(sl, gz), O.mirror_pts(sr, gz), og["radius"], s.k, d,
                                 s.n_qp_pair, groups)
    else:
        want = O.offedge_moments(sl, sr, sl, sr, og["radius"], s.k, d, s.n_qp_pair, groups)
    assert rel_err(out.cpu().numpy(), want) < 1e-12
