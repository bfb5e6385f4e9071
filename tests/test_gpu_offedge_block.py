"""The off-edge block sampler on the GPU against the reference.

``mw_offedge_block`` (through the C ABI, and through
``momwire_b200.accel``'s functions with the reference's own signatures) on
the seven blocks the reference's ``bspline_assemble_offedge_block`` family
returned: within 1e-12 of the largest entry.  A far block of the 4x4 array
(no two wings on one edge) also equals the same block of the full fill."""

import ctypes as C

import numpy as np
import pytest

from blocks import CASES, case
from cases import CASES as STRUCTS
from conftest import rel_err

import momwire_b200
from momwire_b200 import _lib, accel

pytestmark = pytest.mark.gpu


def _via_abi(a, device):
    import torch

    keep = []

    def side(supp, polys, sl, sr, tn, grp):
        t = [torch.from_numpy(np.ascontiguousarray(x)).to(device) for x in
             (supp.astype(np.int32), polys, sl, sr, tn)]
        if grp is not None:
            t.append(torch.from_numpy(grp.astype(np.int32)).to(device))
        keep.extend(t)
        s = _lib.BlockSide(supp.shape[0], t[0].data_ptr(), t[1].data_ptr(), sl.shape[0], t[2].data_ptr(),
                           t[3].data_ptr(), t[4].data_ptr(), t[5].data_ptr() if grp is not None else None)
        return s

    g = a["group"] or (None, None)
    sI = side(a["supp_I"], a["polys_I"], a["segl_I"], a["segr_I"], a["tan_I"], g[0])
    sJ = side(a["supp_J"], a["polys_J"], a["segl_J"], a["segr_J"], a["tan_J"], g[1])
    nI, nJ = a["supp_I"].shape[0], a["supp_J"].shape[0]
    Z = torch.zeros((nI, nJ), dtype=torch.complex128, device=device)
    fr = _lib.Freq(a["k"], a["omega"], a["eps_"], a["mu_"])
    rf = None
    if a["refl"] is not None:
        e, c0, c1 = a["refl"]
        rf = _lib.BlockRefl(e.real, e.imag, c0.real, c0.imag, c1.real, c1.imag)
    t = np.ascontiguousarray(a["t"])
    w = np.ascontiguousarray(a["w"])
    _lib.call("mw_offedge_block", a["degree"], C.byref(sI), C.byref(sJ), a["a2"], C.byref(fr), t.size, t.ctypes.data,
              w.ctypes.data, C.byref(rf) if rf is not None else None, a["a_ek"], Z.data_ptr(), nJ, None)
    return Z.cpu().numpy()


@pytest.mark.parametrize("name", CASES)
def test_block_via_c_abi_matches_reference(name, cuda_device):
    a, want = case(name)
    assert rel_err(_via_abi(a, cuda_device), want) < 1e-12


@pytest.mark.parametrize("name", CASES)
def test_reference_signatures(name, cuda_device):
    a, want = case(name)
    base = (a["supp_I"], a["polys_I"], a["segl_I"], a["segr_I"], a["tan_I"], a["supp_J"], a["polys_J"], a["segl_J"],
            a["segr_J"], a["tan_J"], a["a2"], a["k"], a["omega"], a["eps_"], a["mu_"], a["degree"], a["t"], a["w"])
    if a["group"] is not None and a["refl"] is not None:
        got = accel.bspline_assemble_offedge_block_refl_ek(*base, *a["group"], a["a_ek"], *a["refl"])
    elif a["group"] is not None:
        got = accel.bspline_assemble_offedge_block_ek(*base, *a["group"], a["a_ek"])
    elif a["refl"] is not None:
        got = accel.bspline_assemble_offedge_block_refl(*base, *a["refl"])
    else:
        got = accel.bspline_assemble_offedge_block(*base)
    assert got.shape == want.shape and got.dtype == np.complex128
    assert rel_err(got, want) < 1e-12


def test_far_block_equals_the_fill(cuda_device):
    a, _want = case("free_d2_far")
    s = momwire_b200.BSplineSolver(**STRUCTS["array4x4"]())
    Z = s._compute_Z_operator()
    block = _via_abi(a, cuda_device)
    assert rel_err(block, Z[0:40, 200:262]) < 1e-11


def test_bad_quadrature_order_is_refused(cuda_device):
    a, _want = case("free_d2")
    base = (a["supp_I"], a["polys_I"], a["segl_I"], a["segr_I"], a["tan_I"], a["supp_J"], a["polys_J"], a["segl_J"],
            a["segr_J"], a["tan_J"], a["a2"], a["k"], a["omega"], a["eps_"], a["mu_"], a["degree"])
    t, w = np.polynomial.legendre.leggauss(9)
    with pytest.raises(RuntimeError, match="n_qp > 8"):
        accel.bspline_assemble_offedge_block(*base, 0.5 * (t + 1), 0.5 * w)
