"""The reference's off-edge block assemblers, evaluated on the GPU.

momwire's H-matrix and array-block solvers sample rows, columns and blocks
of Z through four functions of its accelerator module --
``bspline_assemble_offedge_block`` and its ``_refl``, ``_ek`` and
``_refl_ek`` twins (``_accelerators.cpp:1977-2680``, called from
``hmatrix.py:1157-1290`` and ``array_block.py:1143``).  This module offers
the same four functions with the same arguments and the same (nI, nJ)
complex128 result, computed by ``mw_offedge_block`` on the current CUDA
device, so a maintainer can route those calls here (INTEGRATION.md shows
how).  Inputs are host arrays, as the reference takes them; they are
uploaded, the block is filled on the device and copied back.
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib


def _torch():
    import torch

    return torch


def _side(torch, dev, supp, polys, segl, segr, tan, group, keep):
    """Upload one side's tables; ``keep`` holds the tensors alive."""
    supp = np.ascontiguousarray(supp, dtype=np.int32)
    polys = np.ascontiguousarray(polys, dtype=np.float64)
    if supp.ndim != 2 or polys.ndim != 3 or polys.shape[0] != supp.shape[0]:
        raise RuntimeError("support arrays must have shape (n, D+1)")
    arrs = [supp, polys] + [np.ascontiguousarray(a, dtype=np.float64).reshape(-1, 3) for a in (segl, segr, tan)]
    if group is not None:
        arrs.append(np.ascontiguousarray(group, dtype=np.int32))
    t = [torch.from_numpy(a).to(dev) for a in arrs]
    keep.extend(t)
    s = _lib.BlockSide()
    s.n_basis = supp.shape[0]
    s.supp, s.polys = t[0].data_ptr(), t[1].data_ptr()
    s.n_seg = arrs[2].shape[0]
    s.seg_l, s.seg_r, s.tangent = t[2].data_ptr(), t[3].data_ptr(), t[4].data_ptr()
    s.ek_group = t[5].data_ptr() if group is not None else None
    return s


def _block(supp_I, polys_I, segl_I, segr_I, tan_I, supp_J, polys_J, segl_J, segr_J, tan_J, a_squared, k, omega,
           eps_, mu_, max_d, gl_t, gl_w, cancel_flag=0, group=None, a_ek=0.0, refl=None):
    if cancel_flag:
        # the reference polls its flag inside the loop and raises when set
        if C.c_int32.from_address(int(cancel_flag)).value:
            raise RuntimeError("cancelled")
    torch = _torch()
    if not torch.cuda.is_available():
        raise RuntimeError("the off-edge block assembler needs a CUDA device")
    dev = torch.device("cuda", torch.cuda.current_device())
    keep = []
    gI, gJ = group if group is not None else (None, None)
    sI = _side(torch, dev, supp_I, polys_I, segl_I, segr_I, tan_I, gI, keep)
    sJ = _side(torch, dev, supp_J, polys_J, segl_J, segr_J, tan_J, gJ, keep)
    nI, nJ = sI.n_basis, sJ.n_basis
    t = np.ascontiguousarray(gl_t, dtype=np.float64)
    w = np.ascontiguousarray(gl_w, dtype=np.float64)
    if t.size > 8:
        raise RuntimeError("n_qp > 8 not supported (scratch buffer size)")
    Z = torch.empty((max(nI, 1), max(nJ, 1)), dtype=torch.complex128, device=dev)
    fr = _lib.Freq(float(k), float(omega), float(eps_), float(mu_))
    rf = None
    if refl is not None:
        eps_t, c0, c1 = (complex(x) for x in refl)
        rf = _lib.BlockRefl(eps_t.real, eps_t.imag, c0.real, c0.imag, c1.real, c1.imag)
    st = torch.cuda.current_stream(dev).cuda_stream
    _lib.call("mw_offedge_block", int(max_d), C.byref(sI), C.byref(sJ), float(a_squared), C.byref(fr), t.size,
              t.ctypes.data, w.ctypes.data, C.byref(rf) if rf is not None else None, float(a_ek), Z.data_ptr(),
              Z.shape[1], st)
    return Z.cpu().numpy()[:nI, :nJ].copy()


def bspline_assemble_offedge_block(supp_I, polys_I, segl_I, segr_I, tan_I, supp_J, polys_J, segl_J, segr_J, tan_J,
                                   a_squared, k, omega, eps_, mu_, max_d, gl_t, gl_w, cancel_flag=0):
    """Free-space (or, with the J side mirrored, PEC-image) block."""
    return _block(supp_I, polys_I, segl_I, segr_I, tan_I, supp_J, polys_J, segl_J, segr_J, tan_J, a_squared, k,
                  omega, eps_, mu_, max_d, gl_t, gl_w, cancel_flag)


def bspline_assemble_offedge_block_refl(supp_I, polys_I, segl_I, segr_I, tan_I, supp_J, polys_J, segl_J, segr_J,
                                        tan_J, a_squared, k, omega, eps_, mu_, max_d, gl_t, gl_w, eps_t, phi_c0,
                                        phi_c1, cancel_flag=0):
    """Reflection-coefficient image block (J side passed mirrored)."""
    return _block(supp_I, polys_I, segl_I, segr_I, tan_I, supp_J, polys_J, segl_J, segr_J, tan_J, a_squared, k,
                  omega, eps_, mu_, max_d, gl_t, gl_w, cancel_flag, refl=(eps_t, phi_c0, phi_c1))


def bspline_assemble_offedge_block_ek(supp_I, polys_I, segl_I, segr_I, tan_I, supp_J, polys_J, segl_J, segr_J,
                                      tan_J, a_squared, k, omega, eps_, mu_, max_d, gl_t, gl_w, group_I, group_J,
                                      a_ek, cancel_flag=0):
    """Extended-kernel block: NEC's coaxial factor on pairs of equal labels."""
    return _block(supp_I, polys_I, segl_I, segr_I, tan_I, supp_J, polys_J, segl_J, segr_J, tan_J, a_squared, k,
                  omega, eps_, mu_, max_d, gl_t, gl_w, cancel_flag, group=(group_I, group_J), a_ek=a_ek)


def bspline_assemble_offedge_block_refl_ek(supp_I, polys_I, segl_I, segr_I, tan_I, supp_J, polys_J, segl_J, segr_J,
                                           tan_J, a_squared, k, omega, eps_, mu_, max_d, gl_t, gl_w, group_I,
                                           group_J, a_ek, eps_t, phi_c0, phi_c1, cancel_flag=0):
    """Reflection-coefficient image block under the extended kernel."""
    return _block(supp_I, polys_I, segl_I, segr_I, tan_I, supp_J, polys_J, segl_J, segr_J, tan_J, a_squared, k,
                  omega, eps_, mu_, max_d, gl_t, gl_w, cancel_flag, group=(group_I, group_J), a_ek=a_ek,
                  refl=(eps_t, phi_c0, phi_c1))
