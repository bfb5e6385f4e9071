"""CPU oracle for the off-edge block sampler.

TEST INFRASTRUCTURE ONLY: only ``tests/`` import this module, as the
checker of ``mw_offedge_block``.

Restates the reference's fused off-edge assembler
(``bspline_assemble_offedge_block[_refl][_ek]``, ``_accelerators.cpp:1977-2680``):
for bases m in I and n in J, every wing pair (a, b) is integrated with the
n_qp x n_qp Gauss rule of reduced-kernel samples G = exp(-jkR)/(4 pi R),
R = sqrt(|x - y|^2 + a^2) (times NEC's coaxial factor on extended-kernel
pairs of equal labels), contracted with the wings' polynomials and their
derivatives, and weighted by the tangent dot (A term) and 1 (charge term)
-- or, for the reflection-coefficient image with the J side mirrored, by
the Fresnel dyad and c0 + c1 rho_v.  Vectorised over the block.
"""

from __future__ import annotations

import numpy as np

INV4PI = 1.0 / (4.0 * np.pi)


def _ek(R, a, k):
    kr = k * R
    ar2 = (a / R) ** 2
    t1, t2 = 0.25 * ar2 * ar2, 0.5 * ar2
    return (1.0 + t1 * (3.0 - kr * kr) - t2) + 1j * (3.0 * t1 * kr - t2 * kr)


def _fresnel(ci, ti, cj, tj, eps_t):
    d = ci - cj
    hyp = np.hypot(d[..., 0], d[..., 1])
    rmag = np.maximum(np.sqrt(np.sum(d * d, axis=-1)), 1e-30)
    cth = d[..., 2] / rmag
    safe = hyp > 1e-30
    inv = 1.0 / np.where(safe, hyp, 1.0)
    px = np.where(safe, -d[..., 1] * inv, 1.0)
    py = np.where(safe, d[..., 0] * inv, 0.0)
    P = (ti[..., 0] * px + ti[..., 1] * py) * (tj[..., 0] * px + tj[..., 1] * py)
    td = np.sum(ti * tj, axis=-1)
    root = np.sqrt(eps_t - (1.0 - cth * cth) + 0j)
    rv = (eps_t * cth - root) / (eps_t * cth + root)
    rh = (cth - root) / (cth + root)
    return rv * (td - P) - rh * P, rv


def offedge_block(supp_I, polys_I, segl_I, segr_I, tan_I, supp_J, polys_J, segl_J, segr_J, tan_J, a2, k, omega,
                  eps_, mu_, t, w, group=None, a_ek=0.0, refl=None):
    """Z[I, J] (nI, nJ) complex128."""
    d1 = polys_I.shape[2]
    ex = np.arange(d1)
    out = np.zeros((supp_I.shape[0], supp_J.shape[0]), np.complex128)
    for a in range(d1):
        si = supp_I[:, a]
        Li = np.linalg.norm(segr_I[si] - segl_I[si], axis=1)
        xi = (1.0 - t)[None, :, None] * segl_I[si][:, None, :] + t[None, :, None] * segr_I[si][:, None, :]
        ui = Li[:, None] * t[None, :]
        fi = np.einsum("mqp,mp->mq", ui[..., None] ** ex, polys_I[:, a, :]) * (w[None, :] * Li[:, None])
        dfi = np.einsum("mqp,mp->mq", np.where(ex > 0, ex * ui[..., None] ** np.maximum(ex - 1, 0), 0.0),
                        polys_I[:, a, :]) * (w[None, :] * Li[:, None])
        for b in range(d1):
            sj = supp_J[:, b]
            Lj = np.linalg.norm(segr_J[sj] - segl_J[sj], axis=1)
            yj = (1.0 - t)[None, :, None] * segl_J[sj][:, None, :] + t[None, :, None] * segr_J[sj][:, None, :]
            uj = Lj[:, None] * t[None, :]
            fj = np.einsum("nrp,np->nr", uj[..., None] ** ex, polys_J[:, b, :]) * (w[None, :] * Lj[:, None])
            dfj = np.einsum("nrp,np->nr", np.where(ex > 0, ex * uj[..., None] ** np.maximum(ex - 1, 0), 0.0),
                            polys_J[:, b, :]) * (w[None, :] * Lj[:, None])
            diff = xi[:, None, :, None, :] - yj[None, :, None, :, :]
            R = np.sqrt(np.sum(diff * diff, axis=-1) + a2)  # (m, n, q, r)
            G = np.exp(-1j * k * R) * (INV4PI / R)
            if group is not None and a_ek > 0.0:
                gi, gj = group[0][si], group[1][sj]
                elig = (gi[:, None] >= 0) & (gi[:, None] == gj[None, :])
                G = np.where(elig[:, :, None, None], G * _ek(R, a_ek, k), G)
            IA = np.einsum("mq,mnqr,nr->mn", fi, G, fj)
            IP = np.einsum("mq,mnqr,nr->mn", dfi, G, dfj)
            ti, tj = tan_I[si][:, None, :], tan_J[sj][None, :, :]
            if refl is None:
                wa, wp = np.sum(ti * tj, axis=-1), 1.0
            else:
                eps_t, c0, c1 = refl
                ci = 0.5 * (segl_I[si] + segr_I[si])[:, None, :]
                cj = 0.5 * (segl_J[sj] + segr_J[sj])[None, :, :]
                wa, rv = _fresnel(ci, ti, cj, tj, eps_t)
                wp = c0 + c1 * rv
            out += 1j * omega * mu_ * wa * IA + wp * IP / (1j * omega * eps_)
    return out
