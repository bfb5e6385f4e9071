// Image weights of the ground models, per segment pair: shared by the
// Galerkin fill and the enrichment blocks.
#pragma once

#include "common.cuh"

namespace mw {

// Fresnel image weights of one segment pair (_ground_refl.py:63-269 and
// _potential_ground.py:711-810).  ci / ti: observer centre and tangent;
// cjm / tjm: the MIRRORED source centre and tangent.
__device__ __forceinline__ void refl_weights(const double* ci, const double* ti, const double* cjm,
                                             const double* tjm, const mw_ground& gr, cd* wA, cd* wP) {
    double dx = ci[0] - cjm[0];
    double dy = ci[1] - cjm[1];
    double dz = ci[2] - cjm[2];  // = z_i + z_j - 2 gz
    double hyp = hypot(dx, dy);
    double rmag = fmax(sqrt(dx * dx + dy * dy + dz * dz), 1e-30);
    double cth = dz / rmag;
    double px, py;
    if (hyp > 1e-30) {
        double inv = 1.0 / hyp;
        px = -(dy * inv);
        py = dx * inv;
    } else {
        px = 1.0;
        py = 0.0;
    }
    double tmp = ti[0] * px + ti[1] * py;
    double tnp = tjm[0] * px + tjm[1] * py;
    double P = tmp * tnp;
    double td = ti[0] * tjm[0] + ti[1] * tjm[1] + ti[2] * tjm[2];
    cd et{gr.eps_re, gr.eps_im};
    double sin2 = 1.0 - cth * cth;
    cd root = csqrt_p(cd{et.re - sin2, et.im});
    cd ec{et.re * cth, et.im * cth};
    cd rv = cdiv(ec - root, ec + root);
    cd rh = cdiv(cd{cth - root.re, -root.im}, cd{cth + root.re, root.im});
    *wA = (td - P) * rv - P * rh;
    switch (gr.phi_mode) {
        case MW_PHI_RHO_V: *wP = rv; break;
        case MW_PHI_IMAGE: *wP = cdiv(cd{et.re - 1.0, et.im}, cd{et.re + 1.0, et.im}); break;
        case MW_PHI_BLEND: {
            cd im = cdiv(cd{et.re - 1.0, et.im}, cd{et.re + 1.0, et.im});
            *wP = 0.5 * (rv + im);
            break;
        }
        default: {  // MW_PHI_NORMAL
            cd r = csqrt_p(et);
            *wP = cdiv(cd{r.re - 1.0, r.im}, cd{r.re + 1.0, r.im});
        }
    }
}

}  // namespace mw
