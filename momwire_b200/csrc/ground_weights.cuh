// Image weights of the ground models, per segment pair: shared by the
// Galerkin fill, the enrichment blocks and the off-edge block sampler.
#pragma once

#include "common.cuh"

namespace mw {

// The Fresnel dyad of one segment pair (_ground_refl.py:63-269): the A-term
// weight rho_v (t.t' - P) - rho_h P and rho_v itself, from the observer
// centre / tangent ci / ti and the MIRRORED source centre / tangent cjm /
// tjm, eps~ = (er, ei).
__device__ __forceinline__ void refl_dyad(const double* ci, const double* ti, const double* cjm, const double* tjm,
                                          double er, double ei, cd* wA, cd* rv_out) {
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
    cd et{er, ei};
    double sin2 = 1.0 - cth * cth;
    cd root = csqrt_p(cd{et.re - sin2, et.im});
    cd ec{et.re * cth, et.im * cth};
    cd rv = cdiv(ec - root, ec + root);
    cd rh = cdiv(cd{cth - root.re, -root.im}, cd{cth + root.re, root.im});
    *wA = (td - P) * rv - P * rh;
    *rv_out = rv;
}

// Fresnel image weights of one segment pair (_ground_refl.py:63-269 and
// _potential_ground.py:711-810): the dyad and the charge weight of the
// ground's phi mode.  ci / ti: observer centre and tangent; cjm / tjm: the
// MIRRORED source centre and tangent.
__device__ __forceinline__ void refl_weights(const double* ci, const double* ti, const double* cjm,
                                             const double* tjm, const mw_ground& gr, cd* wA, cd* wP) {
    cd rv;
    refl_dyad(ci, ti, cjm, tjm, gr.eps_re, gr.eps_im, wA, &rv);
    const cd et{gr.eps_re, gr.eps_im};
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

// NEC Eq 89 coaxial factor 1 + T1*C2 - T2*C1 of the extended thin-wire
// kernel (_bspline_kernels.py:198), R the reduced distance.
__device__ __forceinline__ cd ek_factor(double R, double a, double k) {
    double kr = k * R;
    double ar = a / R;
    double ar2 = ar * ar;
    double t1 = 0.25 * ar2 * ar2;
    double t2 = 0.5 * ar2;
    // c1 = 1 + j kr ; c2 = 3 c1 - kr^2
    double c2re = 3.0 - kr * kr, c2im = 3.0 * kr;
    return cd{1.0 + t1 * c2re - t2, t1 * c2im - t2 * kr};
}

}  // namespace mw
