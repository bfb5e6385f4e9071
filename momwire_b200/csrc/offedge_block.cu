// Off-edge Galerkin block sampler (FP64), sm_100a.
//
// The reference's H-matrix and array-block solvers compress the far field
// with adaptive cross approximation: they ask for arbitrary rows, columns
// and blocks Z[I, J] of the impedance matrix between two basis sets, and
// its C++ assembler (bspline_assemble_offedge_block[_refl][_ek],
// _accelerators.cpp:1977-2680) evaluates them by plain n_qp x n_qp
// Gauss quadrature of every wing pair -- no same-edge treatment (the
// sampled blocks are well separated) -- fused with the Galerkin combine:
//   Z[m, n] = j w mu sum_ab w_A(a,b) I_A + sum_ab w_Phi(a,b) I_Phi / (j w eps)
//   I_A   = sum_qr w_q w_r  f_m,a(u_q) f_n,b(u_r)  G(R_qr)
//   I_Phi = sum_qr w_q w_r  f'_m,a(u_q) f'_n,b(u_r) G(R_qr)
// with G = exp(-jkR) / (4 pi R), R = sqrt(|x - y|^2 + a^2), f the wing's
// polynomial in local arc length; w_A = the tangent dot and w_Phi = 1, or
// for the reflection-coefficient image (J side passed pre-mirrored) the
// Fresnel dyad and w_Phi = c0 + c1 rho_v; under the extended kernel G takes
// NEC's coaxial factor on pairs with equal non-negative group labels.
//
// Design: one warp per (m, n) basis pair; the warp's lanes split the
// (d+1)^2 wing pairs x n_qp^2 nodes, the pair weights are computed once per
// warp by its first lanes, and a shuffle reduction gives the entry.  Output
// row-major, Z[m * ldz + n], like the reference's (nI, nJ) array.
#include "common.cuh"
#include "ground_weights.cuh"

namespace mw {

constexpr int kObWarps = 8;
constexpr int kObMaxQ = 8;

struct ObSide {
    const int32_t* supp;
    const double* polys;
    const double* seg_l;
    const double* seg_r;
    const double* tan;
    const int32_t* group;
};

struct ObArgs {
    ObSide I, J;
    int nI, nJ, d1;
    double a2, k, omega, eps0, mu0;
    int nq;
    double t[kObMaxQ], w[kObMaxQ];
    int refl;
    double er, ei, c0r, c0i, c1r, c1i;
    double a_ek;  // > 0: extended kernel on eligible pairs
    double* Z;
    int64_t ldz;
};

__device__ __forceinline__ double ob_len(const ObSide& S, int s) {
    const double dx = S.seg_r[3 * s] - S.seg_l[3 * s];
    const double dy = S.seg_r[3 * s + 1] - S.seg_l[3 * s + 1];
    const double dz = S.seg_r[3 * s + 2] - S.seg_l[3 * s + 2];
    return sqrt(dx * dx + dy * dy + dz * dz);
}

// Value and derivative of a wing's polynomial (coefficients c[0..d1-1] of
// u^p) at u.
__device__ __forceinline__ void ob_poly(const double* c, int d1, double u, double* v, double* dv) {
    double p = 0.0, dp = 0.0;
    for (int i = d1 - 1; i >= 0; --i) p = p * u + c[i];
    for (int i = d1 - 1; i >= 1; --i) dp = dp * u + i * c[i];
    *v = p;
    *dv = dp;
}

__global__ void __launch_bounds__(32 * kObWarps) offedge_block_kernel(ObArgs A) {
    __shared__ cd s_wa[kObWarps][16], s_wp[kObWarps][16];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int64_t task = (int64_t)blockIdx.x * kObWarps + wib;
    const bool live = task < (int64_t)A.nI * A.nJ;
    const int m = live ? (int)(task / A.nJ) : 0, n = live ? (int)(task % A.nJ) : 0;
    const int d1 = A.d1, np = d1 * d1;
    // per wing pair: the two weights (zero for a padded wing)
    if (live && lane < np) {
        const int a = lane / d1, b = lane % d1;
        const int si = A.I.supp[m * d1 + a], sj = A.J.supp[n * d1 + b];
        cd wa{0.0, 0.0}, wp{0.0, 0.0};
        if (si >= 0 && sj >= 0) {
            const double* ti = A.I.tan + 3 * si;
            const double* tj = A.J.tan + 3 * sj;
            const double td = ti[0] * tj[0] + ti[1] * tj[1] + ti[2] * tj[2];
            if (!A.refl) {
                wa = cd{td, 0.0};
                wp = cd{1.0, 0.0};
            } else {
                double ci[3], cj[3];
#pragma unroll
                for (int c = 0; c < 3; ++c) {
                    ci[c] = 0.5 * (A.I.seg_l[3 * si + c] + A.I.seg_r[3 * si + c]);
                    cj[c] = 0.5 * (A.J.seg_l[3 * sj + c] + A.J.seg_r[3 * sj + c]);
                }
                cd rv;
                refl_dyad(ci, ti, cj, tj, A.er, A.ei, &wa, &rv);
                wp = cd{A.c0r, A.c0i} + cd{A.c1r, A.c1i} * rv;
            }
        }
        s_wa[wib][lane] = wa;
        s_wp[wib][lane] = wp;
    }
    __syncwarp();
    cd zA{0.0, 0.0}, zP{0.0, 0.0};
    if (live) {
        const int nq = A.nq, nqq = nq * nq;
        for (int idx = lane; idx < np * nqq; idx += 32) {
            const int ab = idx / nqq, qr = idx % nqq;
            const int a = ab / d1, b = ab % d1, q = qr / nq, r = qr % nq;
            const int si = A.I.supp[m * d1 + a], sj = A.J.supp[n * d1 + b];
            if (si < 0 || sj < 0) continue;
            const double Li = ob_len(A.I, si), Lj = ob_len(A.J, sj);
            const double tq = A.t[q], tr = A.t[r];
            double R2 = A.a2;
#pragma unroll
            for (int c = 0; c < 3; ++c) {
                const double x = (1.0 - tq) * A.I.seg_l[3 * si + c] + tq * A.I.seg_r[3 * si + c];
                const double y = (1.0 - tr) * A.J.seg_l[3 * sj + c] + tr * A.J.seg_r[3 * sj + c];
                R2 += (x - y) * (x - y);
            }
            const double R = sqrt(R2);
            double sn, cs;
            sincos(A.k * R, &sn, &cs);
            const double g = 1.0 / (4.0 * kPi * R);
            cd G{cs * g, -sn * g};
            if (A.a_ek > 0.0 && A.I.group != nullptr && A.J.group != nullptr) {
                const int gi = A.I.group[si], gj = A.J.group[sj];
                if (gi >= 0 && gi == gj) G = G * ek_factor(R, A.a_ek, A.k);
            }
            double fi, dfi, fj, dfj;
            ob_poly(A.I.polys + (int64_t)(m * d1 + a) * d1, d1, tq * Li, &fi, &dfi);
            ob_poly(A.J.polys + (int64_t)(n * d1 + b) * d1, d1, tr * Lj, &fj, &dfj);
            const double wq = A.w[q] * Li * A.w[r] * Lj;
            zA = zA + (wq * fi * fj) * (s_wa[wib][ab] * G);
            zP = zP + (wq * dfi * dfj) * (s_wp[wib][ab] * G);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        zA.re += __shfl_xor_sync(0xffffffffu, zA.re, off);
        zA.im += __shfl_xor_sync(0xffffffffu, zA.im, off);
        zP.re += __shfl_xor_sync(0xffffffffu, zP.re, off);
        zP.im += __shfl_xor_sync(0xffffffffu, zP.im, off);
    }
    if (live && lane == 0) {
        const double om_mu = A.omega * A.mu0, inv_om_eps = 1.0 / (A.omega * A.eps0);
        double* out = A.Z + 2 * ((int64_t)m * A.ldz + n);
        out[0] = -om_mu * zA.im + zP.im * inv_om_eps;
        out[1] = om_mu * zA.re - zP.re * inv_om_eps;
    }
}

}  // namespace mw

using namespace mw;

extern "C" mw_status mw_offedge_block(int32_t degree, const mw_block_side* I, const mw_block_side* J,
                                      double a_squared, const mw_freq* freq, int32_t n_qp, const double* gl_t,
                                      const double* gl_w, const mw_block_refl* refl, double a_ek, double* Z,
                                      int64_t ldz, void* stream) {
    MW_REQUIRE(I && J && freq && gl_t && gl_w, "NULL argument");
    MW_REQUIRE(degree == 1 || degree == 2, "max_d must be 1 or 2, got %d", degree);
    MW_REQUIRE(n_qp >= 1 && n_qp <= kObMaxQ, "n_qp > %d not supported (got %d)", kObMaxQ, n_qp);
    MW_REQUIRE(I->n_basis >= 0 && J->n_basis >= 0, "negative basis count");
    MW_REQUIRE(ldz >= (J->n_basis > 0 ? J->n_basis : 1), "ldz smaller than the J-side basis count");
    if (I->n_basis == 0 || J->n_basis == 0) return MW_OK;
    MW_REQUIRE(Z && I->supp && I->polys && I->seg_l && I->seg_r && I->tangent && J->supp && J->polys && J->seg_l &&
                   J->seg_r && J->tangent,
               "NULL side table");
    MW_REQUIRE(!(a_ek > 0.0) || (I->ek_group && J->ek_group), "the extended kernel needs both sides' group labels");
    ObArgs A{};
    A.I = ObSide{I->supp, I->polys, I->seg_l, I->seg_r, I->tangent, I->ek_group};
    A.J = ObSide{J->supp, J->polys, J->seg_l, J->seg_r, J->tangent, J->ek_group};
    A.nI = I->n_basis;
    A.nJ = J->n_basis;
    A.d1 = degree + 1;
    A.a2 = a_squared;
    A.k = freq->k;
    A.omega = freq->omega;
    A.eps0 = freq->eps0;
    A.mu0 = freq->mu0;
    A.nq = n_qp;
    for (int i = 0; i < n_qp; ++i) {
        A.t[i] = gl_t[i];
        A.w[i] = gl_w[i];
    }
    A.refl = refl != nullptr;
    if (refl) {
        A.er = refl->eps_re;
        A.ei = refl->eps_im;
        A.c0r = refl->phi_c0_re;
        A.c0i = refl->phi_c0_im;
        A.c1r = refl->phi_c1_re;
        A.c1i = refl->phi_c1_im;
    }
    A.a_ek = a_ek;
    A.Z = Z;
    A.ldz = ldz;
    const int64_t tasks = (int64_t)A.nI * A.nJ;
    MW_REQUIRE(tasks / kObWarps < (1ll << 31), "block too large");
    cudaStream_t st = as_stream(stream);
    {
        ProfileScope ps(PC_FILL, st, 0.0, 16.0 * (double)tasks);
        offedge_block_kernel<<<(unsigned)((tasks + kObWarps - 1) / kObWarps), 32 * kObWarps, 0, st>>>(A);
    }
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}
