// Galerkin impedance fill for the B-spline thin-wire EFIE (FP64), sm_100a.
//
// Reference algorithm: momwire bspline.py _compute_Z_operator (:3702) with
// _bspline_kernels.py's moment integrals and _accelerators.cpp's assembly.
// Design (B200-first, not a port):
//   * one CTA owns a tile of up to 16 x 16 basis pairs; the segments its
//     bases touch (<= 24 per side) are staged in shared memory together with
//     their Gauss points and weight-folded monomials;
//   * phase A computes the (d+1)^2 moments of every touched segment pair
//     straight into shared memory -- four lanes per pair, one source-side
//     quadrature row each, reduced with warp shuffles; same-edge pairs read
//     the analytic static + smooth Toeplitz table instead;
//   * phase B contracts moments with the basis polynomials into Z and
//     writes the tile column-major with coalesced stores (optionally a
//     complex64 copy for the mixed-precision factorisation).
// The (d+1)^2 x N^2 moment tensor of the reference never exists.
#include <cstdio>

#include "common.cuh"
#include "ground_weights.cuh"

namespace mw {

struct GLParams {
    int nq;
    double t[8];    // nodes on [0,1]
    double w[8];    // weights on [0,1]
    double x20[20]; // 20-point nodes on [-1,1] (static panels)
    double w20[20];
};

static GLParams make_gl(int nq) {
    GLParams g{};
    g.nq = nq;
    const double *t, *w;
    gauss_legendre01(nq, &t, &w);
    for (int i = 0; i < nq; ++i) { g.t[i] = t[i]; g.w[i] = w[i]; }
    gauss_legendre01(20, &t, &w);
    for (int i = 0; i < 20; ++i) { g.x20[i] = 2.0 * t[i] - 1.0; g.w20[i] = 2.0 * w[i]; }
    return g;
}

// fac - fac_static = T1 (3 j kr - kr^2) - T2 (j kr)   (_bspline_kernels.py:225)
__device__ __forceinline__ cd ek_reg_extra(double R, double a, double k) {
    double kr = k * R;
    double ar = a / R;
    double ar2 = ar * ar;
    double t1 = 0.25 * ar2 * ar2;
    double t2 = 0.5 * ar2;
    return cd{-t1 * kr * kr, 3.0 * t1 * kr - t2 * kr};
}

// --------------------------------------------------------------------------
// Same-edge Toeplitz table
// --------------------------------------------------------------------------

// W_pq(t) = int u^p (u - t)^q du over [0,h] ∩ [t, h+t], all terms >= 0.
template <int D>
__device__ __forceinline__ void conv_weights(double h, double t, double W[D + 1][D + 1]) {
    const double binom[3][3] = {{1, 0, 0}, {1, 1, 0}, {1, 2, 1}};
    double at = fabs(t), rest = h - at;
    double tp[D + 1], rp[2 * D + 2];
    tp[0] = 1.0;
    for (int i = 1; i <= D; ++i) tp[i] = tp[i - 1] * at;
    rp[0] = 1.0;
    for (int i = 1; i < 2 * D + 2; ++i) rp[i] = rp[i - 1] * rest;
#pragma unroll
    for (int p = 0; p <= D; ++p)
#pragma unroll
        for (int q = 0; q <= D; ++q) {
            double acc = 0.0;
            if (t >= 0.0) {
                for (int r = 0; r <= p; ++r) {
                    int e = q + r + 1;
                    acc += binom[p][r] * tp[p - r] * rp[e] / e;
                }
            } else {
                for (int r = 0; r <= q; ++r) {
                    int e = p + r + 1;
                    acc += binom[q][r] * tp[q - r] * rp[e] / e;
                }
            }
            W[p][q] = acc;
        }
}

// The static integral of one table row is a sum over Gauss points of
// graded panels on the two half-intervals [-h, 0] and [0, h].  A half whose
// kernel peak c is at least one interval length away is a single 20-point
// panel; otherwise the panels grow geometrically from the end nearest the
// peak: [0, s], [s, 2s], [2s, 4s], ... (s = the radius) until they cover the
// interval.  The peak of every same-edge table entry sits on an end of the
// half interval (c = delta*h with integer delta) or outside it.
__device__ __forceinline__ int half_panels(double lo, double hi, double c, double a, bool& graded,
                                           bool& near_left) {
    const double L = hi - lo;
    const double dist = (c < lo) ? lo - c : (c > hi ? c - hi : 0.0);
    graded = dist < L;
    near_left = fabs(lo - c) <= fabs(hi - c);
    if (!graded) return 1;
    int n = 1;
    for (double s1 = fmax(a, 1e-300); s1 < L; s1 *= 2.0) ++n;
    return n;
}

// Bounds of panel i of a half-interval (see half_panels).
__device__ __forceinline__ void half_panel_bounds(double lo, double hi, double a, bool graded, bool near_left,
                                                  int i, double& x0, double& x1) {
    if (!graded) {
        x0 = lo;
        x1 = hi;
        return;
    }
    const double L = hi - lo, s = fmax(a, 1e-300);
    const double e0 = i == 0 ? 0.0 : fmin(ldexp(s, i - 1), L);
    const double e1 = fmin(ldexp(s, i), L);
    if (near_left) {
        x0 = lo + e0;
        x1 = lo + e1;
    } else {
        x0 = hi - e1;
        x1 = hi - e0;
    }
}

// One Gauss point g of panel [x0, x1] of the static integral:
// acc += half_width w_g K(t - c) W(t), K = 1/R (+ the EK correction).
template <int D, bool EK>
__device__ __forceinline__ void static_point(double x0, double x1, int g, double c, double h, double a,
                                             const GLParams& gl, double acc[D + 1][D + 1]) {
    const double half = 0.5 * (x1 - x0), mid = 0.5 * (x0 + x1);
    const double t = mid + half * gl.x20[g];
    const double x = t - c;
    const double R2 = x * x + a * a;
    const double R = sqrt(R2);
    double K = 1.0 / R;
    if (EK) K += (a * a / (4.0 * R2 * R2 * R)) * (3.0 * a * a - 2.0 * R2);
    double W[D + 1][D + 1];
    conv_weights<D>(h, t, W);
    const double wk = half * gl.w20[g] * K;
#pragma unroll
    for (int p = 0; p <= D; ++p)
#pragma unroll
        for (int q = 0; q <= D; ++q) acc[p][q] += wk * W[p][q];
}

template <int N>
__device__ __forceinline__ void warp_sum(double (&v)[N]) {
#pragma unroll
    for (int i = 0; i < N; ++i)
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v[i] += __shfl_xor_sync(0xffffffffu, v[i], off);
}

// Table modes: kTableFused writes static + smooth parts for one k per
// blockIdx.y; a frequency batch instead runs kTableStatic once (the static
// part is k-independent: it is written, as the real part, into all n_k
// tables) and then kTableSmoothAdd per k, which adds the smooth part.
enum { kTableFused = 0, kTableStatic = 1, kTableSmoothAdd = 2 };
constexpr int kTableThreads = 128;  // one warp per table row

// One warp per same-edge table row: the lanes split the static quadrature
// points and the nq x nq smooth-part samples, then reduce with shuffles.
template <int D, bool EK>
__global__ void __launch_bounds__(kTableThreads) same_edge_table_kernel(
    int n_edge, const int32_t* __restrict__ n_in_edge, const int64_t* __restrict__ table_off,
    const double* __restrict__ hs, const double* __restrict__ radii, int64_t rows, double k0, GLParams gl,
    double* __restrict__ out, const double* __restrict__ kb, int64_t out_stride, int mode = kTableFused,
    int n_k = 1) {
    constexpr int NM = D + 1, NE = NM * NM * 2;
    const int lane = threadIdx.x & 31;
    const int64_t row = blockIdx.x * (int64_t)(kTableThreads / 32) + (threadIdx.x >> 5);
    if (row >= rows) return;  // uniform per warp
    const double k = kb ? kb[blockIdx.y] : k0;
    double* const out0 = out;
    out += blockIdx.y * out_stride;
    // edge owning this row: last e with table_off[e] <= row
    int lo = 0, hi = n_edge - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (table_off[mid] <= row) lo = mid; else hi = mid - 1;
    }
    const int e = lo;
    const int n = n_in_edge[e];
    const int delta = (int)(row - table_off[e]) - (n - 1);
    const double h = hs[e], a = radii[e];
    const double c = delta * h;

    double st[NM * NM];
#pragma unroll
    for (int i = 0; i < NM * NM; ++i) st[i] = 0.0;
    if (mode != kTableSmoothAdd) {
        bool g0, l0, g1, l1;
        const int n0 = half_panels(-h, 0.0, c, a, g0, l0);
        const int n1 = half_panels(0.0, h, c, a, g1, l1);
        double acc[NM][NM];
#pragma unroll
        for (int p = 0; p < NM; ++p)
#pragma unroll
            for (int q = 0; q < NM; ++q) acc[p][q] = 0.0;
        for (int g = lane; g < 20 * (n0 + n1); g += 32) {
            const int pi = g / 20, gi = g - pi * 20;
            double x0, x1;
            if (pi < n0) half_panel_bounds(-h, 0.0, a, g0, l0, pi, x0, x1);
            else         half_panel_bounds(0.0, h, a, g1, l1, pi - n0, x0, x1);
            static_point<D, EK>(x0, x1, gi, c, h, a, gl, acc);
        }
#pragma unroll
        for (int p = 0; p < NM; ++p)
#pragma unroll
            for (int q = 0; q < NM; ++q) st[p * NM + q] = kInv4Pi * acc[p][q];
        warp_sum(st);
    }
    if (mode == kTableStatic) {
        for (int idx = lane; idx < n_k * NE; idx += 32) {
            const int b = idx / NE, x = idx - b * NE;
            out0[b * out_stride + row * NE + x] = (x & 1) ? 0.0 : st[x >> 1];
        }
        return;
    }

    // smooth part: (exp(-jkR) - 1)/(4 pi R) on nq x nq Gauss points
    double rg[NE];
#pragma unroll
    for (int i = 0; i < NE; ++i) rg[i] = 0.0;
    for (int smp = lane; smp < gl.nq * gl.nq; smp += 32) {
        const int qi = smp / gl.nq, ri = smp - qi * gl.nq;
        const double u = gl.t[qi] * h, wu = gl.w[qi] * h;
        const double v = gl.t[ri] * h, wv = gl.w[ri] * h;
        const double x = u - v - c;
        const double R = sqrt(x * x + a * a);
        double s, co, sh, ch;
        sincos(k * R, &s, &co);
        sincos(0.5 * k * R, &sh, &ch);
        // exp(-jkR) - 1 = -2 sin^2(kR/2) - j sin(kR)
        cd num = cd{-2.0 * sh * sh, -s};
        if (EK) num = num * ek_factor(R, a, k) + ek_reg_extra(R, a, k);
        const double g = kInv4Pi / R;
        const cd G = cd{num.re * g, num.im * g};
        double up = wu;
#pragma unroll
        for (int p = 0; p < NM; ++p) {
            double vp = wv;
#pragma unroll
            for (int P = 0; P < NM; ++P) {
                rg[(p * NM + P) * 2 + 0] += up * vp * G.re;
                rg[(p * NM + P) * 2 + 1] += up * vp * G.im;
                vp *= v;
            }
            up *= u;
        }
    }
    warp_sum(rg);
    if (lane < NE) {
        double* o = out + row * NE + lane;
        // rg[lane] with a lane-dependent index: pick it with a static loop
        double mine = 0.0, stat = 0.0;
#pragma unroll
        for (int i = 0; i < NE; ++i)
            if (i == lane) mine = rg[i];
#pragma unroll
        for (int i = 0; i < NM * NM; ++i)
            if (2 * i == lane) stat = st[i];
        if (mode == kTableSmoothAdd) *o += mine;
        else *o = stat + mine;
    }
}

// --------------------------------------------------------------------------
// Pair moments (shared by the fused fill and the standalone moment kernel)
// --------------------------------------------------------------------------

// Per-segment staged data: Gauss points (3 nq), weight-folded powers
// w_q L (u_q)^p (nq*(D+1)), tangent, centre, radius.
template <int D>
struct SegStage {
    static constexpr int NM = D + 1;
    __device__ static int stride(int nq) { return nq * 3 + nq * NM + 7; }
};

template <int D>
__device__ __forceinline__ void stage_segment(double* dst, int nq, const GLParams& gl,
                                              const double* sl, const double* sr, const double* tg,
                                              double a, bool mirror, double gz) {
    constexpr int NM = D + 1;
    double l0 = sl[0], l1 = sl[1], l2 = sl[2];
    double r0 = sr[0], r1 = sr[1], r2 = sr[2];
    double dx = r0 - l0, dy = r1 - l1, dz = r2 - l2;
    double L = sqrt(dx * dx + dy * dy + dz * dz);
    for (int q = 0; q < nq; ++q) {
        double t = gl.t[q];
        double px = (1.0 - t) * l0 + t * r0;
        double py = (1.0 - t) * l1 + t * r1;
        double pz = (1.0 - t) * l2 + t * r2;
        if (mirror) pz = 2.0 * gz - pz;
        dst[q * 3 + 0] = px;
        dst[q * 3 + 1] = py;
        dst[q * 3 + 2] = pz;
        double u = t * L, wp = gl.w[q] * L;
        for (int p = 0; p < NM; ++p) {
            dst[nq * 3 + q * NM + p] = wp;
            wp *= u;
        }
    }
    int o = nq * 3 + nq * NM;
    dst[o + 0] = tg[0];
    dst[o + 1] = tg[1];
    dst[o + 2] = mirror ? -tg[2] : tg[2];
    double cz = 0.5 * (l2 + r2);
    dst[o + 3] = 0.5 * (l0 + r0);
    dst[o + 4] = 0.5 * (l1 + r1);
    dst[o + 5] = mirror ? 2.0 * gz - cz : cz;
    dst[o + 6] = a;
}

// sin x and cos x for |x| <= kPhaseStepMax from their Taylor series through
// x^17 and x^16 (Horner in x^2; coefficients 1/n!).  At |x| = 0.75 the first
// omitted terms, x^19/19! and x^18/18!, are below 1e-18: full double
// precision.
constexpr double kPhaseStepMax = 0.75;
__device__ __forceinline__ void phase_step(double x, double* sx, double* cx) {
    const double t = x * x;
    double c = 1.0 / 20922789888000.0;  // 1/16!
    c = fma(c, t, -1.0 / 87178291200.0);
    c = fma(c, t, 1.0 / 479001600.0);
    c = fma(c, t, -1.0 / 3628800.0);
    c = fma(c, t, 1.0 / 40320.0);
    c = fma(c, t, -1.0 / 720.0);
    c = fma(c, t, 1.0 / 24.0);
    c = fma(c, t, -0.5);
    *cx = fma(c, t, 1.0);
    double s = 1.0 / 355687428096000.0;  // 1/17!
    s = fma(s, t, -1.0 / 1307674368000.0);
    s = fma(s, t, 1.0 / 6227020800.0);
    s = fma(s, t, -1.0 / 39916800.0);
    s = fma(s, t, 1.0 / 362880.0);
    s = fma(s, t, -1.0 / 5040.0);
    s = fma(s, t, 1.0 / 120.0);
    s = fma(s, t, -1.0 / 6.0);
    *sx = fma(s * t, x, x);
}

// Lane `qi` of a pair computes its observer quadrature row and returns its
// share of all (D+1)^2 moments; the caller reduces the shares over lanes.
// NQ > 0: the quadrature order is known at compile time (nq == NQ), so the
// source-point loop unrolls and its independent samples interleave.
template <int D, bool EK, int NQ = 0>
__device__ __forceinline__ void pair_row(const double* si, const double* sj, int nq_rt, int qi,
                                         double k, bool ek_on, cd Jp[D + 1][D + 1]) {
    constexpr int NM = D + 1;
    const int nq = NQ > 0 ? NQ : nq_rt;
#pragma unroll
    for (int p = 0; p < NM; ++p)
#pragma unroll
        for (int P = 0; P < NM; ++P) Jp[p][P] = cd{0.0, 0.0};
    if (qi >= nq) return;
    double a = si[nq * 3 + nq * NM + 6];
    double a2 = a * a;
    double xi = si[qi * 3 + 0], yi = si[qi * 3 + 1], zi = si[qi * 3 + 2];
    cd accP[NM];
#pragma unroll
    for (int P = 0; P < NM; ++P) accP[P] = cd{0.0, 0.0};
    const double* wv = sj + nq * 3;
    double R0 = 0.0, s0 = 0.0, c0 = 1.0;
#pragma unroll
    for (int r = 0; r < (NQ > 0 ? NQ : 8); ++r) {
        if (NQ == 0 && r >= nq) break;
        double dx = xi - sj[r * 3 + 0];
        double dy = yi - sj[r * 3 + 1];
        double dz = zi - sj[r * 3 + 2];
        double R2 = dx * dx + dy * dy + dz * dz + a2;
        // one reciprocal square root serves both R and 1/R
        double iR = rsqrt(R2);
        double R = R2 * iR;
        double s, c;
        // the first source point's phase in full; the others rotate it by
        // k (R - R0), at most k times a segment length, through that angle's
        // Taylor series (phase_step) -- a full sincos where it is wider
        const double x = k * (R - R0);
        if (r == 0 || fabs(x) > kPhaseStepMax) {
            sincos(k * R, &s, &c);
            if (r == 0) {
                R0 = R;
                s0 = s;
                c0 = c;
            }
        } else {
            double sx, cx;
            phase_step(x, &sx, &cx);
            s = s0 * cx + c0 * sx;
            c = c0 * cx - s0 * sx;
        }
        double g = kInv4Pi * iR;
        cd G = cd{c * g, -s * g};
        if (EK && ek_on) G = G * ek_factor(R, a, k);
#pragma unroll
        for (int P = 0; P < NM; ++P) {
            double w = wv[r * NM + P];
            accP[P].re += w * G.re;
            accP[P].im += w * G.im;
        }
    }
    const double* wu = si + nq * 3 + qi * NM;
#pragma unroll
    for (int p = 0; p < NM; ++p) {
        double w = wu[p];
#pragma unroll
        for (int P = 0; P < NM; ++P) Jp[p][P] = cd{w * accP[P].re, w * accP[P].im};
    }
}

template <int D>
__device__ __forceinline__ void reduce4(cd Jp[D + 1][D + 1]) {
#pragma unroll
    for (int p = 0; p <= D; ++p)
#pragma unroll
        for (int P = 0; P <= D; ++P) {
#pragma unroll
            for (int off = 1; off < 4; off <<= 1) {
                Jp[p][P].re += __shfl_xor_sync(0xffffffffu, Jp[p][P].re, off);
                Jp[p][P].im += __shfl_xor_sync(0xffffffffu, Jp[p][P].im, off);
            }
        }
}

// --------------------------------------------------------------------------
// Fused fill kernel
// --------------------------------------------------------------------------

struct FillArgs {
    mw_segments seg;
    mw_basis basis;
    const double* table;
    const int32_t* e_n;        // edges: segments per edge
    const int64_t* e_off;      // edges: table offsets
    mw_ground ground;
    double k, omega, eps0, mu0;
    double* Z;
    int64_t ldz;
    float* Z32;
    int64_t ldz32;
    // frequency batch (blockIdx.z): per-entry k / omega (NULL = the scalars
    // above) and the strides between consecutive tables and matrices
    const double* kb;
    const double* omegab;
    int64_t table_stride, z_stride, z32_stride;
    int nbatch;
};

// One (row tile, column tile) block of Z.  With allow_mirror the tile pair
// is checked for symmetry (every staged segment of both tiles has the same
// radius: the thin-wire kernel uses the observer radius, so only then is the
// Galerkin block of (tc, tr) the transpose of that of (tr, tc)); a symmetric
// pair also writes the transposed block.  Returns whether it did.
template <int D, bool IMAGE, bool EK>
__device__ __forceinline__ bool fill_tile(const FillArgs& A, const GLParams& gl, double* smem, const int tr,
                                          const int tc, const bool allow_mirror) {
    constexpr int NM = D + 1, NMM = NM * NM;
    const int nq = gl.nq;
    const int SD = SegStage<D>::stride(nq);
    const int SMAX = A.basis.max_tile_seg;
    const int TB = A.basis.max_tile_basis;
    const int ns_r = A.basis.tile_ns[tr], ns_c = A.basis.tile_ns[tc];
    const int nb_r = A.basis.tile_nb[tr], nb_c = A.basis.tile_nb[tc];
    const int fb_r = A.basis.tile_first[tr], fb_c = A.basis.tile_first[tc];
    const int bz = blockIdx.z;
    const double kz = A.kb ? A.kb[bz] : A.k;
    const double omz = A.omegab ? A.omegab[bz] : A.omega;
    const double* table = A.table ? A.table + bz * A.table_stride : nullptr;
    // z_stride / z32_stride count complex elements (two scalars each)
    double* Zb = A.Z + 2 * bz * A.z_stride;
    float* Z32b = A.Z32 ? A.Z32 + 2 * bz * A.z32_stride : nullptr;

    double* s_row = smem;                               // SMAX * SD
    double* s_col = s_row + SMAX * SD;                  // SMAX * SD
    double* s_J = s_col + SMAX * SD;                    // SMAX*SMAX*NMM*2
    double* s_W = s_J + (size_t)SMAX * SMAX * NMM * 2;  // image: SMAX*SMAX*4
    double* s_pr = s_W + (IMAGE ? (size_t)SMAX * SMAX * 4 : 0);  // TB*NMM
    double* s_pc = s_pr + TB * NMM;                     // TB*NMM
    double* s_out = s_pc + TB * NMM;                    // TB*TB*2 (mirrored block)
    int* s_int = reinterpret_cast<int*>(s_out + TB * TB * 2);
    int* s_seg_r = s_int;               // SMAX
    int* s_seg_c = s_seg_r + SMAX;      // SMAX
    int* s_edge_r = s_seg_c + SMAX;     // SMAX
    int* s_edge_c = s_edge_r + SMAX;
    int* s_pos_r = s_edge_c + SMAX;
    int* s_pos_c = s_pos_r + SMAX;
    int* s_grp_r = s_pos_c + SMAX;
    int* s_grp_c = s_grp_r + SMAX;
    int* s_loc_r = s_grp_c + SMAX;      // TB*NM
    int* s_loc_c = s_loc_r + TB * NM;   // TB*NM

    const int tid = threadIdx.x;
    const double gz = A.ground.ground_z;

    // ---- staging: segment lists, Gauss points, basis polynomials
    const double r_ref = A.seg.radius[A.basis.tile_seg[(size_t)tr * SMAX]];
    int odd_radius = 0;
    for (int i = tid; i < ns_r; i += blockDim.x) {
        int s = A.basis.tile_seg[(size_t)tr * SMAX + i];
        odd_radius |= A.seg.radius[s] != r_ref;
        s_seg_r[i] = s;
        s_edge_r[i] = A.seg.edge[s];
        s_pos_r[i] = A.seg.pos_in_edge[s];
        s_grp_r[i] = EK ? A.seg.ek_group[s] : 0;
        stage_segment<D>(s_row + i * SD, nq, gl, A.seg.seg_l + 3 * s, A.seg.seg_r + 3 * s,
                         A.seg.tangent + 3 * s, A.seg.radius[s], false, 0.0);
    }
    for (int i = tid; i < ns_c; i += blockDim.x) {
        int s = A.basis.tile_seg[(size_t)tc * SMAX + i];
        odd_radius |= A.seg.radius[s] != r_ref;
        s_seg_c[i] = s;
        s_edge_c[i] = A.seg.edge[s];
        s_pos_c[i] = A.seg.pos_in_edge[s];
        s_grp_c[i] = EK ? (IMAGE ? A.seg.ek_group_img[s] : A.seg.ek_group[s]) : 0;
        stage_segment<D>(s_col + i * SD, nq, gl, A.seg.seg_l + 3 * s, A.seg.seg_r + 3 * s,
                         A.seg.tangent + 3 * s, A.seg.radius[s], IMAGE, gz);
    }
    for (int i = tid; i < nb_r * NMM; i += blockDim.x)
        s_pr[i] = A.basis.polys[(size_t)fb_r * NMM + i];
    for (int i = tid; i < nb_c * NMM; i += blockDim.x)
        s_pc[i] = A.basis.polys[(size_t)fb_c * NMM + i];
    for (int i = tid; i < nb_r * NM; i += blockDim.x) s_loc_r[i] = A.basis.loc[(size_t)fb_r * NM + i];
    for (int i = tid; i < nb_c * NM; i += blockDim.x) s_loc_c[i] = A.basis.loc[(size_t)fb_c * NM + i];
    const bool mirror = __syncthreads_or(odd_radius) == 0 && allow_mirror;

    // ---- phase A: moments of every staged segment pair (4 lanes per pair)
    const int npair = ns_r * ns_c;
    const int lane4 = tid & 3;
    const int ngroups = blockDim.x >> 2;
    const int rounds = (npair + ngroups - 1) / ngroups;
    for (int rd = 0; rd < rounds; ++rd) {
        int pidx = rd * ngroups + (tid >> 2);
        bool valid = pidx < npair;
        int li = valid ? pidx / ns_c : 0;
        int lj = valid ? pidx - li * ns_c : 0;
        bool same_edge = !IMAGE && valid && s_edge_r[li] == s_edge_c[lj];
        cd Jp[NM][NM];
        // every lane of the warp joins the shuffles; invalid/same-edge
        // groups contribute zeros
        if (valid && !same_edge) {
            bool ek_on = EK && (s_grp_r[li] == s_grp_c[lj]);
            if (nq == 4) {
                // the default rule: one observer point per lane
                pair_row<D, EK, 4>(s_row + li * SD, s_col + lj * SD, 4, lane4, kz, ek_on, Jp);
            } else {
                cd Jt[NM][NM];
                pair_row<D, EK>(s_row + li * SD, s_col + lj * SD, nq, lane4, kz, ek_on, Jt);
                cd Jt2[NM][NM];
                pair_row<D, EK>(s_row + li * SD, s_col + lj * SD, nq, lane4 + 4, kz, ek_on, Jt2);
#pragma unroll
                for (int p = 0; p < NM; ++p)
#pragma unroll
                    for (int P = 0; P < NM; ++P) Jp[p][P] = Jt[p][P] + Jt2[p][P];
            }
        } else {
#pragma unroll
            for (int p = 0; p < NM; ++p)
#pragma unroll
                for (int P = 0; P < NM; ++P) Jp[p][P] = cd{0.0, 0.0};
        }
        reduce4<D>(Jp);
        if (valid) {
            double* dst = s_J + (size_t)pidx * NMM * 2;
            if (same_edge) {
                if (lane4 == 0) {
                    int e = s_edge_r[li];
                    int64_t row = A.e_off[e] + (s_pos_c[lj] - s_pos_r[li]) + A.e_n[e] - 1;
                    const double* src = table + row * NMM * 2;
#pragma unroll
                    for (int x = 0; x < NMM * 2; ++x) dst[x] = src[x];
                }
            } else if (lane4 == 0) {
#pragma unroll
                for (int p = 0; p < NM; ++p)
#pragma unroll
                    for (int P = 0; P < NM; ++P) {
                        dst[(p * NM + P) * 2 + 0] = Jp[p][P].re;
                        dst[(p * NM + P) * 2 + 1] = Jp[p][P].im;
                    }
            }
            if (IMAGE && lane4 == 1) {
                // per-pair image weights
                const double* si = s_row + li * SD + nq * 3 + nq * NM;
                const double* sj = s_col + lj * SD + nq * 3 + nq * NM;
                cd wA, wP;
                if (A.ground.model == MW_GROUND_REFL) {
                    refl_weights(si + 3, si, sj + 3, sj, A.ground, &wA, &wP);
                } else {
                    double td = si[0] * sj[0] + si[1] * sj[1] + si[2] * sj[2];
                    if (A.ground.model == MW_GROUND_SOMM_IMAGE) {
                        cd et{A.ground.eps_re, A.ground.eps_im};
                        cd c2 = cdiv(cd{et.re - 1.0, et.im}, cd{et.re + 1.0, et.im});
                        wA = td * c2;
                        wP = c2;
                    } else {
                        wA = cd{td, 0.0};
                        wP = cd{1.0, 0.0};
                    }
                }
                double* w = s_W + (size_t)pidx * 4;
                w[0] = wA.re; w[1] = wA.im; w[2] = wP.re; w[3] = wP.im;
            }
        }
    }
    __syncthreads();

    // ---- phase B: Galerkin contraction into the Z tile
    const double wmu = omz * A.mu0;
    const double inv_weps = 1.0 / (omz * A.eps0);
    for (int pp = tid; pp < TB * TB; pp += blockDim.x) {
        int mi = pp % TB, ni = pp / TB;
        if (mi >= nb_r || ni >= nb_c) continue;
        cd zA{0.0, 0.0}, zP{0.0, 0.0};
        const double* Cm = s_pr + mi * NMM;
        const double* Cn = s_pc + ni * NMM;
        for (int a = 0; a < NM; ++a) {
            int la = s_loc_r[mi * NM + a];
            if (la < 0) continue;
            for (int b = 0; b < NM; ++b) {
                int lb = s_loc_c[ni * NM + b];
                if (lb < 0) continue;
                const double* J = s_J + ((size_t)la * ns_c + lb) * NMM * 2;
                cd inA{0.0, 0.0}, inP{0.0, 0.0};
#pragma unroll
                for (int p = 0; p < NM; ++p) {
                    cd rowA{0.0, 0.0};
#pragma unroll
                    for (int P = 0; P < NM; ++P) {
                        double c = Cn[b * NM + P];
                        rowA.re += c * J[(p * NM + P) * 2 + 0];
                        rowA.im += c * J[(p * NM + P) * 2 + 1];
                    }
                    double cm = Cm[a * NM + p];
                    inA.re += cm * rowA.re;
                    inA.im += cm * rowA.im;
                }
#pragma unroll
                for (int p = 1; p < NM; ++p) {
                    cd rowP{0.0, 0.0};
#pragma unroll
                    for (int P = 1; P < NM; ++P) {
                        double c = P * Cn[b * NM + P];
                        rowP.re += c * J[((p - 1) * NM + (P - 1)) * 2 + 0];
                        rowP.im += c * J[((p - 1) * NM + (P - 1)) * 2 + 1];
                    }
                    double cm = p * Cm[a * NM + p];
                    inP.re += cm * rowP.re;
                    inP.im += cm * rowP.im;
                }
                if (IMAGE) {
                    const double* w = s_W + ((size_t)la * ns_c + lb) * 4;
                    zA = zA + cd{w[0], w[1]} * inA;
                    zP = zP + cd{w[2], w[3]} * inP;
                } else {
                    const double* ti = s_row + la * SD + nq * 3 + nq * NM;
                    const double* tj = s_col + lb * SD + nq * 3 + nq * NM;
                    double td = ti[0] * tj[0] + ti[1] * tj[1] + ti[2] * tj[2];
                    zA.re += td * inA.re;
                    zA.im += td * inA.im;
                    zP = zP + inP;
                }
            }
        }
        // j w mu zA + zP / (j w eps)
        double zre = -wmu * zA.im + inv_weps * zP.im;
        double zim = wmu * zA.re - inv_weps * zP.re;
        if (mirror) {
            s_out[(mi * TB + ni) * 2 + 0] = zre;
            s_out[(mi * TB + ni) * 2 + 1] = zim;
        }
        int64_t m = fb_r + mi, n = fb_c + ni;
        double* zp = Zb + m * 2 + n * A.ldz * 2;
        if (IMAGE) {
            zre = zp[0] - zre;
            zim = zp[1] - zim;
        }
        zp[0] = zre;
        zp[1] = zim;
        if (Z32b) {
            float* z32 = Z32b + m * 2 + n * A.ldz32 * 2;
            z32[0] = (float)zre;
            z32[1] = (float)zim;
        }
    }
    if (!mirror) return false;
    __syncthreads();
    // the transposed block Z[n, m], column tile index fastest (coalesced)
    for (int pp = tid; pp < TB * TB; pp += blockDim.x) {
        int ni = pp % TB, mi = pp / TB;
        if (mi >= nb_r || ni >= nb_c) continue;
        double zre = s_out[(mi * TB + ni) * 2 + 0];
        double zim = s_out[(mi * TB + ni) * 2 + 1];
        int64_t m = fb_r + mi, n = fb_c + ni;
        double* zp = Zb + n * 2 + m * A.ldz * 2;
        if (IMAGE) {
            zre = zp[0] - zre;
            zim = zp[1] - zim;
        }
        zp[0] = zre;
        zp[1] = zim;
        if (Z32b) {
            float* z32 = Z32b + n * 2 + m * A.ldz32 * 2;
            z32[0] = (float)zre;
            z32[1] = (float)zim;
        }
    }
    return true;
}

// Upper-triangle tile pair of block b: tc(tc+1)/2 <= b < (tc+1)(tc+2)/2,
// tr = b - tc(tc+1)/2 <= tc.
__device__ __forceinline__ void tri_pair(int64_t b, int& tr, int& tc) {
    int64_t c = (int64_t)((sqrt(8.0 * (double)b + 1.0) - 1.0) * 0.5);
    while ((c + 1) * (c + 2) / 2 <= b) ++c;
    while (c * (c + 1) / 2 > b) --c;
    tc = (int)c;
    tr = (int)(b - c * (c + 1) / 2);
}

// One block per upper-triangle tile pair (tr <= tc).  A symmetric pair is
// computed once and written to both blocks of Z; otherwise the block also
// computes (tc, tr) itself.  The EK image fill labels direct and mirrored
// segments separately, so it always computes both.
#ifndef MW_FILL_MIN_BLOCKS
#define MW_FILL_MIN_BLOCKS 3  // resident CTAs per SM the register allocation must allow
#endif

template <int D, bool IMAGE, bool EK>
__global__ void __launch_bounds__(256, MW_FILL_MIN_BLOCKS) fill_kernel(FillArgs A, GLParams gl) {
    extern __shared__ double smem[];
    int tr, tc;
    tri_pair((int64_t)blockIdx.x, tr, tc);
    const bool off_diag = tr != tc;
    const bool mirrored = fill_tile<D, IMAGE, EK>(A, gl, smem, tr, tc, off_diag && !(IMAGE && EK));
    if (off_diag && !mirrored) {
        __syncthreads();
        fill_tile<D, IMAGE, EK>(A, gl, smem, tc, tr, false);
    }
}

// --------------------------------------------------------------------------
// Standalone moment tensor (parity tests; the fill never materialises J)
// --------------------------------------------------------------------------

template <int D>
__global__ void offedge_moments_kernel(mw_segments si, mw_segments sj, double k, int mirror, double gz,
                                       const int32_t* gi, const int32_t* gj, GLParams gl,
                                       double* __restrict__ out) {
    constexpr int NM = D + 1;
    int nq = gl.nq;
    int64_t pair = (blockIdx.x * (int64_t)blockDim.x + threadIdx.x) >> 2;
    int lane4 = threadIdx.x & 3;
    int64_t npair = (int64_t)si.n_seg * sj.n_seg;
    bool valid = pair < npair;
    int i = valid ? (int)(pair / sj.n_seg) : 0;
    int j = valid ? (int)(pair - (int64_t)i * sj.n_seg) : 0;
    double bi[8 * 3 + 8 * NM + 7], bj[8 * 3 + 8 * NM + 7];
    cd Jp[NM][NM];
    if (valid) {
        stage_segment<D>(bi, nq, gl, si.seg_l + 3 * i, si.seg_r + 3 * i, si.tangent + 3 * i,
                         si.radius[i], false, 0.0);
        stage_segment<D>(bj, nq, gl, sj.seg_l + 3 * j, sj.seg_r + 3 * j, sj.tangent + 3 * j,
                         sj.radius[j], mirror != 0, gz);
        bool ek_on = gi && gj && gi[i] == gj[j];
        cd J1[NM][NM], J2[NM][NM];
        if (gi && gj) {
            pair_row<D, true>(bi, bj, nq, lane4, k, ek_on, J1);
            pair_row<D, true>(bi, bj, nq, lane4 + 4, k, ek_on, J2);
        } else {
            pair_row<D, false>(bi, bj, nq, lane4, k, false, J1);
            pair_row<D, false>(bi, bj, nq, lane4 + 4, k, false, J2);
        }
#pragma unroll
        for (int p = 0; p < NM; ++p)
#pragma unroll
            for (int P = 0; P < NM; ++P) Jp[p][P] = J1[p][P] + J2[p][P];
    } else {
#pragma unroll
        for (int p = 0; p < NM; ++p)
#pragma unroll
            for (int P = 0; P < NM; ++P) Jp[p][P] = cd{0.0, 0.0};
    }
    reduce4<D>(Jp);
    if (valid && lane4 == 0) {
#pragma unroll
        for (int p = 0; p < NM; ++p)
#pragma unroll
            for (int P = 0; P < NM; ++P) {
                size_t o = (((size_t)p * NM + P) * si.n_seg + i) * sj.n_seg + j;
                out[2 * o + 0] = Jp[p][P].re;
                out[2 * o + 1] = Jp[p][P].im;
            }
    }
}

// --------------------------------------------------------------------------
// Host launchers
// --------------------------------------------------------------------------

static size_t fill_smem_bytes(int D, bool image, int nq, int smax, int tb) {
    int NM = D + 1, NMM = NM * NM;
    int SD = nq * 3 + nq * NM + 7;
    size_t dbl = (size_t)2 * smax * SD + (size_t)smax * smax * NMM * 2 + (image ? (size_t)smax * smax * 4 : 0) +
                 (size_t)2 * tb * NMM + (size_t)tb * tb * 2;
    size_t ints = (size_t)8 * smax + (size_t)2 * tb * NM;
    return dbl * 8 + ints * 4;
}

// Algorithmic flops of one fill: q^2 * 20 per kernel sample group plus the
// (d+1)^2 moment FMAs per segment pair, and the Galerkin contraction per
// basis pair, (d+1)^2 [2 (d+1)^2 + 2 d^2] * 2.
static double fill_flops(int D, int nq, double n_seg, double n_basis) {
    double NM = D + 1;
    double f_pair = nq * nq * 20.0 + NM * NM * nq * nq * 4.0;
    double f_basis = NM * NM * (2.0 * NM * NM + 2.0 * D * D) * 2.0;
    return n_seg * n_seg * f_pair + n_basis * n_basis * f_basis;
}

template <int D, bool IMAGE, bool EK>
static mw_status launch_fill(const FillArgs& A, const GLParams& gl, cudaStream_t st) {
    size_t smem = fill_smem_bytes(D, IMAGE, gl.nq, A.basis.max_tile_seg, A.basis.max_tile_basis);
    auto kern = fill_kernel<D, IMAGE, EK>;
    MW_CHECK_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const int nbz = A.nbatch > 0 ? A.nbatch : 1;
    const int64_t nt = A.basis.n_tile;
    dim3 grid((unsigned)(nt * (nt + 1) / 2), 1, nbz);
    double nb = A.basis.n_basis;
    // flops of the upper-triangle tile pairs (the mirrored blocks are
    // written, not recomputed, when every segment has one radius)
    const double tri = (double)(nt + 1) / (2.0 * (double)nt);
    ProfileScope ps(IMAGE ? PC_FILL_IMAGE : PC_FILL, st, tri * nbz * fill_flops(D, gl.nq, A.seg.n_seg, nb),
                    nbz * nb * nb * (16.0 + (A.Z32 ? 8.0 : 0.0)) * (IMAGE ? 2.0 : 1.0));
    kern<<<grid, 256, smem, st>>>(A, gl);
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

}  // namespace mw

using namespace mw;

static mw_status check_common(const mw_basis* b, int n_qp) {
    MW_REQUIRE(b != nullptr, "basis is NULL");
    MW_REQUIRE(b->degree == 1 || b->degree == 2, "degree must be 1 or 2 (got %d)", b->degree);
    MW_REQUIRE(n_qp >= 1 && n_qp <= 8, "n_qp_pair must be in [1, 8] (got %d)", n_qp);
    MW_REQUIRE(b->max_tile_basis >= 1 && b->max_tile_basis <= MW_MAX_TILE_BASIS,
               "max_tile_basis out of range (%d)", b->max_tile_basis);
    MW_REQUIRE(b->max_tile_seg >= 1 && b->max_tile_seg <= MW_MAX_TILE_SEG, "max_tile_seg out of range (%d)",
               b->max_tile_seg);
    MW_REQUIRE(b->n_tile >= 1, "no basis tiles");
    return MW_OK;
}

extern "C" mw_status mw_same_edge_table(const mw_edges* edges, int32_t degree, int32_t n_qp,
                                        int32_t extended_kernel, double k, double* out, void* stream) {
    MW_REQUIRE(edges && out, "NULL argument");
    MW_REQUIRE(degree == 1 || degree == 2, "degree must be 1 or 2 (got %d)", degree);
    MW_REQUIRE(n_qp >= 1 && n_qp <= 8, "n_qp_pair must be in [1, 8] (got %d)", n_qp);
    if (edges->table_rows == 0) return MW_OK;
    GLParams gl = make_gl(n_qp);
    const int threads = kTableThreads, rows_per_block = kTableThreads / 32;
    int64_t blocks = (edges->table_rows + rows_per_block - 1) / rows_per_block;
    cudaStream_t st = as_stream(stream);
    ProfileScope ps(PC_TABLE, st);
#define MW_TBL(DD, EE)                                                                                 \
    same_edge_table_kernel<DD, EE><<<(unsigned)blocks, threads, 0, st>>>(                                \
        edges->n_edge, edges->n_in_edge, edges->table_off, edges->h, edges->radius, edges->table_rows, k, \
        gl, out, nullptr, 0)
    if (degree == 1) { if (extended_kernel) MW_TBL(1, true); else MW_TBL(1, false); }
    else             { if (extended_kernel) MW_TBL(2, true); else MW_TBL(2, false); }
#undef MW_TBL
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

extern "C" mw_status mw_offedge_moments(const mw_segments* seg_i, const mw_segments* seg_j, int32_t degree,
                                        int32_t n_qp, double k, int32_t mirror, double ground_z,
                                        const int32_t* groups_i, const int32_t* groups_j, double* out,
                                        void* stream) {
    MW_REQUIRE(seg_i && seg_j && out, "NULL argument");
    MW_REQUIRE(degree == 1 || degree == 2, "degree must be 1 or 2 (got %d)", degree);
    MW_REQUIRE(n_qp >= 1 && n_qp <= 8, "n_qp_pair must be in [1, 8] (got %d)", n_qp);
    int64_t npair = (int64_t)seg_i->n_seg * seg_j->n_seg;
    if (npair == 0) return MW_OK;
    GLParams gl = make_gl(n_qp);
    int threads = 256;
    int64_t blocks = (npair * 4 + threads - 1) / threads;
    cudaStream_t st = as_stream(stream);
    if (degree == 1)
        offedge_moments_kernel<1><<<(unsigned)blocks, threads, 0, st>>>(*seg_i, *seg_j, k, mirror, ground_z,
                                                                        groups_i, groups_j, gl, out);
    else
        offedge_moments_kernel<2><<<(unsigned)blocks, threads, 0, st>>>(*seg_i, *seg_j, k, mirror, ground_z,
                                                                        groups_i, groups_j, gl, out);
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

extern "C" mw_status mw_fill_z(const mw_segments* seg, const mw_basis* basis, const double* table,
                               const mw_edges* edges, const mw_freq* freq, int32_t n_qp, double* Z, int64_t ldz,
                               float* Z32, int64_t ldz32, void* stream) {
    MW_REQUIRE(seg && basis && table && edges && freq && Z, "NULL argument");
    mw_status s = check_common(basis, n_qp);
    if (s != MW_OK) return s;
    MW_REQUIRE(ldz >= basis->n_basis, "ldz < n_basis");
    MW_REQUIRE(Z32 == nullptr || ldz32 >= basis->n_basis, "ldz32 < n_basis");
    FillArgs A{};
    A.seg = *seg;
    A.basis = *basis;
    A.table = table;
    A.e_n = edges->n_in_edge;
    A.e_off = edges->table_off;
    A.k = freq->k;
    A.omega = freq->omega;
    A.eps0 = freq->eps0;
    A.mu0 = freq->mu0;
    A.Z = Z;
    A.ldz = ldz;
    A.Z32 = Z32;
    A.ldz32 = ldz32;
    GLParams gl = make_gl(n_qp);
    cudaStream_t st = as_stream(stream);
    bool ek = seg->ek_group != nullptr;
    if (basis->degree == 1) return ek ? launch_fill<1, false, true>(A, gl, st) : launch_fill<1, false, false>(A, gl, st);
    return ek ? launch_fill<2, false, true>(A, gl, st) : launch_fill<2, false, false>(A, gl, st);
}

extern "C" mw_status mw_fill_z_image(const mw_segments* seg, const mw_basis* basis, const mw_ground* ground,
                                     const mw_freq* freq, int32_t n_qp, double* Z, int64_t ldz, float* Z32,
                                     int64_t ldz32, void* stream) {
    MW_REQUIRE(seg && basis && ground && freq && Z, "NULL argument");
    mw_status s = check_common(basis, n_qp);
    if (s != MW_OK) return s;
    MW_REQUIRE(ground->model >= MW_GROUND_PEC && ground->model <= MW_GROUND_SOMM_IMAGE,
               "ground model %d has no image term", ground->model);
    MW_REQUIRE(ldz >= basis->n_basis, "ldz < n_basis");
    bool ek = seg->ek_group != nullptr;
    MW_REQUIRE(!ek || seg->ek_group_img != nullptr, "EK image fill needs ek_group_img labels");
    FillArgs A{};
    A.seg = *seg;
    A.basis = *basis;
    A.ground = *ground;
    A.k = freq->k;
    A.omega = freq->omega;
    A.eps0 = freq->eps0;
    A.mu0 = freq->mu0;
    A.Z = Z;
    A.ldz = ldz;
    A.Z32 = Z32;
    A.ldz32 = ldz32;
    GLParams gl = make_gl(n_qp);
    cudaStream_t st = as_stream(stream);
    if (basis->degree == 1) return ek ? launch_fill<1, true, true>(A, gl, st) : launch_fill<1, true, false>(A, gl, st);
    return ek ? launch_fill<2, true, true>(A, gl, st) : launch_fill<2, true, false>(A, gl, st);
}

extern "C" mw_status mw_fill_z_batch(const mw_segments* seg, const mw_basis* basis, const mw_edges* edges,
                                     int32_t n_k, const double* k_dev, const double* omega_dev, double eps0,
                                     double mu0, int32_t n_qp, int32_t extended_kernel, double ground_z,
                                     int32_t pec_ground, double* table, double* Z, int64_t ldz, int64_t z_stride,
                                     float* Z32, int64_t ldz32, int64_t z32_stride, void* stream) {
    MW_REQUIRE(seg && basis && edges && k_dev && omega_dev && table && Z, "NULL argument");
    MW_REQUIRE(n_k >= 1 && n_k <= 65535, "n_k out of range (%d)", n_k);
    mw_status s = check_common(basis, n_qp);
    if (s != MW_OK) return s;
    MW_REQUIRE(ldz >= basis->n_basis && z_stride >= ldz * basis->n_basis, "bad Z layout");
    MW_REQUIRE(Z32 == nullptr || (ldz32 >= basis->n_basis && z32_stride >= ldz32 * basis->n_basis), "bad Z32 layout");
    const int d = basis->degree;
    const int64_t tstride = edges->table_rows * (d + 1) * (d + 1) * 2;
    GLParams gl = make_gl(n_qp);
    cudaStream_t st = as_stream(stream);
    if (edges->table_rows > 0) {
        ProfileScope ps(PC_TABLE, st);
        const int threads = kTableThreads, rows_per_block = kTableThreads / 32;
        const unsigned bx = (unsigned)((edges->table_rows + rows_per_block - 1) / rows_per_block);
        const bool ek = extended_kernel != 0;
        // the k-independent static part once into every table, then the
        // smooth part per k
#define MW_TBL_B(DD, EE, GRID, MODE)                                                                            \
    same_edge_table_kernel<DD, EE><<<GRID, threads, 0, st>>>(edges->n_edge, edges->n_in_edge, edges->table_off, \
                                                             edges->h, edges->radius, edges->table_rows, 0.0, gl,   \
                                                             table, k_dev, tstride, MODE, n_k)
        for (int mode : {(int)kTableStatic, (int)kTableSmoothAdd}) {
            dim3 grid(bx, mode == kTableStatic ? 1u : (unsigned)n_k);
            if (d == 1) { if (ek) MW_TBL_B(1, true, grid, mode); else MW_TBL_B(1, false, grid, mode); }
            else        { if (ek) MW_TBL_B(2, true, grid, mode); else MW_TBL_B(2, false, grid, mode); }
            MW_CHECK_CUDA(cudaGetLastError());
            count_launch();
        }
#undef MW_TBL_B
    }
    FillArgs A{};
    A.seg = *seg;
    A.basis = *basis;
    A.table = table;
    A.e_n = edges->n_in_edge;
    A.e_off = edges->table_off;
    A.eps0 = eps0;
    A.mu0 = mu0;
    A.Z = Z;
    A.ldz = ldz;
    A.Z32 = Z32;
    A.ldz32 = ldz32;
    A.kb = k_dev;
    A.omegab = omega_dev;
    A.table_stride = tstride;
    A.z_stride = z_stride;
    A.z32_stride = z32_stride;
    A.nbatch = n_k;
    const bool ek = seg->ek_group != nullptr;
    s = (d == 1) ? (ek ? launch_fill<1, false, true>(A, gl, st) : launch_fill<1, false, false>(A, gl, st))
                 : (ek ? launch_fill<2, false, true>(A, gl, st) : launch_fill<2, false, false>(A, gl, st));
    if (s != MW_OK || !pec_ground) return s;
    MW_REQUIRE(!ek || seg->ek_group_img != nullptr, "EK image fill needs ek_group_img labels");
    A.ground.model = MW_GROUND_PEC;
    A.ground.ground_z = ground_z;
    return (d == 1) ? (ek ? launch_fill<1, true, true>(A, gl, st) : launch_fill<1, true, false>(A, gl, st))
                    : (ek ? launch_fill<2, true, true>(A, gl, st) : launch_fill<2, true, false>(A, gl, st));
}
