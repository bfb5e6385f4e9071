// Singular basis enrichment blocks (FP64), sm_100a.
//
// The reference enriches every wire end of a junction of at least
// enrichment_min_k ends with one extra basis on the adjacent segment,
// Phi(u) = u log u (u the normalised distance from the junction) minus, for
// the "stable" variant, a polynomial that keeps both end values zero
// (bspline.py:3048-3693, C++ assemble_Z_enrich at _accelerators.cpp:2997).
// The augmented system is [[Z, Z_pe], [Z_ep, Z_ee]].  Each block entry is a
// Galerkin double sum over n_qp x n_qp Gauss nodes of the reduced kernel
// exp(-jkR) / (4 pi R), R = sqrt(|x - y|^2 + a^2):
//   Z = j w mu w_A sum (wv_x G wv_y) + w_Phi sum (wd_x G wd_y) / (j w eps)
// with wv / wd the node weight times the basis value / arc derivative, and
// w_A / w_Phi the tangent dot and 1 in free space.  A ground subtracts the
// same sums against mirrored sources with its image weights (PEC, Fresnel
// reflection coefficients, the Sommerfeld ground's C2 image).
//
// Design: one warp per (polynomial basis, enrichment basis) pair and one per
// (enrichment, enrichment) pair; lane j owns source node j (its position
// and shape values computed once), loops over the observer nodes of each
// wing, and the warp reduces.  The kernel is symmetric (and the mirror an
// isometry, the image weights symmetric in the pair), so one sum gives both
// Z_pe[m, e] and Z_ep[e, m].  Writes the blocks into the augmented matrix
// (column-major, leading dimension ldz; the polynomial block is the fill's)
// and, when given, their complex64 copy.
#include "common.cuh"
#include "ground_weights.cuh"

namespace mw {

constexpr int kEnrWarps = 8;
constexpr int kEnrMaxD = 3;

struct EnrichArgs {
    const double* seg_l;
    const double* seg_r;
    const double* tan;
    const int32_t* supp;
    const double* polys;
    int d1;  // degree + 1
    int n_poly;
    const int32_t* e_seg;
    const int32_t* e_origin;
    int n_e;
    const double* t01;
    const double* w01;
    int nq;
    double proj[kEnrMaxD + 1];  // subtracted polynomial in u (zeros: raw shape)
    double a2, k, omega, eps0, mu0;
    mw_ground ground;
    int has_ground;
    double* Z;
    int64_t ldz;
    float* Z32;
    int64_t ld32;
};

__device__ __forceinline__ void seg_point(const EnrichArgs& A, int s, double t, double* x) {
#pragma unroll
    for (int c = 0; c < 3; ++c) x[c] = A.seg_l[3 * s + c] + t * (A.seg_r[3 * s + c] - A.seg_l[3 * s + c]);
}

__device__ __forceinline__ double seg_len(const EnrichArgs& A, int s) {
    const double dx = A.seg_r[3 * s] - A.seg_l[3 * s];
    const double dy = A.seg_r[3 * s + 1] - A.seg_l[3 * s + 1];
    const double dz = A.seg_r[3 * s + 2] - A.seg_l[3 * s + 2];
    return sqrt(dx * dx + dy * dy + dz * dz);
}

// Weight * shape value and weight * arc derivative of enrichment basis e at
// node q: u = t (junction at the segment's left end) or 1 - t.
__device__ __forceinline__ void enrich_node(const EnrichArgs& A, int e, int q, double* y, double* wv, double* wd) {
    const int s = A.e_seg[e];
    const double h = seg_len(A, s);
    const double t = A.t01[q];
    const bool left = A.e_origin[e] == 0;
    const double u = left ? t : 1.0 - t;
    const double lu = log(fmax(u, 1e-300));
    double p = 0.0, dp = 0.0;
    for (int i = A.d1 - 1; i >= 0; --i) p = p * u + A.proj[i];
    for (int i = A.d1 - 1; i >= 1; --i) dp = dp * u + i * A.proj[i];
    const double wq = A.w01[q] * h;
    *wv = wq * (u * lu - p);
    *wd = wq * (left ? 1.0 : -1.0) * (lu + 1.0 - dp) / h;
    seg_point(A, s, t, y);
}

__device__ __forceinline__ cd green(const double* x, const double* y, double a2, double k) {
    const double dx = x[0] - y[0], dy = x[1] - y[1], dz = x[2] - y[2];
    const double R = sqrt(dx * dx + dy * dy + dz * dz + a2);
    double sn, cs;
    sincos(k * R, &sn, &cs);
    const double g = 1.0 / (4.0 * kPi * R);
    return cd{cs * g, -sn * g};
}

__device__ __forceinline__ void warp_sum4(cd& a, cd& b) {
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        a.re += __shfl_xor_sync(0xffffffffu, a.re, off);
        a.im += __shfl_xor_sync(0xffffffffu, a.im, off);
        b.re += __shfl_xor_sync(0xffffffffu, b.re, off);
        b.im += __shfl_xor_sync(0xffffffffu, b.im, off);
    }
}

// (w_A, w_Phi) of an observer segment so / source segment ss for the pass:
// free space (image = false) or the ground's image.
__device__ __forceinline__ void pass_weights(const EnrichArgs& A, int so, int ss, bool image, cd* wA, cd* wP) {
    const double* to = A.tan + 3 * so;
    const double* ts = A.tan + 3 * ss;
    if (!image) {
        *wA = cd{to[0] * ts[0] + to[1] * ts[1] + to[2] * ts[2], 0.0};
        *wP = cd{1.0, 0.0};
        return;
    }
    const double tdi = to[0] * ts[0] + to[1] * ts[1] - to[2] * ts[2];  // against the mirrored tangent
    const mw_ground& g = A.ground;
    if (g.model == MW_GROUND_PEC) {
        *wA = cd{tdi, 0.0};
        *wP = cd{1.0, 0.0};
    } else if (g.model == MW_GROUND_SOMM_IMAGE) {
        const cd c2 = cdiv(cd{g.eps_re - 1.0, g.eps_im}, cd{g.eps_re + 1.0, g.eps_im});
        *wA = tdi * c2;
        *wP = c2;
    } else {
        double co[3], cm[3], tm[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            co[c] = 0.5 * (A.seg_l[3 * so + c] + A.seg_r[3 * so + c]);
            cm[c] = 0.5 * (A.seg_l[3 * ss + c] + A.seg_r[3 * ss + c]);
            tm[c] = ts[c];
        }
        cm[2] = 2.0 * g.ground_z - cm[2];
        tm[2] = -tm[2];
        refl_weights(co, to, cm, tm, g, wA, wP);
    }
}

__device__ __forceinline__ cd mix(const EnrichArgs& A, cd wA, cd IA, cd wP, cd IP) {
    // j w mu wA IA + wP IP / (j w eps)
    const cd a = wA * IA, p = wP * IP;
    const double om_mu = A.omega * A.mu0, inv_om_eps = 1.0 / (A.omega * A.eps0);
    return cd{-om_mu * a.im + inv_om_eps * p.im, om_mu * a.re - inv_om_eps * p.re};
}

__device__ __forceinline__ void store(const EnrichArgs& A, int64_t row, int64_t col, cd v) {
    A.Z[2 * (row + col * A.ldz)] = v.re;
    A.Z[2 * (row + col * A.ldz) + 1] = v.im;
    if (A.Z32 != nullptr) {
        A.Z32[2 * (row + col * A.ld32)] = (float)v.re;
        A.Z32[2 * (row + col * A.ld32) + 1] = (float)v.im;
    }
}

__global__ void __launch_bounds__(32 * kEnrWarps) enrich_pe_kernel(EnrichArgs A) {
    const int lane = threadIdx.x & 31;
    const int64_t task = (int64_t)blockIdx.x * kEnrWarps + (threadIdx.x >> 5);
    if (task >= (int64_t)A.n_poly * A.n_e) return;
    const int m = (int)(task / A.n_e), e = (int)(task % A.n_e);
    const int se = A.e_seg[e];
    cd Z{0.0, 0.0};
    for (int a = 0; a < A.d1; ++a) {
        const int sm = A.supp[m * A.d1 + a];
        if (sm < 0) continue;
        const double* c = A.polys + (int64_t)(m * A.d1 + a) * A.d1;
        bool live = false;
        for (int p = 0; p < A.d1; ++p) live = live || c[p] != 0.0;
        if (!live) continue;
        const double hm = seg_len(A, sm);
        for (int pass = 0; pass < 1 + A.has_ground; ++pass) {
            const bool image = pass == 1;
            cd IA{0.0, 0.0}, IP{0.0, 0.0};
            for (int j = lane; j < A.nq; j += 32) {
                double y[3], wv, wd;
                enrich_node(A, e, j, y, &wv, &wd);
                if (image) y[2] = 2.0 * A.ground.ground_z - y[2];
                cd SA{0.0, 0.0}, SP{0.0, 0.0};
                for (int i = 0; i < A.nq; ++i) {
                    double x[3];
                    const double t = A.t01[i];
                    seg_point(A, sm, t, x);
                    const double u = t * hm;
                    double pv = 0.0, dv = 0.0;
                    for (int p = A.d1 - 1; p >= 0; --p) pv = pv * u + c[p];
                    for (int p = A.d1 - 1; p >= 1; --p) dv = dv * u + p * c[p];
                    const double wq = A.w01[i] * hm;
                    const cd G = green(x, y, A.a2, A.k);
                    SA = SA + (wq * pv) * G;
                    SP = SP + (wq * dv) * G;
                }
                IA = IA + wv * SA;
                IP = IP + wd * SP;
            }
            warp_sum4(IA, IP);
            cd wA, wP;
            pass_weights(A, sm, se, image, &wA, &wP);
            const cd z = mix(A, wA, IA, wP, IP);
            Z = image ? Z - z : Z + z;
        }
    }
    if (lane == 0) {
        store(A, m, (int64_t)A.n_poly + e, Z);  // Z_pe[m, e]
        store(A, (int64_t)A.n_poly + e, m, Z);  // Z_ep[e, m]
    }
}

__global__ void __launch_bounds__(32 * kEnrWarps) enrich_ee_kernel(EnrichArgs A) {
    const int lane = threadIdx.x & 31;
    const int task = blockIdx.x * kEnrWarps + (threadIdx.x >> 5);
    if (task >= A.n_e * A.n_e) return;
    const int e = task / A.n_e, f = task % A.n_e;
    cd Z{0.0, 0.0};
    for (int pass = 0; pass < 1 + A.has_ground; ++pass) {
        const bool image = pass == 1;
        cd IA{0.0, 0.0}, IP{0.0, 0.0};
        for (int j = lane; j < A.nq; j += 32) {
            double y[3], wv, wd;
            enrich_node(A, f, j, y, &wv, &wd);
            if (image) y[2] = 2.0 * A.ground.ground_z - y[2];
            cd SA{0.0, 0.0}, SP{0.0, 0.0};
            for (int i = 0; i < A.nq; ++i) {
                double x[3], xv, xd;
                enrich_node(A, e, i, x, &xv, &xd);
                const cd G = green(x, y, A.a2, A.k);
                SA = SA + xv * G;
                SP = SP + xd * G;
            }
            IA = IA + wv * SA;
            IP = IP + wd * SP;
        }
        warp_sum4(IA, IP);
        cd wA, wP;
        pass_weights(A, A.e_seg[e], A.e_seg[f], image, &wA, &wP);
        const cd z = mix(A, wA, IA, wP, IP);
        Z = image ? Z - z : Z + z;
    }
    if (lane == 0) store(A, (int64_t)A.n_poly + e, (int64_t)A.n_poly + f, Z);
}

}  // namespace mw

using namespace mw;

extern "C" mw_status mw_enrich_blocks(const mw_segments* seg, const mw_basis* basis, const mw_enrich* en,
                                      const mw_freq* fr, const mw_ground* ground, double* Z, int64_t ldz,
                                      float* Z32, int64_t ldz32, void* stream) {
    MW_REQUIRE(seg && basis && en && fr && Z, "NULL argument");
    MW_REQUIRE(basis->degree >= 1 && basis->degree <= kEnrMaxD, "degree %d outside 1..%d", basis->degree, kEnrMaxD);
    MW_REQUIRE(en->n_enrich >= 0 && en->n_qp >= 1, "bad enrichment sizes");
    MW_REQUIRE(ldz >= (int64_t)basis->n_basis + en->n_enrich, "ldz smaller than the augmented order");
    MW_REQUIRE(Z32 == nullptr || ldz32 >= (int64_t)basis->n_basis + en->n_enrich, "ldz32 too small");
    if (en->n_enrich == 0) return MW_OK;
    MW_REQUIRE(en->seg && en->origin && en->t01 && en->w01, "NULL enrichment table");
    EnrichArgs A{};
    A.seg_l = seg->seg_l;
    A.seg_r = seg->seg_r;
    A.tan = seg->tangent;
    A.supp = basis->supp;
    A.polys = basis->polys;
    A.d1 = basis->degree + 1;
    A.n_poly = basis->n_basis;
    A.e_seg = en->seg;
    A.e_origin = en->origin;
    A.n_e = en->n_enrich;
    A.t01 = en->t01;
    A.w01 = en->w01;
    A.nq = en->n_qp;
    for (int i = 0; i <= kEnrMaxD; ++i) A.proj[i] = i < A.d1 ? en->proj[i] : 0.0;
    A.a2 = en->radius * en->radius;
    A.k = fr->k;
    A.omega = fr->omega;
    A.eps0 = fr->eps0;
    A.mu0 = fr->mu0;
    A.has_ground = ground != nullptr && ground->model != MW_GROUND_NONE;
    if (A.has_ground) A.ground = *ground;
    A.Z = Z;
    A.ldz = ldz;
    A.Z32 = Z32;
    A.ld32 = ldz32;
    cudaStream_t st = as_stream(stream);
    {
        ProfileScope ps(PC_FILL, st, 0.0, 0.0);
        const int64_t pe = (int64_t)A.n_poly * A.n_e;
        if (pe > 0) {
            enrich_pe_kernel<<<(unsigned)((pe + kEnrWarps - 1) / kEnrWarps), 32 * kEnrWarps, 0, st>>>(A);
            count_launch();
        }
        const int64_t ee = (int64_t)A.n_e * A.n_e;
        enrich_ee_kernel<<<(unsigned)((ee + kEnrWarps - 1) / kEnrWarps), 32 * kEnrWarps, 0, st>>>(A);
        count_launch();
    }
    MW_CHECK_CUDA(cudaGetLastError());
    return MW_OK;
}
