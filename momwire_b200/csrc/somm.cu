// Sommerfeld ground on the GPU (sm_100a): the remainder-surface grid fill,
// the interpolated + projected remainder field and its Galerkin block Q.
//
// Reference path (ground_model="sommerfeld"):
//   grid fill     SommerfeldGrid -> iv_surfaces_direct -> six integrals
//                 (_sommerfeld.py:648-813, :535-584; C++
//                 somm_six_integrals_batch _accelerators.cpp:5792)
//   field         remainder_field_proj / proj_one (_sommerfeld.py:940-1035,
//                 _accelerators.cpp:5906-5963)
//   Galerkin Q    _Z_sommerfeld_remainder (bspline.py:1791-1915) -> C++
//                 sommerfeld_remainder_bspline_Q (_accelerators.cpp:6081-6253)
//
// Grid fill: one warp per node, the 24 Gauss nodes of every contour segment
// spread over lanes 0..23 (warp-uniform control flow, each lane holding the
// same bisection stack), nodes handed out through an atomic counter because
// their cost varies by orders of magnitude (grazing Hankel-form rows).
//
// Q: one CTA per (row tile, column tile) of the fill's basis tiling.  Phase A
// forms the per-segment-pair moments Jc[p][P] = sum_qr W_p(q) F(q, r) W_P(r)
// over n_qp x n_qp Gauss nodes in shared memory (one thread per pair);
// phase B contracts them with the basis polynomials and subtracts Q from the
// Z tile (and refreshes its complex64 copy).  The grid tables are read
// through the read-only cache: a node's four surfaces are one 64-byte line.
#include <vector>

#include "common.cuh"
#include "somm_math.cuh"
#include "somm_proj.cuh"

namespace mw {

using somm::GL24;

// -------------------------------------------------------------- grid fill
struct WarpRule {
    somm::SixParams P;
    double xl, wl;  // this lane's Gauss node and weight (lanes >= 24: 0)
    __device__ void operator()(cd z0, cd z1, cd out[6]) const {
        const cd mid = somm::cscale(z0 + z1, 0.5), half = somm::cscale(z1 - z0, 0.5);
        double v[12];
#pragma unroll
        for (int i = 0; i < 12; ++i) v[i] = 0.0;
        if (wl != 0.0) {
            cd f[6];
            somm::integrand6(P, mid + somm::cscale(half, xl), f);
#pragma unroll
            for (int i = 0; i < 6; ++i) {
                v[2 * i] = f[i].re * wl;
                v[2 * i + 1] = f[i].im * wl;
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
#pragma unroll
            for (int i = 0; i < 12; ++i) v[i] += __shfl_xor_sync(0xffffffffu, v[i], off);
#pragma unroll
        for (int i = 0; i < 6; ++i) out[i] = cd{v[2 * i], v[2 * i + 1]} * half;
    }
};

struct SurfArgs {
    int64_t n;
    const double *r1, *rho, *h, *theta;
    const double *eps_re, *eps_im;  // per-node eps~, or NULL: eps_t for all
    cd eps_t;
    double k2, omega, mu, rtol;
    double2* out;  // (n, 4) complex
    unsigned long long* next;
};

__global__ void __launch_bounds__(128) somm_surfaces_kernel(SurfArgs A, GL24 gl) {
    const int lane = threadIdx.x & 31;
    WarpRule rule;
    rule.xl = lane < somm::kGaussN ? gl.x[lane] : 0.0;
    rule.wl = lane < somm::kGaussN ? gl.w[lane] : 0.0;
    for (;;) {
        unsigned long long node = 0;
        if (lane == 0) node = atomicAdd(A.next, 1ull);
        node = __shfl_sync(0xffffffffu, node, 0);
        if (node >= (unsigned long long)A.n) break;
        cd s[4];
        const cd et = A.eps_re ? cd{A.eps_re[node], A.eps_im[node]} : A.eps_t;
        somm::surfaces(rule, et, A.k2, A.omega, A.mu, A.r1[node], A.rho[node], A.h[node], A.theta[node], A.rtol, s);
        if (lane < 4) A.out[node * 4 + lane] = make_double2(s[lane].re, s[lane].im);
    }
}

static GL24 make_gl24() {
    GL24 g{};
    const double *t, *w;
    gauss_legendre01(somm::kGaussN, &t, &w);
    for (int i = 0; i < somm::kGaussN; ++i) {
        g.x[i] = 2.0 * t[i] - 1.0;
        g.w[i] = 2.0 * w[i];
    }
    return g;
}

__global__ void field_proj_kernel(GridDev G, double gz, double k, int64_t n_obs, const double* __restrict__ obs,
                                  const double* __restrict__ t_obs, int64_t n_src, const double* __restrict__ src,
                                  const double* __restrict__ t_src, double2* __restrict__ out) {
    const int64_t total = n_obs * n_src;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t m = q / n_src, n = q - m * n_src;
        const SrcTangent ts = split_tangent(t_src[3 * n], t_src[3 * n + 1], t_src[3 * n + 2]);
        const cd v = proj_one(G, gz, k, obs[3 * m], obs[3 * m + 1], obs[3 * m + 2], t_obs[3 * m], t_obs[3 * m + 1],
                              t_obs[3 * m + 2], src[3 * n], src[3 * n + 1], src[3 * n + 2], ts);
        out[q] = make_double2(v.re, v.im);
    }
}

// --------------------------------------------------------------- Galerkin Q
constexpr int kQMaxNq = 8;

struct QArgs {
    mw_segments seg;
    mw_basis basis;
    GridDev G;
    double gz, k;
    int nq;
    double tq[kQMaxNq], wq[kQMaxNq];  // nodes / weights on [0, 1]
    double* Z;
    int64_t ldz;
    float* Z32;
    int64_t ldz32;
};

// per staged segment: nq nodes (3 each), W[p][q] ((d+1) x nq), tangent (3),
// source tangent split (4)
__host__ __device__ constexpr int q_seg_stride(int NM, int nq) { return nq * 3 + NM * nq + 7; }

template <int D>
static size_t q_smem_bytes(int nq, int smax, int tb) {
    constexpr int NM = D + 1, NMM = NM * NM;
    return sizeof(double) * ((size_t)2 * smax * q_seg_stride(NM, nq) + (size_t)smax * smax * NMM * 2 + 2 * tb * NMM) +
           sizeof(int) * (2 * tb * NM);
}

template <int D>
__device__ __forceinline__ void q_stage(double* dst, const QArgs& A, int s) {
    constexpr int NM = D + 1;
    const int nq = A.nq;
    const double* l = A.seg.seg_l + 3 * s;
    const double* r = A.seg.seg_r + 3 * s;
    const double dx = r[0] - l[0], dy = r[1] - l[1], dz = r[2] - l[2];
    const double L = sqrt(dx * dx + dy * dy + dz * dz);
    for (int q = 0; q < nq; ++q) {
        const double t = A.tq[q];
        dst[3 * q + 0] = l[0] + t * dx;
        dst[3 * q + 1] = l[1] + t * dy;
        dst[3 * q + 2] = l[2] + t * dz;
        const double u = L * t;
        double wp = L * A.wq[q];
        for (int p = 0; p < NM; ++p) {
            dst[nq * 3 + p * nq + q] = wp;
            wp *= u;
        }
    }
    const double* tg = A.seg.tangent + 3 * s;
    double* o = dst + nq * 3 + NM * nq;
    o[0] = tg[0];
    o[1] = tg[1];
    o[2] = tg[2];
    const SrcTangent ts = split_tangent(tg[0], tg[1], tg[2]);
    o[3] = ts.ux;
    o[4] = ts.uy;
    o[5] = ts.th;
    o[6] = ts.tz;
}

template <int D>
__global__ void __launch_bounds__(256) somm_q_kernel(QArgs A) {
    constexpr int NM = D + 1, NMM = NM * NM;
    extern __shared__ double qsm[];
    const int nq = A.nq;
    const int SD = q_seg_stride(NM, nq);
    const int SMAX = A.basis.max_tile_seg, TB = A.basis.max_tile_basis;
    const int tr = blockIdx.y, tc = blockIdx.x;
    const int ns_r = A.basis.tile_ns[tr], ns_c = A.basis.tile_ns[tc];
    const int nb_r = A.basis.tile_nb[tr], nb_c = A.basis.tile_nb[tc];
    const int fb_r = A.basis.tile_first[tr], fb_c = A.basis.tile_first[tc];
    double* s_row = qsm;
    double* s_col = s_row + SMAX * SD;
    double* s_J = s_col + SMAX * SD;                   // SMAX*SMAX*NMM complex
    double* s_pr = s_J + (size_t)SMAX * SMAX * NMM * 2;
    double* s_pc = s_pr + TB * NMM;
    int* s_loc_r = reinterpret_cast<int*>(s_pc + TB * NMM);
    int* s_loc_c = s_loc_r + TB * NM;
    const int tid = threadIdx.x;
    for (int i = tid; i < ns_r; i += blockDim.x) q_stage<D>(s_row + i * SD, A, A.basis.tile_seg[(size_t)tr * SMAX + i]);
    for (int i = tid; i < ns_c; i += blockDim.x) q_stage<D>(s_col + i * SD, A, A.basis.tile_seg[(size_t)tc * SMAX + i]);
    for (int i = tid; i < nb_r * NMM; i += blockDim.x) s_pr[i] = A.basis.polys[(size_t)fb_r * NMM + i];
    for (int i = tid; i < nb_c * NMM; i += blockDim.x) s_pc[i] = A.basis.polys[(size_t)fb_c * NMM + i];
    for (int i = tid; i < nb_r * NM; i += blockDim.x) s_loc_r[i] = A.basis.loc[(size_t)fb_r * NM + i];
    for (int i = tid; i < nb_c * NM; i += blockDim.x) s_loc_c[i] = A.basis.loc[(size_t)fb_c * NM + i];
    __syncthreads();

    // phase A: Jc of every staged segment pair
    for (int pidx = tid; pidx < ns_r * ns_c; pidx += blockDim.x) {
        const int li = pidx / ns_c, lj = pidx - li * ns_c;
        const double* so = s_row + li * SD;
        const double* ss = s_col + lj * SD;
        const double* to = so + nq * 3 + NM * nq;
        const double* tsv = ss + nq * 3 + NM * nq;
        const SrcTangent ts{tsv[3], tsv[4], tsv[5], tsv[6]};
        cd J[NM][NM];
#pragma unroll
        for (int p = 0; p < NM; ++p)
#pragma unroll
            for (int P = 0; P < NM; ++P) J[p][P] = cd{0.0, 0.0};
        for (int q = 0; q < nq; ++q) {
            cd row[NM];
#pragma unroll
            for (int P = 0; P < NM; ++P) row[P] = cd{0.0, 0.0};
            for (int r = 0; r < nq; ++r) {
                const cd F = proj_one(A.G, A.gz, A.k, so[3 * q], so[3 * q + 1], so[3 * q + 2], to[0], to[1], to[2],
                                      ss[3 * r], ss[3 * r + 1], ss[3 * r + 2], ts);
#pragma unroll
                for (int P = 0; P < NM; ++P) {
                    const double w = ss[nq * 3 + P * nq + r];
                    row[P].re += F.re * w;
                    row[P].im += F.im * w;
                }
            }
#pragma unroll
            for (int p = 0; p < NM; ++p) {
                const double w = so[nq * 3 + p * nq + q];
#pragma unroll
                for (int P = 0; P < NM; ++P) {
                    J[p][P].re += w * row[P].re;
                    J[p][P].im += w * row[P].im;
                }
            }
        }
        double* dst = s_J + (size_t)pidx * NMM * 2;
#pragma unroll
        for (int p = 0; p < NM; ++p)
#pragma unroll
            for (int P = 0; P < NM; ++P) {
                dst[(p * NM + P) * 2] = J[p][P].re;
                dst[(p * NM + P) * 2 + 1] = J[p][P].im;
            }
    }
    __syncthreads();

    // phase B: Q = sum_ab C_m J C_n; Z -= Q
    for (int pp = tid; pp < TB * TB; pp += blockDim.x) {
        const int mi = pp % TB, ni = pp / TB;
        if (mi >= nb_r || ni >= nb_c) continue;
        cd Q{0.0, 0.0};
        const double* Cm = s_pr + mi * NMM;
        const double* Cn = s_pc + ni * NMM;
        for (int a = 0; a < NM; ++a) {
            const int la = s_loc_r[mi * NM + a];
            if (la < 0) continue;
            for (int b = 0; b < NM; ++b) {
                const int lb = s_loc_c[ni * NM + b];
                if (lb < 0) continue;
                const double* J = s_J + ((size_t)la * ns_c + lb) * NMM * 2;
#pragma unroll
                for (int p = 0; p < NM; ++p) {
                    cd rowv{0.0, 0.0};
#pragma unroll
                    for (int P = 0; P < NM; ++P) {
                        const double c = Cn[b * NM + P];
                        rowv.re += c * J[(p * NM + P) * 2];
                        rowv.im += c * J[(p * NM + P) * 2 + 1];
                    }
                    const double cm = Cm[a * NM + p];
                    Q.re += cm * rowv.re;
                    Q.im += cm * rowv.im;
                }
            }
        }
        const int64_t m = fb_r + mi, n = fb_c + ni;
        double* zp = A.Z + 2 * (m + n * A.ldz);
        const double zr = zp[0] - Q.re, zi = zp[1] - Q.im;
        zp[0] = zr;
        zp[1] = zi;
        if (A.Z32) {
            float* z32 = A.Z32 + 2 * (m + n * A.ldz32);
            z32[0] = (float)zr;
            z32[1] = (float)zi;
        }
    }
}

// ------------------------------------------------------ image-point extent
// max over endpoint pairs of |obs - image(src)|; products and sums rounded
// one by one (no fused multiply-add) so the value matches a plain host
// evaluation bit for bit.
__global__ void max_image_distance_kernel(int n_seg, const double* __restrict__ seg_l,
                                          const double* __restrict__ seg_r, double gz, unsigned long long* out) {
    const int64_t n = 2 * (int64_t)n_seg;
    const int64_t total = n * n;
    double best = 0.0;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = q / n, j = q - i * n;
        const double* a = i < n_seg ? seg_l + 3 * i : seg_r + 3 * (i - n_seg);
        const double* b = j < n_seg ? seg_l + 3 * j : seg_r + 3 * (j - n_seg);
        const double dx = __dsub_rn(a[0], b[0]), dy = __dsub_rn(a[1], b[1]);
        const double hz = __dadd_rn(__dsub_rn(a[2], gz), __dsub_rn(b[2], gz));
        const double s = __dadd_rn(__dadd_rn(__dmul_rn(dx, dx), __dmul_rn(dy, dy)), __dmul_rn(hz, hz));
        best = fmax(best, __dsqrt_rn(s));
    }
    for (int off = 16; off > 0; off >>= 1) best = fmax(best, __shfl_xor_sync(0xffffffffu, best, off));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(best));
}

static GridDev grid_dev(const mw_somm_grid* g) {
    GridDev G{};
    G.n_region = g->n_region;
    for (int r = 0; r < 6; ++r) {
        const int rr = r < g->n_region ? r : g->n_region - 1;
        G.n_r[r] = g->n_r[rr];
        G.n_th[r] = g->n_th[rr];
        G.off[r] = g->offset[rr];
        G.r0[r] = g->r0[rr];
        G.dr[r] = g->dr[rr];
        G.th0[r] = g->th0[rr];
        G.dth[r] = g->dth[rr];
    }
    G.r1_max = g->r1_max;
    G.r_break = g->r_break;
    G.th_split = g->th_split;
    // four-region grids route every clamped query near
    G.r_near = g->n_region == 6 ? g->r_near : g->r1_max;
    G.tiny = 1e-12 * g->r1_max;
    G.vscale = g->value_scale;
    G.vals = reinterpret_cast<const double2*>(g->vals);
    return G;
}

static mw_status check_grid(const mw_somm_grid* g) {
    MW_REQUIRE(g != nullptr && g->vals != nullptr, "grid is NULL");
    MW_REQUIRE(g->n_region == 4 || g->n_region == 6, "grid must have 4 or 6 regions (got %d)", g->n_region);
    for (int r = 0; r < g->n_region; ++r)
        MW_REQUIRE(g->n_r[r] >= 4 && g->n_th[r] >= 4 && g->dr[r] > 0.0 && g->dth[r] > 0.0 && g->offset[r] >= 0,
                   "grid region %d malformed", r);
    MW_REQUIRE(g->r1_max > 0.0, "grid r1_max must be positive");
    return MW_OK;
}

}  // namespace mw

using namespace mw;

extern "C" size_t mw_somm_surfaces_workspace_size(void) { return 256; }

static mw_status launch_surfaces(int64_t n_nodes, const double* r1, const double* rho, const double* h,
                                 const double* theta, const double* eps_re_v, const double* eps_im_v, double eps_re,
                                 double eps_im, double k2, double omega, double mu, double rtol, double* out,
                                 void* workspace, void* stream) {
    MW_REQUIRE(n_nodes >= 0, "n_nodes must be >= 0");
    if (n_nodes == 0) return MW_OK;
    MW_REQUIRE(r1 && rho && h && theta && out && workspace, "NULL argument");
    MW_REQUIRE(k2 > 0.0 && rtol > 0.0, "k2 and rtol must be positive");
    cudaStream_t st = as_stream(stream);
    SurfArgs A{n_nodes, r1, rho, h, theta, eps_re_v, eps_im_v, cd{eps_re, eps_im}, k2, omega, mu, rtol,
               reinterpret_cast<double2*>(out), reinterpret_cast<unsigned long long*>(workspace)};
    MW_CHECK_CUDA(cudaMemsetAsync(workspace, 0, sizeof(unsigned long long), st));
    int dev = 0, sms = 148;
    MW_CHECK_CUDA(cudaGetDevice(&dev));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t warps = n_nodes < (int64_t)sms * 16 ? n_nodes : (int64_t)sms * 16;
    {
        ProfileScope ps(PC_SOMM_GRID, st);
        somm_surfaces_kernel<<<(unsigned)((warps + 3) / 4), 128, 0, st>>>(A, make_gl24());
    }
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

extern "C" mw_status mw_somm_surfaces(int64_t n_nodes, const double* r1, const double* rho, const double* h,
                                      const double* theta, double eps_re, double eps_im, double k2, double omega,
                                      double mu, double rtol, double* out, void* workspace, void* stream) {
    return launch_surfaces(n_nodes, r1, rho, h, theta, nullptr, nullptr, eps_re, eps_im, k2, omega, mu, rtol, out,
                           workspace, stream);
}

extern "C" mw_status mw_somm_surfaces_eps(int64_t n_nodes, const double* r1, const double* rho, const double* h,
                                          const double* theta, const double* eps_re, const double* eps_im, double k2,
                                          double omega, double mu, double rtol, double* out, void* workspace,
                                          void* stream) {
    MW_REQUIRE(eps_re && eps_im, "NULL eps arrays");
    return launch_surfaces(n_nodes, r1, rho, h, theta, eps_re, eps_im, 0.0, 0.0, k2, omega, mu, rtol, out, workspace,
                           stream);
}

extern "C" mw_status mw_somm_field_proj(int64_t n_obs, const double* obs, const double* t_obs, int64_t n_src,
                                        const double* src, const double* t_src, double ground_z, double k,
                                        const mw_somm_grid* grid, double* out, void* stream) {
    MW_REQUIRE(n_obs >= 0 && n_src >= 0, "sizes must be >= 0");
    if (n_obs == 0 || n_src == 0) return MW_OK;
    MW_REQUIRE(obs && t_obs && src && t_src && out, "NULL argument");
    mw_status s = check_grid(grid);
    if (s != MW_OK) return s;
    cudaStream_t st = as_stream(stream);
    const int64_t total = n_obs * n_src;
    const unsigned blocks = (unsigned)((total + 255) / 256 < 148 * 32 ? (total + 255) / 256 : 148 * 32);
    field_proj_kernel<<<blocks, 256, 0, st>>>(grid_dev(grid), ground_z, k, n_obs, obs, t_obs, n_src, src, t_src,
                                               reinterpret_cast<double2*>(out));
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

extern "C" mw_status mw_somm_remainder_q(const mw_segments* seg, const mw_basis* basis, const mw_somm_grid* grid,
                                         int32_t n_qp, double ground_z, double k, double* Z, int64_t ldz, float* Z32,
                                         int64_t ldz32, void* stream) {
    MW_REQUIRE(seg && basis && Z, "NULL argument");
    MW_REQUIRE(basis->degree == 1 || basis->degree == 2, "degree must be 1 or 2");
    MW_REQUIRE(n_qp >= 1 && n_qp <= kQMaxNq, "n_qp_sommerfeld must be in [1, %d] (got %d)", kQMaxNq, n_qp);
    MW_REQUIRE(basis->max_tile_seg >= 1 && basis->max_tile_seg <= MW_MAX_TILE_SEG &&
                   basis->max_tile_basis >= 1 && basis->max_tile_basis <= MW_MAX_TILE_BASIS && basis->n_tile >= 1,
               "bad basis tiling");
    MW_REQUIRE(ldz >= basis->n_basis && (Z32 == nullptr || ldz32 >= basis->n_basis), "leading dimension too small");
    mw_status s = check_grid(grid);
    if (s != MW_OK) return s;
    cudaStream_t st = as_stream(stream);
    QArgs A{};
    A.seg = *seg;
    A.basis = *basis;
    A.G = grid_dev(grid);
    A.gz = ground_z;
    A.k = k;
    A.nq = n_qp;
    const double *t, *w;
    gauss_legendre01(n_qp, &t, &w);
    for (int i = 0; i < n_qp; ++i) {
        A.tq[i] = t[i];
        A.wq[i] = w[i];
    }
    A.Z = Z;
    A.ldz = ldz;
    A.Z32 = Z32;
    A.ldz32 = ldz32;
    const int d = basis->degree;
    const size_t smem = d == 1 ? q_smem_bytes<1>(n_qp, basis->max_tile_seg, basis->max_tile_basis)
                               : q_smem_bytes<2>(n_qp, basis->max_tile_seg, basis->max_tile_basis);
    dim3 grid2(basis->n_tile, basis->n_tile);
    const double nn = (double)seg->n_seg * n_qp;
    ProfileScope ps(PC_SOMM_Q, st, nn * nn * 420.0, 16.0 * 2.0 * basis->n_basis * basis->n_basis);
    if (d == 1) {
        MW_CHECK_CUDA(cudaFuncSetAttribute(somm_q_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        somm_q_kernel<1><<<grid2, 256, smem, st>>>(A);
    } else {
        MW_CHECK_CUDA(cudaFuncSetAttribute(somm_q_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        somm_q_kernel<2><<<grid2, 256, smem, st>>>(A);
    }
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

extern "C" mw_status mw_max_image_distance(int32_t n_seg, const double* seg_l, const double* seg_r, double ground_z,
                                           double* out, void* stream) {
    MW_REQUIRE(n_seg >= 1 && seg_l && seg_r && out, "bad arguments");
    cudaStream_t st = as_stream(stream);
    MW_CHECK_CUDA(cudaMemsetAsync(out, 0, sizeof(double), st));
    const int64_t total = 4 * (int64_t)n_seg * n_seg;
    const unsigned blocks = (unsigned)((total + 255) / 256 < 148 * 8 ? (total + 255) / 256 : 148 * 8);
    max_image_distance_kernel<<<blocks, 256, 0, st>>>(n_seg, seg_l, seg_r, ground_z,
                                                      reinterpret_cast<unsigned long long*>(out));
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}
