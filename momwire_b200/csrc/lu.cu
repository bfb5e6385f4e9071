// Dense complex128 LU with partial pivoting and triangular solves (sm_100a).
//
// Replaces LAPACK zgetrf/zgetrs reached through scipy.linalg.solve in
// momwire (bspline.py:2971-2989).  Right-looking blocked algorithm:
//   panel   : one cooperative kernel per NB-column panel; the rows are split
//             over all SMs, one bounded grid barrier per column; pivot
//             candidates and their rows travel through double-buffered
//             slots so a column costs exactly one barrier;
//   laswp   : row interchanges outside the panel;
//   trsm    : U12 = L11^-1 A12 with L11 staged in shared memory;
//   gemm    : A22 -= L21 U12, register-tiled complex FP64 (4 DFMA per
//             complex multiply-add), the bulk of the (8/3) n^3 flops.
// Pivot choice follows LAPACK's izamax: max |re| + |im|, first index wins.
#include <cstdio>

#include "common.cuh"

namespace mw {

constexpr int kNB = 64;          // panel width
constexpr int kPanelThreads = 256;

struct PanelWs {
    unsigned int counter;  // grid barrier arrivals
    int err;               // device status (MW_ERR_TIMEOUT)
    int pad[2];
};

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Bounded grid barrier; returns false (for every thread of the CTA) when
// the wait gave up, after recording MW_ERR_TIMEOUT.
__device__ bool grid_sync_bounded(PanelWs* ws, unsigned int target) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(&ws->counter, 1u);
        int ok = 1;
        long long spins = 0;
        while (ld_acquire(&ws->counter) < target) {
            if (ws->err) { ok = 0; break; }
            if (++spins > (1ll << 24)) {
                atomicExch(&ws->err, MW_ERR_TIMEOUT);
                ok = 0;
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

__device__ __forceinline__ double cabs1(cd z) { return fabs(z.re) + fabs(z.im); }

struct PanelArgs {
    cd* A;
    int64_t lda;
    int64_t n;
    int64_t j0;
    int jb;
    int rcap;  // slab leading dimension (rows per CTA)
    int32_t* ipiv;
    int32_t* info;
    PanelWs* ws;
    // slot buffers, double buffered: [2][G] values, [2][G] indices,
    // [2][G][jb] candidate rows, [2][jb] current row
    double* slot_val;
    int64_t* slot_idx;
    cd* slot_row;
    cd* cur_row;
};

// Block-wide argmax of (value, row): larger value wins, smaller row on ties.
__device__ __forceinline__ void argmax_merge(double& v, int64_t& i, double v2, int64_t i2) {
    if (v2 > v || (v2 == v && i2 < i)) {
        v = v2;
        i = i2;
    }
}

__device__ void block_argmax(double& v, int64_t& i, double* s_v, int64_t* s_i) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        double v2 = __shfl_xor_sync(0xffffffffu, v, off);
        int64_t i2 = __shfl_xor_sync(0xffffffffu, i, off);
        argmax_merge(v, i, v2, i2);
    }
    if (lane == 0) {
        s_v[warp] = v;
        s_i[warp] = i;
    }
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        v = lane < nw ? s_v[lane] : -1.0;
        i = lane < nw ? s_i[lane] : INT64_MAX;
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            double v2 = __shfl_xor_sync(0xffffffffu, v, off);
            int64_t i2 = __shfl_xor_sync(0xffffffffu, i, off);
            argmax_merge(v, i, v2, i2);
        }
        if (lane == 0) {
            s_v[0] = v;
            s_i[0] = i;
        }
    }
    __syncthreads();
    v = s_v[0];
    i = s_i[0];
    __syncthreads();
}

// Panel factorisation of rows [j0, n) x columns [j0, j0+jb).  Each CTA keeps
// its contiguous row slab of the panel in shared memory for the whole panel
// (column-major, leading dimension rcap) and writes it back at the end.
__global__ void __launch_bounds__(kPanelThreads) panel_kernel(PanelArgs P) {
    extern __shared__ cd slab[];
    __shared__ double s_v[kPanelThreads / 32];
    __shared__ int64_t s_i[kPanelThreads / 32];
    __shared__ cd s_piv[kNB];
    __shared__ cd s_cur[kNB];
    __shared__ int64_t s_p;
    __shared__ double s_pv;
    __shared__ int s_bg;

    const int G = gridDim.x;
    const int g = blockIdx.x;
    const int tid = threadIdx.x;
    const int64_t m = P.n - P.j0;
    const int64_t per = (m + G - 1) / G;
    const int64_t r0 = P.j0 + g * per;
    const int64_t r1 = min(P.n, r0 + per);
    const int R = (int)max((int64_t)0, r1 - r0);
    const int rcap = P.rcap;
    const int jb = P.jb;
    cd* A = P.A;
    const int64_t lda = P.lda;

    for (int idx = tid; idx < R * jb; idx += blockDim.x) {
        int i = idx % R, x = idx / R;
        slab[x * rcap + i] = A[(r0 + i) + (P.j0 + x) * lda];
    }
    __syncthreads();

    for (int jj = 0; jj < jb; ++jj) {
        const int64_t c = P.j0 + jj;
        const int buf = jj & 1;
        const int i0 = (int)max((int64_t)0, c - r0);  // first local row >= c
        // 1. local argmax of |re| + |im| in column c
        double best = -1.0;
        int64_t bidx = INT64_MAX;
        for (int i = i0 + tid; i < R; i += blockDim.x) argmax_merge(best, bidx, cabs1(slab[jj * rcap + i]), r0 + i);
        block_argmax(best, bidx, s_v, s_i);
        // 2. publish the candidate and (owner of row c) the current row c
        if (tid == 0) {
            P.slot_val[buf * G + g] = best;
            P.slot_idx[buf * G + g] = bidx;
        }
        if (bidx != INT64_MAX)
            for (int x = tid; x < jb; x += blockDim.x)
                P.slot_row[((size_t)buf * G + g) * kNB + x] = slab[x * rcap + (int)(bidx - r0)];
        if (c >= r0 && c < r1)
            for (int x = tid; x < jb; x += blockDim.x) P.cur_row[buf * kNB + x] = slab[x * rcap + (int)(c - r0)];
        // 3. one barrier per column
        if (!grid_sync_bounded(P.ws, (unsigned)(jj + 1) * G)) return;
        // 4. global pivot from the G candidates (warp 0)
        if (tid < 32) {
            double bv = -1.0;
            int64_t bi = INT64_MAX;
            int bg = 0;
            for (int x = tid; x < G; x += 32) {
                double v = __ldcg(&P.slot_val[buf * G + x]);
                int64_t i = (int64_t)__ldcg(reinterpret_cast<const long long*>(&P.slot_idx[buf * G + x]));
                if (i == INT64_MAX) continue;
                if (v > bv || (v == bv && i < bi)) { bv = v; bi = i; bg = x; }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                double v2 = __shfl_xor_sync(0xffffffffu, bv, off);
                int64_t i2 = __shfl_xor_sync(0xffffffffu, bi, off);
                int g2 = __shfl_xor_sync(0xffffffffu, bg, off);
                if (v2 > bv || (v2 == bv && i2 < bi)) { bv = v2; bi = i2; bg = g2; }
            }
            if (tid == 0) {
                s_p = bi;
                s_pv = bv;
                s_bg = bg;
                if (g == 0) P.ipiv[c] = (int32_t)(bi + 1);
            }
        }
        __syncthreads();
        const int64_t p = s_p;
        const int bg = s_bg;
        for (int x = tid; x < jb; x += blockDim.x) {
            // L2-coherent loads: these slots were written by other CTAs
            double2 a = __ldcg(reinterpret_cast<const double2*>(P.slot_row) + ((size_t)buf * G + bg) * kNB + x);
            double2 b = __ldcg(reinterpret_cast<const double2*>(P.cur_row) + buf * kNB + x);
            s_piv[x] = cd{a.x, a.y};
            s_cur[x] = cd{b.x, b.y};
        }
        __syncthreads();
        // 5. swap rows c <-> p inside the slab
        if (p != c) {
            if (c >= r0 && c < r1)
                for (int x = tid; x < jb; x += blockDim.x) slab[x * rcap + (int)(c - r0)] = s_piv[x];
            if (p >= r0 && p < r1)
                for (int x = tid; x < jb; x += blockDim.x) slab[x * rcap + (int)(p - r0)] = s_cur[x];
        }
        __syncthreads();
        // 6. scale below the pivot, then rank-1 update of the panel
        if (s_pv == 0.0) {
            if (g == 0 && tid == 0 && P.info[0] == 0) P.info[0] = (int32_t)(c + 1);
            continue;  // LAPACK: no scaling, no update for an exact zero pivot
        }
        const int is = (int)max((int64_t)0, c + 1 - r0);
        const int nr = R - is;
        if (nr > 0) {
            const cd inv = cdiv(cd{1.0, 0.0}, s_piv[jj]);
            for (int i = is + tid; i < R; i += blockDim.x) slab[jj * rcap + i] = slab[jj * rcap + i] * inv;
            __syncthreads();
            const int ncol = jb - jj - 1;
            for (int idx = tid; idx < nr * ncol; idx += blockDim.x) {
                int i = is + idx % nr, x = jj + 1 + idx / nr;
                slab[x * rcap + i] = slab[x * rcap + i] - slab[jj * rcap + i] * s_piv[x];
            }
        }
        __syncthreads();
    }
    for (int idx = tid; idx < R * jb; idx += blockDim.x) {
        int i = idx % R, x = idx / R;
        A[(r0 + i) + (P.j0 + x) * lda] = slab[x * rcap + i];
    }
}

__global__ void laswp_kernel(cd* A, int64_t lda, int64_t col0, int64_t ncols, const int32_t* ipiv, int64_t k1,
                             int64_t k2) {
    int64_t col = col0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (col >= col0 + ncols) return;
    cd* a = A + col * lda;
    for (int64_t i = k1; i < k2; ++i) {
        int64_t p = ipiv[i] - 1;
        if (p != i) {
            cd t = a[i];
            a[i] = a[p];
            a[p] = t;
        }
    }
}

// X (jb x ncols, leading dim ldx) <- L^-1 X with L unit lower (jb x jb),
// or U^-1 X with U upper non-unit.  32 columns per CTA.
template <bool UPPER>
__global__ void __launch_bounds__(256) trsm_kernel(const cd* T, int64_t ldt, cd* X, int64_t ldx, int jb,
                                                   int64_t ncols) {
    extern __shared__ cd trsm_smem[];
    cd(*sT)[kNB + 1] = reinterpret_cast<cd(*)[kNB + 1]>(trsm_smem);
    cd(*sX)[33] = reinterpret_cast<cd(*)[33]>(trsm_smem + kNB * (kNB + 1));
    const int tid = threadIdx.x;
    const int64_t c0 = blockIdx.x * 32;
    const int nc = (int)((ncols - c0) < 32 ? (ncols - c0) : 32);
    for (int i = tid; i < jb * jb; i += blockDim.x) {
        int r = i % jb, cc = i / jb;
        sT[r][cc] = T[r + cc * ldt];
    }
    for (int i = tid; i < jb * nc; i += blockDim.x) {
        int r = i % jb, cc = i / jb;
        sX[r][cc] = X[r + (c0 + cc) * ldx];
    }
    __syncthreads();
    if (!UPPER) {
        for (int k = 0; k < jb; ++k) {
            for (int i = tid; i < (jb - k - 1) * nc; i += blockDim.x) {
                int r = k + 1 + i % (jb - k - 1), cc = i / (jb - k - 1);
                sX[r][cc] = sX[r][cc] - sT[r][k] * sX[k][cc];
            }
            __syncthreads();
        }
    } else {
        for (int k = jb - 1; k >= 0; --k) {
            if (tid < nc) sX[k][tid] = cdiv(sX[k][tid], sT[k][k]);
            __syncthreads();
            for (int i = tid; i < k * nc; i += blockDim.x) {
                int r = i % k, cc = i / k;
                sX[r][cc] = sX[r][cc] - sT[r][k] * sX[k][cc];
            }
            __syncthreads();
        }
    }
    for (int i = tid; i < jb * nc; i += blockDim.x) {
        int r = i % jb, cc = i / jb;
        X[r + (c0 + cc) * ldx] = sX[r][cc];
    }
}

// C = alpha op(A) op(B) + beta C, complex128, column-major.
// 128 x 64 output tile per CTA, 256 threads, 8 x 4 complex per thread,
// K staged through shared memory 8 at a time.
constexpr int GM = 128, GN = 64, GK = 8;

template <bool TA, bool TB>
__global__ void __launch_bounds__(256) zgemm_kernel(int64_t m, int64_t n, int64_t k, cd alpha, const cd* __restrict__ A,
                                                    int64_t lda, const cd* __restrict__ B, int64_t ldb, cd beta,
                                                    cd* __restrict__ C, int64_t ldc) {
    __shared__ cd sA[GK][GM + 1];
    __shared__ cd sB[GK][GN + 1];
    const int tid = threadIdx.x;
    const int64_t m0 = blockIdx.x * (int64_t)GM, n0 = blockIdx.y * (int64_t)GN;
    const int tx = tid % 16, ty = tid / 16;  // rows tx + 16*i, cols ty + 16*j
    cd acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = cd{0.0, 0.0};

    for (int64_t k0 = 0; k0 < k; k0 += GK) {
        // stage A tile (GM x GK) and B tile (GK x GN)
        for (int i = tid; i < GM * GK; i += 256) {
            int r = TA ? i / GK : i % GM;
            int kk = TA ? i % GK : i / GM;
            int64_t gr = m0 + r, gk = k0 + kk;
            cd v{0.0, 0.0};
            if (gr < m && gk < k) v = TA ? A[gk + gr * lda] : A[gr + gk * lda];
            sA[kk][r] = v;
        }
        for (int i = tid; i < GK * GN; i += 256) {
            int kk = TB ? i / GN : i % GK;
            int cc = TB ? i % GN : i / GK;
            int64_t gk = k0 + kk, gc = n0 + cc;
            cd v{0.0, 0.0};
            if (gk < k && gc < n) v = TB ? B[gc + gk * ldb] : B[gk + gc * ldb];
            sB[kk][cc] = v;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < GK; ++kk) {
            cd a[8], b[4];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = sA[kk][tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = sB[kk][ty + 16 * j];
#pragma unroll
            for (int i = 0; i < 8; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    acc[i][j].re = fma(a[i].re, b[j].re, acc[i][j].re);
                    acc[i][j].re = fma(-a[i].im, b[j].im, acc[i][j].re);
                    acc[i][j].im = fma(a[i].re, b[j].im, acc[i][j].im);
                    acc[i][j].im = fma(a[i].im, b[j].re, acc[i][j].im);
                }
        }
        __syncthreads();
    }
    const bool beta_zero = (beta.re == 0.0 && beta.im == 0.0);
#pragma unroll
    for (int j = 0; j < 4; ++j) {
        int64_t gc = n0 + ty + 16 * j;
        if (gc >= n) continue;
#pragma unroll
        for (int i = 0; i < 8; ++i) {
            int64_t gr = m0 + tx + 16 * i;
            if (gr >= m) continue;
            cd v = alpha * acc[i][j];
            cd* cp = C + gr + gc * ldc;
            if (!beta_zero) v = v + beta * (*cp);
            *cp = v;
        }
    }
}

constexpr size_t kTrsmSmem = sizeof(cd) * (kNB * (kNB + 1) + kNB * 33);

static mw_status trsm_setup() {
    static bool done = false;
    if (!done) {
        MW_CHECK_CUDA(cudaFuncSetAttribute(trsm_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsmSmem));
        MW_CHECK_CUDA(cudaFuncSetAttribute(trsm_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsmSmem));
        done = true;
    }
    return MW_OK;
}

mw_status zgemm_launch(bool ta, bool tb, int64_t m, int64_t n, int64_t k, cd alpha, const cd* A, int64_t lda,
                       const cd* B, int64_t ldb, cd beta, cd* C, int64_t ldc, cudaStream_t st) {
    if (m <= 0 || n <= 0) return MW_OK;
    dim3 grid((unsigned)((m + GM - 1) / GM), (unsigned)((n + GN - 1) / GN));
    ProfileScope ps(PC_ZGEMM, st, 8.0 * (double)m * n * k, 16.0 * ((double)m * k + (double)k * n + 2.0 * m * n));
    if (!ta && !tb) zgemm_kernel<false, false><<<grid, 256, 0, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else if (ta && !tb) zgemm_kernel<true, false><<<grid, 256, 0, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else if (!ta && tb) zgemm_kernel<false, true><<<grid, 256, 0, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else zgemm_kernel<true, true><<<grid, 256, 0, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

constexpr size_t kPanelSmemMax = 200 * 1024;  // slab bytes per CTA

static int panel_sms() {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(panel_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelSmemMax);
        if (sms < 1) sms = 1;
    }
    return sms;
}

static size_t ws_layout(int G, size_t* off_val, size_t* off_idx, size_t* off_row, size_t* off_cur);

// Factor the panel rows [j0, n) x columns [j0, j0+jb) with partial pivoting.
// One cooperative launch when every CTA's row slab fits in shared memory;
// otherwise split the columns in two and recurse (left half, then update and
// factor the right half, then apply the right half's swaps to the left).
static mw_status panel_factor(cd* A, int64_t lda, int64_t n, int64_t j0, int jb, int32_t* ipiv, int32_t* info,
                              char* ws, cudaStream_t st) {
    const int sms = panel_sms();
    const int64_t m = n - j0;
    int64_t want = (m + 31) / 32;  // at least 32 rows per CTA
    int G = (int)(want < sms ? want : sms);
    if (G < 1) G = 1;
    const int64_t per = (m + G - 1) / G;
    const size_t smem = (size_t)per * jb * sizeof(cd);
    if (smem > kPanelSmemMax) {
        MW_REQUIRE(jb > 1, "matrix too large for the panel kernel (%lld rows per CTA)", (long long)per);
        const int h = jb / 2;
        mw_status s = panel_factor(A, lda, n, j0, h, ipiv, info, ws, st);
        if (s != MW_OK) return s;
        laswp_kernel<<<(unsigned)((jb - h + 127) / 128), 128, 0, st>>>(A, lda, j0 + h, jb - h, ipiv, j0, j0 + h);
        trsm_kernel<false><<<(unsigned)((jb - h + 31) / 32), 256, kTrsmSmem, st>>>(
            A + j0 + j0 * lda, lda, A + j0 + (j0 + h) * lda, lda, h, jb - h);
        count_launch(2);
        s = zgemm_launch(false, false, m - h, jb - h, h, cd{-1.0, 0.0}, A + (j0 + h) + j0 * lda, lda,
                         A + j0 + (j0 + h) * lda, lda, cd{1.0, 0.0}, A + (j0 + h) + (j0 + h) * lda, lda, st);
        if (s != MW_OK) return s;
        s = panel_factor(A, lda, n, j0 + h, jb - h, ipiv, info, ws, st);
        if (s != MW_OK) return s;
        laswp_kernel<<<(unsigned)((h + 127) / 128), 128, 0, st>>>(A, lda, j0, h, ipiv, j0 + h, j0 + jb);
        count_launch();
        MW_CHECK_CUDA(cudaGetLastError());
        return MW_OK;
    }
    size_t ov, oi, orow, ocur;
    ws_layout(G, &ov, &oi, &orow, &ocur);
    PanelWs* pws = reinterpret_cast<PanelWs*>(ws);
    // reset the barrier counter only; the error word stays sticky
    MW_CHECK_CUDA(cudaMemsetAsync(&pws->counter, 0, sizeof(unsigned int), st));
    PanelArgs P;
    P.A = A;
    P.lda = lda;
    P.n = n;
    P.j0 = j0;
    P.jb = jb;
    P.rcap = (int)per;
    P.ipiv = ipiv;
    P.info = info;
    P.ws = pws;
    P.slot_val = reinterpret_cast<double*>(ws + ov);
    P.slot_idx = reinterpret_cast<int64_t*>(ws + oi);
    P.slot_row = reinterpret_cast<cd*>(ws + orow);
    P.cur_row = reinterpret_cast<cd*>(ws + ocur);
    void* args[] = {&P};
    {
        ProfileScope ps(PC_PANEL, st, 4.0 * (double)m * jb * jb, 32.0 * (double)m * jb);
        MW_CHECK_CUDA(cudaLaunchCooperativeKernel((void*)panel_kernel, dim3(G), dim3(kPanelThreads), args, smem, st));
    }
    count_launch();
    return MW_OK;
}

static size_t ws_layout(int G, size_t* off_val, size_t* off_idx, size_t* off_row, size_t* off_cur) {
    size_t o = 256;  // PanelWs + padding
    *off_val = o;
    o += sizeof(double) * 2 * G;
    o = (o + 255) & ~size_t(255);
    *off_idx = o;
    o += sizeof(int64_t) * 2 * G;
    o = (o + 255) & ~size_t(255);
    *off_row = o;
    o += sizeof(cd) * 2 * (size_t)G * kNB;
    o = (o + 255) & ~size_t(255);
    *off_cur = o;
    o += sizeof(cd) * 2 * kNB;
    return (o + 255) & ~size_t(255);
}

}  // namespace mw

using namespace mw;

extern "C" size_t mw_getrf_workspace_size(int64_t n) {
    size_t a, b, c, d;
    (void)n;
    return ws_layout(1024, &a, &b, &c, &d);  // enough for any grid up to 1024 CTAs
}

extern "C" mw_status mw_zgetrf(int64_t n, double* Ad, int64_t lda, int32_t* ipiv, int32_t* info, void* workspace,
                               size_t workspace_bytes, const volatile int32_t* cancel, void* stream) {
    MW_REQUIRE(n >= 0 && lda >= (n > 0 ? n : 1), "bad n/lda");
    MW_REQUIRE(Ad && ipiv && info && workspace, "NULL argument");
    MW_REQUIRE(workspace_bytes >= mw_getrf_workspace_size(n), "workspace too small");
    cudaStream_t st = as_stream(stream);
    cd* A = reinterpret_cast<cd*>(Ad);
    char* ws = reinterpret_cast<char*>(workspace);
    MW_CHECK_CUDA(cudaMemsetAsync(info, 0, 2 * sizeof(int32_t), st));
    MW_CHECK_CUDA(cudaMemsetAsync(ws, 0, sizeof(PanelWs), st));
    { mw_status s0 = trsm_setup(); if (s0 != MW_OK) return s0; }
    PanelWs* pws = reinterpret_cast<PanelWs*>(ws);
    for (int64_t j0 = 0; j0 < n; j0 += kNB) {
        if (cancel && *cancel) {
            set_error("factorisation cancelled");
            return MW_ERR_CANCELLED;
        }
        int jb = (int)((n - j0) < kNB ? (n - j0) : kNB);
        {
            mw_status s = panel_factor(A, lda, n, j0, jb, ipiv, info, ws, st);
            if (s != MW_OK) return s;
        }
        int64_t left = j0, right = n - j0 - jb;
        if (left > 0) {
            ProfileScope ps(PC_LASWP, st, 0.0, 64.0 * (double)jb * left);
            laswp_kernel<<<(unsigned)((left + 127) / 128), 128, 0, st>>>(A, lda, 0, left, ipiv, j0, j0 + jb);
            count_launch();
        }
        if (right > 0) {
            {
                ProfileScope ps(PC_LASWP, st, 0.0, 64.0 * (double)jb * right);
                laswp_kernel<<<(unsigned)((right + 127) / 128), 128, 0, st>>>(A, lda, j0 + jb, right, ipiv, j0,
                                                                             j0 + jb);
            }
            cd* A11 = A + j0 + j0 * lda;
            cd* A12 = A + j0 + (j0 + jb) * lda;
            {
                ProfileScope ps(PC_TRSM, st, 4.0 * (double)jb * jb * right, 32.0 * (double)jb * right);
                trsm_kernel<false><<<(unsigned)((right + 31) / 32), 256, kTrsmSmem, st>>>(A11, lda, A12, lda, jb,
                                                                                         right);
            }
            count_launch(2);  // laswp + trsm
            cd* A21 = A + (j0 + jb) + j0 * lda;
            cd* A22 = A + (j0 + jb) + (j0 + jb) * lda;
            mw_status s = zgemm_launch(false, false, right, right, jb, cd{-1.0, 0.0}, A21, lda, A12, lda,
                                       cd{1.0, 0.0}, A22, lda, st);
            if (s != MW_OK) return s;
        }
        MW_CHECK_CUDA(cudaGetLastError());
    }
    // a barrier timeout anywhere is reported in info[1]
    MW_CHECK_CUDA(cudaMemcpyAsync(info + 1, &pws->err, sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    return MW_OK;
}

extern "C" mw_status mw_zgetrs(int64_t n, int64_t nrhs, const double* LUd, int64_t lda, const int32_t* ipiv,
                               double* Bd, int64_t ldb, void* stream) {
    MW_REQUIRE(n >= 0 && nrhs >= 0 && lda >= (n > 0 ? n : 1) && ldb >= (n > 0 ? n : 1), "bad sizes");
    MW_REQUIRE(LUd && ipiv && Bd, "NULL argument");
    if (n == 0 || nrhs == 0) return MW_OK;
    cudaStream_t st = as_stream(stream);
    const cd* LU = reinterpret_cast<const cd*>(LUd);
    cd* B = reinterpret_cast<cd*>(Bd);
    {
        mw_status s0 = trsm_setup();
        if (s0 != MW_OK) return s0;
    }
    laswp_kernel<<<(unsigned)((nrhs + 127) / 128), 128, 0, st>>>(B, ldb, 0, nrhs, ipiv, 0, n);
    count_launch();
    unsigned cb = (unsigned)((nrhs + 31) / 32);
    for (int64_t j0 = 0; j0 < n; j0 += kNB) {
        int jb = (int)((n - j0) < kNB ? (n - j0) : kNB);
        trsm_kernel<false><<<cb, 256, kTrsmSmem, st>>>(LU + j0 + j0 * lda, lda, B + j0, ldb, jb, nrhs);
        count_launch();
        int64_t rest = n - j0 - jb;
        if (rest > 0) {
            mw_status s = zgemm_launch(false, false, rest, nrhs, jb, cd{-1.0, 0.0}, LU + (j0 + jb) + j0 * lda, lda,
                                       B + j0, ldb, cd{1.0, 0.0}, B + j0 + jb, ldb, st);
            if (s != MW_OK) return s;
        }
    }
    int64_t last = ((n - 1) / kNB) * kNB;
    for (int64_t j0 = last; j0 >= 0; j0 -= kNB) {
        int jb = (int)((n - j0) < kNB ? (n - j0) : kNB);
        trsm_kernel<true><<<cb, 256, kTrsmSmem, st>>>(LU + j0 + j0 * lda, lda, B + j0, ldb, jb, nrhs);
        count_launch();
        if (j0 > 0) {
            mw_status s = zgemm_launch(false, false, j0, nrhs, jb, cd{-1.0, 0.0}, LU + j0 * lda, lda, B + j0, ldb,
                                       cd{1.0, 0.0}, B, ldb, st);
            if (s != MW_OK) return s;
        }
    }
    MW_CHECK_CUDA(cudaGetLastError());
    return MW_OK;
}

extern "C" mw_status mw_zgemm(int32_t transA, int32_t transB, int64_t m, int64_t n, int64_t k, double alpha_re,
                              double alpha_im, const double* A, int64_t lda, const double* B, int64_t ldb,
                              double beta_re, double beta_im, double* C, int64_t ldc, void* stream) {
    MW_REQUIRE(m >= 0 && n >= 0 && k >= 0, "negative size");
    MW_REQUIRE(A && B && C, "NULL argument");
    return zgemm_launch(transA != 0, transB != 0, m, n, k, cd{alpha_re, alpha_im}, reinterpret_cast<const cd*>(A),
                        lda, reinterpret_cast<const cd*>(B), ldb, cd{beta_re, beta_im}, reinterpret_cast<cd*>(C),
                        ldc, as_stream(stream));
}
