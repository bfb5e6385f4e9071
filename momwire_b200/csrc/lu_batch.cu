// Batched mixed-precision solves for frequency sweeps (sm_100a).
//
// The swept port solve of the reference (bspline.py:4181-4440:
// _swept_batched_z_chunks + _solve_with_kcl_swept_ports, a stacked
// numpy.linalg.solve over the k axis) factorises one small complex matrix per
// frequency.  Here a whole batch of same-order matrices (one structure at
// many frequencies) is factorised together in complex64:
//   panel   one CTA per matrix, the panel (rows j0..n, 8-32 columns) resident
//           in shared memory; pivot search, swap, scale and rank-1 update
//           synchronise with __syncthreads only;
//   update  the batched tcgen05 3xTF32 update of cgemm_tc.cu over all
//           matrices' tiles in one persistent launch;
// then every matrix is solved and refined in FP64 against its own Z
// (X += LU32 \ (B - Z X)) until the largest relative correction of the whole
// batch is below tol.
#include <cmath>
#include <vector>

#include "common.cuh"

namespace mw {

mw_status cgemm_tc_update_batched(int64_t m, int64_t n, int64_t k, int batch, const cf* A, int64_t lda, int64_t sa,
                                  const cf* B, int64_t ldb, int64_t sb, cf* C, int64_t ldc, int64_t sc, void* ws,
                                  size_t ws_bytes, int* err, cudaStream_t st, int max_ctas);
size_t cgemm_tc_workspace_batched(int64_t m, int64_t n, int64_t k, int batch);

constexpr int kBNB = 16;       // default panel width of the batched factorisation
constexpr int kBNBMax = 32;    // widest panel of the batched factorisation (<= kBOuter)
constexpr int kBOuter = 64;    // block of the batched factorisation: the trailing update's k
constexpr int kBSB = 64;       // block size of the batched triangular solves
constexpr int kBThreads = 256;

__device__ __forceinline__ void amax_merge(double& v, int& i, double v2, int i2) {
    if (v2 > v || (v2 == v && i2 < i)) {
        v = v2;
        i = i2;
    }
}

// One CTA factors the panel rows [j0, n) x columns [j0, j0+jb) of its matrix.
__global__ void __launch_bounds__(kBThreads) panel1_kernel(cf* A, int64_t lda, int64_t stride, int n, int j0, int jb,
                                                           int32_t* ipiv, int32_t* info) {
    extern __shared__ __align__(16) unsigned char p1_smem[];
    cf* slab = reinterpret_cast<cf*>(p1_smem);
    __shared__ double s_v[kBThreads / 32];
    __shared__ int s_i[kBThreads / 32];
    __shared__ int s_p;
    __shared__ double s_pv;
    const int b = blockIdx.x, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    A += (int64_t)b * stride;
    ipiv += (int64_t)b * n;
    const int m = n - j0;
    for (int q = tid; q < m * jb; q += blockDim.x) {
        const int i = q % m, x = q / m;
        slab[x * m + i] = A[(j0 + i) + (int64_t)(j0 + x) * lda];
    }
    __syncthreads();
    for (int jj = 0; jj < jb; ++jj) {
        double best = -1.0;
        int bi = 0x7fffffff;
        for (int i = jj + tid; i < m; i += blockDim.x) amax_merge(best, bi, cabs1(slab[jj * m + i]), i);
#pragma unroll
        for (int off = 16; off > 0; off >>= 1)
            amax_merge(best, bi, __shfl_xor_sync(0xffffffffu, best, off), __shfl_xor_sync(0xffffffffu, bi, off));
        if (lane == 0) {
            s_v[warp] = best;
            s_i[warp] = bi;
        }
        __syncthreads();
        if (warp == 0) {
            best = lane < kBThreads / 32 ? s_v[lane] : -1.0;
            bi = lane < kBThreads / 32 ? s_i[lane] : 0x7fffffff;
#pragma unroll
            for (int off = 16; off > 0; off >>= 1)
                amax_merge(best, bi, __shfl_xor_sync(0xffffffffu, best, off), __shfl_xor_sync(0xffffffffu, bi, off));
            if (lane == 0) {
                s_p = bi;
                s_pv = best;
                ipiv[j0 + jj] = j0 + bi + 1;
            }
        }
        __syncthreads();
        const int p = s_p;
        if (p != jj)
            for (int x = tid; x < jb; x += blockDim.x) {
                const cf t = slab[x * m + jj];
                slab[x * m + jj] = slab[x * m + p];
                slab[x * m + p] = t;
            }
        __syncthreads();
        if (s_pv == 0.0) {
            if (tid == 0 && info[b] == 0) info[b] = j0 + jj + 1;
            continue;
        }
        const cf inv = cdiv(cf{1.f, 0.f}, slab[jj * m + jj]);
        // rows in the threads: scale the multiplier and update its row
        for (int i = jj + 1 + tid; i < m; i += blockDim.x) {
            const cf l = slab[jj * m + i] * inv;
            slab[jj * m + i] = l;
            for (int x = jj + 1; x < jb; ++x) slab[x * m + i] = slab[x * m + i] - l * slab[x * m + jj];
        }
        __syncthreads();
    }
    for (int q = tid; q < m * jb; q += blockDim.x) {
        const int i = q % m, x = q / m;
        A[(j0 + i) + (int64_t)(j0 + x) * lda] = slab[x * m + i];
    }
}

template <class T>
__global__ void laswp_batched_kernel(T* A, int64_t lda, int64_t stride, int col0, int ncols, const int32_t* ipiv,
                                     int n, int k1, int k2) {
    const int col = col0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= col0 + ncols) return;
    T* a = A + (int64_t)blockIdx.y * stride + (int64_t)col * lda;
    const int32_t* pv = ipiv + (int64_t)blockIdx.y * n;
    for (int i = k1; i < k2; ++i) {
        const int p = pv[i] - 1;
        if (p != i) {
            const T t = a[i];
            a[i] = a[p];
            a[p] = t;
        }
    }
}

__device__ __forceinline__ cf shfl_cf(cf v, int src) {
    return cf{__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src)};
}

// X <- L^-1 X (unit lower) or U^-1 X (upper) for the jb x jb diagonal block
// at T (jb <= 64); a warp per column at a time, batch on blockIdx.y.
constexpr int kTrsmColsPerWarp = 8;
template <bool UPPER>
__global__ void __launch_bounds__(256) trsm_batched_kernel(const cf* Tm, int64_t ldt, int64_t ts, cf* X, int64_t ldx,
                                                           int64_t xs, int jb, int ncols) {
    __shared__ cf sT[64][65];
    __shared__ cf sD[64];  // U: reciprocals of the diagonal
    Tm += (int64_t)blockIdx.y * ts;
    X += (int64_t)blockIdx.y * xs;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (UPPER && tid < jb) sD[tid] = cdiv(cf{1.f, 0.f}, Tm[tid + (int64_t)tid * ldt]);
    for (int i = tid; i < jb * jb; i += blockDim.x) {
        const int r = i % jb, c = i / jb;
        sT[r][c] = Tm[r + (int64_t)c * ldt];
    }
    __syncthreads();
    // each warp solves kTrsmColsPerWarp columns in turn (the staged triangle
    // serves 8 x kTrsmColsPerWarp consecutive columns)
    for (int cc = 0; cc < kTrsmColsPerWarp; ++cc) {
        const int col = (blockIdx.x * kTrsmColsPerWarp + cc) * 8 + warp;
        if (col >= ncols) return;  // whole warp leaves together
        cf* x = X + (int64_t)col * ldx;
        cf x0 = lane < jb ? x[lane] : cf{0.f, 0.f};
        cf x1 = lane + 32 < jb ? x[lane + 32] : cf{0.f, 0.f};
        if (!UPPER) {
            for (int k = 0; k < jb; ++k) {
                const cf xk = shfl_cf(k < 32 ? x0 : x1, k & 31);
                if (lane > k && lane < jb) x0 = x0 - sT[lane][k] * xk;
                if (lane + 32 > k && lane + 32 < jb) x1 = x1 - sT[lane + 32][k] * xk;
            }
        } else {
            for (int k = jb - 1; k >= 0; --k) {
                if (k < 32) {
                    if (lane == k) x0 = x0 * sD[k];
                } else if (lane == k - 32) {
                    x1 = x1 * sD[k];
                }
                const cf xk = shfl_cf(k < 32 ? x0 : x1, k & 31);
                if (lane < k) x0 = x0 - sT[lane][k] * xk;
                if (lane + 32 < k) x1 = x1 - sT[lane + 32][k] * xk;
            }
        }
        if (lane < jb) x[lane] = x0;
        if (lane + 32 < jb) x[lane + 32] = x1;
    }
}

static dim3 trsm_batched_grid(int ncols, int batch) {
    return dim3((unsigned)((ncols + 8 * kTrsmColsPerWarp - 1) / (8 * kTrsmColsPerWarp)), (unsigned)batch);
}

// Y (m x nr) -= A (m x k) X (k x nr), complex64, batch on blockIdx.y;
// one thread per row (k <= 64, nr small).
__global__ void gemm_small_batched_kernel(const cf* A, int64_t lda, int64_t as, const cf* X, int64_t ldx, int64_t xs,
                                          cf* Y, int64_t ldy, int64_t ys, int m, int k, int nr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= m) return;
    A += (int64_t)blockIdx.y * as;
    X += (int64_t)blockIdx.y * xs;
    Y += (int64_t)blockIdx.y * ys;
    for (int c = 0; c < nr; ++c) {
        cf acc{0.f, 0.f};
        for (int l = 0; l < k; ++l) acc = acc + A[i + (int64_t)l * lda] * X[l + (int64_t)c * ldx];
        Y[i + (int64_t)c * ldy] = Y[i + (int64_t)c * ldy] - acc;
    }
}

// R = B - Z X  (complex128; B shared across the batch when bs == 0)
__global__ void resid_batched_kernel(const cd* Z, int64_t ldz, int64_t zs, const cd* X, int64_t ldx, int64_t xs,
                                     const cd* B, int64_t ldb, int64_t bs, cd* R, int64_t ldr, int64_t rs, int n,
                                     int nr) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Z += (int64_t)blockIdx.y * zs;
    X += (int64_t)blockIdx.y * xs;
    B += (int64_t)blockIdx.y * bs;
    R += (int64_t)blockIdx.y * rs;
    for (int c = 0; c < nr; ++c) {
        double ar = 0.0, ai = 0.0;
        const cd* x = X + (int64_t)c * ldx;
        for (int j = 0; j < n; ++j) {
            const cd z = Z[i + (int64_t)j * ldz];
            const cd v = x[j];
            ar = fma(z.re, v.re, ar);
            ar = fma(-z.im, v.im, ar);
            ai = fma(z.re, v.im, ai);
            ai = fma(z.im, v.re, ai);
        }
        const cd bb = B[i + (int64_t)c * ldb];
        R[i + (int64_t)c * ldr] = cd{bb.re - ar, bb.im - ai};
    }
}

__global__ void narrow_batched_kernel(const cd* R, cf* R32, int64_t total) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x)
        R32[q] = cf{(float)R[q].re, (float)R[q].im};
}

// X += C; per-matrix max |C| and max |X| (|re| + |im|) into cm / xm.
__global__ void accum_batched_kernel(const cf* C, cd* X, int64_t per, double* cm, double* xm) {
    const int b = blockIdx.y;
    double mc = 0.0, mx = 0.0;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < per; q += (int64_t)gridDim.x * blockDim.x) {
        const cf c = C[b * per + q];
        cd x = X[b * per + q];
        x.re += (double)c.re;
        x.im += (double)c.im;
        X[b * per + q] = x;
        mc = fmax(mc, fabs((double)c.re) + fabs((double)c.im));
        mx = fmax(mx, fabs(x.re) + fabs(x.im));
    }
    for (int off = 16; off > 0; off >>= 1) {
        mc = fmax(mc, __shfl_xor_sync(0xffffffffu, mc, off));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(reinterpret_cast<unsigned long long*>(cm + b), (unsigned long long)__double_as_longlong(mc));
        atomicMax(reinterpret_cast<unsigned long long*>(xm + b), (unsigned long long)__double_as_longlong(mx));
    }
}

static size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

struct BatchWs {
    void* tc;
    size_t tc_bytes;
    int* tc_err;
    cd* R;
    cf* R32;
    double* norms;  // [2][batch]
};

static size_t batch_ws_bytes(int n, int nrhs, int batch) {
    return al256(cgemm_tc_workspace_batched(n, n, kBOuter, batch)) + 256 + al256((size_t)batch * n * nrhs * 16) +
           al256((size_t)batch * n * nrhs * 8) + al256((size_t)batch * 16);
}

static BatchWs batch_ws(void* ws, int n, int nrhs, int batch) {
    char* w = static_cast<char*>(ws);
    BatchWs b;
    b.tc = w;
    b.tc_bytes = cgemm_tc_workspace_batched(n, n, kBOuter, batch);
    w += al256(b.tc_bytes);
    b.tc_err = reinterpret_cast<int*>(w);
    w += 256;
    b.R = reinterpret_cast<cd*>(w);
    w += al256((size_t)batch * n * nrhs * 16);
    b.R32 = reinterpret_cast<cf*>(w);
    w += al256((size_t)batch * n * nrhs * 8);
    b.norms = reinterpret_cast<double*>(w);
    return b;
}

static mw_status cgetrf_batched(int n, int batch, cf* A, int64_t lda, int64_t stride, int32_t* ipiv, int32_t* info,
                                const BatchWs& w, int pw, cudaStream_t st) {
    const size_t slab_max = (size_t)n * pw * sizeof(cf);
    MW_REQUIRE(slab_max <= 200 * 1024, "order %d too large for a batched panel of %d columns", n, pw);
    static bool attr = false;
    if (!attr) {
        MW_CHECK_CUDA(cudaFuncSetAttribute(panel1_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
        attr = true;
    }
    // Blocked right-looking factorisation: kBOuter-column blocks, each
    // factored as pw-column panels (one CTA per matrix) whose updates stay
    // inside the block; the rest of the matrix then takes the block's row
    // interchanges, one triangular solve and ONE tensor-core update with
    // k = kBOuter (a pw-wide k would underuse the tensor pipe).
    for (int J0 = 0; J0 < n; J0 += kBOuter) {
        const int bw = (n - J0) < kBOuter ? (n - J0) : kBOuter;
        for (int j0 = J0; j0 < J0 + bw; j0 += pw) {
            const int jb = (J0 + bw - j0) < pw ? (J0 + bw - j0) : pw;
            {
                ProfileScope ps(PC_PANEL, st, 4.0 * (double)(n - j0) * jb * jb * batch);
                panel1_kernel<<<batch, kBThreads, (size_t)(n - j0) * jb * sizeof(cf), st>>>(A, lda, stride, n, j0, jb,
                                                                                            ipiv, info);
                count_launch();
            }
            if (j0 > 0) {
                ProfileScope ps(PC_LASWP, st);
                laswp_batched_kernel<cf><<<dim3((j0 + 127) / 128, batch), 128, 0, st>>>(A, lda, stride, 0, j0, ipiv,
                                                                                        n, j0, j0 + jb);
                count_launch();
            }
            const int inner = J0 + bw - j0 - jb;  // block columns right of this panel
            if (inner > 0) {
                {
                    ProfileScope ps(PC_LASWP, st);
                    laswp_batched_kernel<cf><<<dim3((inner + 127) / 128, batch), 128, 0, st>>>(
                        A, lda, stride, j0 + jb, inner, ipiv, n, j0, j0 + jb);
                }
                cf* A11 = A + j0 + (int64_t)j0 * lda;
                cf* A12 = A + j0 + (int64_t)(j0 + jb) * lda;
                {
                    ProfileScope ps(PC_TRSM, st, 4.0 * (double)jb * jb * inner * batch);
                    trsm_batched_kernel<false><<<trsm_batched_grid(inner, batch), 256, 0, st>>>(A11, lda, stride, A12,
                                                                                             lda, stride, jb, inner);
                }
                count_launch(2);
                mw_status s = cgemm_tc_update_batched(n - j0 - jb, inner, jb, batch, A + (j0 + jb) + (int64_t)j0 * lda,
                                                      lda, stride, A12, lda, stride,
                                                      A + (j0 + jb) + (int64_t)(j0 + jb) * lda, lda, stride, w.tc,
                                                      w.tc_bytes, w.tc_err, st, 0);
                if (s != MW_OK) return s;
            }
        }
        const int right = n - J0 - bw;
        if (right > 0) {
            {
                ProfileScope ps(PC_LASWP, st);
                laswp_batched_kernel<cf><<<dim3((right + 127) / 128, batch), 128, 0, st>>>(
                    A, lda, stride, J0 + bw, right, ipiv, n, J0, J0 + bw);
            }
            cf* A11 = A + J0 + (int64_t)J0 * lda;
            cf* A12 = A + J0 + (int64_t)(J0 + bw) * lda;
            {
                ProfileScope ps(PC_TRSM, st, 4.0 * (double)bw * bw * right * batch);
                trsm_batched_kernel<false><<<trsm_batched_grid(right, batch), 256, 0, st>>>(A11, lda, stride, A12, lda,
                                                                                         stride, bw, right);
            }
            count_launch(2);
            mw_status s = cgemm_tc_update_batched(right, right, bw, batch, A + (J0 + bw) + (int64_t)J0 * lda, lda,
                                                  stride, A12, lda, stride, A + (J0 + bw) + (int64_t)(J0 + bw) * lda,
                                                  lda, stride, w.tc, w.tc_bytes, w.tc_err, st, 0);
            if (s != MW_OK) return s;
        }
        MW_CHECK_CUDA(cudaGetLastError());
    }
    return MW_OK;
}

// In-place solve of the batch's B (n x nr each, column-major, ld n).
static mw_status cgetrs_batched(int n, int nr, int batch, const cf* LU, int64_t lda, int64_t stride,
                                const int32_t* ipiv, cf* B, cudaStream_t st) {
    const int64_t bs = (int64_t)n * nr;
    ProfileScope ps(PC_ZGEMM, st, 8.0 * (double)n * n * nr * batch);  // the whole batched getrs
    laswp_batched_kernel<cf><<<dim3((nr + 127) / 128, batch), 128, 0, st>>>(B, n, bs, 0, nr, ipiv, n, 0, n);
    count_launch();
    for (int j0 = 0; j0 < n; j0 += kBSB) {
        const int jb = (n - j0) < kBSB ? (n - j0) : kBSB;
        trsm_batched_kernel<false><<<trsm_batched_grid(nr, batch), 256, 0, st>>>(LU + j0 + (int64_t)j0 * lda, lda, stride,
                                                                             B + j0, n, bs, jb, nr);
        count_launch();
        const int rest = n - j0 - jb;
        if (rest > 0) {
            gemm_small_batched_kernel<<<dim3((rest + 127) / 128, batch), 128, 0, st>>>(
                LU + (j0 + jb) + (int64_t)j0 * lda, lda, stride, B + j0, n, bs, B + j0 + jb, n, bs, rest, jb, nr);
            count_launch();
        }
    }
    for (int j0 = ((n - 1) / kBSB) * kBSB; j0 >= 0; j0 -= kBSB) {
        const int jb = (n - j0) < kBSB ? (n - j0) : kBSB;
        trsm_batched_kernel<true><<<trsm_batched_grid(nr, batch), 256, 0, st>>>(LU + j0 + (int64_t)j0 * lda, lda, stride,
                                                                            B + j0, n, bs, jb, nr);
        count_launch();
        if (j0 > 0) {
            gemm_small_batched_kernel<<<dim3((j0 + 127) / 128, batch), 128, 0, st>>>(
                LU + (int64_t)j0 * lda, lda, stride, B + j0, n, bs, B, n, bs, j0, jb, nr);
            count_launch();
        }
    }
    MW_CHECK_CUDA(cudaGetLastError());
    return MW_OK;
}

}  // namespace mw

using namespace mw;

extern "C" size_t mw_zgesv_mixed_batched_workspace_size(int32_t n, int32_t nrhs, int32_t batch) {
    return batch_ws_bytes(n, nrhs, batch);
}

extern "C" mw_status mw_zgesv_mixed_batched(int32_t n, int32_t nrhs, int32_t batch, int32_t panel_width,
                                            const double* Z, int64_t ldz,
                                            int64_t z_stride, float* Z32, int64_t ldz32, int64_t z32_stride,
                                            int32_t* ipiv, int32_t* info, const double* B, int64_t ldb,
                                            int64_t b_stride, double* X, double tol, int32_t max_iter, void* workspace,
                                            size_t workspace_bytes, int32_t* iterations, double* last_correction,
                                            void* stream) {
    MW_REQUIRE(n >= 1 && nrhs >= 1 && batch >= 1 && batch <= 65535, "bad sizes");
    MW_REQUIRE(Z && Z32 && ipiv && info && B && X && workspace, "NULL argument");
    MW_REQUIRE(ldz >= n && ldz32 >= n && ldb >= n, "leading dimension too small");
    MW_REQUIRE(workspace_bytes >= batch_ws_bytes(n, nrhs, batch), "workspace too small");
    cudaStream_t st = as_stream(stream);
    BatchWs w = batch_ws(workspace, n, nrhs, batch);
    MW_CHECK_CUDA(cudaMemsetAsync(info, 0, sizeof(int32_t) * batch, st));
    MW_CHECK_CUDA(cudaMemsetAsync(w.tc_err, 0, sizeof(int), st));
    cf* Z32c = reinterpret_cast<cf*>(Z32);
    const int pw = panel_width > 0 ? panel_width : kBNB;
    MW_REQUIRE((pw == 8 || pw == 16 || pw == 32) && pw <= kBNBMax, "panel_width must be 8, 16 or 32 (got %d)", pw);
    mw_status s = cgetrf_batched(n, batch, Z32c, ldz32, z32_stride, ipiv, info, w, pw, st);
    if (s != MW_OK) return s;
    const int64_t per = (int64_t)n * nrhs;
    const int64_t tot = per * batch;
    cd* Xc = reinterpret_cast<cd*>(X);
    const cd* Zc = reinterpret_cast<const cd*>(Z);
    const cd* Bc = reinterpret_cast<const cd*>(B);
    // R = B (X = 0): the residual kernel with X = 0 would read Z; copy B instead
    MW_CHECK_CUDA(cudaMemsetAsync(Xc, 0, sizeof(cd) * tot, st));
    for (int b = 0; b < batch; ++b)
        MW_CHECK_CUDA(cudaMemcpy2DAsync(w.R + (int64_t)b * per, sizeof(cd) * n, Bc + (int64_t)b * b_stride,
                                        sizeof(cd) * ldb, sizeof(cd) * n, nrhs, cudaMemcpyDeviceToDevice, st));
    std::vector<double> hn(2 * (size_t)batch), prev((size_t)batch, 0.0);
    std::vector<int32_t> hinfo(batch);
    double corr = INFINITY;
    int it = 0;
    const unsigned g1 = (unsigned)((tot + 255) / 256 < 8192 ? (tot + 255) / 256 : 8192);
    for (;; ++it) {
        narrow_batched_kernel<<<g1, 256, 0, st>>>(w.R, w.R32, tot);
        count_launch();
        s = cgetrs_batched(n, nrhs, batch, Z32c, ldz32, z32_stride, ipiv, w.R32, st);
        if (s != MW_OK) return s;
        MW_CHECK_CUDA(cudaMemsetAsync(w.norms, 0, sizeof(double) * 2 * batch, st));
        {
            ProfileScope ps(PC_REFINE, st, 2.0 * (double)tot, 40.0 * (double)tot);
            dim3 g((unsigned)((per + 255) / 256 < 64 ? (per + 255) / 256 : 64), (unsigned)batch);
            accum_batched_kernel<<<g, 256, 0, st>>>(w.R32, Xc, per, w.norms, w.norms + batch);
            count_launch();
        }
        MW_CHECK_CUDA(cudaMemcpyAsync(hn.data(), w.norms, sizeof(double) * 2 * batch, cudaMemcpyDeviceToHost, st));
        int tce = 0;
        if (it == 0) {
            MW_CHECK_CUDA(cudaMemcpyAsync(hinfo.data(), info, sizeof(int32_t) * batch, cudaMemcpyDeviceToHost, st));
            MW_CHECK_CUDA(cudaMemcpyAsync(&tce, w.tc_err, sizeof(int), cudaMemcpyDeviceToHost, st));
        }
        MW_CHECK_CUDA(cudaStreamSynchronize(st));
        if (it == 0) {
            if (tce != 0) {
                set_error("batched factorisation: a bounded device wait timed out");
                return MW_ERR_TIMEOUT;
            }
            for (int b = 0; b < batch; ++b)
                if (hinfo[b] > 0) {
                    set_error("matrix %d of the batch: exact zero pivot at column %d", b, hinfo[b]);
                    return MW_ERR_SINGULAR;
                }
        }
        // as mw_zgesv_mixed: the relative correction, or once corrections
        // contract (q <= 1/2) the error estimated to remain, r q
        corr = 0.0;
        for (int b = 0; b < batch; ++b) {
            const double xm = hn[batch + b];
            const double r = xm > 0.0 ? hn[b] / xm : (hn[b] > 0.0 ? INFINITY : 0.0);
            double v = r;
            if (it > 0 && prev[b] > 0.0 && r <= 0.5 * prev[b]) v = fmin(r, r * (r / prev[b]));
            prev[b] = r;
            if (!(v <= corr)) corr = v;
        }
        if (corr <= tol || it >= max_iter) break;
        {
            ProfileScope ps(PC_REFINE, st, 8.0 * (double)n * n * nrhs * batch, 16.0 * (double)n * n * batch);
            resid_batched_kernel<<<dim3((n + 127) / 128, batch), 128, 0, st>>>(Zc, ldz, z_stride, Xc, n, per, Bc, ldb,
                                                                               b_stride, w.R, n, per, n, nrhs);
            count_launch();
        }
    }
    if (iterations) *iterations = it;
    if (last_correction) *last_correction = corr;
    if (!(corr <= tol)) {
        set_error("batched refinement did not reach tol %.3g in %d steps (last correction %.3g)", tol, it, corr);
        return MW_ERR_SINGULAR;
    }
    return MW_OK;
}
