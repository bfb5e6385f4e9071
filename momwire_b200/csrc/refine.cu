// Mixed-precision solve with FP64 iterative refinement (sm_100a).
//
// Solves Z X = B (complex128) from a complex64 LU of the same matrix:
//   X0 = LU32 \ B;  repeat  R = B - Z X (FP64),  C = LU32 \ R,  X += C
// until, for every column, the relative correction r = ||C||_inf / ||X||_inf
// or -- once successive corrections contract by q = r / r_prev <= 1/2 -- the
// error estimated to remain after it, r q, is <= tol.  The factors come
// from mw_cgetrf (tensor-core trailing updates, 3xTF32); the residual uses
// the FP64 Z.  The reference solves in complex128 LAPACK
// (bspline.py:2971-2989); this path adds nothing to its algebra.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <vector>

#include "common.cuh"

namespace mw {
mw_status zgemm_launch(bool ta, bool tb, int64_t m, int64_t n, int64_t k, cd alpha, const cd* A, int64_t lda,
                       const cd* B, int64_t ldb, cd beta, cd* C, int64_t ldc, cudaStream_t st, int max_ctas,
                       void* split_ws, size_t split_ws_bytes);
size_t zgemm_split_ws_bytes(int64_t m, int64_t n);
mw_status zgemm_split_ws_init(void* split_ws, cudaStream_t st);

__global__ void to_c64_kernel(const cd* __restrict__ src, int64_t lds, cf* __restrict__ dst, int64_t ldd, int64_t n,
                              int64_t ncol) {
    const int64_t total = n * ncol;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = q % n, j = q / n;
        const cd v = src[i + j * lds];
        dst[i + j * ldd] = cf{(float)v.re, (float)v.im};
    }
}

// X += C (widened), and per-column max-abs of C and of the new X.
__global__ void accumulate_kernel(const cf* __restrict__ C, int64_t ldc, cd* __restrict__ X, int64_t ldx, int64_t n,
                                  double* __restrict__ cmax, double* __restrict__ xmax) {
    const int64_t j = blockIdx.y;
    double mc = 0.0, mx = 0.0;
    for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const cf c = C[i + j * ldc];
        cd x = X[i + j * ldx];
        x.re += (double)c.re;
        x.im += (double)c.im;
        X[i + j * ldx] = x;
        mc = fmax(mc, fabs((double)c.re) + fabs((double)c.im));
        mx = fmax(mx, fabs(x.re) + fabs(x.im));
    }
    for (int off = 16; off > 0; off >>= 1) {
        mc = fmax(mc, __shfl_xor_sync(0xffffffffu, mc, off));
        mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, off));
    }
    if ((threadIdx.x & 31) == 0) {
        // non-negative doubles order like their bit patterns
        atomicMax(reinterpret_cast<unsigned long long*>(cmax + j), (unsigned long long)__double_as_longlong(mc));
        atomicMax(reinterpret_cast<unsigned long long*>(xmax + j), (unsigned long long)__double_as_longlong(mx));
    }
}

__global__ void copy_c128_kernel(const cd* __restrict__ src, int64_t lds, cd* __restrict__ dst, int64_t ldd, int64_t n,
                                 int64_t ncol) {
    const int64_t total = n * ncol;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t i = q % n, j = q / n;
        dst[i + j * ldd] = src[i + j * lds];
    }
}

static unsigned grid_for(int64_t total) {
    int64_t b = (total + 255) / 256;
    return (unsigned)(b < 4096 ? (b < 1 ? 1 : b) : 4096);
}

}  // namespace mw

using namespace mw;

extern "C" size_t mw_cgetrf_workspace_size(int64_t n, int64_t nrhs_max);
extern "C" mw_status mw_cgetrf(int64_t n, float* A, int64_t lda, int32_t* ipiv, int32_t* info, void* workspace,
                               size_t workspace_bytes, int64_t nrhs_max, const volatile int32_t* cancel, void* stream);
extern "C" mw_status mw_cgetrs(int64_t n, int64_t nrhs, const float* LU, int64_t lda, const int32_t* ipiv, float* B,
                               int64_t ldb, void* workspace, size_t workspace_bytes, void* stream);

namespace mw {
mw_status cgetrf_forward(int64_t n, float* Ad, int64_t lda, int32_t* ipiv, int32_t* info, void* workspace,
                         size_t workspace_bytes, float* Bd, int64_t ldb, int64_t nrhs, const volatile int32_t* cancel,
                         void* stream, bool static_pivot);
mw_status cgetrs_upper(int64_t n, int64_t nrhs, const float* LUd, int64_t lda, float* Bd, int64_t ldb, void* workspace,
                       size_t workspace_bytes, void* stream);
size_t cgetrs_ops_bytes(int64_t n, int64_t nrhs);
mw_status cgetrs_ops_prepare(int64_t n, const float* LUd, int64_t lda, void* ops, void* stream);
mw_status cgetrs_upper_ops(int64_t n, int64_t nrhs, const float* LUd, int64_t lda, float* Bd, int64_t ldb,
                           const void* ops, void* workspace, size_t workspace_bytes, void* stream);
mw_status cgetrs_ops(int64_t n, int64_t nrhs, const float* LUd, int64_t lda, const int32_t* ipiv, float* Bd,
                     int64_t ldb, const void* ops, void* workspace, size_t workspace_bytes, void* stream,
                     bool static_pivot);
}  // namespace mw

static size_t al256(size_t x) { return (x + 255) & ~size_t(255); }

namespace {
// Pivoting of the complex64 factorisation: 0 pivots within each diagonal
// block (static pivoting) and falls back to partial pivoting, 1 partial
// pivoting only.
std::atomic<int> g_pivot_mode{0};
// What the last mw_zgesv_mixed on this host thread used: 0 static pivots,
// 1 partial pivoting, 2 static pivots rejected then partial pivoting.
thread_local int g_last_pivoting = -1;
// the largest |L21| of the last static-pivot factorisation (0 when none)
thread_local double g_last_growth = 0.0;
// the controlling relative correction of every refinement step of the last
// call (the initial solve first)
thread_local std::vector<double> g_last_history;
// A static-pivot factorisation is kept while every |L21| (|re| + |im|) stays
// within this bound (partial pivoting keeps |L| <= 1); the FP64 refinement
// then has to converge as well.
constexpr float kStaticLmaxBound = 64.0f;
}  // namespace

extern "C" int32_t mw_set_mixed_pivoting(int32_t mode) {
    if (mode != 0 && mode != 1) {
        set_error("pivoting mode must be 0 (static with fallback) or 1 (partial), got %d", mode);
        return MW_ERR_INVALID;
    }
    return g_pivot_mode.exchange(mode);
}

extern "C" int32_t mw_last_mixed_pivoting(void) { return g_last_pivoting; }

extern "C" double mw_last_mixed_growth(void) { return g_last_growth; }

extern "C" int32_t mw_last_mixed_history(double* out, int32_t max_n) {
    const int32_t n = (int32_t)g_last_history.size();
    for (int32_t i = 0; i < n && i < max_n; ++i) out[i] = g_last_history[i];
    return n;
}

extern "C" size_t mw_zgesv_mixed_workspace_size(int64_t n, int64_t nrhs) {
    return al256(mw_cgetrf_workspace_size(n, nrhs)) + al256((size_t)n * nrhs * 16) + al256((size_t)n * nrhs * 8) +
           al256((size_t)nrhs * 16) + al256(zgemm_split_ws_bytes(n, nrhs)) + al256(cgetrs_ops_bytes(n, nrhs));
}

extern "C" mw_status mw_zgesv_mixed(int64_t n, int64_t nrhs, const double* Z, int64_t ldz, float* Z32, int64_t ldz32,
                                    int32_t* ipiv, const double* B, int64_t ldb, double* X, int64_t ldx, double tol,
                                    int32_t max_iter, void* workspace, size_t workspace_bytes, int32_t* info,
                                    int32_t* iterations, double* last_correction, const volatile int32_t* cancel,
                                    void* stream) {
    MW_REQUIRE(n >= 1 && nrhs >= 1 && ldz >= n && ldz32 >= n && ldb >= n && ldx >= n, "bad sizes");
    MW_REQUIRE(Z && Z32 && ipiv && B && X && workspace && info, "NULL argument");
    MW_REQUIRE(max_iter >= 0, "max_iter < 0");
    MW_REQUIRE(workspace_bytes >= mw_zgesv_mixed_workspace_size(n, nrhs), "workspace too small");
    cudaStream_t st = as_stream(stream);
    char* w = static_cast<char*>(workspace);
    const size_t lu_ws = mw_cgetrf_workspace_size(n, nrhs);
    void* ws_lu = w;
    cd* R = reinterpret_cast<cd*>(w + al256(lu_ws));
    cf* R32 = reinterpret_cast<cf*>(w + al256(lu_ws) + al256((size_t)n * nrhs * 16));
    double* norms = reinterpret_cast<double*>(w + al256(lu_ws) + al256((size_t)n * nrhs * 16) +
                                              al256((size_t)n * nrhs * 8));
    // the residual product's K-split partials (counts zeroed here, reset by
    // the kernel after each use)
    void* split_ws = reinterpret_cast<char*>(norms) + al256((size_t)nrhs * 16);
    const size_t split_bytes = zgemm_split_ws_bytes(n, nrhs);
    if (mw_status s0 = zgemm_split_ws_init(split_ws, st); s0 != MW_OK) return s0;
    // the solves' block operators of the factors (rebuilt after each factorisation)
    void* ops = static_cast<char*>(split_ws) + al256(split_bytes);
    const cd* Zc = reinterpret_cast<const cd*>(Z);
    const cd* Bc = reinterpret_cast<const cd*>(B);
    cd* Xc = reinterpret_cast<cd*>(X);
    const int64_t tot = n * nrhs;

    bool static_pivot = g_pivot_mode.load() == 0;
    bool fell_back = false;
    double corr = INFINITY;
    int it = 0;
    std::vector<double> hn(2 * nrhs), prev(nrhs, 0.0);
    for (int attempt = 0;; ++attempt) {
        if (attempt > 0) {
            // partial pivoting after a rejected static-pivot factorisation:
            // Z32 again from the FP64 Z (the same rounding as the fill's)
            static_pivot = false;
            fell_back = true;
            to_c64_kernel<<<grid_for(n * n), 256, 0, st>>>(Zc, ldz, reinterpret_cast<cf*>(Z32), ldz32, n, n);
            count_launch();
        }
        // the first solve's right-hand sides ride through the factorisation
        // (complex64 B, forward-substituted as the trailing columns are updated)
        to_c64_kernel<<<grid_for(tot), 256, 0, st>>>(Bc, ldb, R32, n, n, nrhs);
        count_launch();
        mw_status s;
        {
            ProfileScope ps(PC_FACTOR, st, 8.0 / 3.0 * (double)n * n * n + 4.0 * (double)n * n * nrhs, 0.0);
            s = cgetrf_forward(n, Z32, ldz32, ipiv, info, ws_lu, lu_ws, reinterpret_cast<float*>(R32), n, nrhs,
                               cancel, stream, static_pivot);
        }
        if (s != MW_OK) return s;
        int32_t hinfo[2] = {0, 0};
        unsigned int hws[4] = {0, 0, 0, 0};  // the panel status block at the start of the workspace
        MW_CHECK_CUDA(cudaMemcpyAsync(hinfo, info, sizeof(hinfo), cudaMemcpyDeviceToHost, st));
        MW_CHECK_CUDA(cudaMemcpyAsync(hws, ws_lu, sizeof(hws), cudaMemcpyDeviceToHost, st));
        MW_CHECK_CUDA(cudaStreamSynchronize(st));
        if (hinfo[1] != 0) {
            set_error("factorisation: a bounded device wait timed out");
            return MW_ERR_TIMEOUT;
        }
        if (static_pivot) {
            float lmax;
            std::memcpy(&lmax, &hws[2], sizeof(float));
            g_last_growth = lmax;
            if (!(lmax <= kStaticLmaxBound) || hinfo[0] > 0) continue;  // growth too large or singular block
        }
        if (hinfo[0] > 0) {
            set_error("exact zero pivot at column %d", hinfo[0]);
            return MW_ERR_SINGULAR;
        }
        // X = 0, R = B
        MW_CHECK_CUDA(cudaMemsetAsync(norms, 0, sizeof(double) * 2 * nrhs, st));
        MW_CHECK_CUDA(cudaMemset2DAsync(Xc, sizeof(cd) * ldx, 0, sizeof(cd) * n, nrhs, st));
        copy_c128_kernel<<<grid_for(tot), 256, 0, st>>>(Bc, ldb, R, n, n, nrhs);
        count_launch();
        corr = INFINITY;
        std::fill(prev.begin(), prev.end(), 0.0);
        g_last_history.clear();
        for (it = 0;; ++it) {
            if (cancel && *cancel) {
                set_error("solve cancelled");
                return MW_ERR_CANCELLED;
            }
            if (it == 0) {
                // R32 holds L^-1 P B from the factorisation
                ProfileScope ps(PC_SOLVE, st, 4.0 * (double)n * n * nrhs, 0.0);
                s = cgetrs_ops_prepare(n, Z32, ldz32, ops, stream);
                if (s != MW_OK) return s;
                s = cgetrs_upper_ops(n, nrhs, Z32, ldz32, reinterpret_cast<float*>(R32), n, ops, ws_lu, lu_ws, stream);
            } else {
                {
                    ProfileScope ps(PC_REFINE, st, 0.0, 24.0 * (double)tot);
                    to_c64_kernel<<<grid_for(tot), 256, 0, st>>>(R, n, R32, n, n, nrhs);
                    count_launch();
                }
                ProfileScope ps(PC_SOLVE, st, 8.0 * (double)n * n * nrhs, 0.0);
                s = cgetrs_ops(n, nrhs, Z32, ldz32, ipiv, reinterpret_cast<float*>(R32), n, ops, ws_lu, lu_ws, stream,
                               static_pivot);
            }
            if (s != MW_OK) return s;
            MW_CHECK_CUDA(cudaMemsetAsync(norms, 0, sizeof(double) * 2 * nrhs, st));
            {
                ProfileScope ps(PC_REFINE, st, 2.0 * (double)tot, 40.0 * (double)tot);
                dim3 g((unsigned)((n + 255) / 256 < 64 ? (n + 255) / 256 : 64), (unsigned)nrhs);
                accumulate_kernel<<<g, 256, 0, st>>>(R32, n, Xc, ldx, n, norms, norms + nrhs);
                count_launch();
            }
            MW_CHECK_CUDA(cudaMemcpyAsync(hn.data(), norms, sizeof(double) * 2 * nrhs, cudaMemcpyDeviceToHost, st));
            MW_CHECK_CUDA(cudaStreamSynchronize(st));
            // per column: the relative correction r, and once corrections
            // contract (q = r / r_prev <= 1/2), the error left after this one,
            // about r q.  The initial solve counts as the first correction: it
            // starts from X = 0, so its error was the whole solution (r = 1) and
            // the first refinement correction r_1 measures the contraction
            // itself.  The controlling value is the smaller of r and r q,
            // maximised over the columns.
            corr = 0.0;
            for (int64_t j = 0; j < nrhs; ++j) {
                double xm = hn[nrhs + j];
                double r = xm > 0.0 ? hn[j] / xm : (hn[j] > 0.0 ? INFINITY : 0.0);
                double v = r;
                if (it > 0 && prev[j] > 0.0 && r <= 0.5 * prev[j]) v = fmin(r, r * (r / prev[j]));
                prev[j] = r;
                if (!(v <= corr)) corr = v;  // NaN-propagating max
            }
            g_last_history.push_back(corr);
            if (corr <= tol || it >= max_iter) break;
            // R = B - Z X   (FP64)
            copy_c128_kernel<<<grid_for(tot), 256, 0, st>>>(Bc, ldb, R, n, n, nrhs);
            count_launch();
            s = zgemm_launch(false, false, n, nrhs, n, cd{-1.0, 0.0}, Zc, ldz, Xc, ldx, cd{1.0, 0.0}, R, n, st, 0,
                             split_ws, split_bytes);
            if (s != MW_OK) return s;
        }
        if (corr <= tol || !static_pivot) break;
        // the static-pivot factors did not refine to tol: partial pivoting
    }
    g_last_pivoting = static_pivot ? 0 : (fell_back ? 2 : 1);
    if (iterations) *iterations = it;
    if (last_correction) *last_correction = corr;
    if (!(corr <= tol)) {
        set_error("iterative refinement did not reach tol %.3g in %d steps (last correction %.3g)", tol, it, corr);
        return MW_ERR_SINGULAR;
    }
    return MW_OK;
}
