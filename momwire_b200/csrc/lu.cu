// Dense complex LU with partial pivoting and triangular solves (sm_100a).
//
// Replaces LAPACK zgetrf/zgetrs reached through scipy.linalg.solve in
// momwire (bspline.py:2971-2989).  Right-looking blocked algorithm, generic
// in the element type (complex128 for the plain path, complex64 for the
// mixed-precision path):
//   panel   : one cooperative kernel per panel; rows split over the CTAs,
//             each CTA's row slab kept in shared memory for the whole panel,
//             one all-to-all pivot exchange per column -- complex128: a
//             bounded grid barrier and double-buffered slots; complex64:
//             self-validating tagged records read in one batch (no fence);
//             panels whose slabs would not fit are split in two and
//             recursed;
//   laswp   : row interchanges outside the panel;
//   trsm    : triangular leaves with the triangle staged lane-major in
//             shared memory, each optionally applying the block solved
//             before it (the next-block update of a blocked sweep);
//   update  : A22 -= L21 U12 -- complex128: register-tiled FP64 GEMM;
//             complex64: tcgen05 tensor cores, 3xTF32 (cgemm_tc.cu).
// Pivot choice follows LAPACK's izamax: max |re| + |im|, first index wins
// (complex64: the float sum, as LAPACK's icamax).
#include <cstdio>
#include <cstdlib>
#include <type_traits>

#include "common.cuh"
#include "tc_layout.cuh"
#include "waits.cuh"

namespace mw {

// tensor-core update (cgemm_tc.cu)
mw_status cgemm_tc_update(int64_t m, int64_t n, int64_t k, const cf* A, int64_t lda, const cf* B, int64_t ldb, cf* C,
                          int64_t ldc, void* ws, size_t ws_bytes, int* err, cudaStream_t st, int max_ctas);
size_t cgemm_tc_workspace(int64_t m, int64_t n, int64_t k);
TcPlanes tc_planes(void* ws, int64_t m_max, int64_t n_max, int64_t k);
mw_status cgemm_tc_prepacked(int64_t m, int64_t n, int64_t k, const TcPlanes& pl, cf* C, int64_t ldc, int* err,
                             cudaStream_t st, int max_ctas);
mw_status tc_pack_a(int64_t m, int64_t k, const cf* A, int64_t lda, float* a_hi, float* a_lo, cudaStream_t st,
                    int batch = 1, int64_t a_stride = 0, int64_t p_stride = 0);
size_t tc_pack_a_bytes(int64_t m, int64_t k);
size_t tc_pack_b_bytes(int64_t k, int64_t n);
mw_status cgemm_tc_prepacked2(int64_t m, int64_t n, int64_t k1, const TcPlanes& pl1, int64_t k2, const TcPlanes& pl2,
                              cf* C, int64_t ldc, int* err, cudaStream_t st, int max_ctas);

// static-pivot panel of the complex64 path (lu_static.cu)
mw_status static_panel_c64(cf* A, int64_t lda, int64_t n, int64_t j0, int jb, int32_t* ipiv, int32_t* info,
                           PanelWs* ws, cf* inv_diag, int32_t* perm, const TcPlanes* pack_a, cudaStream_t st);
void static_permute_c64(cf* A, int64_t lda, int64_t row0, int jb, int64_t col0, int64_t ncols, const int32_t* perm,
                        cudaStream_t st);
void static_left_permute_c64(cf* A, int64_t lda, int64_t n, const int32_t* perm_all, cudaStream_t st);
void static_rows_permute_c64(cf* B, int64_t ldb, int64_t n, int64_t ncols, const int32_t* perm_all,
                             cudaStream_t st);

constexpr int kNB = 64;         // panel half width (rank-1 work per cooperative panel)
constexpr int kOuterNB = 128;   // getrf block: panel width and trailing-update k
constexpr int kPanelMaxJb = 128;
constexpr int kPanelThreads = 256;

__device__ __forceinline__ cd ldcg_c(const cd* p) {
    double2 v = __ldcg(reinterpret_cast<const double2*>(p));
    return cd{v.x, v.y};
}
__device__ __forceinline__ cf ldcg_c(const cf* p) {
    float2 v = __ldcg(reinterpret_cast<const float2*>(p));
    return cf{v.x, v.y};
}

struct PanelArgs {
    void* A;
    int64_t lda;
    int64_t n;
    int64_t j0;
    int jb;
    int rcap;  // slab leading dimension (rows per CTA)
    int32_t* ipiv;
    int32_t* info;
    PanelWs* ws;
    // double-buffered slots: [2][G] values, [2][G] indices (complex64: the
    // key words), [2][G][kPanelMaxJb] candidate rows (complex64: the tagged
    // records, candidate rows then row c), [2][kPanelMaxJb] current row
    double* slot_val;
    int64_t* slot_idx;
    void* slot_row;
    void* cur_row;
};

__device__ __forceinline__ void argmax_merge(double& v, int64_t& i, double v2, int64_t i2) {
    if (v2 > v || (v2 == v && i2 < i)) {
        v = v2;
        i = i2;
    }
}

// Block-wide argmax of (value, row): larger value wins, smaller row on ties.
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
template <class T>
__global__ void __launch_bounds__(kPanelThreads) panel_kernel(PanelArgs P) {
    extern __shared__ __align__(16) unsigned char panel_smem[];
    T* slab = reinterpret_cast<T*>(panel_smem);
    __shared__ double s_v[kPanelThreads / 32];
    __shared__ int64_t s_i[kPanelThreads / 32];
    __shared__ T s_piv[kPanelMaxJb];
    __shared__ T s_cur[kPanelMaxJb];
    __shared__ int64_t s_p;
    __shared__ double s_pv;

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
    T* A = static_cast<T*>(P.A);
    T* slot_row = static_cast<T*>(P.slot_row);
    T* cur_row = static_cast<T*>(P.cur_row);
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
                slot_row[((size_t)buf * G + g) * kPanelMaxJb + x] = slab[x * rcap + (int)(bidx - r0)];
        if (c >= r0 && c < r1)
            for (int x = tid; x < jb; x += blockDim.x) cur_row[buf * kPanelMaxJb + x] = slab[x * rcap + (int)(c - r0)];
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
                if (g == 0) P.ipiv[c] = (int32_t)(bi + 1);
            }
            bg = __shfl_sync(0xffffffffu, bg, 0);
            // the same warp fetches the pivot row and the current row (L2-
            // coherent loads: other CTAs wrote them)
            for (int x = tid; x < jb; x += 32) {
                s_piv[x] = ldcg_c(slot_row + ((size_t)buf * G + bg) * kPanelMaxJb + x);
                s_cur[x] = ldcg_c(cur_row + buf * kPanelMaxJb + x);
            }
        }
        __syncthreads();
        const int64_t p = s_p;
        if (s_pv == 0.0 && g == 0 && tid == 0 && P.info[0] == 0) P.info[0] = (int32_t)(c + 1);
        // 5-6. rows in the threads: the owners of rows c and p swap them;
        // every row below c is scaled by the pivot and updated with the
        // pivot row (LAPACK: an exact zero pivot is neither divided by nor
        // applied)
        const bool apply = s_pv != 0.0;
        const T inv = apply ? cdiv(cone<T>(), s_piv[jj]) : cone<T>();
        // the swap, one column per thread, then the scale and rank-1 update
        // with two threads per row (the two halves of the block, alternate
        // columns); each half reads the multiplier from the pivot column
        if (p != c) {
            const int lc0 = (c >= r0 && c < r1) ? (int)(c - r0) : -1;
            const int lp0 = (p >= r0 && p < r1) ? (int)(p - r0) : -1;
            for (int x = tid; x < jb; x += blockDim.x) {
                if (lc0 >= 0) slab[x * rcap + lc0] = s_piv[x];
                if (lp0 >= 0) slab[x * rcap + lp0] = s_cur[x];
            }
            __syncthreads();
        }
        if (apply) {
            constexpr int kHalf = kPanelThreads / 2;
            const int par = tid / kHalf;
            for (int i = i0 + (tid % kHalf); i < R; i += kHalf) {
                if (r0 + i == c) continue;
                const T l = slab[jj * rcap + i] * inv;
                for (int x = jj + 1 + par; x < jb; x += 2) slab[x * rcap + i] = slab[x * rcap + i] - l * s_piv[x];
            }
            __syncthreads();
            // the multipliers last: both halves read column jj above
            for (int i = i0 + tid; i < R; i += blockDim.x)
                if (r0 + i != c) slab[jj * rcap + i] = slab[jj * rcap + i] * inv;
        }
        __syncthreads();
    }
    for (int idx = tid; idx < R * jb; idx += blockDim.x) {
        int i = idx % R, x = idx / R;
        A[(r0 + i) + (P.j0 + x) * lda] = slab[x * rcap + i];
    }
}

// Complex64 panel with self-validating exchange records.  Every word a CTA
// publishes carries the column it belongs to, so no fence orders the
// publication and a reader needs no second round trip:
//   key  : one 64-bit word per CTA [seq 8 | float(|re|+|im|) bits 32 |
//          2^24-1 - (row - j0) 24]; largest key wins (largest value, then
//          smallest row: LAPACK's izamax rule at float resolution);
//   rows : the CTA's candidate row (zeros when it has none) and, from the
//          owner of row c, row c itself, each element as two 64-bit words
//          [tag 32 | float bits 32] with tag = c + 1.
// Each CTA reads all G keys and all G + 1 rows in one batch of relaxed
// loads (G <= kC64MaxGrid, so at most 33 rows of 64 elements), re-reading a
// word until its tag matches (bounded), and takes the winner's row from
// shared memory.  The key's float rounding can only change the choice
// between candidates within one float ulp of each other, which the FP64
// refinement of the mixed path absorbs.  The record area is cleared at the
// start of a factorisation, so a word from an earlier one never matches.
constexpr int kC64MaxGrid = 32;
constexpr int kC64RecStride = kC64MaxGrid * kPanelMaxJb;  // 16-byte elements per buffer
constexpr int kC64Items = ((kC64MaxGrid + 1) * kNB + kPanelThreads - 1) / kPanelThreads;

__device__ __forceinline__ unsigned long long ld_relaxed_u64(const unsigned long long* p) {
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed_u64(unsigned long long* p, unsigned long long v) {
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}
__device__ __forceinline__ void ld_tagged(const unsigned long long* p, unsigned long long& a, unsigned long long& b) {
    asm volatile("ld.relaxed.gpu.global.v2.u64 {%0, %1}, [%2];" : "=l"(a), "=l"(b) : "l"(p) : "memory");
}
__device__ __forceinline__ void st_tagged(unsigned long long* p, cf v, unsigned int tag) {
    const unsigned long long a = ((unsigned long long)tag << 32) | __float_as_uint(v.re);
    const unsigned long long b = ((unsigned long long)tag << 32) | __float_as_uint(v.im);
    asm volatile("st.relaxed.gpu.global.v2.u64 [%0], {%1, %2};" ::"l"(p), "l"(a), "l"(b) : "memory");
}

// 1 / z for the complex64 panel: z scaled by the reciprocal of its larger
// component (so |z|^2 neither overflows nor underflows; tiny z take Smith's
// form), then two correctly
// rounded reciprocals instead of Smith's three divisions -- a few ulp, which
// the FP64 refinement of the mixed path absorbs.
__device__ __forceinline__ cf crcp_scaled(cf z) {
    const float s = fmaxf(fabsf(z.re), fabsf(z.im));
    if (s < 1e-30f) return cdiv(cone<cf>(), z);  // 1/s would overflow: Smith's form
    const float rs = __frcp_rn(s);
    const float a = z.re * rs, b = z.im * rs;
    const float t = rs * __frcp_rn(a * a + b * b);
    return cf{a * t, -b * t};
}

// The exchange of column jj+1 overlaps the bulk of column jj's update: once
// column jj's pivot is known, every CTA updates column jj+1 of its rows,
// finds its candidate for jj+1, finishes that candidate row (and, on the
// owner, row c+1) over the remaining columns, publishes them, and only then
// updates the rest of its rows while the other CTAs' records arrive.
__global__ void __launch_bounds__(kPanelThreads) panel_kernel_c64(PanelArgs P) {
    extern __shared__ __align__(16) unsigned char panel_smem[];
    cf* slab = reinterpret_cast<cf*>(panel_smem);
    __shared__ double s_v[kPanelThreads / 32];
    __shared__ int64_t s_i[kPanelThreads / 32];
    // per column parity: G candidate rows, then row c (two buffers, so the
    // next column's records land while the bulk update still reads these)
    __shared__ cf s_rows[2][(kC64MaxGrid + 1) * kNB];
    __shared__ unsigned long long s_bk;
    __shared__ int s_bg;
    __shared__ unsigned int s_wfb[kPanelThreads / 32], s_wrow[kPanelThreads / 32];

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
    cf* A = static_cast<cf*>(P.A);
    unsigned long long* rec = static_cast<unsigned long long*>(P.slot_row);  // [2][kC64RecStride] x 2 words
    unsigned long long* words = reinterpret_cast<unsigned long long*>(P.slot_idx);  // [2][G]
    const int64_t lda = P.lda;
    const int n_items = (G + 1) * jb;

    for (int idx = tid; idx < R * jb; idx += blockDim.x) {
        int i = idx % R, x = idx / R;
        slab[x * rcap + i] = A[(r0 + i) + (P.j0 + x) * lda];
    }
    __syncthreads();

    // Publish the records of column cc (candidate local row lb or -1 with
    // value best, local row lc of cc or -1).  Thread x writes element x of
    // the candidate row, thread jb + x element x of row cc, the last thread
    // the key; a caller that finishes rows lb / lc first keeps the same
    // thread-to-column mapping, so no barrier is needed in between.
    auto publish = [&](int64_t cc, int lb, int lc, double best) {
        const int nbuf = (int)((cc - P.j0) & 1);
        const unsigned int tag = (unsigned int)(cc + 1);
        unsigned long long* rb = rec + (size_t)nbuf * kC64RecStride * 2;
        if (tid < jb) {
            const cf v = lb >= 0 ? slab[tid * rcap + lb] : cf{0.0f, 0.0f};
            st_tagged(rb + (size_t)(g * jb + tid) * 2, v, tag);
        } else if (tid < 2 * jb) {
            if (lc >= 0) st_tagged(rb + (size_t)(G * jb + (tid - jb)) * 2, slab[(tid - jb) * rcap + lc], tag);
        }
        if (tid == kPanelThreads - 1) {
            const unsigned long long seq = (unsigned long long)((cc + 1) % 255 + 1);
            unsigned long long key = 0;  // no candidate: loses to every row
            if (lb >= 0) {
                const unsigned int fb = __float_as_uint((float)best);
                key = ((unsigned long long)fb << 24) | (unsigned long long)(0xFFFFFFll - (r0 + lb - P.j0));
            }
            st_relaxed_u64(words + (size_t)nbuf * G + g, (seq << 56) | key);
        }
    };

    {
        double best = -1.0;
        int64_t bidx = INT64_MAX;
        for (int i = tid; i < R; i += blockDim.x) argmax_merge(best, bidx, cabs1(slab[i]), r0 + i);
        block_argmax(best, bidx, s_v, s_i);
        publish(P.j0, bidx != INT64_MAX ? (int)(bidx - r0) : -1, (P.j0 >= r0 && P.j0 < r1) ? (int)(P.j0 - r0) : -1,
                best);
    }
    for (int jj = 0; jj < jb; ++jj) {
        const int64_t c = P.j0 + jj;
        const int buf = jj & 1;
        const unsigned int tag = (unsigned int)(c + 1);
        // 1..255, never the 0 the slots are cleared to; a stale word in a
        // slot is at most 2 * kNB + 2 columns old, so it never matches
        const unsigned long long seq = (unsigned long long)((c + 1) % 255 + 1);
        const unsigned long long* rb = rec + (size_t)buf * kC64RecStride * 2;
        // every load of the column in flight at once, then the re-reads
        unsigned long long wa[kC64Items], wb[kC64Items];
#pragma unroll
        for (int k = 0; k < kC64Items; ++k) {
            const int idx = tid + k * kPanelThreads;
            if (idx < n_items) ld_tagged(rb + (size_t)idx * 2, wa[k], wb[k]);
        }
        unsigned long long kw = 0;
        if (tid < G) kw = ld_relaxed_u64(words + (size_t)buf * G + tid);
        int ok = 1;
        long long spins = 0;
        auto give_up = [&]() {
            if ((++spins & 1023) == 0 && (spins > (1ll << 24) || *(volatile int*)&P.ws->err)) {
                atomicExch(&P.ws->err, MW_ERR_TIMEOUT);
                ok = 0;
            }
            return !ok;
        };
#pragma unroll
        for (int k = 0; k < kC64Items; ++k) {
            const int idx = tid + k * kPanelThreads;
            if (idx < n_items && ok) {
                while ((unsigned int)(wa[k] >> 32) != tag || (unsigned int)(wb[k] >> 32) != tag) {
                    if (give_up()) break;
                    ld_tagged(rb + (size_t)idx * 2, wa[k], wb[k]);
                }
                s_rows[buf][idx] = cf{__uint_as_float((unsigned int)wa[k]), __uint_as_float((unsigned int)wb[k])};
            }
        }
        if (tid < G && ok)
            while ((kw >> 56) != seq) {
                if (give_up()) break;
                kw = ld_relaxed_u64(words + (size_t)buf * G + tid);
            }
        if (tid < 32) {
            // largest key: largest value bits, then largest inverted row;
            // the lowest lane on (impossible) full ties
            const unsigned long long key = tid < G ? (kw & 0x00FFFFFFFFFFFFFFull) : 0ull;
            const unsigned int fb = (unsigned int)(key >> 24), lo = (unsigned int)(key & 0xFFFFFFull);
            const unsigned int mfb = __reduce_max_sync(0xffffffffu, fb);
            const unsigned int mlo = __reduce_max_sync(0xffffffffu, fb == mfb ? lo : 0u);
            const unsigned int win = __ballot_sync(0xffffffffu, fb == mfb && lo == mlo);
            if (tid == 0) {
                s_bk = ((unsigned long long)mfb << 24) | mlo;
                s_bg = __ffs(win) - 1;
            }
        }
        // (this barrier also ends the previous column's bulk update)
        if (!__syncthreads_and(ok)) return;  // a wait gave up: the error word is set
        const unsigned long long bk = s_bk;
        const cf* s_piv = s_rows[buf] + s_bg * jb;
        const cf* s_cur = s_rows[buf] + G * jb;
        const int64_t p = P.j0 + (0xFFFFFFll - (int64_t)(bk & 0xFFFFFFull));
        const bool zero = ((bk >> 24) & 0xFFFFFFFFull) == 0ull;  // |pivot| == 0
        // LAPACK: an exact zero pivot is neither divided by nor applied
        const bool apply = !zero;
        const cf inv = apply ? crcp_scaled(s_piv[jj]) : cone<cf>();
        const int i0 = (int)max((int64_t)0, c - r0);
        const bool last = jj + 1 >= jb;
        // 1. swap rows c and p (one column per thread; row p's columns jj
        // and jj+1 belong to its row thread below), scale column jj below c,
        // update column jj+1
        if (p != c) {
            const int lc0 = (c >= r0 && c < r1) ? (int)(c - r0) : -1;
            const int lp0 = (p >= r0 && p < r1) ? (int)(p - r0) : -1;
            for (int x = tid; x < jb; x += blockDim.x) {
                if (lc0 >= 0) slab[x * rcap + lc0] = s_piv[x];
                if (lp0 >= 0 && x != jj && x != jj + 1) slab[x * rcap + lp0] = s_cur[x];
            }
        }
        // the candidate of column jj+1 among this thread's rows (all > c):
        // largest float |re|+|im| (LAPACK's scabs1), then smallest row
        unsigned int bfb = 0u, brow = 0xFFFFFFFFu;
        for (int i = i0 + tid; i < R; i += blockDim.x) {
            const int64_t gr = r0 + i;
            if (gr == c) continue;
            const bool swapped = gr == p && p != c;
            // both loads ahead of the stores
            const cf a0 = swapped ? s_cur[jj] : slab[jj * rcap + i];
            const cf a1 = last ? cf{0.0f, 0.0f} : (swapped ? s_cur[jj + 1] : slab[(jj + 1) * rcap + i]);
            cf n1 = a1;
            if (!apply) {
                if (swapped) {
                    slab[jj * rcap + i] = a0;
                    if (!last) slab[(jj + 1) * rcap + i] = a1;
                }
            } else {
                const cf l = a0 * inv;
                slab[jj * rcap + i] = l;
                if (!last) {
                    n1 = a1 - l * s_piv[jj + 1];
                    slab[(jj + 1) * rcap + i] = n1;
                }
            }
            const unsigned int fb = __float_as_uint(fabsf(n1.re) + fabsf(n1.im));
            if (fb > bfb || brow == 0xFFFFFFFFu) {  // rows ascend: ties keep the first
                bfb = fb;
                brow = (unsigned int)i;
            }
        }
        {
            const unsigned int mfb = __reduce_max_sync(0xffffffffu, brow == 0xFFFFFFFFu ? 0u : bfb);
            const unsigned int mrow =
                __reduce_min_sync(0xffffffffu, (brow != 0xFFFFFFFFu && bfb == mfb) ? brow : 0xFFFFFFFFu);
            if ((tid & 31) == 0) {
                s_wfb[tid >> 5] = mfb;
                s_wrow[tid >> 5] = mrow;
            }
        }
        __syncthreads();
        if (last) {
            if (g == 0 && tid == 0) {
                P.ipiv[c] = (int32_t)(p + 1);
                if (zero && P.info[0] == 0) P.info[0] = (int32_t)(c + 1);
            }
            break;
        }
        // 2. the candidate row for column jj+1 and row c+1, finished over the
        // remaining columns by the threads that publish them
        const int64_t cn = c + 1;
        unsigned int cfb, crow;
        {
            // every warp combines the eight warp results itself
            const int ln = tid & 31;
            const unsigned int f = ln < kPanelThreads / 32 ? s_wfb[ln] : 0u;
            const unsigned int r = ln < kPanelThreads / 32 ? s_wrow[ln] : 0xFFFFFFFFu;
            cfb = __reduce_max_sync(0xffffffffu, r != 0xFFFFFFFFu ? f : 0u);
            crow = __reduce_min_sync(0xffffffffu, (r != 0xFFFFFFFFu && f == cfb) ? r : 0xFFFFFFFFu);
        }
        const double best = (double)__uint_as_float(cfb);
        const int64_t bidx = crow != 0xFFFFFFFFu ? r0 + crow : INT64_MAX;
        const int lb = bidx != INT64_MAX ? (int)(bidx - r0) : -1;
        const int lc = (cn >= r0 && cn < r1) ? (int)(cn - r0) : -1;
        if (apply) {
            if (tid < jb) {
                if (lb >= 0 && tid >= jj + 2) slab[tid * rcap + lb] = slab[tid * rcap + lb] - slab[jj * rcap + lb] * s_piv[tid];
            } else if (tid < 2 * jb) {
                const int x = tid - jb;
                if (lc >= 0 && lc != lb && x >= jj + 2)
                    slab[x * rcap + lc] = slab[x * rcap + lc] - slab[jj * rcap + lc] * s_piv[x];
            }
        }
        // (row lc == lb: the candidate's thread finished it; its row-c
        // element is read by thread jb + x after the barrier in phase 3)
        if (lc >= 0 && lc == lb) __syncthreads();
        publish(cn, lb, lc, best);
        if (g == 0 && tid == 0) {
            P.ipiv[c] = (int32_t)(p + 1);
            if (zero && P.info[0] == 0) P.info[0] = (int32_t)(c + 1);
        }
        // 3. the rest of column jj's update while the other CTAs publish:
        // two threads per row (the two halves of the block), alternate columns
        if (apply) {
            constexpr int kHalf = kPanelThreads / 2;
            const int par = tid / kHalf;
            for (int i = i0 + (tid % kHalf); i < R; i += kHalf) {
                const int64_t gr = r0 + i;
                if (gr <= c || i == lb || i == lc) continue;
                const cf l = slab[jj * rcap + i];
                int x = jj + 2 + par;
                // four columns' loads ahead of their stores
                for (; x + 6 < jb; x += 8) {
                    const cf a0 = slab[x * rcap + i], a1 = slab[(x + 2) * rcap + i];
                    const cf a2 = slab[(x + 4) * rcap + i], a3 = slab[(x + 6) * rcap + i];
                    const cf p0 = s_piv[x], p1 = s_piv[x + 2], p2 = s_piv[x + 4], p3 = s_piv[x + 6];
                    slab[x * rcap + i] = a0 - l * p0;
                    slab[(x + 2) * rcap + i] = a1 - l * p1;
                    slab[(x + 4) * rcap + i] = a2 - l * p2;
                    slab[(x + 6) * rcap + i] = a3 - l * p3;
                }
                for (; x < jb; x += 2) slab[x * rcap + i] = slab[x * rcap + i] - l * s_piv[x];
            }
        }
    }
    for (int idx = tid; idx < R * jb; idx += blockDim.x) {
        int i = idx % R, x = idx / R;
        A[(r0 + i) + (P.j0 + x) * lda] = slab[x * rcap + i];
    }
}

template <class T>
__global__ void laswp_kernel(T* A, int64_t lda, int64_t col0, int64_t ncols, const int32_t* ipiv, int64_t k1,
                             int64_t k2) {
    int64_t col = col0 + blockIdx.x * (int64_t)blockDim.x + threadIdx.x;
    if (col >= col0 + ncols) return;
    T* a = A + col * lda;
    for (int64_t i = k1; i < k2; ++i) {
        int64_t p = ipiv[i] - 1;
        if (p != i) {
            T t = a[i];
            a[i] = a[p];
            a[p] = t;
        }
    }
}

__device__ __forceinline__ cd shfl_c(cd v, int src) {
    return cd{__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src)};
}
__device__ __forceinline__ cf shfl_c(cf v, int src) {
    return cf{__shfl_sync(0xffffffffu, v.re, src), __shfl_sync(0xffffffffu, v.im, src)};
}

// Rows of a triangular-solve leaf in the multi-right-hand-side solve:
// 128 for complex64 (its staged triangle, 132 KB, fits shared memory; half
// the sequential steps of 64-row leaves), 64 for complex128.  The
// factorisation's own block-row solves (thousands of columns) keep 64-row
// leaves, whose 33 KB lets several CTAs share an SM.
template <class T>
struct GetrsLeaf {
    static constexpr int value = 64;
};
template <>
struct GetrsLeaf<cf> {
    static constexpr int value = 128;
};

// X (jb x ncols, leading dim ldx) <- L^-1 X with L unit lower (jb x jb),
// or U^-1 X with U upper non-unit (jb <= leaf).  The CTA stages the triangle
// in shared memory; each warp then owns NC columns of X in registers (lane l
// holds rows RP*l .. RP*l+RP-1 of each) and substitutes with warp shuffles
// only, every staged triangle element read once for all of them.  Wide
// solves take NC = 4 (a quarter of the CTAs stage the triangle); narrow
// ones, whose latency sits on the critical path, NC = 1 (more CTAs).
constexpr int kTrsmWarps = 8;
// Packed-B output of a leaf (complex64 only): the solved rows also written
// as the B operand of a tensor-core update, rows at K offset kap0 / 2 of an
// inner dimension of b_nks stages.
struct LeafPack {
    float* b_hi = nullptr;
    float* b_lo = nullptr;
    int b_nks = 0;
    int kap0 = 0;
};
// A batch of independent solves in one launch (blockIdx.y = member b): the
// triangle of member b at Tm + b t_step, its right-hand sides at X + b
// x_step, its order min(jb, n - b L).  n = 0: a single solve.
struct TrsmBatch {
    int64_t t_step = 0;
    int64_t x_step = 0;
    int64_t n = 0;
};

template <class T, bool UPPER, int L, int NC>
__global__ void __launch_bounds__(32 * kTrsmWarps) trsm_kernel(const T* Tm, int64_t ldt, T* X, int64_t ldx, int jb,
                                                               int64_t ncols, const T* Aoff, int64_t ldo, const T* Xp,
                                                               int K, LeafPack pk, TrsmBatch bt) {
    // Lane l owns rows RP*l .. RP*l+RP-1 of the block, so a RP x RP diagonal
    // block is solved inside one lane; its RP results reach the other lanes
    // in RP independent shuffles and every lane applies the RP x RP update:
    // 32 short dependent chains instead of L long ones.  The triangle is
    // staged as S[block kb][a*RP + b][lane] = T(RP*lane + a, RP*kb + b), so
    // a lane's loads are consecutive across the warp (no bank conflicts).
    // Accumulation order per row is the substitution order (columns
    // ascending for L, descending for U).
    // With K > 0 the leaf first applies the block solved before it,
    // X -= Aoff (jb x K) * Xp (K rows of the same columns), staged in the
    // same lane-major form -- the next-block update of a blocked sweep, done
    // where its result is consumed.
    constexpr int RP = L / 32;
    static_assert(RP * 32 == L, "leaf order must be a multiple of 32");
    if (bt.n > 0) {
        Tm += blockIdx.y * bt.t_step;
        X += blockIdx.y * bt.x_step;
        const int64_t left = bt.n - (int64_t)blockIdx.y * L;
        if (left < jb) jb = (int)left;
    }
    extern __shared__ __align__(16) unsigned char trsm_smem[];
    T* S = reinterpret_cast<T*>(trsm_smem);
    T* sD = S + L * L;  // U: reciprocals of the diagonal (zero beyond jb)
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const T zero{};
    if (UPPER && tid < L) sD[tid] = tid < jb ? cdiv(cone<T>(), Tm[tid + (int64_t)tid * ldt]) : zero;
    // Stage rows < nr, columns < nc of M (leading dimension ld) into S
    // lane-major -- all of it (part 0), the strict upper (1) or strict lower
    // (-1) triangle -- zero elsewhere; sixteen loads in flight per thread
    // before the shared-memory stores.  Lane slots are swizzled by the row
    // phase a (slot = lane ^ a*32/RP): the RP phases of a warp's consecutive
    // rows land in different banks, and a lane's reads stay a permutation of
    // the 32 slots.
    auto stage = [&](const T* M, int64_t ld, int nr, int nc, int part) {
        constexpr int kU = 16;
        for (int base = 0; base < L * L; base += kU * (int)blockDim.x) {
            T t[kU];
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int i = base + u * (int)blockDim.x + tid;
                const int r = i % L, c = i / L;
                const bool need = i < L * L && r < nr && c < nc && (part == 0 || (part > 0 ? r < c : r > c));
                t[u] = need ? M[r + (int64_t)c * ld] : zero;
            }
#pragma unroll
            for (int u = 0; u < kU; ++u) {
                const int i = base + u * (int)blockDim.x + tid;
                if (i < L * L) {
                    const int r = i % L, c = i / L;
                    S[((c / RP) * RP * RP + (r % RP) * RP + (c % RP)) * 32 + ((r / RP) ^ ((r % RP) * (32 / RP)))] = t[u];
                }
            }
        }
    };
    const int64_t col0 = ((int64_t)blockIdx.x * kTrsmWarps + warp) * NC;
    const bool active = col0 < ncols;  // (a whole warp; it stays for the barriers)
    bool cok[NC];
#pragma unroll
    for (int q = 0; q < NC; ++q) cok[q] = col0 + q < ncols;
    T v[NC][RP];
#pragma unroll
    for (int q = 0; q < NC; ++q)
#pragma unroll
        for (int a = 0; a < RP; ++a)
            v[q][a] = cok[q] && RP * lane + a < jb ? X[(col0 + q) * ldx + RP * lane + a] : zero;
    if (K > 0) {
        stage(Aoff, ldo, jb, K, 0);
        __syncthreads();
        if (active) {
            T xp[NC][RP];
#pragma unroll
            for (int q = 0; q < NC; ++q)
#pragma unroll
                for (int a = 0; a < RP; ++a)
                    xp[q][a] = cok[q] && RP * lane + a < K ? Xp[(col0 + q) * ldx + RP * lane + a] : zero;
            const int nkq = (K + RP - 1) / RP;
            for (int kb = 0; kb < nkq; ++kb) {
                const T* Sk = S + kb * RP * RP * 32;
                T xb[NC][RP];
#pragma unroll
                for (int q = 0; q < NC; ++q)
#pragma unroll
                    for (int b = 0; b < RP; ++b) xb[q][b] = shfl_c(xp[q][b], kb);
#pragma unroll
                for (int a = 0; a < RP; ++a)
#pragma unroll
                    for (int b = 0; b < RP; ++b) {
                        const T sab = Sk[(a * RP + b) * 32 + (lane ^ (a * (32 / RP)))];
#pragma unroll
                        for (int q = 0; q < NC; ++q) v[q][a] = v[q][a] - sab * xb[q][b];
                    }
            }
        }
        __syncthreads();  // S is the triangle's from here
    }
    // the strict triangle the solve reads
    stage(Tm, ldt, jb, jb, UPPER ? 1 : -1);
    __syncthreads();
    if (!active) return;  // whole warp leaves together
    const int nkb = (jb + RP - 1) / RP;
    if (!UPPER) {
        for (int kb = 0; kb < nkb; ++kb) {
            const T* Sk = S + kb * RP * RP * 32;
            T xb[NC][RP];
#pragma unroll
            for (int q = 0; q < NC; ++q)
#pragma unroll
                for (int b = 0; b < RP; ++b) xb[q][b] = zero;
            if (lane == kb) {
#pragma unroll
                for (int a = 0; a < RP; ++a) {
#pragma unroll
                    for (int q = 0; q < NC; ++q) {
                        T t = v[q][a];
#pragma unroll
                        for (int b = 0; b < a; ++b)
                            t = t - Sk[(a * RP + b) * 32 + (lane ^ (a * (32 / RP)))] * xb[q][b];
                        xb[q][a] = t;
                        v[q][a] = t;
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < NC; ++q)
#pragma unroll
                for (int b = 0; b < RP; ++b) xb[q][b] = shfl_c(xb[q][b], kb);
            if (lane > kb) {
#pragma unroll
                for (int a = 0; a < RP; ++a)
#pragma unroll
                    for (int b = 0; b < RP; ++b) {
                        const T sab = Sk[(a * RP + b) * 32 + (lane ^ (a * (32 / RP)))];
#pragma unroll
                        for (int q = 0; q < NC; ++q) v[q][a] = v[q][a] - sab * xb[q][b];
                    }
            }
        }
    } else {
        for (int kb = nkb - 1; kb >= 0; --kb) {
            const T* Sk = S + kb * RP * RP * 32;
            T xb[NC][RP];
#pragma unroll
            for (int q = 0; q < NC; ++q)
#pragma unroll
                for (int b = 0; b < RP; ++b) xb[q][b] = zero;
            if (lane == kb) {
#pragma unroll
                for (int a = RP - 1; a >= 0; --a) {
#pragma unroll
                    for (int q = 0; q < NC; ++q) {
                        T t = v[q][a];
#pragma unroll
                        for (int b = RP - 1; b > a; --b)
                            t = t - Sk[(a * RP + b) * 32 + (lane ^ (a * (32 / RP)))] * xb[q][b];
                        xb[q][a] = t * sD[RP * lane + a];
                        v[q][a] = xb[q][a];
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < NC; ++q)
#pragma unroll
                for (int b = 0; b < RP; ++b) xb[q][b] = shfl_c(xb[q][b], kb);
            if (lane < kb) {
#pragma unroll
                for (int a = 0; a < RP; ++a)
#pragma unroll
                    for (int b = RP - 1; b >= 0; --b) {
                        const T sab = Sk[(a * RP + b) * 32 + (lane ^ (a * (32 / RP)))];
#pragma unroll
                        for (int q = 0; q < NC; ++q) v[q][a] = v[q][a] - sab * xb[q][b];
                    }
            }
        }
    }
#pragma unroll
    for (int q = 0; q < NC; ++q)
        if (cok[q]) {
#pragma unroll
            for (int a = 0; a < RP; ++a)
                if (RP * lane + a < jb) X[(col0 + q) * ldx + RP * lane + a] = v[q][a];
        }
    if constexpr (std::is_same<T, cf>::value && RP % 2 == 0) {
        if (pk.b_hi != nullptr) {
            // rows RP*lane .. +RP-1 are real K rows kap0 + 2 RP lane .. (re, im
            // interleaved), whole 16-byte chunks; rows past jb carry zeros
#pragma unroll
            for (int q = 0; q < NC; ++q)
                if (cok[q]) {
#pragma unroll
                    for (int a = 0; a < RP; a += 2) {
                        const int64_t kap4 = pk.kap0 + 2 * (RP * lane + a);
                        if (kap4 < (int64_t)pk.b_nks * TC_KS)
                            tc_store_b4(pk.b_hi, pk.b_lo, pk.b_nks, col0 + q, kap4,
                                        make_float4(v[q][a].re, v[q][a].im, v[q][a + 1].re, v[q][a + 1].im));
                    }
                }
        }
    }
}

template <class T, int L>
constexpr size_t trsm_smem_bytes() {
    return sizeof(T) * (L * (L + 1) + L);
}

// columns at which a solve switches to four columns per warp: enough CTAs
// remain to cover the SMs twice
constexpr int64_t kTrsmWide = 4 * 8 * 2 * 148;

template <class T, int L, int NC>
static mw_status trsm_attr() {
    MW_CHECK_CUDA(cudaFuncSetAttribute(trsm_kernel<T, false, L, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)trsm_smem_bytes<T, L>()));
    MW_CHECK_CUDA(cudaFuncSetAttribute(trsm_kernel<T, true, L, NC>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)trsm_smem_bytes<T, L>()));
    return MW_OK;
}

template <class T>
static mw_status trsm_setup() {
    static bool done = false;
    if (!done) {
        constexpr int GL = GetrsLeaf<T>::value;
        mw_status s = trsm_attr<T, kNB, 1>();
        if (s == MW_OK) s = trsm_attr<T, kNB, 4>();
        if (s == MW_OK) s = trsm_attr<T, GL, 1>();
        if (s == MW_OK) s = trsm_attr<T, GL, 4>();
        if (s != MW_OK) return s;
        done = true;
    }
    return MW_OK;
}

template <class T, bool UPPER, int L = kNB>
static void trsm_launch(const T* Tm, int64_t ldt, T* X, int64_t ldx, int jb, int64_t ncols, cudaStream_t st,
                        const T* Aoff = nullptr, int64_t ldo = 0, const T* Xp = nullptr, int K = 0,
                        LeafPack pk = LeafPack{}, TrsmBatch bt = TrsmBatch{}, unsigned batch = 1) {
    ProfileScope ps(PC_TRSM, st, (4.0 * (double)jb * jb * ncols + 8.0 * (double)jb * K * ncols) * batch,
                    2.0 * sizeof(T) * (double)jb * ncols * batch);
    if (ncols >= kTrsmWide || batch > 1) {
        const int64_t per_cta = (int64_t)kTrsmWarps * 4;
        const dim3 grid((unsigned)((ncols + per_cta - 1) / per_cta), batch);
        trsm_kernel<T, UPPER, L, 4><<<grid, 32 * kTrsmWarps, trsm_smem_bytes<T, L>(), st>>>(
            Tm, ldt, X, ldx, jb, ncols, Aoff, ldo, Xp, K, pk, bt);
    } else {
        trsm_kernel<T, UPPER, L, 1><<<(unsigned)((ncols + kTrsmWarps - 1) / kTrsmWarps), 32 * kTrsmWarps,
                                      trsm_smem_bytes<T, L>(), st>>>(Tm, ldt, X, ldx, jb, ncols, Aoff, ldo, Xp, K,
                                                                     pk, bt);
    }
    count_launch();
}

template <class T>
static void laswp_launch(T* A, int64_t lda, int64_t col0, int64_t ncols, const int32_t* ipiv, int64_t k1, int64_t k2,
                         cudaStream_t st) {
    if (ncols <= 0) return;
    ProfileScope ps(PC_LASWP, st, 0.0, 4.0 * sizeof(T) * (double)(k2 - k1) * ncols);
    laswp_kernel<T><<<(unsigned)((ncols + 127) / 128), 128, 0, st>>>(A, lda, col0, ncols, ipiv, k1, k2);
    count_launch();
}

// --------------------------------------------------------------- FP64 GEMM
// C = alpha op(A) op(B) + beta C, complex128, column-major.  128 x 64 tile
// per CTA, 256 threads, 8 x 4 complex per thread; K staged 8 at a time
// through a two-slot shared-memory ring with register prefetch of the next
// slice while the current one is consumed.
constexpr int GM = 128, GN = 64, GK = 8;
constexpr size_t kZgemmSmem = sizeof(cd) * 2 * (GK * (GM + 1) + GK * (GN + 1));

template <bool TA, bool TB>
__global__ void __launch_bounds__(256) zgemm_kernel(int64_t m, int64_t n, int64_t k, cd alpha, const cd* __restrict__ A,
                                                    int64_t lda, const cd* __restrict__ B, int64_t ldb, cd beta,
                                                    cd* __restrict__ C, int64_t ldc) {
    extern __shared__ __align__(16) unsigned char zg_smem[];
    cd* sA0 = reinterpret_cast<cd*>(zg_smem);             // [2][GK][GM+1]
    cd* sB0 = sA0 + 2 * GK * (GM + 1);                     // [2][GK][GN+1]
    const int tid = threadIdx.x;
    const int64_t m0 = blockIdx.x * (int64_t)GM, n0 = blockIdx.y * (int64_t)GN;
    const int tx = tid % 16, ty = tid / 16;  // rows tx + 16*i, cols ty + 16*j
    constexpr int LA = GM * GK / 256, LB = GK * GN / 256;
    cd acc[8][4];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j] = cd{0.0, 0.0};

    cd ra[LA], rb[LB];
    auto fetch = [&](int64_t k0) {
#pragma unroll
        for (int u = 0; u < LA; ++u) {
            int i = tid + u * 256;
            int r = TA ? i / GK : i % GM;
            int kk = TA ? i % GK : i / GM;
            int64_t gr = m0 + r, gk = k0 + kk;
            ra[u] = (gr < m && gk < k) ? (TA ? A[gk + gr * lda] : A[gr + gk * lda]) : cd{0.0, 0.0};
        }
#pragma unroll
        for (int u = 0; u < LB; ++u) {
            int i = tid + u * 256;
            int kk = TB ? i / GN : i % GK;
            int cc = TB ? i % GN : i / GK;
            int64_t gk = k0 + kk, gc = n0 + cc;
            rb[u] = (gk < k && gc < n) ? (TB ? B[gc + gk * ldb] : B[gk + gc * ldb]) : cd{0.0, 0.0};
        }
    };
    auto stash = [&](int slot) {
        cd* sA = sA0 + slot * GK * (GM + 1);
        cd* sB = sB0 + slot * GK * (GN + 1);
#pragma unroll
        for (int u = 0; u < LA; ++u) {
            int i = tid + u * 256;
            int r = TA ? i / GK : i % GM;
            int kk = TA ? i % GK : i / GM;
            sA[kk * (GM + 1) + r] = ra[u];
        }
#pragma unroll
        for (int u = 0; u < LB; ++u) {
            int i = tid + u * 256;
            int kk = TB ? i / GN : i % GK;
            int cc = TB ? i % GN : i / GK;
            sB[kk * (GN + 1) + cc] = rb[u];
        }
    };

    fetch(0);
    stash(0);
    __syncthreads();
    int slot = 0;
    for (int64_t k0 = 0; k0 < k; k0 += GK) {
        const bool more = k0 + GK < k;
        if (more) fetch(k0 + GK);
        const cd* sA = sA0 + slot * GK * (GM + 1);
        const cd* sB = sB0 + slot * GK * (GN + 1);
#pragma unroll
        for (int kk = 0; kk < GK; ++kk) {
            cd a[8], b[4];
#pragma unroll
            for (int i = 0; i < 8; ++i) a[i] = sA[kk * (GM + 1) + tx + 16 * i];
#pragma unroll
            for (int j = 0; j < 4; ++j) b[j] = sB[kk * (GN + 1) + ty + 16 * j];
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
        if (more) stash(slot ^ 1);
        __syncthreads();
        slot ^= 1;
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

// FP64 tensor path (sm_100 has no tcgen05 kind for fp64; DMMA
// mma.sync.m8n8k4.f64 is the fp64 tensor route).  CTA tile 128 x 64
// complex, 8 warps as 4 (M) x 2 (N), warp tile 32 x 32 complex = 4 x 4
// blocks of 8 x 8.  Each block takes three real MMAs per k-step of 4
// (the 3M product):
//   X += Ar Br,  Y += Ai Bi,  W += (Ar + Ai)(Br + Bi);  Cr = X - Y,  Ci = W - X - Y
// -- a quarter fewer MMAs than the four-product form, at an error bound on
// each part of a few units of 2^-53 times sum |A||B|, far below what the
// complex64 refinement needs of its residual.  K is staged 16 complex at a
// time through a three-slot shared-memory ring filled by cp.async (no
// staging registers: the three accumulator sets need them).
constexpr int DM_M = 128, DM_N = 64, DM_K = 16, DM_STAGES = 3;
constexpr int DM_PA = DM_M + 2;   // sA[kk][row] row stride (complex): the 4 kk rows of a load fall on distinct banks
constexpr int DM_PB = DM_K + 4;   // sB[col][kk] stride (complex): 8 columns x 4 kk of a load on distinct banks
constexpr int DM_SA = DM_K * DM_PA, DM_SB = DM_N * DM_PB;  // per slot
constexpr size_t kDmmaSmem = sizeof(cd) * DM_STAGES * (DM_SA + DM_SB);

__device__ __forceinline__ void dmma(double& d0, double& d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// 16-byte global -> shared copy; zero-filled when !valid (src then unread)
__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(s), "l"(src), "r"(valid ? 16 : 0) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// The last, partial wave of output tiles may be split along K (chosen by
// zgemm_launch): tiles [0, full) are computed whole; every tile from `full`
// on is cut into `splits` K chunks of whole DM_K steps, one work unit each.
// A chunk's partial sum goes to `part` in the threads' fragment order; the
// unit that brings its tile's count to `splits` adds the chunks in chunk
// order (the same sum whichever unit finishes last), applies alpha and beta,
// writes C and resets the count to zero for the next launch.  No unit waits
// on another.
struct DmSplit {
    unsigned int* count;  // one per split tile, zero between launches
    cd* part;             // [split tiles * splits][DM_M * DM_N]
    int64_t full;
    int splits;
};
constexpr int kDmSplitMaxUnits = 256;
constexpr size_t kDmSplitCountBytes = sizeof(unsigned int) * kDmSplitMaxUnits;

template <bool TA, bool TB>
__global__ void __launch_bounds__(256, 1) zgemm_dmma_kernel(int64_t m, int64_t n, int64_t k, cd alpha,
                                                            const cd* __restrict__ A, int64_t lda,
                                                            const cd* __restrict__ B, int64_t ldb, cd beta,
                                                            cd* __restrict__ C, int64_t ldc, DmSplit split) {
    extern __shared__ __align__(16) unsigned char dm_smem[];
    __shared__ int s_last;
    cd* sA0 = reinterpret_cast<cd*>(dm_smem);  // [DM_STAGES][DM_K][DM_PA]
    cd* sB0 = sA0 + DM_STAGES * DM_SA;         // [DM_STAGES][DM_N][DM_PB]
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wm = warp & 3, wn = warp >> 2;
    const int gid = lane >> 2, tig = lane & 3;
    constexpr int LA = DM_M * DM_K / 256, LB = DM_K * DM_N / 256;
    // persistent over the work units (the grid may be capped to leave SMs
    // to a concurrent kernel)
    const int64_t n_mt = (m + DM_M - 1) / DM_M;
    const int64_t n_tiles = n_mt * ((n + DM_N - 1) / DM_N);
    const int64_t n_units = split.full + (n_tiles - split.full) * split.splits;
    const int64_t kchunk = ((k + DM_K - 1) / DM_K + split.splits - 1) / split.splits * DM_K;
    for (int64_t unit = blockIdx.x; unit < n_units; unit += gridDim.x) {
    int64_t tile = unit, kb = 0, ke = k;
    int chunk = -1;
    if (unit >= split.full) {
        const int64_t v = unit - split.full;
        tile = split.full + v / split.splits;
        chunk = (int)(v % split.splits);
        kb = chunk * kchunk;
        ke = kb + kchunk < k ? kb + kchunk : k;
    }
    const int64_t m0 = (tile % n_mt) * DM_M, n0 = (tile / n_mt) * DM_N;
    double x[4][4][2], y[4][4][2], w[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) x[i][j][h] = y[i][j][h] = w[i][j][h] = 0.0;

    // stage K columns [k0, k0 + DM_K) of the tile into `slot`
    auto load = [&](int slot, int64_t k0) {
        cd* sA = sA0 + slot * DM_SA;
        cd* sB = sB0 + slot * DM_SB;
#pragma unroll
        for (int u = 0; u < LA; ++u) {
            const int i = tid + u * 256;
            const int r = TA ? i / DM_K : i % DM_M;
            const int kk = TA ? i % DM_K : i / DM_M;
            const int64_t gr = m0 + r, gk = k0 + kk;
            const bool ok = gr < m && gk < ke;
            cp_async16(sA + kk * DM_PA + r, ok ? (TA ? A + gk + gr * lda : A + gr + gk * lda) : A, ok);
        }
#pragma unroll
        for (int u = 0; u < LB; ++u) {
            const int i = tid + u * 256;
            const int kk = TB ? i / DM_N : i % DM_K;
            const int cc = TB ? i % DM_N : i / DM_K;
            const int64_t gk = k0 + kk, gc = n0 + cc;
            const bool ok = gk < ke && gc < n;
            cp_async16(sB + cc * DM_PB + kk, ok ? (TB ? B + gc + gk * ldb : B + gk + gc * ldb) : B, ok);
        }
    };

    const int64_t nk = kb < ke ? (ke - kb + DM_K - 1) / DM_K : 0;  // K steps of this unit
#pragma unroll
    for (int s = 0; s < DM_STAGES - 1; ++s) {
        if (s < nk) load(s, kb + s * DM_K);
        cp_async_commit();
    }
    for (int64_t t = 0; t < nk; ++t) {
        cp_async_wait<DM_STAGES - 2>();  // step t has landed
        __syncthreads();                  // and every warp is done with step t - 1's slot
        const int64_t tn = t + DM_STAGES - 1;
        if (tn < nk) load((int)(tn % DM_STAGES), kb + tn * DM_K);
        cp_async_commit();
        const int slot = (int)(t % DM_STAGES);
        const cd* sA = sA0 + slot * DM_SA;
        const cd* sB = sB0 + slot * DM_SB;
#pragma unroll
        for (int k4 = 0; k4 < DM_K; k4 += 4) {
            double ar[4], ai[4], as[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const cd a = sA[(k4 + tig) * DM_PA + wm * 32 + i * 8 + gid];
                ar[i] = a.re;
                ai[i] = a.im;
                as[i] = a.re + a.im;
            }
#pragma unroll
            for (int j = 0; j < 4; ++j) {
                const cd b = sB[(wn * 32 + j * 8 + gid) * DM_PB + k4 + tig];
                const double bs = b.re + b.im;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    dmma(x[i][j][0], x[i][j][1], ar[i], b.re);
                    dmma(y[i][j][0], y[i][j][1], ai[i], b.im);
                    dmma(w[i][j][0], w[i][j][1], as[i], bs);
                }
            }
        }
    }
    cp_async_wait<0>();
    __syncthreads();  // the ring is free for the next unit
    // Cr = X - Y into x, Ci = W - X - Y into w
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const double xv = x[i][j][h], yv = y[i][j][h];
                x[i][j][h] = xv - yv;
                w[i][j][h] -= xv + yv;
            }
    const bool beta_zero = (beta.re == 0.0 && beta.im == 0.0);
    if (chunk >= 0) {
        // partial sum of a split tile: element e of this thread at e * 256 + tid
        const int64_t st = tile - split.full;
        cd* P = split.part + (st * split.splits + chunk) * (DM_M * DM_N);
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int h = 0; h < 2; ++h) P[((i * 4 + j) * 2 + h) * 256 + tid] = cd{x[i][j][h], w[i][j][h]};
        __threadfence();
        __syncthreads();
        if (tid == 0) s_last = atomicAdd(split.count + st, 1u) == (unsigned)split.splits - 1;
        __syncthreads();
        if (!s_last) continue;
        __threadfence();
        const cd* P0 = split.part + st * split.splits * (DM_M * DM_N);
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
            for (int j = 0; j < 4; ++j)
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    double sr = 0.0, si = 0.0;
                    for (int c = 0; c < split.splits; ++c) {
                        const double2 v = __ldcg(reinterpret_cast<const double2*>(
                            P0 + (int64_t)c * (DM_M * DM_N) + ((i * 4 + j) * 2 + h) * 256 + tid));
                        sr += v.x;
                        si += v.y;
                    }
                    x[i][j][h] = sr;
                    w[i][j][h] = si;
                }
        if (tid == 0) split.count[st] = 0u;
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int64_t gr = m0 + wm * 32 + i * 8 + gid;
        if (gr >= m) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int64_t gc = n0 + wn * 32 + j * 8 + 2 * tig + h;
                if (gc >= n) continue;
                cd v = alpha * cd{x[i][j][h], w[i][j][h]};
                cd* cp = C + gr + gc * ldc;
                if (!beta_zero) v = v + beta * (*cp);
                *cp = v;
            }
    }
    }  // units
}

mw_status zgemm_launch_simt(bool ta, bool tb, int64_t m, int64_t n, int64_t k, cd alpha, const cd* A, int64_t lda,
                            const cd* B, int64_t ldb, cd beta, cd* C, int64_t ldc, cudaStream_t st);

// Workspace for splitting the DMMA kernel's last wave of an m x n product
// along K: the tile counts, then one partial tile per work unit.
size_t zgemm_split_ws_bytes(int64_t m, int64_t n) {
    const int64_t tiles = ((m + DM_M - 1) / DM_M) * ((n + DM_N - 1) / DM_N);
    const int64_t units = 16 * tiles < kDmSplitMaxUnits ? 16 * tiles : kDmSplitMaxUnits;
    return kDmSplitCountBytes + (size_t)units * DM_M * DM_N * sizeof(cd);
}

mw_status zgemm_split_ws_init(void* split_ws, cudaStream_t st) {
    MW_CHECK_CUDA(cudaMemsetAsync(split_ws, 0, kDmSplitCountBytes, st));
    return MW_OK;
}

static int dmma_sms() {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms < 1) sms = 1;
    }
    return sms;
}

// Shape dispatch (measured on B200, 16x16 dipole array): the register-tiled
// DFMA kernel wins on the LU's rank-64 updates (16.4 vs 13.8 TFLOP/s: short
// K, epilogue-bound), the DMMA kernel on long-K products such as the
// refinement residual Z X (14.4 vs 9.6 TFLOP/s).  The DMMA kernel runs one
// CTA per SM over its tiles; given a workspace (zgemm_split_ws_bytes, counts
// zeroed once), a last wave that would leave SMs idle is split along K so
// that it fills them: the residual of the 16x16 array has 328 tiles on 148
// SMs, 2 whole waves and 32 tiles cut into 4 chunks each.
mw_status zgemm_launch(bool ta, bool tb, int64_t m, int64_t n, int64_t k, cd alpha, const cd* A, int64_t lda,
                       const cd* B, int64_t ldb, cd beta, cd* C, int64_t ldc, cudaStream_t st, int max_ctas,
                       void* split_ws, size_t split_ws_bytes) {
    if (m <= 0 || n <= 0) return MW_OK;
    if (k < 128) return zgemm_launch_simt(ta, tb, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, st);
    {
        static bool attr = false;
        if (!attr) {
            MW_CHECK_CUDA(cudaFuncSetAttribute(zgemm_dmma_kernel<false, false>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDmmaSmem));
            MW_CHECK_CUDA(cudaFuncSetAttribute(zgemm_dmma_kernel<true, false>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDmmaSmem));
            MW_CHECK_CUDA(cudaFuncSetAttribute(zgemm_dmma_kernel<false, true>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDmmaSmem));
            MW_CHECK_CUDA(cudaFuncSetAttribute(zgemm_dmma_kernel<true, true>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDmmaSmem));
            attr = true;
        }
        // one CTA per SM (register-bound); a cap leaves SMs to other work
        const int64_t tiles = ((m + DM_M - 1) / DM_M) * ((n + DM_N - 1) / DM_N);
        int64_t ctas = dmma_sms();
        if (max_ctas > 0 && ctas > max_ctas) ctas = max_ctas;
        DmSplit split{nullptr, nullptr, tiles, 1};
        const int64_t tail = tiles % ctas;
        if (split_ws && tail > 0 && split_ws_bytes > kDmSplitCountBytes) {
            const int64_t room = (int64_t)((split_ws_bytes - kDmSplitCountBytes) / (DM_M * DM_N * sizeof(cd)));
            int64_t s = ctas / tail;
            const int64_t ksteps = (k + DM_K - 1) / DM_K;
            if (s > ksteps) s = ksteps;
            if (tail * s > room) s = room / tail;
            if (tail * s > kDmSplitMaxUnits) s = kDmSplitMaxUnits / tail;
            if (s >= 2) s = (ksteps + (ksteps + s - 1) / s - 1) / ((ksteps + s - 1) / s);  // no empty chunk
            if (s >= 2) {
                split.count = static_cast<unsigned int*>(split_ws);
                split.part = reinterpret_cast<cd*>(static_cast<char*>(split_ws) + kDmSplitCountBytes);
                split.full = tiles - tail;
                split.splits = (int)s;
            }
        }
        const int64_t units = split.full + (tiles - split.full) * split.splits;
        dim3 grid((unsigned)(units < ctas ? units : ctas));
        ProfileScope ps(PC_ZGEMM, st, 8.0 * (double)m * n * k, 16.0 * ((double)m * k + (double)k * n + 2.0 * m * n));
        if (!ta && !tb)
            zgemm_dmma_kernel<false, false><<<grid, 256, kDmmaSmem, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                             split);
        else if (ta && !tb)
            zgemm_dmma_kernel<true, false><<<grid, 256, kDmmaSmem, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                             split);
        else if (!ta && tb)
            zgemm_dmma_kernel<false, true><<<grid, 256, kDmmaSmem, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                             split);
        else
            zgemm_dmma_kernel<true, true><<<grid, 256, kDmmaSmem, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc,
                                                                             split);
        MW_CHECK_CUDA(cudaGetLastError());
        count_launch();
        return MW_OK;
    }
}

// The register-tiled DFMA kernel: the products with k < 128 (the FP64
// panels' half-width updates, a KCL Schur step with few constraint rows).
mw_status zgemm_launch_simt(bool ta, bool tb, int64_t m, int64_t n, int64_t k, cd alpha, const cd* A, int64_t lda,
                            const cd* B, int64_t ldb, cd beta, cd* C, int64_t ldc, cudaStream_t st) {
    if (m <= 0 || n <= 0) return MW_OK;
    static bool attr = false;
    if (!attr) {
        MW_CHECK_CUDA(cudaFuncSetAttribute(zgemm_kernel<false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kZgemmSmem));
        MW_CHECK_CUDA(cudaFuncSetAttribute(zgemm_kernel<true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kZgemmSmem));
        MW_CHECK_CUDA(cudaFuncSetAttribute(zgemm_kernel<false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kZgemmSmem));
        MW_CHECK_CUDA(cudaFuncSetAttribute(zgemm_kernel<true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kZgemmSmem));
        attr = true;
    }
    dim3 grid((unsigned)((m + GM - 1) / GM), (unsigned)((n + GN - 1) / GN));
    ProfileScope ps(PC_ZGEMM, st, 8.0 * (double)m * n * k, 16.0 * ((double)m * k + (double)k * n + 2.0 * m * n));
    if (!ta && !tb) zgemm_kernel<false, false><<<grid, 256, kZgemmSmem, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else if (ta && !tb) zgemm_kernel<true, false><<<grid, 256, kZgemmSmem, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else if (!ta && tb) zgemm_kernel<false, true><<<grid, 256, kZgemmSmem, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    else zgemm_kernel<true, true><<<grid, 256, kZgemmSmem, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc);
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

// --------------------------------------------------------------- driver
constexpr size_t kPanelSmemMax = 192 * 1024;  // slab bytes per CTA (beside 34 KB of static buffers)

template <class T>
static int panel_sms() {
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        cudaFuncSetAttribute(panel_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelSmemMax);
        cudaFuncSetAttribute(panel_kernel_c64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kPanelSmemMax);
        if (sms < 1) sms = 1;
    }
    return sms;
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
    o += sizeof(cd) * 2 * (size_t)G * kPanelMaxJb;
    o = (o + 255) & ~size_t(255);
    *off_cur = o;
    o += sizeof(cd) * 2 * kPanelMaxJb;
    return (o + 255) & ~size_t(255);
}

constexpr int kMaxPanelGrid = 1024;

// Trailing update C -= A B of a block (type-specific engine).
struct Updater {
    // complex64 only: tensor-core workspace and the CTAs an update may hold
    void* tc_ws = nullptr;
    size_t tc_ws_bytes = 0;
    int* tc_err = nullptr;
    int max_ctas = 0;
    int64_t ws_m = 0, ws_n = 0;  // the largest update the workspace was laid out for (k = kOuterNB)
};

static mw_status block_update(const cd* A, int64_t lda, const cd* B, int64_t ldb, cd* C, int64_t ldc, int64_t m,
                              int64_t n, int64_t k, const Updater& u, cudaStream_t st) {
    return zgemm_launch(false, false, m, n, k, cd{-1.0, 0.0}, A, lda, B, ldb, cd{1.0, 0.0}, C, ldc, st, u.max_ctas,
                        nullptr, 0);
}

// C -= A B from operands already in the updater's planes (complex64).
template <class T>
static mw_status update_prepacked(int64_t m, int64_t n, int64_t k, const TcPlanes& pl, T* C, int64_t ldc,
                                  const Updater& u, cudaStream_t st) {
    if constexpr (std::is_same<T, cf>::value) {
        MW_REQUIRE(m <= u.ws_m && n <= u.ws_n && k <= kOuterNB, "prepacked update larger than its planes");
        return cgemm_tc_prepacked(m, n, k, pl, C, ldc, u.tc_err, st, u.max_ctas);
    } else {
        (void)m, (void)n, (void)k, (void)pl, (void)C, (void)ldc, (void)u, (void)st;
        set_error("prepacked update is complex64 only");
        return MW_ERR_INVALID;
    }
}

static mw_status block_update(const cf* A, int64_t lda, const cf* B, int64_t ldb, cf* C, int64_t ldc, int64_t m,
                              int64_t n, int64_t k, const Updater& u, cudaStream_t st) {
    return cgemm_tc_update(m, n, k, A, lda, B, ldb, C, ldc, u.tc_ws, u.tc_ws_bytes, u.tc_err, st, u.max_ctas);
}

// X <- L^-1 X for a unit lower triangle of any order, in kNB-row diagonal
// blocks: each leaf applies the block just before it itself (the leaf
// kernel's fused update), blocks further back -- orders above 2 kNB only --
// reach it through one block update.
template <class T>
static mw_status trsm_lower_blocked(const T* L, int64_t ldl, T* X, int64_t ldx, int jb, int64_t ncols,
                                    const Updater& up, cudaStream_t st, const TcPlanes* pack = nullptr) {
    // with `pack` (complex64, jb <= 2 kNB) the solved rows are also written
    // as the packed B operand of the update with inner dimension jb
    for (int b0 = 0; b0 < jb; b0 += kNB) {
        const int bb = (jb - b0) < kNB ? (jb - b0) : kNB;
        LeafPack pk;
        if (pack != nullptr) {
            pk.b_hi = pack->b_hi;
            pk.b_lo = pack->b_lo;
            pk.b_nks = tc_n_ks(jb);
            pk.kap0 = 2 * b0;
        }
        if (b0 >= 2 * kNB) {
            const int k = b0 - kNB;  // blocks 0 .. b0-kNB-1
            mw_status s = block_update(L + b0, ldl, X, ldx, X + b0, ldx, bb, ncols, k, up, st);
            if (s != MW_OK) return s;
        }
        if (b0 == 0) {
            trsm_launch<T, false>(L, ldl, X, ldx, bb, ncols, st, nullptr, 0, nullptr, 0, pk);
        } else {
            const int p0 = b0 - kNB;
            trsm_launch<T, false>(L + b0 + (int64_t)b0 * ldl, ldl, X + b0, ldx, bb, ncols, st,
                                  L + b0 + (int64_t)p0 * ldl, ldl, X + p0, kNB, pk);
        }
    }
    return MW_OK;
}

// Factor the panel rows [j0, n) x columns [j0, j0+jb) with partial pivoting.
// One cooperative launch when every CTA's row slab fits in shared memory;
// otherwise split the columns in two and recurse (left half, then update and
// factor the right half, then apply the right half's swaps to the left).
template <class T>
static mw_status panel_factor(T* A, int64_t lda, int64_t n, int64_t j0, int jb, int32_t* ipiv, int32_t* info, char* ws,
                              const Updater& up, cudaStream_t st, int grid_cap = 0) {
    const int sms = panel_sms<T>();
    const int64_t m = n - j0;
    // fewer, fatter CTAs: the per-column grid barrier costs grow with the
    // number of participants, the per-CTA work is small either way
    int64_t want = (m + 127) / 128;  // at least 128 rows per CTA
    int G = (int)(want < sms ? want : sms);
    if (grid_cap > 0 && G > grid_cap) G = grid_cap;
    if (G > kMaxPanelGrid) G = kMaxPanelGrid;
    // the complex64 kernel reads every CTA's candidate row each column
    if (std::is_same<T, cf>::value && G > kC64MaxGrid) G = kC64MaxGrid;
    if (G < 1) G = 1;
    const int64_t per = (m + G - 1) / G;
    const size_t smem = (size_t)per * jb * sizeof(T);
    // panels wider than kNB are factored as two halves (the per-column
    // rank-1 work stays kNB wide; the halves meet in one small update)
    if (smem > kPanelSmemMax || jb > kNB) {
        MW_REQUIRE(jb > 1, "matrix too large for the panel kernel (%lld rows per CTA)", (long long)per);
        const int h = jb / 2;
        mw_status s = panel_factor<T>(A, lda, n, j0, h, ipiv, info, ws, up, st, grid_cap);
        if (s != MW_OK) return s;
        laswp_launch<T>(A, lda, j0 + h, jb - h, ipiv, j0, j0 + h, st);
        trsm_launch<T, false>(A + j0 + j0 * lda, lda, A + j0 + (j0 + h) * lda, lda, h, jb - h, st);
        s = block_update(A + (j0 + h) + j0 * lda, lda, A + j0 + (j0 + h) * lda, lda, A + (j0 + h) + (j0 + h) * lda,
                         lda, m - h, jb - h, h, up, st);
        if (s != MW_OK) return s;
        s = panel_factor<T>(A, lda, n, j0 + h, jb - h, ipiv, info, ws, up, st, grid_cap);
        if (s != MW_OK) return s;
        laswp_launch<T>(A, lda, j0, h, ipiv, j0 + h, j0 + jb, st);
        MW_CHECK_CUDA(cudaGetLastError());
        return MW_OK;
    }
    size_t ov, oi, orow, ocur;
    // fixed offsets (sized for the largest grid): a CTA's exchange slot stays
    // at one address for the whole factorisation
    ws_layout(kMaxPanelGrid, &ov, &oi, &orow, &ocur);
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
    P.slot_row = ws + orow;
    P.cur_row = ws + ocur;
    void* args[] = {&P};
    {
        ProfileScope ps(PC_PANEL, st, 4.0 * (double)m * jb * jb, 2.0 * sizeof(T) * (double)m * jb);
        void* kern = std::is_same<T, cf>::value ? (void*)panel_kernel_c64 : (void*)panel_kernel<T>;
        MW_CHECK_CUDA(cudaLaunchCooperativeKernel(kern, dim3(G), dim3(kPanelThreads), args, smem, st));
    }
    count_launch();
    return MW_OK;
}

// Right-looking blocked LU of an n x n column-major matrix.
template <class T>
static mw_status getrf(int64_t n, T* A, int64_t lda, int32_t* ipiv, int32_t* info, char* ws,
                       const volatile int32_t* cancel, const Updater& up, cudaStream_t st) {
    MW_CHECK_CUDA(cudaMemsetAsync(info, 0, 2 * sizeof(int32_t), st));
    MW_CHECK_CUDA(cudaMemsetAsync(ws, 0, sizeof(PanelWs), st));
    {
        size_t ov, oi, orow, ocur;
        ws_layout(kMaxPanelGrid, &ov, &oi, &orow, &ocur);
        MW_CHECK_CUDA(cudaMemsetAsync(ws + oi, 0, sizeof(int64_t) * 2 * kMaxPanelGrid, st));
        // and the complex64 panel's tagged records (no tag from an earlier
        // factorisation may match)
        MW_CHECK_CUDA(cudaMemsetAsync(ws + orow, 0, sizeof(unsigned long long) * 2 * 2 * kC64RecStride, st));
    }
    {
        mw_status s0 = trsm_setup<T>();
        if (s0 != MW_OK) return s0;
    }
    PanelWs* pws = reinterpret_cast<PanelWs*>(ws);
    for (int64_t j0 = 0; j0 < n; j0 += kOuterNB) {
        if (cancel && *cancel) {
            set_error("factorisation cancelled");
            return MW_ERR_CANCELLED;
        }
        const int jb = (int)((n - j0) < kOuterNB ? (n - j0) : kOuterNB);
        mw_status s = panel_factor<T>(A, lda, n, j0, jb, ipiv, info, ws, up, st);
        if (s != MW_OK) return s;
        const int64_t left = j0, right = n - j0 - jb;
        laswp_launch<T>(A, lda, 0, left, ipiv, j0, j0 + jb, st);
        if (right > 0) {
            laswp_launch<T>(A, lda, j0 + jb, right, ipiv, j0, j0 + jb, st);
            T* A11 = A + j0 + j0 * lda;
            T* A12 = A + j0 + (j0 + jb) * lda;
            trsm_lower_blocked<T>(A11, lda, A12, lda, jb, right, up, st);
            s = block_update(A + (j0 + jb) + j0 * lda, lda, A12, lda, A + (j0 + jb) + (j0 + jb) * lda, lda, right, right,
                             jb, up, st);
            if (s != MW_OK) return s;
        }
        MW_CHECK_CUDA(cudaGetLastError());
    }
    // a barrier timeout anywhere is reported in info[1]
    MW_CHECK_CUDA(cudaMemcpyAsync(info + 1, &pws->err, sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    return MW_OK;
}

// ------------------------------------------------------------ look-ahead
// Right-looking LU with a look-ahead of one block (both precisions).
// The factorisation splits into two streams:
//   main   panel j (<= kLaPanelCtas CTAs), then the update of block j+1's
//          columns only (a narrow GEMM on as many CTAs), so that panel j+1
//          can start at once; the panels' row swaps on the columns left of
//          them are applied at the end, in panel order (the trail stream
//          still reads the previous panel's rows while the next one runs);
//   trail  the row swaps, triangular solve and tensor-core update of every
//          column right of block j+1, on the remaining SMs.
// Panel j waits only for trail j-2 (the last update that touched its
// columns), so each panel runs under the previous block's big update.  The
// two streams use separate packed-operand workspaces; events order them.
constexpr int kLaPanelCtas = 32;

// SMs the complex64 factorisation's critical chain keeps free of the bulk
// updates: kLaPanelCtas, or $MOMWIRE_B200_MAIN_SMS (8 .. 120) for tuning.
static int main_sms() {
    static int v = -1;
    if (v < 0) {
        v = kLaPanelCtas;
        if (const char* e = getenv("MOMWIRE_B200_MAIN_SMS")) {
            const int x = atoi(e);
            if (x >= 8 && x <= 120) v = x;
        }
    }
    return v;
}

struct AuxStreams {
    cudaStream_t trail = nullptr;
    cudaStream_t critical = nullptr;  // highest priority: the chain the other stream feeds
    cudaEvent_t ev_main = nullptr;  // main -> trail
    cudaEvent_t ev_trail[4] = {};   // trail j -> main (ring)
    cudaEvent_t ev_handover = nullptr, ev_back = nullptr;  // caller <-> critical
};

// one set per host thread and device: concurrent factorisations from
// different threads never share the trail stream or its events
static mw_status aux_streams(AuxStreams** out) {
    static thread_local AuxStreams per_dev[64];
    int dev = 0;
    MW_CHECK_CUDA(cudaGetDevice(&dev));
    MW_REQUIRE(dev >= 0 && dev < 64, "device index out of range");
    AuxStreams& a = per_dev[dev];
    if (!a.trail) {
        int least = 0, greatest = 0;
        MW_CHECK_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        MW_CHECK_CUDA(cudaStreamCreateWithFlags(&a.trail, cudaStreamNonBlocking));
        MW_CHECK_CUDA(cudaStreamCreateWithPriority(&a.critical, cudaStreamNonBlocking, greatest));
        MW_CHECK_CUDA(cudaEventCreateWithFlags(&a.ev_main, cudaEventDisableTiming));
        for (auto& e : a.ev_trail) MW_CHECK_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        MW_CHECK_CUDA(cudaEventCreateWithFlags(&a.ev_handover, cudaEventDisableTiming));
        MW_CHECK_CUDA(cudaEventCreateWithFlags(&a.ev_back, cudaEventDisableTiming));
    }
    *out = &a;
    return MW_OK;
}

// The critical chain of a two-stream routine (panels, leaves) runs on the
// highest-priority stream, so that the CTA scheduler hands it the first SMs
// that free up while the bulk updates fill the rest: the caller's stream
// hands over (everything queued on it first) ...
static mw_status critical_begin(AuxStreams* ax, cudaStream_t caller, cudaStream_t* out) {
    MW_CHECK_CUDA(cudaEventRecord(ax->ev_handover, caller));
    MW_CHECK_CUDA(cudaStreamWaitEvent(ax->critical, ax->ev_handover, 0));
    *out = ax->critical;
    return MW_OK;
}

// ... and waits for it at the end.
static mw_status critical_end(AuxStreams* ax, cudaStream_t caller) {
    MW_CHECK_CUDA(cudaEventRecord(ax->ev_back, ax->critical));
    MW_CHECK_CUDA(cudaStreamWaitEvent(caller, ax->ev_back, 0));
    return MW_OK;
}

template <class T>
static mw_status getrf_lookahead(int64_t n, T* A, int64_t lda, int32_t* ipiv, int32_t* info, char* ws,
                                 const volatile int32_t* cancel, const Updater& up_main, const Updater& up_trail,
                                 cudaStream_t st, T* Baug = nullptr, int64_t ldb = 0, int64_t nrhs = 0,
                                 int32_t* perm_all = nullptr) {
    // static pivots when the caller passes room for every block's row order
    const bool static_pivot = perm_all != nullptr;
    MW_CHECK_CUDA(cudaMemsetAsync(info, 0, 2 * sizeof(int32_t), st));
    MW_CHECK_CUDA(cudaMemsetAsync(ws, 0, sizeof(PanelWs), st));
    {
        // the panel exchange words start cleared (no stale sequence number)
        size_t ov, oi, orow, ocur;
        ws_layout(kMaxPanelGrid, &ov, &oi, &orow, &ocur);
        MW_CHECK_CUDA(cudaMemsetAsync(ws + oi, 0, sizeof(int64_t) * 2 * kMaxPanelGrid, st));
        // and the complex64 panel's tagged records (no tag from an earlier
        // factorisation may match)
        MW_CHECK_CUDA(cudaMemsetAsync(ws + orow, 0, sizeof(unsigned long long) * 2 * 2 * kC64RecStride, st));
    }
    {
        mw_status s0 = trsm_setup<T>();
        if (s0 != MW_OK) return s0;
    }
    AuxStreams* ax = nullptr;
    {
        mw_status s0 = aux_streams(&ax);
        if (s0 != MW_OK) return s0;
    }
    cudaStream_t tr = ax->trail;
    PanelWs* pws = reinterpret_cast<PanelWs*>(ws);
    const int64_t nb = (n + kOuterNB - 1) / kOuterNB;
    const cudaStream_t caller = st;
    {
        mw_status s0 = critical_begin(ax, caller, &st);
        if (s0 != MW_OK) return s0;
    }
    // the trail stream starts after everything already queued on st
    MW_CHECK_CUDA(cudaEventRecord(ax->ev_main, st));
    MW_CHECK_CUDA(cudaStreamWaitEvent(tr, ax->ev_main, 0));
    for (int64_t j = 0; j < nb; ++j) {
        if (cancel && *cancel) {
            // let both streams finish what they were given before returning
            MW_CHECK_CUDA(cudaStreamSynchronize(tr));
            MW_CHECK_CUDA(cudaStreamSynchronize(st));
            set_error("factorisation cancelled");
            return MW_ERR_CANCELLED;
        }
        const int64_t j0 = j * kOuterNB;
        const int jb = (int)((n - j0) < kOuterNB ? (n - j0) : kOuterNB);
        if (j >= 2) MW_CHECK_CUDA(cudaStreamWaitEvent(st, ax->ev_trail[(j - 2) & 3], 0));
        mw_status s;
        // static pivots: the block's interchanges never leave it, so they
        // reach the columns beside it as one parallel row permutation (each
        // block's row order kept, for the columns left of it at the end)
        int32_t* perm = nullptr;
        // static pivots, complex64: the panel's L21 and each solved block
        // row are written straight into the tensor-core operand planes, so
        // the updates run without a packing pass.  L21 of even panels lives
        // in the trail updater's A planes, of odd ones in the main
        // updater's: panel j + 2 overwrites them only after trail j, the
        // last reader, has finished (the wait on ev_trail above).
        bool prepacked = false;
        TcPlanes pl_main{}, pl_trail{};
        if constexpr (std::is_same<T, cf>::value) {
            if (static_pivot) {
                size_t ov, oi, orow, ocur;
                ws_layout(kMaxPanelGrid, &ov, &oi, &orow, &ocur);
                perm = perm_all + j0;
                prepacked = up_main.tc_ws != nullptr && up_trail.tc_ws != nullptr && jb == kOuterNB;
                if (prepacked) {
                    pl_main = tc_planes(up_main.tc_ws, up_main.ws_m, up_main.ws_n, kOuterNB);
                    pl_trail = tc_planes(up_trail.tc_ws, up_trail.ws_m, up_trail.ws_n, kOuterNB);
                    const TcPlanes& own = (j & 1) ? pl_main : pl_trail;
                    pl_main.a_hi = pl_trail.a_hi = own.a_hi;
                    pl_main.a_lo = pl_trail.a_lo = own.a_lo;
                }
                s = static_panel_c64(A, lda, n, j0, jb, ipiv, info, pws, reinterpret_cast<cf*>(ws + ocur), perm,
                                     prepacked ? &pl_main : nullptr, st);
            } else {
                s = panel_factor<T>(A, lda, n, j0, jb, ipiv, info, ws, up_main, st, kLaPanelCtas);
            }
        } else {
            s = panel_factor<T>(A, lda, n, j0, jb, ipiv, info, ws, up_main, st, kLaPanelCtas);
        }
        if (s != MW_OK) return s;
        auto swap_rows = [&](T* M, int64_t ldm, int64_t col0, int64_t ncols, cudaStream_t sx) {
            if constexpr (std::is_same<T, cf>::value) {
                if (perm != nullptr) {
                    static_permute_c64(M, ldm, j0, jb, col0, ncols, perm, sx);
                    return;
                }
            }
            laswp_launch<T>(M, ldm, col0, ncols, ipiv, j0, j0 + jb, sx);
        };
        MW_CHECK_CUDA(cudaEventRecord(ax->ev_main, st));
        // (the swaps of panel j on the columns left of it wait until the
        // end: trail j-1 may still be reading those rows of panel j-1)
        const int64_t c1 = j0 + jb;                                       // next block
        const int64_t jbn = (n - c1) < kOuterNB ? (n - c1) : kOuterNB;
        const int64_t c2 = c1 + jbn;                                      // rest
        if (jbn > 0) {
            if (j >= 1) MW_CHECK_CUDA(cudaStreamWaitEvent(st, ax->ev_trail[(j - 1) & 3], 0));
            swap_rows(A, lda, c1, jbn, st);
            s = trsm_lower_blocked<T>(A + j0 + j0 * lda, lda, A + j0 + c1 * lda, lda, jb, jbn, up_main, st,
                                      prepacked ? &pl_main : nullptr);
            if (s != MW_OK) return s;
            s = prepacked ? update_prepacked(n - c1, jbn, jb, pl_main, A + c1 + c1 * lda, lda, up_main, st)
                          : block_update(A + c1 + j0 * lda, lda, A + j0 + c1 * lda, lda, A + c1 + c1 * lda, lda,
                                         n - c1, jbn, jb, up_main, st);
            if (s != MW_OK) return s;
        }
        // trail: everything right of the next block, after panel j
        MW_CHECK_CUDA(cudaStreamWaitEvent(tr, ax->ev_main, 0));
        if (n - c2 > 0) {
            swap_rows(A, lda, c2, n - c2, tr);
            s = trsm_lower_blocked<T>(A + j0 + j0 * lda, lda, A + j0 + c2 * lda, lda, jb, n - c2, up_trail, tr,
                                      prepacked ? &pl_trail : nullptr);
            if (s != MW_OK) return s;
            s = prepacked ? update_prepacked(n - c1, n - c2, jb, pl_trail, A + c1 + c2 * lda, lda, up_trail, tr)
                          : block_update(A + c1 + j0 * lda, lda, A + j0 + c2 * lda, lda, A + c1 + c2 * lda, lda,
                                         n - c1, n - c2, jb, up_trail, tr);
            if (s != MW_OK) return s;
        }
        if (Baug != nullptr && nrhs > 0) {
            // right-hand sides carried as extra columns right of the matrix:
            // this panel's interchanges, L11^-1 on its rows, L21 update below
            // (L21 stays as it is until the deferred left interchanges at the
            // end, which the later rows of Baug then mirror in its own swaps)
            swap_rows(Baug, ldb, 0, nrhs, tr);
            const bool pk_rhs = prepacked && n - c1 > 0;
            s = trsm_lower_blocked<T>(A + j0 + j0 * lda, lda, Baug + j0, ldb, jb, nrhs, up_trail, tr,
                                      pk_rhs ? &pl_trail : nullptr);
            if (s != MW_OK) return s;
            if (n - c1 > 0) {
                s = pk_rhs ? update_prepacked(n - c1, nrhs, jb, pl_trail, Baug + c1, ldb, up_trail, tr)
                           : block_update(A + c1 + j0 * lda, lda, Baug + j0, ldb, Baug + c1, ldb, n - c1, nrhs, jb,
                                          up_trail, tr);
                if (s != MW_OK) return s;
            }
        }
        MW_CHECK_CUDA(cudaEventRecord(ax->ev_trail[j & 3], tr));
        MW_CHECK_CUDA(cudaGetLastError());
    }
    if (nb > 0) MW_CHECK_CUDA(cudaStreamWaitEvent(st, ax->ev_trail[(nb - 1) & 3], 0));
    // every panel's row swaps on the columns left of it, in panel order (the
    // static path's stay inside their blocks: one launch for all of them)
    bool left_done = false;
    if constexpr (std::is_same<T, cf>::value) {
        if (static_pivot) {
            static_left_permute_c64(A, lda, n, perm_all, st);
            left_done = true;
        }
    }
    for (int64_t j = 1; j < nb && !left_done; ++j) {
        const int64_t j0 = j * kOuterNB;
        const int jb = (int)((n - j0) < kOuterNB ? (n - j0) : kOuterNB);
        laswp_launch<T>(A, lda, 0, j0, ipiv, j0, j0 + jb, st);
    }
    MW_CHECK_CUDA(cudaMemcpyAsync(info + 1, &pws->err, sizeof(int32_t), cudaMemcpyDeviceToDevice, st));
    return critical_end(ax, caller);
}

// One triangular sweep over the right-hand sides B with look-ahead.  Step i
// runs leaf block i on the caller's stream, which first applies the block
// solved at step i-1 (the leaf kernel's fused update), then a second stream
// applies block i's solution to the blocks from i+2 on.  Block j thus gets
// block j-1 inside its leaf and every earlier block from the second stream;
// the second stream's update of step k writes blocks >= k+2, so leaf i
// waits only for step i-2's, and the streams never write the same rows at
// once.  upper = false: X <- L^-1 X (unit lower, blocks in order);
// upper = true: X <- U^-1 X (blocks in reverse).
template <class T>
static mw_status trsm_sweep(bool upper, int64_t n, int64_t nrhs, const T* LU, int64_t lda, T* B, int64_t ldb,
                            const Updater& up_main, const Updater& up_rest, cudaStream_t st) {
    constexpr int LF = GetrsLeaf<T>::value;
    (void)up_main;
    if (n <= 0 || nrhs <= 0) return MW_OK;
    AuxStreams* ax = nullptr;
    {
        mw_status s0 = aux_streams(&ax);
        if (s0 != MW_OK) return s0;
    }
    cudaStream_t tr = ax->trail;
    const int64_t nblk = (n + LF - 1) / LF;
    const cudaStream_t caller = st;
    {
        mw_status s0 = critical_begin(ax, caller, &st);
        if (s0 != MW_OK) return s0;
    }
    auto blk0 = [&](int64_t b) { return b * LF < n ? b * LF : n; };
    auto blk1 = [&](int64_t b) { return (b + 1) * LF < n ? (b + 1) * LF : n; };
    // the second stream starts after everything queued on st
    MW_CHECK_CUDA(cudaEventRecord(ax->ev_main, st));
    MW_CHECK_CUDA(cudaStreamWaitEvent(tr, ax->ev_main, 0));
    for (int64_t i = 0; i < nblk; ++i) {
        const int64_t b = upper ? nblk - 1 - i : i;
        const int64_t r0 = blk0(b), r1 = blk1(b);
        const int jb = (int)(r1 - r0);
        // the blocks before i-1 reach this leaf's rows on the second stream
        if (i >= 2) MW_CHECK_CUDA(cudaStreamWaitEvent(st, ax->ev_trail[(i - 2) & 3], 0));
        const T* Aoff = nullptr;
        const T* Xp = nullptr;
        int K = 0;
        if (i >= 1) {  // the block solved at step i-1
            const int64_t q = upper ? b + 1 : b - 1;
            const int64_t q0 = blk0(q), q1 = blk1(q);
            Aoff = LU + r0 + q0 * lda;
            Xp = B + q0;
            K = (int)(q1 - q0);
        }
        if (upper) trsm_launch<T, true, LF>(LU + r0 + r0 * lda, lda, B + r0, ldb, jb, nrhs, st, Aoff, lda, Xp, K);
        else trsm_launch<T, false, LF>(LU + r0 + r0 * lda, lda, B + r0, ldb, jb, nrhs, st, Aoff, lda, Xp, K);
        MW_CHECK_CUDA(cudaEventRecord(ax->ev_main, st));
        mw_status s;
        if (!upper) {
            const int64_t f0 = blk0(b + 2);
            if (f0 < n) {  // blocks i+2.., on the second stream
                MW_CHECK_CUDA(cudaStreamWaitEvent(tr, ax->ev_main, 0));
                s = block_update(LU + f0 + r0 * lda, lda, B + r0, ldb, B + f0, ldb, n - f0, nrhs, jb, up_rest, tr);
                if (s != MW_OK) return s;
            }
        } else if (b >= 2) {  // the blocks above block b-1, on the second stream
            const int64_t f1 = blk0(b - 1);
            MW_CHECK_CUDA(cudaStreamWaitEvent(tr, ax->ev_main, 0));
            s = block_update(LU + r0 * lda, lda, B + r0, ldb, B, ldb, f1, nrhs, jb, up_rest, tr);
            if (s != MW_OK) return s;
        }
        MW_CHECK_CUDA(cudaEventRecord(ax->ev_trail[i & 3], tr));
    }
    MW_CHECK_CUDA(cudaEventRecord(ax->ev_main, tr));
    MW_CHECK_CUDA(cudaStreamWaitEvent(st, ax->ev_main, 0));
    MW_CHECK_CUDA(cudaGetLastError());
    return critical_end(ax, caller);
}

// ------------------------------------------------ sweeps on block operators
// The complex64 solves' triangular sweeps with each 128-row leaf turned into
// one product.  Steps s = 0, 1, ... of a sweep take the blocks in order (L:
// b = s) or in reverse (U: b = nblk - 1 - s).  A second stream applies the
// solved blocks to the blocks further on two steps at a time: pair k, after
// the leaf of step 2k + 1, applies steps 2k and 2k + 1 to the blocks of the
// steps from 2k + 3 on, as one tensor-core update with a two-part inner
// dimension.  A leaf therefore folds in what no pair has applied yet: the
// step before it, and at even steps the one before that too.  With T the
// triangle (unit lower L or upper U of the factors) and q1, q2 the blocks
// of those steps:
//     M_b = T_bb^-1 [ I | -T_b,q1 | -T_b,q2 ]           (128 x 384, column-major)
// built once per factorisation (sweep_ops_prepare: the right-hand sides,
// zero where a step has no q1 or q2, then one batched leaf solve per
// triangle), so that the leaf is one product
//     X_b = M_b [ B_b ; X_q1 ; X_q2 ]
// with no dependent substitution chain.  The same preparation packs every
// block column of the factors as the updates' A operand; each leaf writes
// X_b as the packed B operand of its pair's update, into one of four plane
// sets by step (mod 4): the update of pair k reads the sets of steps 2k and
// 2k + 1, which are written again only at steps 2k + 4 and 2k + 5, after
// leaf 2k + 3 has waited for that update.  Leaf s waits for pair
// floor((s - 3) / 2), the last one that reaches its rows.
constexpr int kOpsB = 128;        // block order (the complex64 solve leaf)
constexpr int kOpsK = 3 * kOpsB;  // columns of an operator
constexpr int kOpsCols = 4;       // right-hand sides per leaf CTA
static_assert(kOpsB == GetrsLeaf<cf>::value, "operator blocks are the solve's leaf blocks");

// the packed A operand of one block column, all n rows (one plane, hi or lo)
static size_t ops_colplane_bytes(int64_t n) { return tc_pack_a_bytes(n, kOpsB); }
// one packed B plane of a leaf's output (128 rows, nrhs columns)
static size_t ops_xplane_bytes(int64_t nrhs) { return (tc_pack_b_bytes(kOpsB, nrhs) + 1023) & ~size_t(1023); }

size_t sweep_ops_bytes(int64_t n, int64_t nrhs) {
    const int64_t nblk = (n + kOpsB - 1) / kOpsB;
    // the L operators, the U operators, every block column of the factors
    // as packed A operand (hi, lo), four plane sets of leaf outputs (hi, lo)
    return 2 * (size_t)nblk * kOpsB * kOpsK * sizeof(cf) + 2 * (size_t)nblk * ops_colplane_bytes(n) +
           8 * ops_xplane_bytes(nrhs);
}

// Every block's [I | -T_b,q1 | -T_b,q2] (sweep order of the triangle given
// by `upper`): rows past the block's order, and columns past a block's, zero.
// One CTA per block.
__global__ void __launch_bounds__(256) ops_rhs_kernel(const cf* __restrict__ LU, int64_t lda, int64_t n, int upper,
                                                      cf* __restrict__ M) {
    const int64_t nblk = (n + kOpsB - 1) / kOpsB;
    const int64_t b = blockIdx.x;
    const int64_t s = upper ? nblk - 1 - b : b;  // sweep step
    auto block_at = [&](int64_t step) { return upper ? nblk - 1 - step : step; };
    auto order = [&](int64_t blk) { return (int)(n - blk * kOpsB < kOpsB ? n - blk * kOpsB : kOpsB); };
    const int jb = order(b);
    const int64_t q1 = s >= 1 ? block_at(s - 1) : -1;
    const int64_t q2 = (s >= 2 && (s & 1) == 0) ? block_at(s - 2) : -1;
    const int jq1 = q1 >= 0 ? order(q1) : 0, jq2 = q2 >= 0 ? order(q2) : 0;
    cf* Mb = M + b * kOpsB * kOpsK;
    for (int i = threadIdx.x; i < kOpsB * kOpsK; i += blockDim.x) {
        const int r = i % kOpsB, c = i / kOpsB;
        const int part = c / kOpsB, cc = c % kOpsB;
        cf v{0.0f, 0.0f};
        if (r < jb) {
            if (part == 0) {
                if (cc == r) v = cf{1.0f, 0.0f};
            } else {
                const int64_t q = part == 1 ? q1 : q2;
                const int jq = part == 1 ? jq1 : jq2;
                if (cc < jq) {
                    const cf t = LU[(b * kOpsB + r) + (q * kOpsB + cc) * lda];
                    v = cf{-t.re, -t.im};
                }
            }
        }
        Mb[i] = v;
    }
}

// X_b (rows < jb of this CTA's kOpsCols columns, in place) = M_b [X_b ; X_q1 ;
// X_q2] with X_q1, X_q2 the jq1, jq2 rows of the blocks folded in (0: none);
// with b_hi set, X_b also as a packed B operand (inner dimension jb, b_nks
// stages).  M_b streams through shared memory in 32-column chunks (32 KB,
// contiguous in M_b), two in flight by cp.async, so two CTAs fit an SM and
// the leaf's CTAs take one wave of the SMs a concurrent update leaves;
// thread (r, g) accumulates row r of columns 2 g, 2 g + 1, reading its M_b
// row conflict-free and the right-hand sides as broadcasts.
constexpr int kOpsChunk = 32;
constexpr size_t kLeafOpsSmem = sizeof(cf) * (2 * (size_t)kOpsChunk * kOpsB + (size_t)kOpsK * kOpsCols +
                                              (size_t)kOpsCols * (kOpsB + 1));
__global__ void __launch_bounds__(256, 1) leaf_ops_kernel(const cf* __restrict__ Mb, cf* __restrict__ X, int64_t ldx,
                                                          int jb, const cf* __restrict__ Xq1, int jq1,
                                                          const cf* __restrict__ Xq2, int jq2, int64_t ncols,
                                                          float* __restrict__ b_hi, float* __restrict__ b_lo,
                                                          int b_nks) {
    extern __shared__ __align__(16) unsigned char lo_smem[];
    cf* sM = reinterpret_cast<cf*>(lo_smem);  // [2][kOpsChunk][kOpsB]
    cf* sR = sM + 2 * kOpsChunk * kOpsB;       // [kOpsK][kOpsCols]
    cf* sO = sR + kOpsK * kOpsCols;            // [kOpsCols][kOpsB + 1]
    const int tid = threadIdx.x;
    const int parts = 1 + (jq1 > 0 ? 1 : 0) + (jq2 > 0 ? 1 : 0);
    const int nchunk = parts * kOpsB / kOpsChunk;
    // chunk c: columns [c kOpsChunk, (c + 1) kOpsChunk) of M_b, one contiguous
    // 32 KB run; eight 16-byte copies per thread
    auto fetch = [&](int c) {
        const char* src = reinterpret_cast<const char*>(Mb + (size_t)c * kOpsChunk * kOpsB);
        char* dst = reinterpret_cast<char*>(sM + (size_t)(c & 1) * kOpsChunk * kOpsB);
        constexpr int n16 = kOpsChunk * kOpsB * (int)sizeof(cf) / 16;
#pragma unroll
        for (int u = 0; u < n16 / 256; ++u) {
            const int q = tid + 256 * u;
            cp_async16(dst + 16 * q, src + 16 * q, true);
        }
        cp_async_commit();
    };
    fetch(0);
    if (nchunk > 1) fetch(1);
    const int64_t c0 = (int64_t)blockIdx.x * kOpsCols;
    for (int i = tid; i < parts * kOpsB * kOpsCols; i += blockDim.x) {
        const int k = i % (parts * kOpsB), c = i / (parts * kOpsB);
        const int64_t col = c0 + c;
        const int part = k / kOpsB, kk = k % kOpsB;
        cf v{0.0f, 0.0f};
        if (col < ncols) {
            if (part == 0) {
                if (kk < jb) v = X[kk + col * ldx];
            } else if (part == 1) {
                if (kk < jq1) v = Xq1[kk + col * ldx];
            } else if (kk < jq2) {
                v = Xq2[kk + col * ldx];
            }
        }
        sR[k * kOpsCols + c] = v;
    }
    const int r = tid & (kOpsB - 1), g = tid >> 7;
    cf acc0{0.0f, 0.0f}, acc1{0.0f, 0.0f};
    for (int c = 0; c < nchunk; ++c) {
        if (c + 1 < nchunk) cp_async_wait<1>();
        else cp_async_wait<0>();
        __syncthreads();  // chunk c (and, the first time, sR) visible to all
        const cf* m = sM + (size_t)(c & 1) * kOpsChunk * kOpsB + r;
        const cf* x = sR + (size_t)c * kOpsChunk * kOpsCols + 2 * g;
#pragma unroll 16
        for (int k = 0; k < kOpsChunk; ++k) {
            const cf mk = m[k * kOpsB];
            const float4 xx = *reinterpret_cast<const float4*>(x + k * kOpsCols);
            acc0 = acc0 + mk * cf{xx.x, xx.y};
            acc1 = acc1 + mk * cf{xx.z, xx.w};
        }
        __syncthreads();  // every thread is done with this slot
        if (c + 2 < nchunk) fetch(c + 2);
    }
    sO[(2 * g) * (kOpsB + 1) + r] = r < jb ? acc0 : cf{0.0f, 0.0f};
    sO[(2 * g + 1) * (kOpsB + 1) + r] = r < jb ? acc1 : cf{0.0f, 0.0f};
    __syncthreads();
    for (int i = tid; i < kOpsB * kOpsCols; i += blockDim.x) {
        const int rr = i % kOpsB, c = i / kOpsB;
        const int64_t col = c0 + c;
        if (col < ncols && rr < jb) X[rr + col * ldx] = sO[c * (kOpsB + 1) + rr];
    }
    if (b_hi != nullptr) {
        // real K rows 2 rr (re) and 2 rr + 1 (im): rows 2p and 2p + 1 of the
        // block make one 16-byte chunk; rows past jb carry zeros
        for (int i = tid; i < (kOpsB / 2) * kOpsCols; i += blockDim.x) {
            const int p = i % (kOpsB / 2), c = i / (kOpsB / 2);
            const int64_t col = c0 + c;
            const int64_t kap4 = 4 * (int64_t)p;
            if (col < ncols && kap4 < (int64_t)b_nks * TC_KS) {
                const cf v0 = sO[c * (kOpsB + 1) + 2 * p], v1 = sO[c * (kOpsB + 1) + 2 * p + 1];
                tc_store_b4(b_hi, b_lo, b_nks, col, kap4, make_float4(v0.re, v0.im, v1.re, v1.im));
            }
        }
    }
}

// Both triangles' operators and the packed block columns of the factors LU
// (n x n, complex64) into `ops` (sweep_ops_bytes(n, nrhs)).
static mw_status sweep_ops_prepare(int64_t n, const cf* LU, int64_t lda, cf* ops, cudaStream_t st) {
    if (n <= 0) return MW_OK;
    {
        mw_status s0 = trsm_setup<cf>();
        if (s0 != MW_OK) return s0;
    }
    const int64_t nblk = (n + kOpsB - 1) / kOpsB;
    MW_REQUIRE(nblk <= 65535, "too many blocks for one batched launch");
    cf* ML = ops;
    cf* MU = ops + nblk * kOpsB * kOpsK;
    {
        ProfileScope ps(PC_MISC, st);
        ops_rhs_kernel<<<(unsigned)nblk, 256, 0, st>>>(LU, lda, n, 0, ML);
        ops_rhs_kernel<<<(unsigned)nblk, 256, 0, st>>>(LU, lda, n, 1, MU);
        count_launch(2);
    }
    const TrsmBatch bt{(int64_t)kOpsB * (lda + 1), (int64_t)kOpsB * kOpsK, n};
    trsm_launch<cf, false, kOpsB>(LU, lda, ML, kOpsB, kOpsB, kOpsK, st, nullptr, 0, nullptr, 0, LeafPack{}, bt,
                                  (unsigned)nblk);
    trsm_launch<cf, true, kOpsB>(LU, lda, MU, kOpsB, kOpsB, kOpsK, st, nullptr, 0, nullptr, 0, LeafPack{}, bt,
                                 (unsigned)nblk);
    // every block column, all rows, as the packed A operand (inner dimension
    // its width): the full columns in one launch, a partial last one apart
    char* cpl = reinterpret_cast<char*>(ops + 2 * nblk * kOpsB * kOpsK);
    const size_t pa = ops_colplane_bytes(n);
    const int64_t nfull = n / kOpsB;
    mw_status s = tc_pack_a(n, kOpsB, LU, lda, reinterpret_cast<float*>(cpl), reinterpret_cast<float*>(cpl + pa), st,
                            (int)nfull, (int64_t)kOpsB * lda, (int64_t)(2 * pa / sizeof(float)));
    if (s != MW_OK) return s;
    if (nblk > nfull) {
        char* c = cpl + nfull * 2 * pa;
        s = tc_pack_a(n, n - nfull * kOpsB, LU + nfull * kOpsB * lda, lda, reinterpret_cast<float*>(c),
                      reinterpret_cast<float*>(c + pa), st);
        if (s != MW_OK) return s;
    }
    MW_CHECK_CUDA(cudaGetLastError());
    return MW_OK;
}

// One triangular sweep over the right-hand sides B (nrhs columns, at most
// the nrhs the operator region was sized for) on the operators: leaf s on
// the caller's stream, the update of pair k on the second stream after
// leaf 2k + 1.
static mw_status trsm_sweep_ops(bool upper, int64_t n, int64_t nrhs, const cf* LU, int64_t lda, cf* B, int64_t ldb,
                                const cf* ops, int64_t nrhs_ops, const Updater& up_rest, cudaStream_t st) {
    if (n <= 0 || nrhs <= 0) return MW_OK;
    MW_REQUIRE(nrhs <= nrhs_ops, "more right-hand sides than the operator region holds");
    static bool attr = false;
    if (!attr) {
        MW_CHECK_CUDA(cudaFuncSetAttribute(leaf_ops_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kLeafOpsSmem));
        attr = true;
    }
    AuxStreams* ax = nullptr;
    {
        mw_status s0 = aux_streams(&ax);
        if (s0 != MW_OK) return s0;
    }
    cudaStream_t tr = ax->trail;
    const int64_t nblk = (n + kOpsB - 1) / kOpsB;
    const cf* M = ops + (upper ? nblk * kOpsB * kOpsK : 0);
    const char* cpl = reinterpret_cast<const char*>(ops + 2 * nblk * kOpsB * kOpsK);
    const size_t pa = ops_colplane_bytes(n);
    char* xpl = const_cast<char*>(cpl) + nblk * 2 * pa;  // four plane sets of leaf outputs
    const size_t px = ops_xplane_bytes(nrhs_ops);
    auto xhi = [&](int64_t s) { return reinterpret_cast<float*>(xpl + (s & 3) * 2 * px); };
    auto xlo = [&](int64_t s) { return reinterpret_cast<float*>(xpl + (s & 3) * 2 * px + px); };
    const cudaStream_t caller = st;
    {
        mw_status s0 = critical_begin(ax, caller, &st);
        if (s0 != MW_OK) return s0;
    }
    auto block_at = [&](int64_t s) { return upper ? nblk - 1 - s : s; };
    auto blk0 = [&](int64_t b) { return b * kOpsB < n ? b * kOpsB : n; };
    auto blk1 = [&](int64_t b) { return (b + 1) * kOpsB < n ? (b + 1) * kOpsB : n; };
    MW_CHECK_CUDA(cudaEventRecord(ax->ev_main, st));
    MW_CHECK_CUDA(cudaStreamWaitEvent(tr, ax->ev_main, 0));
    const unsigned leaf_grid = (unsigned)((nrhs + kOpsCols - 1) / kOpsCols);
    for (int64_t s = 0; s < nblk; ++s) {
        const int64_t b = block_at(s);
        const int64_t r0 = blk0(b);
        const int jb = (int)(blk1(b) - r0);
        // the last pair that reaches this block's rows
        if (s >= 3) MW_CHECK_CUDA(cudaStreamWaitEvent(st, ax->ev_trail[((s - 3) / 2) & 3], 0));
        const cf* X1 = nullptr;
        const cf* X2 = nullptr;
        int j1 = 0, j2 = 0;
        if (s >= 1) {
            const int64_t q = block_at(s - 1);
            X1 = B + blk0(q);
            j1 = (int)(blk1(q) - blk0(q));
        }
        if (s >= 2 && (s & 1) == 0) {
            const int64_t q = block_at(s - 2);
            X2 = B + blk0(q);
            j2 = (int)(blk1(q) - blk0(q));
        }
        {
            ProfileScope ps(PC_TRSM, st, 8.0 * (double)jb * (jb + j1 + j2) * nrhs, 8.0 * (double)(jb + j1 + j2) * kOpsB);
            leaf_ops_kernel<<<leaf_grid, 256, kLeafOpsSmem, st>>>(M + b * kOpsB * kOpsK, B + r0, ldb, jb, X1, j1, X2,
                                                                   j2, nrhs, xhi(s), xlo(s), tc_n_ks(jb));
            count_launch();
        }
        if ((s & 1) == 0) continue;
        // pair (s - 1, s) to the blocks of steps s + 2 on: rows from f0 (L)
        // or below f1 (U)
        MW_CHECK_CUDA(cudaEventRecord(ax->ev_main, st));
        const int64_t bp = block_at(s - 1);
        const int jp = (int)(blk1(bp) - blk0(bp));
        const int64_t f0 = upper ? 0 : blk0(b + 2);
        const int64_t f1 = upper ? (b >= 2 ? blk0(b - 1) : 0) : n;
        if (f1 > f0) {
            MW_CHECK_CUDA(cudaStreamWaitEvent(tr, ax->ev_main, 0));
            // block columns bp and b from row f0: f0 / 64 m-blocks into their planes
            auto col = [&](int64_t blk, int k, float** hi, float** lo) {
                const int64_t off = (2 * f0 / TC_M) * (int64_t)tc_n_ks(k) * TC_M * TC_KS;
                *hi = const_cast<float*>(reinterpret_cast<const float*>(cpl + blk * 2 * pa)) + off;
                *lo = const_cast<float*>(reinterpret_cast<const float*>(cpl + blk * 2 * pa + pa)) + off;
            };
            TcPlanes p1{}, p2{};
            col(bp, jp, &p1.a_hi, &p1.a_lo);
            col(b, jb, &p2.a_hi, &p2.a_lo);
            p1.b_hi = xhi(s - 1);
            p1.b_lo = xlo(s - 1);
            p2.b_hi = xhi(s);
            p2.b_lo = xlo(s);
            mw_status rs = cgemm_tc_prepacked2(f1 - f0, nrhs, jp, p1, jb, p2, B + f0, ldb, up_rest.tc_err, tr,
                                               up_rest.max_ctas);
            if (rs != MW_OK) return rs;
        }
        MW_CHECK_CUDA(cudaEventRecord(ax->ev_trail[((s - 1) / 2) & 3], tr));
    }
    MW_CHECK_CUDA(cudaEventRecord(ax->ev_main, tr));
    MW_CHECK_CUDA(cudaStreamWaitEvent(st, ax->ev_main, 0));
    MW_CHECK_CUDA(cudaGetLastError());
    return critical_end(ax, caller);
}

// X <- U^-1 X (the back substitution of a solve).
template <class T>
static mw_status getrs_upper(int64_t n, int64_t nrhs, const T* LU, int64_t lda, T* B, int64_t ldb,
                             const Updater& up_main, const Updater& up, cudaStream_t st) {
    return trsm_sweep<T>(true, n, nrhs, LU, lda, B, ldb, up_main, up, st);
}

// Solve A X = B from the factors (forward with unit L, back with U).
template <class T>
static mw_status getrs(int64_t n, int64_t nrhs, const T* LU, int64_t lda, const int32_t* ipiv, T* B, int64_t ldb,
                       const Updater& up_main, const Updater& up, cudaStream_t st) {
    {
        mw_status s0 = trsm_setup<T>();
        if (s0 != MW_OK) return s0;
    }
    laswp_launch<T>(B, ldb, 0, nrhs, ipiv, 0, n, st);
    mw_status s = trsm_sweep<T>(false, n, nrhs, LU, lda, B, ldb, up_main, up, st);
    if (s != MW_OK) return s;
    return trsm_sweep<T>(true, n, nrhs, LU, lda, B, ldb, up_main, up, st);
}

static size_t panel_ws_bytes() {
    size_t a, b, c, d;
    return ws_layout(kMaxPanelGrid, &a, &b, &c, &d);
}

// Workspace of the complex64 path: panel slots, then the tensor-core
// operand planes for the largest update (m = n, n = n, k = kOuterNB), then the
// device status word.
static size_t cgetrf_perm_offset(int64_t n, int64_t nrhs_max) {
    int64_t w = n > nrhs_max ? n : nrhs_max;
    // panel slots | trail-stream operand planes | status word | main-stream
    // operand planes (k at most kOuterNB; at most kOuterNB columns wide in
    // the factorisation, nrhs_max wide in the solves) | static pivot orders
    const int64_t wm = nrhs_max > kOuterNB ? nrhs_max : kOuterNB;
    const size_t o = panel_ws_bytes() + 1024 + ((cgemm_tc_workspace(n, w, kOuterNB) + 255) & ~size_t(255)) + 256 +
                     cgemm_tc_workspace(n, wm, kOuterNB) + 1024;
    return (o + 255) & ~size_t(255);
}

static size_t cgetrf_ws_bytes(int64_t n, int64_t nrhs_max) {
    return cgetrf_perm_offset(n, nrhs_max) + sizeof(int32_t) * (size_t)(n > 0 ? n : 1) + 256;
}

static Updater tc_updater(char* ws, size_t ws_bytes, int64_t n, int64_t nrhs_max) {
    Updater u;
    size_t p = (panel_ws_bytes() + 1023) & ~size_t(1023);
    int64_t w = n > nrhs_max ? n : nrhs_max;
    u.tc_ws = ws + p;
    u.tc_ws_bytes = cgemm_tc_workspace(n, w, kOuterNB);
    u.ws_m = n;
    u.ws_n = w;
    u.tc_err = reinterpret_cast<int*>(ws + p + ((u.tc_ws_bytes + 255) & ~size_t(255)));
    (void)ws_bytes;
    return u;
}

// The main-stream updater of the look-ahead factorisation: its own operand
// planes (after the trail region and the status word), the shared status
// word, and the panel's CTA budget.
// info[1] = the panel's wait status, else the tensor-core kernels'
__global__ void merge_status_kernel(int32_t* out, const int* panel_err, const int* tc_err) {
    const int a = *panel_err;
    *out = a != 0 ? a : *tc_err;
}

static Updater tc_updater_main(char* ws, int64_t n, int64_t nrhs_max) {
    Updater t = tc_updater(ws, 0, n, nrhs_max);
    Updater u;
    char* base = static_cast<char*>(t.tc_ws) + ((t.tc_ws_bytes + 255) & ~size_t(255)) + 256;
    u.tc_ws = reinterpret_cast<void*>((reinterpret_cast<uintptr_t>(base) + 1023) & ~uintptr_t(1023));
    u.ws_m = n;
    u.ws_n = nrhs_max > kOuterNB ? nrhs_max : kOuterNB;
    u.tc_ws_bytes = cgemm_tc_workspace(u.ws_m, u.ws_n, kOuterNB);
    u.tc_err = t.tc_err;
    u.max_ctas = main_sms();
    return u;
}

}  // namespace mw

using namespace mw;

extern "C" size_t mw_getrf_workspace_size(int64_t n) {
    (void)n;
    return panel_ws_bytes();
}

extern "C" mw_status mw_zgetrf(int64_t n, double* Ad, int64_t lda, int32_t* ipiv, int32_t* info, void* workspace,
                               size_t workspace_bytes, const volatile int32_t* cancel, void* stream) {
    MW_REQUIRE(n >= 0 && lda >= (n > 0 ? n : 1), "bad n/lda");
    MW_REQUIRE(Ad && ipiv && info && workspace, "NULL argument");
    MW_REQUIRE(workspace_bytes >= mw_getrf_workspace_size(n), "workspace too small");
    Updater up_main, up_trail;
    up_main.max_ctas = kLaPanelCtas;
    up_trail.max_ctas = panel_sms<cd>() - kLaPanelCtas;
    ProfileScope ps(PC_FACTOR, as_stream(stream), 8.0 / 3.0 * (double)n * n * n, 0.0);
    return getrf_lookahead<cd>(n, reinterpret_cast<cd*>(Ad), lda, ipiv, info, static_cast<char*>(workspace), cancel,
                               up_main, up_trail, as_stream(stream));
}

extern "C" mw_status mw_zgetrs(int64_t n, int64_t nrhs, const double* LUd, int64_t lda, const int32_t* ipiv,
                               double* Bd, int64_t ldb, void* stream) {
    MW_REQUIRE(n >= 0 && nrhs >= 0 && lda >= (n > 0 ? n : 1) && ldb >= (n > 0 ? n : 1), "bad sizes");
    MW_REQUIRE(LUd && ipiv && Bd, "NULL argument");
    if (n == 0 || nrhs == 0) return MW_OK;
    Updater up_main, up_rest;
    up_main.max_ctas = kLaPanelCtas;                  // leaves and next-block updates
    up_rest.max_ctas = panel_sms<cd>() - kLaPanelCtas;  // the rest, beside them
    ProfileScope ps(PC_SOLVE, as_stream(stream), 8.0 * (double)n * n * nrhs, 0.0);
    return getrs<cd>(n, nrhs, reinterpret_cast<const cd*>(LUd), lda, ipiv, reinterpret_cast<cd*>(Bd), ldb, up_main,
                     up_rest, as_stream(stream));
}

extern "C" size_t mw_cgetrf_workspace_size(int64_t n, int64_t nrhs_max) { return cgetrf_ws_bytes(n, nrhs_max); }

extern "C" mw_status mw_cgetrf(int64_t n, float* Ad, int64_t lda, int32_t* ipiv, int32_t* info, void* workspace,
                               size_t workspace_bytes, int64_t nrhs_max, const volatile int32_t* cancel, void* stream) {
    MW_REQUIRE(n >= 0 && lda >= (n > 0 ? n : 1) && nrhs_max >= 0, "bad n/lda");
    MW_REQUIRE(Ad && ipiv && info && workspace, "NULL argument");
    MW_REQUIRE(workspace_bytes >= cgetrf_ws_bytes(n, nrhs_max), "workspace too small");
    char* ws = static_cast<char*>(workspace);
    Updater up = tc_updater(ws, workspace_bytes, n, nrhs_max);
    Updater up_main = tc_updater_main(ws, n, nrhs_max);
    up.max_ctas = panel_sms<cf>() - main_sms();  // the trail stream leaves the panel its SMs
    cudaStream_t st = as_stream(stream);
    MW_CHECK_CUDA(cudaMemsetAsync(up.tc_err, 0, sizeof(int), st));
    mw_status s = getrf_lookahead<cf>(n, reinterpret_cast<cf*>(Ad), lda, ipiv, info, ws, cancel, up_main, up, st);
    if (s != MW_OK) return s;
    // info[1]: a panel wait's timeout, else a tensor-core one
    merge_status_kernel<<<1, 1, 0, st>>>(info + 1, &reinterpret_cast<PanelWs*>(ws)->err, up.tc_err);
    count_launch();
    MW_CHECK_CUDA(cudaGetLastError());
    return MW_OK;
}

namespace mw {
// Complex64 factorisation that also carries nrhs right-hand sides (B, ld
// ldb, permuted and overwritten with L^-1 P B) through the trail stream;
// the forward substitution of the first solve then costs no extra pass.
mw_status cgetrf_forward(int64_t n, float* Ad, int64_t lda, int32_t* ipiv, int32_t* info, void* workspace,
                         size_t workspace_bytes, float* Bd, int64_t ldb, int64_t nrhs, const volatile int32_t* cancel,
                         void* stream, bool static_pivot) {
    MW_REQUIRE(n >= 0 && lda >= (n > 0 ? n : 1) && nrhs >= 0 && ldb >= (n > 0 ? n : 1), "bad sizes");
    MW_REQUIRE(Ad && ipiv && info && workspace && (nrhs == 0 || Bd), "NULL argument");
    MW_REQUIRE(workspace_bytes >= cgetrf_ws_bytes(n, nrhs), "workspace too small");
    char* ws = static_cast<char*>(workspace);
    Updater up = tc_updater(ws, workspace_bytes, n, nrhs);
    Updater up_main = tc_updater_main(ws, n, nrhs);
    up.max_ctas = panel_sms<cf>() - main_sms();
    cudaStream_t st = as_stream(stream);
    MW_CHECK_CUDA(cudaMemsetAsync(up.tc_err, 0, sizeof(int), st));
    int32_t* perm_all = static_pivot ? reinterpret_cast<int32_t*>(ws + cgetrf_perm_offset(n, nrhs)) : nullptr;
    mw_status s = getrf_lookahead<cf>(n, reinterpret_cast<cf*>(Ad), lda, ipiv, info, ws, cancel, up_main, up, st,
                                      reinterpret_cast<cf*>(Bd), ldb, nrhs, perm_all);
    if (s != MW_OK) return s;
    merge_status_kernel<<<1, 1, 0, st>>>(info + 1, &reinterpret_cast<PanelWs*>(ws)->err, up.tc_err);
    count_launch();
    MW_CHECK_CUDA(cudaGetLastError());
    return MW_OK;
}

// B <- U^-1 B with the factors of cgetrf_forward.
mw_status cgetrs_upper(int64_t n, int64_t nrhs, const float* LUd, int64_t lda, float* Bd, int64_t ldb, void* workspace,
                       size_t workspace_bytes, void* stream) {
    MW_REQUIRE(workspace_bytes >= cgetrf_ws_bytes(n, nrhs), "workspace too small");
    if (n == 0 || nrhs == 0) return MW_OK;
    {
        mw_status s0 = trsm_setup<cf>();
        if (s0 != MW_OK) return s0;
    }
    char* ws = static_cast<char*>(workspace);
    Updater up = tc_updater(ws, workspace_bytes, n, nrhs);
    Updater up_main = tc_updater_main(ws, n, nrhs);
    up.max_ctas = panel_sms<cf>() - main_sms();
    return getrs_upper<cf>(n, nrhs, reinterpret_cast<const cf*>(LUd), lda, reinterpret_cast<cf*>(Bd), ldb, up_main,
                           up, as_stream(stream));
}

// The block operators of the complex64 factors in LUd (after every row
// interchange: the output of cgetrf_forward or mw_cgetrf) into `ops`
// (cgetrs_ops_bytes(n, nrhs) bytes), for cgetrs_upper_ops and cgetrs_ops
// with up to nrhs right-hand sides.
size_t cgetrs_ops_bytes(int64_t n, int64_t nrhs) { return sweep_ops_bytes(n, nrhs); }

mw_status cgetrs_ops_prepare(int64_t n, const float* LUd, int64_t lda, void* ops, void* stream) {
    MW_REQUIRE(n >= 0 && lda >= (n > 0 ? n : 1) && LUd && ops, "bad arguments");
    return sweep_ops_prepare(n, reinterpret_cast<const cf*>(LUd), lda, static_cast<cf*>(ops), as_stream(stream));
}

// cgetrs_upper on the block operators of the same factors.
mw_status cgetrs_upper_ops(int64_t n, int64_t nrhs, const float* LUd, int64_t lda, float* Bd, int64_t ldb,
                           const void* ops, void* workspace, size_t workspace_bytes, void* stream) {
    MW_REQUIRE(workspace_bytes >= cgetrf_ws_bytes(n, nrhs), "workspace too small");
    if (n == 0 || nrhs == 0) return MW_OK;
    char* ws = static_cast<char*>(workspace);
    Updater up = tc_updater(ws, workspace_bytes, n, nrhs);
    up.max_ctas = panel_sms<cf>() - main_sms();
    return trsm_sweep_ops(true, n, nrhs, reinterpret_cast<const cf*>(LUd), lda, reinterpret_cast<cf*>(Bd), ldb,
                          static_cast<const cf*>(ops), nrhs, up, as_stream(stream));
}

// mw_cgetrs on the block operators of the same factors: the interchanges
// (a static-pivot factorisation's as one parallel block permutation, from
// the row orders it left in the workspace), then the forward and the back
// sweep.
mw_status cgetrs_ops(int64_t n, int64_t nrhs, const float* LUd, int64_t lda, const int32_t* ipiv, float* Bd,
                     int64_t ldb, const void* ops, void* workspace, size_t workspace_bytes, void* stream,
                     bool static_pivot) {
    MW_REQUIRE(workspace_bytes >= cgetrf_ws_bytes(n, nrhs), "workspace too small");
    if (n == 0 || nrhs == 0) return MW_OK;
    char* ws = static_cast<char*>(workspace);
    Updater up = tc_updater(ws, workspace_bytes, n, nrhs);
    up.max_ctas = panel_sms<cf>() - main_sms();
    cudaStream_t st = as_stream(stream);
    cf* B = reinterpret_cast<cf*>(Bd);
    const cf* LU = reinterpret_cast<const cf*>(LUd);
    if (static_pivot) {
        static_rows_permute_c64(B, ldb, n, nrhs, reinterpret_cast<const int32_t*>(ws + cgetrf_perm_offset(n, nrhs)),
                                st);
    } else {
        laswp_launch<cf>(B, ldb, 0, nrhs, ipiv, 0, n, st);
    }
    mw_status s = trsm_sweep_ops(false, n, nrhs, LU, lda, B, ldb, static_cast<const cf*>(ops), nrhs, up, st);
    if (s != MW_OK) return s;
    return trsm_sweep_ops(true, n, nrhs, LU, lda, B, ldb, static_cast<const cf*>(ops), nrhs, up, st);
}
}  // namespace mw

extern "C" mw_status mw_cgetrs(int64_t n, int64_t nrhs, const float* LUd, int64_t lda, const int32_t* ipiv, float* Bd,
                               int64_t ldb, void* workspace, size_t workspace_bytes, void* stream) {
    MW_REQUIRE(n >= 0 && nrhs >= 0 && lda >= (n > 0 ? n : 1) && ldb >= (n > 0 ? n : 1), "bad sizes");
    MW_REQUIRE(LUd && ipiv && Bd && workspace, "NULL argument");
    MW_REQUIRE(workspace_bytes >= cgetrf_ws_bytes(n, nrhs), "workspace too small");
    if (n == 0 || nrhs == 0) return MW_OK;
    char* ws = static_cast<char*>(workspace);
    Updater up = tc_updater(ws, workspace_bytes, n, nrhs);
    Updater up_main = tc_updater_main(ws, n, nrhs);
    up.max_ctas = panel_sms<cf>() - main_sms();  // the rest updates leave the leaves their SMs
    return getrs<cf>(n, nrhs, reinterpret_cast<const cf*>(LUd), lda, ipiv, reinterpret_cast<cf*>(Bd), ldb, up_main, up,
                     as_stream(stream));
}

extern "C" mw_status mw_zgemm(int32_t transA, int32_t transB, int64_t m, int64_t n, int64_t k, double alpha_re,
                              double alpha_im, const double* A, int64_t lda, const double* B, int64_t ldb,
                              double beta_re, double beta_im, double* C, int64_t ldc, void* stream) {
    MW_REQUIRE(m >= 0 && n >= 0 && k >= 0, "negative size");
    MW_REQUIRE(A && B && C, "NULL argument");
    return zgemm_launch(transA != 0, transB != 0, m, n, k, cd{alpha_re, alpha_im}, reinterpret_cast<const cd*>(A),
                        lda, reinterpret_cast<const cd*>(B), ldb, cd{beta_re, beta_im}, reinterpret_cast<cd*>(C), ldc,
                        as_stream(stream), 0, nullptr, 0);
}
