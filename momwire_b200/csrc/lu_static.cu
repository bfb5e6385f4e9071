// Static-pivot panel of the complex64 LU (sm_100a).
//
// The mixed-precision path factors Z in complex64 and refines the solution
// against the FP64 Z, so its factors need only be a good preconditioner,
// not LAPACK's partial-pivoting factors.  Pivoting is therefore restricted
// to the rows of each 128 x 128 diagonal block ("static pivoting", Li and
// Demmel 1998: factor with pivots chosen locally, recover accuracy by
// iterative refinement): the panel no longer needs a pivot search over all
// the rows below it, so it has no grid-wide exchange per column.  A panel is
//   sp_diag_kernel  one CTA factors the diagonal block in registers with
//                   partial pivoting among its own rows (row interchanges
//                   kept as a row arrangement, written back once), and
//   sp_l21_kernel   every row below is solved against the block's upper
//                   factor, L21 = A21 U11^-1, four warps per 32 rows.
// The growth the restriction allows is measured: sp_l21_kernel raises the
// largest |L21| (|re| + |im|) into PanelWs::lmax_bits, and an exact zero
// pivot sets it to +inf.  The caller refactors with full partial pivoting
// when it exceeds its bound, and the FP64 refinement checks the result.
// Galerkin thin-wire impedance matrices are strongly diagonal: partial
// pivoting rarely leaves the diagonal block on them (no interchange at all
// on the planar dipole arrays, a few per cent of columns on Yagis, where
// the local pivot's |L| stays below 3).
#include "common.cuh"
#include "tc_layout.cuh"
#include "waits.cuh"

namespace mw {

constexpr int kSpB = 128;          // diagonal block order
constexpr int kSpDiagThreads = 512;  // 128 rows x 4 groups of 32 columns
constexpr int kSpUStride = kSpB + 2;  // complex elements per shared-memory row of U (16-byte aligned)

namespace {

__device__ __forceinline__ cf crcp_sp(cf z) {
    // 1 / z with z scaled by its larger component (|z|^2 neither overflows
    // nor underflows); two reciprocals instead of Smith's three divisions
    const float s = fmaxf(fabsf(z.re), fabsf(z.im));
    if (s < 1e-30f) return cdiv(cone<cf>(), z);
    const float rs = __frcp_rn(s);
    const float a = z.re * rs, b = z.im * rs;
    const float t = rs * __frcp_rn(a * a + b * b);
    return cf{a * t, -b * t};
}

__device__ __forceinline__ float cabs1f(cf z) { return fabsf(z.re) + fabsf(z.im); }

constexpr int kSpLD = kSpB + 2;  // column stride of the staged block (complex; 16-byte aligned columns)
constexpr int kSpPW = 32;        // panel width inside the block
constexpr size_t kSpDiagSmem = sizeof(cf) * (size_t)kSpB * kSpLD;

// U12 = L11^-1 A12 on the rows of the panel at c0 (unit lower L11), one
// thread per later column; `t` is the caller's index among the threads
// that take part (the others pass t < 0).
__device__ __forceinline__ void sp_u12(cf* S, int c0, int jb, int t) {
    const int t0 = c0 + kSpPW;
    const int nt = jb - t0;
    if (t < 0 || t >= nt) return;
    cf* col = S + (t0 + t) * kSpLD + c0;
    cf x[kSpPW];
#pragma unroll
    for (int i = 0; i < kSpPW; ++i) x[i] = col[i];
#pragma unroll
    for (int i = 1; i < kSpPW; ++i) {
        cf v = x[i];
#pragma unroll
        for (int jj = 0; jj < i; ++jj) v = v - S[(c0 + jj) * kSpLD + c0 + i] * x[jj];
        x[i] = v;
    }
#pragma unroll
    for (int i = 0; i < kSpPW; ++i) col[i] = x[i];
}

// A22 -= L21 U12 over rows and columns c0+32 .. jb-1 in 4 x 2 register
// tiles (all threads of the block).
__device__ __forceinline__ void sp_a22(cf* S, int c0, int jb, int tid) {
    const int t0 = c0 + kSpPW;
    const int nt = jb - t0;
    if (nt <= 0) return;
    const int ntr = (nt + 3) / 4, ntc = (nt + 1) / 2;
    for (int tile = tid; tile < ntr * ntc; tile += kSpDiagThreads) {
        const int i0 = t0 + 4 * (tile % ntr), jc = t0 + 2 * (tile / ntr);
        cf acc[4][2];
#pragma unroll
        for (int b2 = 0; b2 < 2; ++b2)
#pragma unroll
            for (int a4 = 0; a4 < 4; ++a4) acc[a4][b2] = S[(jc + b2) * kSpLD + i0 + a4];
#pragma unroll 4
        for (int jj = 0; jj < kSpPW; ++jj) {
            const cf* lcol = S + (c0 + jj) * kSpLD + i0;
            const float4 l01 = *reinterpret_cast<const float4*>(lcol);
            const float4 l23 = *reinterpret_cast<const float4*>(lcol + 2);
            const cf l[4] = {cf{l01.x, l01.y}, cf{l01.z, l01.w}, cf{l23.x, l23.y}, cf{l23.z, l23.w}};
            const cf u0 = S[jc * kSpLD + c0 + jj], u1 = S[(jc + 1) * kSpLD + c0 + jj];
#pragma unroll
            for (int a4 = 0; a4 < 4; ++a4) {
                acc[a4][0] = acc[a4][0] - l[a4] * u0;
                acc[a4][1] = acc[a4][1] - l[a4] * u1;
            }
        }
#pragma unroll
        for (int b2 = 0; b2 < 2; ++b2)
#pragma unroll
            for (int a4 = 0; a4 < 4; ++a4) S[(jc + b2) * kSpLD + i0 + a4] = acc[a4][b2];
    }
}

// The later columns of a factored 32-column panel: U12, then A22 (all
// threads; the caller synchronises after it).
__device__ __forceinline__ void sp_trailing(cf* S, int c0, int jb, int tid) {
    if (jb - (c0 + kSpPW) <= 0) return;
    sp_u12(S, c0, jb, tid);
    __syncthreads();
    sp_a22(S, c0, jb, tid);
}

// Factor A[j0 .. j0+jb) x [j0 .. j0+jb) in place, pivots among these rows
// only: a blocked LU of the block staged in shared memory (column major),
// 32 columns at a time.
//   first   without interchanges: warps 0-3 hold the panel's rows in
//           registers (thread r = row r); per column the pivot row, whose
//           values are final, is published in shared memory, one 128-thread
//           named barrier, then every row below takes its multiplier and
//           updates its panel columns.  Kept when every pivot is nonzero and
//           every |l| (|re| + |im|) stays within kSpNoPivotBound -- on the
//           strongly diagonal Galerkin blocks partial pivoting would keep
//           the diagonal anyway, and the factors are then the same.
//   else    the block is staged again and factored with partial pivoting
//           among its rows: thread (r, s) holds row r's panel columns
//           8s .. 8s+7, every thread takes part in every column, rows are
//           interchanged physically (registers for the panel, shared memory
//           for the other columns); two block barriers per column.
// Each panel is followed by its U12 and A22 updates (sp_trailing).
constexpr float kSpNoPivotBound = 2.0f;

__global__ void __launch_bounds__(kSpDiagThreads, 1)
    sp_diag_kernel(cf* __restrict__ A, int64_t lda, int64_t j0, int jb, int32_t* __restrict__ ipiv,
                   int32_t* __restrict__ info, cf* __restrict__ inv_diag, int32_t* __restrict__ perm, PanelWs* ws) {
    extern __shared__ __align__(16) unsigned char sp_diag_smem[];
    cf* S = reinterpret_cast<cf*>(sp_diag_smem);  // S[col * kSpLD + row]
    __shared__ cf s_col[2][kSpB];                 // column c of every row (by column parity)
    __shared__ unsigned long long s_key[2][4];
    __shared__ __align__(16) cf s_u[2][kSpPW];    // the pivot row's panel values
    __shared__ cf s_rc[2][kSpPW];                 // row c's panel values before the interchange
    __shared__ int s_row_at[kSpB];                // original row at each position
    __shared__ cf s_inv[kSpB];
    __shared__ int s_bad;
    const int tid = threadIdx.x;
    const int lane = tid & 31;
    for (int base = 0; base < kSpB * kSpB; base += 8 * kSpDiagThreads) {
        cf t[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int idx = base + u * kSpDiagThreads + tid;
            const int rr = idx % kSpB, col = idx / kSpB;
            t[u] = (rr < jb && col < jb) ? A[(j0 + rr) + (j0 + col) * lda] : cf{0.0f, 0.0f};
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int idx = base + u * kSpDiagThreads + tid;
            S[(idx / kSpB) * kSpLD + idx % kSpB] = t[u];
        }
    }
    if (tid == 0) s_bad = 0;
    __syncthreads();
    // ---- without interchanges
    for (int c0 = 0; c0 < jb; c0 += kSpPW) {
        const int nck = (jb - c0) < kSpPW ? (jb - c0) : kSpPW;
        const int warp = tid >> 5;
        float lmax = 0.0f;
        bool bad = false;
        // (1) the panel's 32 x 32 diagonal sub-block by warp 0, lane = row
        // c0 + lane: the pivot row is read in place (broadcast), one warp
        // synchronisation per column
        if (warp == 0) {
            cf* row = S + c0 + lane;
            for (int cc = 0; cc < nck; ++cc) {
                __syncwarp();
                const int c = c0 + cc;
                const cf piv = S[c * kSpLD + c];
                const float pa = cabs1f(piv);
                bad = bad || !(pa > 0.0f);
                const cf inv = pa > 0.0f ? crcp_sp(piv) : cone<cf>();
                if (lane == cc) s_inv[c] = inv;
                if (lane > cc && lane < nck) {
                    const cf l = row[c * kSpLD] * inv;
                    row[c * kSpLD] = l;
                    lmax = fmaxf(lmax, cabs1f(l));
#pragma unroll 4
                    for (int q = cc + 1; q < nck; ++q)
                        row[(c0 + q) * kSpLD] = row[(c0 + q) * kSpLD] - l * S[(c0 + q) * kSpLD + c];
                }
            }
        }
        __syncthreads();
        // (2) in parallel: the rows below the sub-block, L = A U11^-1 (warps
        // 0-3, a row each, right-looking along the row), and the columns
        // right of it, U12 = L11^-1 A12 (warps 4-7, a column each)
        const int t0 = c0 + kSpPW;
        if (tid < kSpB) {
            const int R = t0 + tid;
            if (R < jb) {
                cf* row = S + R;
                for (int jj = 0; jj < nck; ++jj) {
                    const cf l = row[(c0 + jj) * kSpLD] * s_inv[c0 + jj];
                    row[(c0 + jj) * kSpLD] = l;
                    lmax = fmaxf(lmax, cabs1f(l));
#pragma unroll 4
                    for (int q = jj + 1; q < nck; ++q)
                        row[(c0 + q) * kSpLD] = row[(c0 + q) * kSpLD] - l * S[(c0 + q) * kSpLD + c0 + jj];
                }
            }
        } else if (tid < 2 * kSpB) {
            sp_u12(S, c0, jb, tid - kSpB);
        }
        // NaN-safe: a NaN multiplier fails the comparison
        if (bad || !(lmax <= kSpNoPivotBound)) atomicOr(&s_bad, 1);
        __syncthreads();
        if (s_bad) break;
        // (3) the trailing block
        sp_a22(S, c0, jb, tid);
        __syncthreads();
    }
    if (!s_bad) {
        for (int c = tid; c < jb; c += kSpDiagThreads) {
            ipiv[j0 + c] = (int32_t)(j0 + c + 1);
            inv_diag[c] = s_inv[c];
            perm[c] = c;
        }
    } else {
        // ---- partial pivoting among the block's rows, from the block as
        // it came
        __syncthreads();
        for (int base = 0; base < kSpB * kSpB; base += 8 * kSpDiagThreads) {
            cf t[8];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int idx = base + u * kSpDiagThreads + tid;
                const int rr = idx % kSpB, col = idx / kSpB;
                t[u] = (rr < jb && col < jb) ? A[(j0 + rr) + (j0 + col) * lda] : cf{0.0f, 0.0f};
            }
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const int idx = base + u * kSpDiagThreads + tid;
                S[(idx / kSpB) * kSpLD + idx % kSpB] = t[u];
            }
        }
        if (tid < kSpB) s_row_at[tid] = tid;
        __syncthreads();
        const int r = tid & (kSpB - 1);
        const int sg = tid >> 7;  // panel column group: columns 8 sg .. 8 sg + 7 of the panel
        const int wig = (tid >> 5) & 3;
        for (int c0 = 0; c0 < jb; c0 += kSpPW) {
            const int nck = (jb - c0) < kSpPW ? (jb - c0) : kSpPW;
            cf pr[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) pr[q] = S[(c0 + 8 * sg + q) * kSpLD + r];
#pragma unroll 1
            for (int cc = 0; cc < nck; ++cc) {
                const int c = c0 + cc, scol = cc >> 3, qc = cc & 7, par = cc & 1;
                if (sg == scol) {
                    cf v = pr[0];
#pragma unroll
                    for (int q = 1; q < 8; ++q)
                        if (q == qc) v = pr[q];
                    s_col[par][r] = v;
                    // largest |re| + |im| among rows c .. jb-1, then the smallest
                    // row (LAPACK's icamax); the low bits carry the row
                    unsigned long long key = 0;
                    if (r >= c && r < jb)
                        key = ((unsigned long long)__float_as_uint(cabs1f(v)) << 32) |
                              ((unsigned long long)(0xFFFFu - (unsigned int)r) << 16) | (unsigned long long)r;
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) {
                        const unsigned long long o = __shfl_xor_sync(0xffffffffu, key, off);
                        key = o > key ? o : key;
                    }
                    if (lane == 0) s_key[par][wig] = key;
                }
                __syncthreads();
                unsigned long long best = s_key[par][0];
#pragma unroll
                for (int w = 1; w < 4; ++w) best = s_key[par][w] > best ? s_key[par][w] : best;
                const int p = (int)(best & 0xFFFFull);
                const bool zero = (best >> 32) == 0ull;
                const cf inv = zero ? cone<cf>() : crcp_sp(s_col[par][p]);
                if (r == p) {
#pragma unroll
                    for (int q = 0; q < 8; ++q) s_u[par][8 * sg + q] = pr[q];
                }
                if (r == c) {
#pragma unroll
                    for (int q = 0; q < 8; ++q) s_rc[par][8 * sg + q] = pr[q];
                }
                // the interchange in the columns outside the panel, one column
                // per thread
                if (p != c && tid < kSpB && (tid < c0 || tid >= c0 + kSpPW)) {
                    cf* col = S + tid * kSpLD;
                    const cf t0 = col[c];
                    col[c] = col[p];
                    col[p] = t0;
                }
                if (tid == 0) {
                    ipiv[j0 + c] = (int32_t)(j0 + p + 1);
                    if (zero) {
                        if (info[0] == 0) info[0] = (int32_t)(j0 + c + 1);
                        atomicExch(&ws->lmax_bits, 0x7f800000u);  // +inf: the block is singular
                    }
                    inv_diag[c] = inv;
                    const int t0 = s_row_at[c];
                    s_row_at[c] = s_row_at[p];
                    s_row_at[p] = t0;
                }
                __syncthreads();  // s_u, s_rc complete
                if (r == c) {
#pragma unroll
                    for (int q = 0; q < 8; ++q) pr[q] = s_u[par][8 * sg + q];
                } else if (r == p) {
#pragma unroll
                    for (int q = 0; q < 8; ++q) pr[q] = s_rc[par][8 * sg + q];
                }
                if (r > c && r < jb && !zero) {
                    // row p now holds row c's old values
                    const cf l = (r == p ? s_col[par][c] : s_col[par][r]) * inv;
#pragma unroll
                    for (int q = 0; q < 8; ++q) {
                        const int pc = 8 * sg + q;
                        if (pc == cc) pr[q] = l;
                        else if (pc > cc) pr[q] = pr[q] - l * s_u[par][pc];
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < 8; ++q) S[(c0 + 8 * sg + q) * kSpLD + r] = pr[q];
            __syncthreads();
            sp_trailing(S, c0, jb, tid);
            __syncthreads();
        }

        // the block's rows in pivot order: position i holds original row s_row_at[i]
        if (tid < jb) perm[tid] = s_row_at[tid];
    }
    __syncthreads();
    for (int base = 0; base < kSpB * kSpB; base += kSpDiagThreads) {
        const int idx = base + tid;
        const int rr = idx % kSpB, col = idx / kSpB;
        if (rr < jb && col < jb) A[(j0 + rr) + (j0 + col) * lda] = S[col * kSpLD + rr];
    }
}

// Rows [row0, row0 + jb) of columns [col0, col0 + ncols) rearranged in
// place, row row0 + i taking the old row row0 + perm[i]: one warp per
// column, all of the column's rows read before any is written.  Applies a
// diagonal block's interchanges to the columns beside it in one parallel
// pass (the interchanges never leave the block).
__global__ void __launch_bounds__(256) sp_permute_kernel(cf* __restrict__ A, int64_t lda, int64_t row0, int jb,
                                                         int64_t col0, int64_t ncols,
                                                         const int32_t* __restrict__ perm) {
    const int lane = threadIdx.x & 31;
    const int64_t col = col0 + (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (col >= col0 + ncols) return;
    cf* a = A + col * lda + row0;
    cf v[kSpB / 32];
#pragma unroll
    for (int u = 0; u < kSpB / 32; ++u) {
        const int i = lane + 32 * u;
        v[u] = i < jb ? a[perm[i]] : cf{0.0f, 0.0f};
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < kSpB / 32; ++u) {
        const int i = lane + 32 * u;
        if (i < jb) a[i] = v[u];
    }
}

// L21 = A21 U11^-1 for the rows below the diagonal block.  Four warps share
// 32 rows: lane i holds row i, warp w its columns 32w .. 32w+31 in
// registers.  The solve proceeds by column chunks: in phase k warp k
// finishes chunk k lane-locally (x_j = a_j / U_jj, then a_l -= x_j U_jl for
// the later columns of the chunk) and publishes it in shared memory; after
// one barrier the warps of later chunks remove it from theirs (a 32 x 32
// block product per lane).  No shuffles, no divergence; U11 (upper
// triangle of the factored block) is staged row-major in shared memory and
// read as broadcasts.  The largest |L21| goes to ws->lmax_bits.
constexpr int kSpGroups = 2;                     // 32-row groups per CTA
constexpr int kSpL21Threads = 32 * 4 * kSpGroups;
constexpr int kSpXStride = 33;                   // complex elements per row of the exchange buffer

__device__ __forceinline__ void load_u2(const cf* __restrict__ src, cf& u0, cf& u1) {
    const float4 v = *reinterpret_cast<const float4*>(src);
    u0 = cf{v.x, v.y};
    u1 = cf{v.z, v.w};
}

__global__ void __launch_bounds__(kSpL21Threads, 1)
    sp_l21_kernel(cf* __restrict__ A, int64_t lda, int64_t j0, int jb, int64_t row_end,
                  const cf* __restrict__ inv_diag, PanelWs* ws, float* __restrict__ a_hi, float* __restrict__ a_lo) {
    extern __shared__ __align__(16) unsigned char sp_smem[];
    cf* sU = reinterpret_cast<cf*>(sp_smem);                 // [kSpB][kSpUStride]
    cf* sInv = sU + (size_t)kSpB * kSpUStride;               // [kSpB]
    cf* sX = sInv + kSpB;                                    // [2][kSpGroups][32][kSpXStride]
    const int tid = threadIdx.x;
    // staged with sixteen loads in flight per thread before the stores
    constexpr int kU = 16;
    for (int base = 0; base < kSpB * kSpB; base += kU * kSpL21Threads) {
        cf t[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int idx = base + u * kSpL21Threads + tid;
            const int j = idx % kSpB, col = idx / kSpB;  // coalesced down each column
            t[u] = (idx < kSpB * kSpB && j <= col && col < jb) ? A[(j0 + j) + (j0 + col) * lda] : cf{0.0f, 0.0f};
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int idx = base + u * kSpL21Threads + tid;
            if (idx < kSpB * kSpB) sU[(idx % kSpB) * kSpUStride + idx / kSpB] = t[u];
        }
    }
    for (int j = tid; j < kSpB; j += blockDim.x) sInv[j] = j < jb ? inv_diag[j] : cf{0.0f, 0.0f};
    const int lane = tid & 31, warp = tid >> 5;
    const int w = warp & 3;          // column chunk of this warp
    const int grp = warp >> 2;       // 32-row group
    const int64_t row = j0 + jb + ((int64_t)blockIdx.x * kSpGroups + grp) * 32 + lane;
    const bool row_ok = row < row_end;
    cf a[32];
#pragma unroll
    for (int l = 0; l < 32; ++l) {
        const int col = 32 * w + l;
        a[l] = (row_ok && col < jb) ? A[row + (j0 + col) * lda] : cf{0.0f, 0.0f};
    }
    __syncthreads();
    float lmax = 0.0f;
    const int nchunks = (jb + 31) / 32;
    for (int k = 0; k < nchunks; ++k) {
        cf* xb = sX + ((size_t)((k & 1) * kSpGroups + grp) * 32 + lane) * kSpXStride;
        if (w == k) {
#pragma unroll
            for (int j = 0; j < 32; ++j) {
                const cf* urow = sU + (size_t)(32 * k + j) * kSpUStride + 32 * k;
                const cf x = a[j] * sInv[32 * k + j];
                a[j] = x;
                lmax = fmaxf(lmax, cabs1f(x));
#pragma unroll
                for (int l0 = (j + 1) & ~1; l0 < 32; l0 += 2) {
                    cf u0, u1;
                    load_u2(urow + l0, u0, u1);
                    if (l0 > j) a[l0] = a[l0] - x * u0;
                    a[l0 + 1] = a[l0 + 1] - x * u1;
                }
            }
#pragma unroll
            for (int j = 0; j < 32; ++j) xb[j] = a[j];
        }
        __syncthreads();
        if (w > k) {
            for (int j = 0; j < 32; ++j) {
                const cf* urow = sU + (size_t)(32 * k + j) * kSpUStride + 32 * w;
                const cf x = xb[j];
#pragma unroll
                for (int l0 = 0; l0 < 32; l0 += 2) {
                    cf u0, u1;
                    load_u2(urow + l0, u0, u1);
                    a[l0] = a[l0] - x * u0;
                    a[l0 + 1] = a[l0 + 1] - x * u1;
                }
            }
        }
    }
    if (row_ok) {
#pragma unroll
        for (int l = 0; l < 32; ++l) {
            const int col = 32 * w + l;
            if (col < jb) A[row + (j0 + col) * lda] = a[l];
        }
    }
    if (a_hi != nullptr) {
        // L21 also as the packed operand of the trailing updates (rows from
        // j0 + jb, inner dimension jb): each complex l is the 2 x 2 block
        // [[re, -im], [im, re]]; rows past the matrix and columns past jb
        // hold zeros, so that the tiles they pad contribute nothing
        const int n_ks = tc_n_ks(jb);
        const int64_t rho = 2 * (row - (j0 + jb));
#pragma unroll
        for (int l = 0; l < 32; l += 2) {
            const int64_t kap4 = 2 * (32 * w + l);
            if (kap4 < (int64_t)n_ks * TC_KS) {
                const cf v0 = a[l], v1 = a[l + 1];
                tc_store_a4(a_hi, a_lo, n_ks, rho, kap4, make_float4(v0.re, -v0.im, v1.re, -v1.im));
                tc_store_a4(a_hi, a_lo, n_ks, rho + 1, kap4, make_float4(v0.im, v0.re, v1.im, v1.re));
            }
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, off));
    // NaN-safe: a NaN compares false and raises the bound to +inf
    if (lane == 0) atomicMax(&ws->lmax_bits, (lmax == lmax) ? __float_as_uint(lmax) : 0x7f800000u);
}

}  // namespace

// The panel of columns [j0, j0+jb) (jb <= 128) over rows [j0, n): the
// diagonal block factored with pivots among its own rows, then L21.
// `inv_diag`: 128 complex64 of device scratch for the reciprocal pivots;
// `perm` (128 int32) receives the block's rows in pivot order; with
// `pack_a` set, L21 is also written as the packed A operand (hi / lo
// planes) of the updates that follow.
mw_status static_panel_c64(cf* A, int64_t lda, int64_t n, int64_t j0, int jb, int32_t* ipiv, int32_t* info,
                           PanelWs* ws, cf* inv_diag, int32_t* perm, const TcPlanes* pack_a, cudaStream_t st) {
    MW_REQUIRE(jb >= 1 && jb <= kSpB, "static panel width %d outside 1..%d", jb, kSpB);
    static bool configured = false;
    const size_t smem = sizeof(cf) * ((size_t)kSpB * kSpUStride + kSpB + (size_t)2 * kSpGroups * 32 * kSpXStride);
    if (!configured) {
        MW_CHECK_CUDA(cudaFuncSetAttribute(sp_l21_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        MW_CHECK_CUDA(cudaFuncSetAttribute(sp_diag_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)kSpDiagSmem));
        configured = true;
    }
    {
        ProfileScope ps(PC_PANEL, st, 8.0 * (double)jb * jb * jb / 3.0, 16.0 * (double)jb * jb);
        sp_diag_kernel<<<1, kSpDiagThreads, kSpDiagSmem, st>>>(A, lda, j0, jb, ipiv, info, inv_diag, perm, ws);
        count_launch();
    }
    {
        const int64_t rows = n - j0 - jb;
        ProfileScope ps(PC_L21, st, 4.0 * (double)rows * jb * jb, 16.0 * (double)rows * jb);
        if (rows > 0) {
            const int64_t per_cta = (int64_t)kSpGroups * 32;
            const unsigned grid = (unsigned)((rows + per_cta - 1) / per_cta);
            sp_l21_kernel<<<grid, kSpL21Threads, smem, st>>>(A, lda, j0, jb, n, inv_diag, ws,
                                                             pack_a ? pack_a->a_hi : nullptr,
                                                             pack_a ? pack_a->a_lo : nullptr);
            count_launch();
        }
    }
    MW_CHECK_CUDA(cudaGetLastError());
    return MW_OK;
}

// Every block's interchanges applied to the columns left of it (the L
// factors of the earlier blocks), all blocks in one launch: blockIdx.y + 1
// is the block, blockIdx.x a chunk of eight columns.  `perm_all` holds the
// n rows in pivot order, block by block.
__global__ void __launch_bounds__(256) sp_left_permute_kernel(cf* __restrict__ A, int64_t lda, int64_t n,
                                                              const int32_t* __restrict__ perm_all) {
    const int64_t j0 = ((int64_t)blockIdx.y + 1) * kSpB;
    const int jb = (int)((n - j0) < kSpB ? (n - j0) : kSpB);
    const int lane = threadIdx.x & 31;
    const int64_t col = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (col >= j0) return;
    const int32_t* perm = perm_all + j0;
    cf* a = A + col * lda + j0;
    cf v[kSpB / 32];
#pragma unroll
    for (int u = 0; u < kSpB / 32; ++u) {
        const int i = lane + 32 * u;
        v[u] = i < jb ? a[perm[i]] : cf{0.0f, 0.0f};
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < kSpB / 32; ++u) {
        const int i = lane + 32 * u;
        if (i < jb) a[i] = v[u];
    }
}

void static_left_permute_c64(cf* A, int64_t lda, int64_t n, const int32_t* perm_all, cudaStream_t st) {
    const int64_t nb = (n + kSpB - 1) / kSpB;
    if (nb < 2) return;
    const int64_t last0 = (nb - 1) * kSpB;  // widest left part
    ProfileScope ps(PC_LASWP, st, 0.0, sizeof(cf) * (double)n * n);
    dim3 grid((unsigned)((last0 + 7) / 8), (unsigned)(nb - 1));
    sp_left_permute_kernel<<<grid, 256, 0, st>>>(A, lda, n, perm_all);
    count_launch();
}

// Every block's interchanges applied to columns [0, ncols) of B (n rows, a
// solve's right-hand sides): the whole row permutation of a static-pivot
// factorisation in one parallel pass (the interchanges never leave their
// block).  blockIdx.y is the block, one warp per column.
__global__ void __launch_bounds__(256) sp_block_permute_kernel(cf* __restrict__ B, int64_t ldb, int64_t n,
                                                               int64_t ncols, const int32_t* __restrict__ perm_all) {
    const int64_t j0 = (int64_t)blockIdx.y * kSpB;
    const int jb = (int)((n - j0) < kSpB ? (n - j0) : kSpB);
    const int lane = threadIdx.x & 31;
    const int64_t col = (int64_t)blockIdx.x * 8 + (threadIdx.x >> 5);
    if (col >= ncols) return;
    const int32_t* perm = perm_all + j0;
    cf* a = B + col * ldb + j0;
    cf v[kSpB / 32];
#pragma unroll
    for (int u = 0; u < kSpB / 32; ++u) {
        const int i = lane + 32 * u;
        v[u] = i < jb ? a[perm[i]] : cf{0.0f, 0.0f};
    }
    __syncwarp();
#pragma unroll
    for (int u = 0; u < kSpB / 32; ++u) {
        const int i = lane + 32 * u;
        if (i < jb) a[i] = v[u];
    }
}

void static_rows_permute_c64(cf* B, int64_t ldb, int64_t n, int64_t ncols, const int32_t* perm_all,
                             cudaStream_t st) {
    const int64_t nb = (n + kSpB - 1) / kSpB;
    if (nb < 1 || ncols <= 0) return;
    ProfileScope ps(PC_LASWP, st, 0.0, 2.0 * sizeof(cf) * (double)n * ncols);
    dim3 grid((unsigned)((ncols + 7) / 8), (unsigned)nb);
    sp_block_permute_kernel<<<grid, 256, 0, st>>>(B, ldb, n, ncols, perm_all);
    count_launch();
}

// The block's interchanges applied to columns [col0, col0 + ncols).
void static_permute_c64(cf* A, int64_t lda, int64_t row0, int jb, int64_t col0, int64_t ncols, const int32_t* perm,
                        cudaStream_t st) {
    if (ncols <= 0) return;
    ProfileScope ps(PC_LASWP, st, 0.0, 2.0 * sizeof(cf) * (double)jb * ncols);
    sp_permute_kernel<<<(unsigned)((ncols + 7) / 8), 256, 0, st>>>(A, lda, row0, jb, col0, ncols, perm);
    count_launch();
}

}  // namespace mw
