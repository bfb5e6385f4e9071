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

constexpr size_t kSpDiagSmem = sizeof(cf) * (kSpB * 33 + 3 * 32 * 33);

__device__ __forceinline__ void group_sync(int id) {
    // the 128 threads (four warps) of one column group
    asm volatile("bar.sync %0, 128;" ::"r"(id) : "memory");
}

// Factor A[j0 .. j0+jb) x [j0 .. j0+jb) in place with partial pivoting among
// these rows, blocked by 32-column chunks.  Thread (r, g) holds row r's
// columns 32g .. 32g+31 (chunk g) in registers.  Chunk k is factored by its
// own four warps alone (rank-1 updates inside the chunk, two group
// barriers per column); then every later chunk g takes the chunk's U rows
// (the pivot rows' chunk-g values, solved with the chunk's unit lower
// triangle by one warp) and removes the chunk from its unpivoted rows with
// one 32 x 32 block product per row.  A chosen pivot row keeps its place in
// registers (its later columns become its U row); rows move once, when the
// block is written back in pivot order.
__global__ void __launch_bounds__(kSpDiagThreads, 1)
    sp_diag_kernel(cf* __restrict__ A, int64_t lda, int64_t j0, int jb, int32_t* __restrict__ ipiv,
                   int32_t* __restrict__ info, cf* __restrict__ inv_diag, int32_t* __restrict__ perm, PanelWs* ws) {
    __shared__ cf s_col[kSpB];                 // column c of every row
    __shared__ cf s_u[32];                     // the pivot row's chunk values
    // dynamic: chunk k of every row (L values of the unpivoted rows), then
    // the U rows of chunk k's pivots in each later chunk
    extern __shared__ __align__(16) unsigned char sp_diag_smem[];
    auto s_L = reinterpret_cast<cf(*)[33]>(sp_diag_smem);                          // [kSpB][33]
    auto s_Ug = reinterpret_cast<cf(*)[32][33]>(sp_diag_smem + sizeof(cf) * kSpB * 33);  // [3][32][33]
    __shared__ unsigned long long s_wkey[4];
    __shared__ int s_piv[32];                  // physical rows chosen in chunk k
    __shared__ int s_pos_of[kSpB];             // current position of each physical row
    __shared__ int s_row_at[kSpB];             // physical row at each position
    const int tid = threadIdx.x;
    const int r = tid & (kSpB - 1);
    const int g = tid >> 7;
    const int lane = tid & 31;
    const int wig = (tid >> 5) & 3;  // warp within its column group
    cf a[32];
#pragma unroll
    for (int i = 0; i < 32; ++i) {
        const int col = 32 * g + i;
        a[i] = (r < jb && col < jb) ? A[(j0 + r) + (j0 + col) * lda] : cf{0.0f, 0.0f};
    }
    bool active = r < jb;
    if (tid < kSpB) {
        s_pos_of[tid] = tid;
        s_row_at[tid] = tid;
    }
    __syncthreads();
    const int nchunk = (jb + 31) / 32;
    for (int k = 0; k < nchunk; ++k) {
        const int nck = (jb - 32 * k) < 32 ? (jb - 32 * k) : 32;  // columns in chunk k
        if (g == k) {
            // ---- (a) chunk k, by its own four warps
#pragma unroll
            for (int cc = 0; cc < 32; ++cc) {
                if (cc < nck) {
                    const int c = 32 * k + cc;
                    const cf v = a[cc];
                    s_col[r] = v;
                    // largest |re| + |im| among the rows not yet chosen, then
                    // the smallest position (LAPACK's icamax on the arranged
                    // rows); the low bits carry the physical row
                    unsigned long long key = 0;
                    if (active)
                        key = ((unsigned long long)__float_as_uint(cabs1f(v)) << 32) |
                              ((unsigned long long)(0xFFFFu - (unsigned int)s_pos_of[r]) << 16) |
                              (unsigned long long)r;
#pragma unroll
                    for (int off = 16; off > 0; off >>= 1) {
                        const unsigned long long o = __shfl_xor_sync(0xffffffffu, key, off);
                        key = o > key ? o : key;
                    }
                    if (lane == 0) s_wkey[wig] = key;
                    group_sync(1 + k);
                    unsigned long long best = s_wkey[0];
#pragma unroll
                    for (int w = 1; w < 4; ++w) best = s_wkey[w] > best ? s_wkey[w] : best;
                    const int p = (int)(best & 0xFFFFull);
                    const int pos_best = (int)(0xFFFFu - (unsigned int)((best >> 16) & 0xFFFFull));
                    const bool zero = (best >> 32) == 0ull;
                    const cf inv = zero ? cone<cf>() : crcp_sp(s_col[p]);
                    if (r == p) {
#pragma unroll
                        for (int l = cc; l < 32; ++l) s_u[l] = a[l];
                        active = false;
                        s_piv[cc] = p;
                    }
                    const cf lr = (active && !zero) ? s_col[r] * inv : cf{0.0f, 0.0f};
                    if (tid == 128 * k) {
                        // the interchange LAPACK makes: positions c and pos_best
                        ipiv[j0 + c] = (int32_t)(j0 + pos_best + 1);
                        if (zero) {
                            if (info[0] == 0) info[0] = (int32_t)(j0 + c + 1);
                            atomicExch(&ws->lmax_bits, 0x7f800000u);  // +inf: the block is singular
                        }
                        inv_diag[c] = inv;
                        const int pc = s_row_at[c];
                        s_row_at[c] = p;
                        s_row_at[pos_best] = pc;
                        s_pos_of[p] = c;
                        s_pos_of[pc] = pos_best;
                    }
                    group_sync(1 + k);  // s_u, s_pos_of complete; s_col and s_wkey read
                    if (active && !zero) {
                        a[cc] = lr;
#pragma unroll
                        for (int l = cc + 1; l < 32; ++l) a[l] = a[l] - lr * s_u[l];
                    }
                }
            }
#pragma unroll
            for (int l = 0; l < 32; ++l) s_L[r][l] = a[l];
        }
        __syncthreads();  // chunk k factored: s_L and s_piv published
        if (g > k) {
            // rows chosen in chunk k stop updating; the chunk's pivot rows
            // publish their chunk-g values (row i of the U block)
            int my_i = -1;
            for (int i = 0; i < nck; ++i)
                if (s_piv[i] == r) my_i = i;
            if (my_i >= 0) {
                active = false;
#pragma unroll
                for (int l = 0; l < 32; ++l) s_Ug[g - k - 1][my_i][l] = a[l];
            }
            group_sync(1 + g);
            if (wig == 0) {
                // U = L_kk^-1 (pivot rows): lane l solves column l, the rows
                // already solved read back from shared memory
                for (int i = 1; i < nck; ++i) {
                    const int pi = s_piv[i];
                    cf t = s_Ug[g - k - 1][i][lane];
                    for (int jj = 0; jj < i; ++jj) t = t - s_L[pi][jj] * s_Ug[g - k - 1][jj][lane];
                    s_Ug[g - k - 1][i][lane] = t;
                }
            }
            group_sync(1 + g);
            if (my_i >= 0) {
#pragma unroll
                for (int l = 0; l < 32; ++l) a[l] = s_Ug[g - k - 1][my_i][l];
            }
            // the block product, by whole warps that still hold unpivoted rows
            if (__any_sync(0xffffffffu, active) && active) {
                for (int jj = 0; jj < nck; ++jj) {
                    const cf x = s_L[r][jj];
                    const cf* urow = &s_Ug[g - k - 1][jj][0];
#pragma unroll
                    for (int l = 0; l < 32; ++l) a[l] = a[l] - x * urow[l];
                }
            }
        } else if (g < k) {
            // earlier chunks: only the chosen rows change state
            for (int i = 0; i < nck; ++i)
                if (s_piv[i] == r) active = false;
        }
        __syncthreads();  // s_L, s_Ug and s_piv free for the next chunk
    }
    if (r < jb) {
        const int pos = s_pos_of[r];
        const int64_t row = j0 + pos;
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            const int col = 32 * g + i;
            if (col < jb) A[row + (j0 + col) * lda] = a[i];
        }
        // the block's rows in pivot order: position pos holds row r
        if (g == 0) perm[pos] = r;
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
                  const cf* __restrict__ inv_diag, PanelWs* ws) {
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
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) lmax = fmaxf(lmax, __shfl_xor_sync(0xffffffffu, lmax, off));
    // NaN-safe: a NaN compares false and raises the bound to +inf
    if (lane == 0) atomicMax(&ws->lmax_bits, (lmax == lmax) ? __float_as_uint(lmax) : 0x7f800000u);
}

}  // namespace

// The panel of columns [j0, j0+jb) (jb <= 128) over rows [j0, n): the
// diagonal block factored with pivots among its own rows, then L21.
// `inv_diag`: 128 complex64 of device scratch for the reciprocal pivots;
// `perm` (128 int32) receives the block's rows in pivot order.
mw_status static_panel_c64(cf* A, int64_t lda, int64_t n, int64_t j0, int jb, int32_t* ipiv, int32_t* info,
                           PanelWs* ws, cf* inv_diag, int32_t* perm, cudaStream_t st) {
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
            sp_l21_kernel<<<grid, kSpL21Threads, smem, st>>>(A, lda, j0, jb, n, inv_diag, ws);
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

// The block's interchanges applied to columns [col0, col0 + ncols).
void static_permute_c64(cf* A, int64_t lda, int64_t row0, int jb, int64_t col0, int64_t ncols, const int32_t* perm,
                        cudaStream_t st) {
    if (ncols <= 0) return;
    ProfileScope ps(PC_LASWP, st, 0.0, 2.0 * sizeof(cf) * (double)jb * ncols);
    sp_permute_kernel<<<(unsigned)((ncols + 7) / 8), 256, 0, st>>>(A, lda, row0, jb, col0, ncols, perm);
    count_launch();
}

}  // namespace mw
