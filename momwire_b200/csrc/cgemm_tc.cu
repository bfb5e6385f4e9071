// Tensor-core complex update C -= A B for the mixed-precision LU (sm_100a).
//
// C is complex64, column-major.  The product is carried out as the real GEMM
//     C_real (2m x n)  -=  Ahat (2m x 2k) * Breal (2k x n)
// where C_real interleaves re/im down each column (the memory of C itself),
// Ahat holds each complex a as the 2x2 block [[re, -im], [im, re]] and
// Breal interleaves re/im of B down each column.  Every fp32 operand is split
// as x = hi + lo with hi = tf32(x), and the MMA sums hi*hi + hi*lo + lo*hi
// ("3xTF32"), which keeps fp32-level accuracy at tensor-core rate.
//
// Kernel structure (one persistent CTA per SM, 64 + 32 x TC_EPI_WARPS threads):
//   warp 0      producer: cp.async.bulk copies of pre-tiled operand stages
//               into a TC_STAGES-deep shared-memory ring (mbarrier complete_tx);
//   warp 1      allocates 512 TMEM columns; one lane issues tcgen05.mma
//               (M=128, N=256, K=8, kind::tf32) into one of two TMEM
//               accumulators and commits to mbarriers;
//   warps 2..   epilogue: tcgen05.ld the accumulator, C -= D with coalesced
//               loads/stores (two warps per TMEM lane quadrant, each half
//               of the columns, so twice the loads are in flight), then
//               hand the accumulator back.
// Operands are packed by the two pack kernels below into the shared-memory
// image of a K-major, no-swizzle UMMA tile: [block][stage][chunk][row][4],
// so each stage block is one contiguous bulk copy.
// Every wait is bounded; on a timeout the kernel records MW_ERR_TIMEOUT,
// lets each role finish without further work, and frees its TMEM.
#include <cstdint>

#include "common.cuh"
#include "tc_common.cuh"
#include "tc_layout.cuh"

namespace mw {

#ifndef MW_TC_STAGES
#define MW_TC_STAGES 4
#endif
#ifndef MW_TC_EPI_WARPS
#define MW_TC_EPI_WARPS 8
#endif
constexpr int TC_STAGES = MW_TC_STAGES;             // depth of the shared-memory ring
constexpr int TC_STAGE_BYTES = 2 * TC_A_BYTES + 2 * TC_B_BYTES;
constexpr int TC_EPI_WARPS = MW_TC_EPI_WARPS;       // 4 or 8: each TMEM lane quadrant by 1 or 2 warps
constexpr int TC_THREADS = 64 + 32 * TC_EPI_WARPS;
static_assert(TC_KS % 8 == 0, "a stage holds whole K=8 MMA steps");
static_assert(TC_EPI_WARPS == 4 || TC_EPI_WARPS == 8, "epilogue warps cover the four TMEM lane quadrants");
static_assert(TC_STAGES * TC_STAGE_BYTES <= 200 * 1024, "operand ring exceeds shared memory");
constexpr uint32_t TC_TMEM_COLS = 512;              // two 256-column accumulators

struct TcArgs {
    const float* a_hi;
    const float* a_lo;
    const float* b_hi;
    const float* b_lo;
    float* C;          // complex64 column-major, viewed as floats
    int64_t ldc;       // in complex elements
    int64_t m_real;    // 2 * complex rows
    int64_t n;         // columns
    int n_mb, n_nb, n_ks;
    int* err;
    // batch of independent updates: strides between consecutive C
    // matrices (floats) and packed operand planes (floats)
    int batch;
    int64_t c_stride;
    int64_t a_pstride, b_pstride;
    // two-part inner dimension: stages [0, n_ks1) from the planes above,
    // stages [n_ks1, n_ks) from these (each part packed on its own, with its
    // own stage count); n_ks1 = 0: one part
    const float* a_hi2 = nullptr;
    const float* a_lo2 = nullptr;
    const float* b_hi2 = nullptr;
    const float* b_lo2 = nullptr;
    int n_ks1 = 0;
};

// ---------------------------------------------------------------- kernel
__global__ void __launch_bounds__(TC_THREADS, 1) cgemm_tc_kernel(TcArgs P) {
    extern __shared__ __align__(1024) uint8_t tc_smem[];
    __shared__ __align__(8) uint64_t bar_full[TC_STAGES], bar_empty[TC_STAGES];
    __shared__ __align__(8) uint64_t bar_accf[2], bar_acce[2], bar_done;
    __shared__ uint32_t s_tmem;

    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    const int per_mat = P.n_mb * P.n_nb;
    const int n_tiles = per_mat * (P.batch > 0 ? P.batch : 1);
    int* err = P.err;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_STAGES; ++s) {
            mbar_init(&bar_full[s], 1);
            mbar_init(&bar_empty[s], 1);
        }
        for (int a = 0; a < 2; ++a) {
            mbar_init(&bar_accf[a], 1);
            mbar_init(&bar_acce[a], TC_EPI_WARPS);
        }
        mbar_init(&bar_done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 1) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&s_tmem)),
                     "r"(TC_TMEM_COLS)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem_base = s_tmem;

    if (warp == 0) {
        // ------------------------------------------------ producer
        if (lane == 0) {
            int slot = 0;
            // phase bit of each slot's empty barrier (bit s), all 1 at start;
            // slots fill round-robin from 0, so `issued` counts every slot
            uint32_t ph_empty = (1u << TC_STAGES) - 1u;
            long long issued = 0;
            bool dead = false;
            for (int t = blockIdx.x; t < n_tiles && !dead; t += gridDim.x) {
                const int bt = t / per_mat, tr = t - bt * per_mat;
                const int mb = tr % P.n_mb, nb = tr / P.n_mb;
                const int nks1 = P.n_ks1 > 0 ? P.n_ks1 : P.n_ks;
                for (int ks = 0; ks < P.n_ks; ++ks) {
                    if (!mbar_wait(&bar_empty[slot], (ph_empty >> slot) & 1u, err)) { dead = true; break; }
                    ph_empty ^= 1u << slot;
                    uint8_t* st = tc_smem + (size_t)slot * TC_STAGE_BYTES;
                    const bool second = ks >= nks1;
                    const int kp = second ? ks - nks1 : ks;             // stage within its part
                    const int nkp = second ? P.n_ks - nks1 : nks1;      // stages of its part
                    const size_t ao = (size_t)bt * P.a_pstride + ((size_t)mb * nkp + kp) * (TC_A_BYTES / 4);
                    const size_t bo = (size_t)bt * P.b_pstride + ((size_t)nb * nkp + kp) * (TC_B_BYTES / 4);
                    mbar_expect_tx(&bar_full[slot], TC_STAGE_BYTES);
                    bulk_g2s(st, (second ? P.a_hi2 : P.a_hi) + ao, TC_A_BYTES, &bar_full[slot]);
                    bulk_g2s(st + TC_A_BYTES, (second ? P.a_lo2 : P.a_lo) + ao, TC_A_BYTES, &bar_full[slot]);
                    bulk_g2s(st + 2 * TC_A_BYTES, (second ? P.b_hi2 : P.b_hi) + bo, TC_B_BYTES, &bar_full[slot]);
                    bulk_g2s(st + 2 * TC_A_BYTES + TC_B_BYTES, (second ? P.b_lo2 : P.b_lo) + bo, TC_B_BYTES,
                             &bar_full[slot]);
                    issued += 1;
                    slot = (slot + 1) % TC_STAGES;
                }
            }
            // drain: the last copy issued into each slot must have landed
            // before the CTA exits (the k-th fill of a slot completes phase
            // k-1 of its full barrier); bounded, and independent of the MMA
            // side so that it also ends when another role gave up
            for (int s = 0; s < TC_STAGES; ++s) {
                const long long fills = issued / TC_STAGES + (s < issued % TC_STAGES ? 1 : 0);
                if (fills == 0) continue;
                for (long long it = 0; it < TC_SPIN_LIMIT; ++it)
                    if (mbar_try_wait(&bar_full[s], (uint32_t)((fills - 1) & 1))) break;
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        // ------------------------------------------------ MMA issuer
        if (lane == 0) {
            const uint32_t idesc = idesc_tf32(TC_M, TC_N);
            int slot = 0;
            uint32_t ph_full = 0;  // phase bit of each slot's full barrier (bit s)
            uint32_t ph_acce[2] = {1, 1};
            bool dead = false;
            int lt = 0;
            for (int t = blockIdx.x; t < n_tiles && !dead; t += gridDim.x, ++lt) {
                const int acc = lt & 1;
                if (!mbar_wait(&bar_acce[acc], ph_acce[acc], err)) { dead = true; break; }
                ph_acce[acc] ^= 1;
                tc_fence_after();
                const uint32_t tmem_d = tmem_base + acc * TC_N;
                for (int ks = 0; ks < P.n_ks; ++ks) {
                    if (!mbar_wait(&bar_full[slot], (ph_full >> slot) & 1u, err)) { dead = true; break; }
                    ph_full ^= 1u << slot;
                    tc_fence_after();
                    const uint32_t st = smem_u32(tc_smem + (size_t)slot * TC_STAGE_BYTES);
                    const uint32_t a_hi = st, a_lo = st + TC_A_BYTES;
                    const uint32_t b_hi = st + 2 * TC_A_BYTES, b_lo = b_hi + TC_B_BYTES;
#pragma unroll
                    for (int kk = 0; kk < TC_KS / 8; ++kk) {
                        // one MMA step = two 16-byte K chunks
                        const uint32_t ao = kk * 2 * (TC_M * 16), bo = kk * 2 * (TC_N * 16);
                        const uint64_t dah = umma_desc(a_hi + ao, TC_M * 16, 128);
                        const uint64_t dal = umma_desc(a_lo + ao, TC_M * 16, 128);
                        const uint64_t dbh = umma_desc(b_hi + bo, TC_N * 16, 128);
                        const uint64_t dbl = umma_desc(b_lo + bo, TC_N * 16, 128);
                        const uint32_t first = (ks == 0 && kk == 0) ? 0u : 1u;
                        mma_tf32(tmem_d, dah, dbh, idesc, first);
                        mma_tf32(tmem_d, dah, dbl, idesc, 1u);
                        mma_tf32(tmem_d, dal, dbh, idesc, 1u);
                    }
                    mma_commit(&bar_empty[slot]);  // stage reusable once these MMAs finish
                    slot = (slot + 1) % TC_STAGES;
                }
                if (!dead) mma_commit(&bar_accf[acc]);
            }
            // teardown: no MMA may still be reading shared memory or writing
            // TMEM when the CTA frees them (commit tracks all prior MMAs)
            mma_commit(&bar_done);
            for (long long it = 0; it < TC_SPIN_LIMIT; ++it)
                if (mbar_try_wait(&bar_done, 0)) break;
        }
        __syncwarp();
    } else {
        // ------------------------------------------------ epilogue (warps 2..)
        const int quad = warp & 3;  // TMEM lane quadrant this warp may access
        // with eight epilogue warps, two share a quadrant and split its columns
        constexpr int kCols = TC_N * 4 / TC_EPI_WARPS;
        const int cbeg = ((warp - 2) / 4) * kCols;
        uint32_t ph_accf[2] = {0, 0};
        bool dead = false;
        int lt = 0;
        for (int t = blockIdx.x; t < n_tiles && !dead; t += gridDim.x, ++lt) {
            const int acc = lt & 1;
            const int bt = t / per_mat, tr = t - bt * per_mat;
            const int mb = tr % P.n_mb, nb = tr / P.n_mb;
            bool ok = true;
            if (lane == 0) ok = mbar_wait(&bar_accf[acc], ph_accf[acc], err);
            ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
            if (!ok) { dead = true; break; }
            ph_accf[acc] ^= 1;
            tc_fence_after();
            const int64_t r = (int64_t)mb * TC_M + quad * 32 + lane;  // real row
            const uint32_t taddr = tmem_base + ((uint32_t)(quad * 32) << 16) + acc * TC_N;
            // 32 columns per round: all loads of C issue before any store so
            // that they overlap (a store may alias the next load otherwise)
            for (int c0 = cbeg; c0 < cbeg + kCols; c0 += 32) {
                float v[32], old[32];
                tmem_ld16(taddr + c0, v);
                tmem_ld16(taddr + c0 + 16, v + 16);
                const int64_t col0 = (int64_t)nb * TC_N + c0;
                const bool row_ok = r < P.m_real;
                float* cbase = P.C + (int64_t)bt * P.c_stride + r + col0 * 2 * P.ldc;
                const int64_t cstep = 2 * P.ldc;
#pragma unroll
                for (int e = 0; e < 32; ++e)
                    old[e] = (row_ok && col0 + e < P.n) ? __ldcs(cbase + e * cstep) : 0.f;
#pragma unroll
                for (int e = 0; e < 32; ++e)
                    if (row_ok && col0 + e < P.n) __stcs(cbase + e * cstep, old[e] - v[e]);
            }
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&bar_acce[acc]);
        }
    }
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem_base), "r"(TC_TMEM_COLS)
                     : "memory");
    }
}

// -------------------------------------------------------------- packing

// Ahat (2m x 2k, from complex A at A + (i + l*lda)) packed as
// [mb][ks][chunk TC_CHUNKS][row 128][4]; zero beyond (2m, 2k).
__global__ void pack_a_kernel(const cf* __restrict__ A, int64_t lda, int64_t m, int64_t k, int n_mb, int n_ks,
                              float* __restrict__ hi, float* __restrict__ lo, int64_t a_stride, int64_t p_stride) {
    const int64_t total = (int64_t)n_mb * n_ks * TC_CHUNKS * TC_M;  // float4 slots
    A += blockIdx.y * a_stride;  // batch entry
    hi += blockIdx.y * p_stride;
    lo += blockIdx.y * p_stride;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int row = (int)(q % TC_M);
        int64_t rest = q / TC_M;
        const int ch = (int)(rest % TC_CHUNKS);
        rest /= TC_CHUNKS;
        const int ks = (int)(rest % n_ks);
        const int mb = (int)(rest / n_ks);
        const int64_t rho = (int64_t)mb * TC_M + row;  // real row
        const int64_t kap0 = (int64_t)ks * TC_KS + ch * 4;
        float4 vh, vl;
        float* ph = &vh.x;
        float* pl = &vl.x;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int64_t kap = kap0 + e;
            float x = 0.f;
            if (rho < 2 * m && kap < 2 * k) {
                const cf a = A[(rho >> 1) + (kap >> 1) * lda];
                const int t = (int)(rho & 1), s = (int)(kap & 1);
                x = (t == 0) ? (s == 0 ? a.re : -a.im) : (s == 0 ? a.im : a.re);
            }
            const float h = tf32_hi(x);
            ph[e] = h;
            pl[e] = x - h;
        }
        reinterpret_cast<float4*>(hi)[q] = vh;
        reinterpret_cast<float4*>(lo)[q] = vl;
    }
}

// Breal^T (n x 2k, from complex B at B + (l + j*ldb)) packed as
// [nb][ks][chunk TC_CHUNKS][row 256][4]; zero beyond (n, 2k).
__global__ void pack_b_kernel(const cf* __restrict__ B, int64_t ldb, int64_t k, int64_t n, int n_nb, int n_ks,
                              float* __restrict__ hi, float* __restrict__ lo, int64_t b_stride, int64_t p_stride) {
    const int64_t total = (int64_t)n_nb * n_ks * TC_CHUNKS * TC_N;
    B += blockIdx.y * b_stride;  // batch entry
    hi += blockIdx.y * p_stride;
    lo += blockIdx.y * p_stride;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < total; q += (int64_t)gridDim.x * blockDim.x) {
        const int row = (int)(q % TC_N);
        int64_t rest = q / TC_N;
        const int ch = (int)(rest % TC_CHUNKS);
        rest /= TC_CHUNKS;
        const int ks = (int)(rest % n_ks);
        const int nb = (int)(rest / n_ks);
        const int64_t j = (int64_t)nb * TC_N + row;
        const int64_t kap0 = (int64_t)ks * TC_KS + ch * 4;
        float4 vh, vl;
        float* ph = &vh.x;
        float* pl = &vl.x;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
            const int64_t kap = kap0 + e;
            float x = 0.f;
            if (j < n && kap < 2 * k) {
                const cf b = B[(kap >> 1) + j * ldb];
                x = (kap & 1) ? b.im : b.re;
            }
            const float h = tf32_hi(x);
            ph[e] = h;
            pl[e] = x - h;
        }
        reinterpret_cast<float4*>(hi)[q] = vh;
        reinterpret_cast<float4*>(lo)[q] = vl;
    }
}

size_t tc_pack_a_bytes(int64_t m, int64_t k) {
    int64_t n_mb = (2 * m + TC_M - 1) / TC_M, n_ks = (2 * k + TC_KS - 1) / TC_KS;
    return (size_t)n_mb * n_ks * TC_A_BYTES;
}
size_t tc_pack_b_bytes(int64_t k, int64_t n) {
    int64_t n_nb = (n + TC_N - 1) / TC_N, n_ks = (2 * k + TC_KS - 1) / TC_KS;
    return (size_t)n_nb * n_ks * TC_B_BYTES;
}

// Batched: C_b (m x n, complex64 col-major) -= A_b (m x k) B_b (k x n) for
// b < batch, matrices `sa`, `sb`, `sc` complex elements apart; packed
// planes in `ws` (a_hi | a_lo | b_hi | b_lo, each 1 KB aligned, batch-major).
mw_status cgemm_tc_update_batched(int64_t m, int64_t n, int64_t k, int batch, const cf* A, int64_t lda, int64_t sa,
                                  const cf* B, int64_t ldb, int64_t sb, cf* C, int64_t ldc, int64_t sc, void* ws,
                                  size_t ws_bytes, int* err, cudaStream_t st, int max_ctas) {
    if (m <= 0 || n <= 0 || k <= 0 || batch <= 0) return MW_OK;
    const int n_mb = (int)((2 * m + TC_M - 1) / TC_M);
    const int n_nb = (int)((n + TC_N - 1) / TC_N);
    const int n_ks = (int)((2 * k + TC_KS - 1) / TC_KS);
    const size_t ab = tc_pack_a_bytes(m, k), bb = tc_pack_b_bytes(k, n);
    auto al = [](size_t x) { return (x + 1023) & ~size_t(1023); };
    MW_REQUIRE(2 * al(ab * batch) + 2 * al(bb * batch) <= ws_bytes, "tensor-core GEMM workspace too small");
    MW_REQUIRE(batch <= 65535, "batch too large");
    char* w = static_cast<char*>(ws);
    float* a_hi = reinterpret_cast<float*>(w);
    float* a_lo = reinterpret_cast<float*>(w + al(ab * batch));
    float* b_hi = reinterpret_cast<float*>(w + 2 * al(ab * batch));
    float* b_lo = reinterpret_cast<float*>(w + 2 * al(ab * batch) + al(bb * batch));
    {
        ProfileScope ps(PC_MISC, st);
        int64_t qa = (int64_t)n_mb * n_ks * TC_CHUNKS * TC_M, qb = (int64_t)n_nb * n_ks * TC_CHUNKS * TC_N;
        dim3 ga((unsigned)((qa + 255) / 256), (unsigned)batch), gb((unsigned)((qb + 255) / 256), (unsigned)batch);
        pack_a_kernel<<<ga, 256, 0, st>>>(A, lda, m, k, n_mb, n_ks, a_hi, a_lo, sa, (int64_t)(ab / 4));
        pack_b_kernel<<<gb, 256, 0, st>>>(B, ldb, k, n, n_nb, n_ks, b_hi, b_lo, sb, (int64_t)(bb / 4));
        count_launch(2);
    }
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        MW_CHECK_CUDA(cudaFuncSetAttribute(cgemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           TC_STAGES * TC_STAGE_BYTES));
    }
    TcArgs P{a_hi, a_lo, b_hi, b_lo, reinterpret_cast<float*>(C), ldc, 2 * m, n, n_mb, n_nb, n_ks, err,
             batch,    2 * sc, (int64_t)(ab / 4), (int64_t)(bb / 4)};
    const int64_t tiles = (int64_t)n_mb * n_nb * batch;
    MW_REQUIRE(tiles < (1ll << 31), "too many tiles");
    const int cap = (max_ctas > 0 && max_ctas < sms) ? max_ctas : sms;  // CTAs (= SMs) this update may hold
    const int grid = tiles < cap ? (int)tiles : cap;
    {
        // bytes: C read and written (complex64) plus the hi / lo operand
        // planes (Ahat 2m x 2k, Breal 2k x n, fp32 each)
        ProfileScope ps(PC_CGEMM_TC, st, 8.0 * (double)m * n * k * batch,
                        (16.0 * (double)m * n + 32.0 * (double)m * k + 16.0 * (double)k * n) * batch);
        cgemm_tc_kernel<<<grid, TC_THREADS, TC_STAGES * TC_STAGE_BYTES, st>>>(P);
    }
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

// The four planes inside a workspace laid out as cgemm_tc_workspace(m_max,
// n_max, k) lays it out; updates of any m <= m_max, n <= n_max, k may use
// them (the blocks of a plane keep their offsets).
TcPlanes tc_planes(void* ws, int64_t m_max, int64_t n_max, int64_t k) {
    auto al = [](size_t x) { return (x + 1023) & ~size_t(1023); };
    const size_t ab = tc_pack_a_bytes(m_max, k), bb = tc_pack_b_bytes(k, n_max);
    char* w = static_cast<char*>(ws);
    return TcPlanes{reinterpret_cast<float*>(w), reinterpret_cast<float*>(w + al(ab)),
                    reinterpret_cast<float*>(w + 2 * al(ab)), reinterpret_cast<float*>(w + 2 * al(ab) + al(bb))};
}

// A (m x k complex64, column-major) into the hi / lo A planes of an update
// with inner dimension k (the B operand is packed elsewhere); `batch`
// matrices at A + b a_stride into planes at a_hi / a_lo + b p_stride floats.
mw_status tc_pack_a(int64_t m, int64_t k, const cf* A, int64_t lda, float* a_hi, float* a_lo, cudaStream_t st,
                    int batch, int64_t a_stride, int64_t p_stride) {
    if (m <= 0 || k <= 0 || batch <= 0) return MW_OK;
    MW_REQUIRE(batch <= 65535, "batch too large");
    const int n_mb = (int)((2 * m + TC_M - 1) / TC_M);
    const int n_ks = tc_n_ks(k);
    const int64_t qa = (int64_t)n_mb * n_ks * TC_CHUNKS * TC_M;
    int64_t blocks = (qa + 255) / 256;
    if (blocks > 65535) blocks = 65535;  // the kernel strides over the rest
    ProfileScope ps(PC_MISC, st);
    pack_a_kernel<<<dim3((unsigned)blocks, (unsigned)batch), 256, 0, st>>>(A, lda, m, k, n_mb, n_ks, a_hi, a_lo,
                                                                           a_stride, p_stride);
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

mw_status cgemm_tc_prepacked(int64_t m, int64_t n, int64_t k, const TcPlanes& pl, cf* C, int64_t ldc, int* err,
                             cudaStream_t st, int max_ctas);

// C (m x n complex64) -= A1 B1 + A2 B2 from operands already packed, part p
// in planes pl<p> for an inner dimension k<p>: one launch for both parts.
mw_status cgemm_tc_prepacked2(int64_t m, int64_t n, int64_t k1, const TcPlanes& pl1, int64_t k2, const TcPlanes& pl2,
                              cf* C, int64_t ldc, int* err, cudaStream_t st, int max_ctas) {
    if (m <= 0 || n <= 0 || k1 <= 0) return MW_OK;
    if (k2 <= 0) return cgemm_tc_prepacked(m, n, k1, pl1, C, ldc, err, st, max_ctas);
    const int n_mb = (int)((2 * m + TC_M - 1) / TC_M);
    const int n_nb = (int)((n + TC_N - 1) / TC_N);
    const int nks1 = tc_n_ks(k1), nks2 = tc_n_ks(k2);
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        MW_CHECK_CUDA(cudaFuncSetAttribute(cgemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           TC_STAGES * TC_STAGE_BYTES));
    }
    TcArgs P{pl1.a_hi, pl1.a_lo, pl1.b_hi, pl1.b_lo, reinterpret_cast<float*>(C), ldc, 2 * m, n, n_mb, n_nb,
             nks1 + nks2, err, 1, 0, 0, 0, pl2.a_hi, pl2.a_lo, pl2.b_hi, pl2.b_lo, nks1};
    const int64_t tiles = (int64_t)n_mb * n_nb;
    MW_REQUIRE(tiles < (1ll << 31), "too many tiles");
    const int cap = (max_ctas > 0 && max_ctas < sms) ? max_ctas : sms;
    const int grid = tiles < cap ? (int)tiles : cap;
    {
        const double k = (double)(k1 + k2);
        ProfileScope ps(PC_CGEMM_TC, st, 8.0 * (double)m * n * k, 16.0 * (double)m * n + 32.0 * (double)m * k +
                                                                      16.0 * k * n);
        cgemm_tc_kernel<<<grid, TC_THREADS, TC_STAGES * TC_STAGE_BYTES, st>>>(P);
    }
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

// C (m x n complex64, column-major) -= A B from operands already packed in
// the planes (for an inner dimension k): no packing pass.
mw_status cgemm_tc_prepacked(int64_t m, int64_t n, int64_t k, const TcPlanes& pl, cf* C, int64_t ldc, int* err,
                             cudaStream_t st, int max_ctas) {
    if (m <= 0 || n <= 0 || k <= 0) return MW_OK;
    const int n_mb = (int)((2 * m + TC_M - 1) / TC_M);
    const int n_nb = (int)((n + TC_N - 1) / TC_N);
    const int n_ks = tc_n_ks(k);
    static int sms = 0;
    if (sms == 0) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        MW_CHECK_CUDA(cudaFuncSetAttribute(cgemm_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           TC_STAGES * TC_STAGE_BYTES));
    }
    TcArgs P{pl.a_hi, pl.a_lo, pl.b_hi, pl.b_lo, reinterpret_cast<float*>(C), ldc, 2 * m, n, n_mb, n_nb, n_ks, err,
             1, 0, 0, 0};
    const int64_t tiles = (int64_t)n_mb * n_nb;
    MW_REQUIRE(tiles < (1ll << 31), "too many tiles");
    const int cap = (max_ctas > 0 && max_ctas < sms) ? max_ctas : sms;
    const int grid = tiles < cap ? (int)tiles : cap;
    {
        ProfileScope ps(PC_CGEMM_TC, st, 8.0 * (double)m * n * k,
                        16.0 * (double)m * n + 32.0 * (double)m * k + 16.0 * (double)k * n);
        cgemm_tc_kernel<<<grid, TC_THREADS, TC_STAGES * TC_STAGE_BYTES, st>>>(P);
    }
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

mw_status cgemm_tc_update(int64_t m, int64_t n, int64_t k, const cf* A, int64_t lda, const cf* B, int64_t ldb, cf* C,
                          int64_t ldc, void* ws, size_t ws_bytes, int* err, cudaStream_t st, int max_ctas) {
    return cgemm_tc_update_batched(m, n, k, 1, A, lda, 0, B, ldb, 0, C, ldc, 0, ws, ws_bytes, err, st, max_ctas);
}

size_t cgemm_tc_workspace_batched(int64_t m, int64_t n, int64_t k, int batch) {
    auto al = [](size_t x) { return (x + 1023) & ~size_t(1023); };
    return 2 * al(tc_pack_a_bytes(m, k) * batch) + 2 * al(tc_pack_b_bytes(k, n) * batch);
}

size_t cgemm_tc_workspace(int64_t m, int64_t n, int64_t k) {
    auto al = [](size_t x) { return (x + 1023) & ~size_t(1023); };
    return 2 * al(tc_pack_a_bytes(m, k)) + 2 * al(tc_pack_b_bytes(k, n));
}

}  // namespace mw

using namespace mw;

extern "C" size_t mw_cgemm_tc_workspace_size(int64_t m, int64_t n, int64_t k) { return cgemm_tc_workspace(m, n, k); }

extern "C" mw_status mw_cgemm_tc_sub(int64_t m, int64_t n, int64_t k, const float* A, int64_t lda, const float* B,
                                     int64_t ldb, float* C, int64_t ldc, void* workspace, size_t workspace_bytes,
                                     int32_t* status, void* stream) {
    MW_REQUIRE(m >= 0 && n >= 0 && k >= 0, "negative size");
    MW_REQUIRE(A && B && C && workspace && status, "NULL argument");
    MW_REQUIRE(lda >= m && ldb >= k && ldc >= m, "leading dimension too small");
    return cgemm_tc_update(m, n, k, reinterpret_cast<const cf*>(A), lda, reinterpret_cast<const cf*>(B), ldb,
                           reinterpret_cast<cf*>(C), ldc, workspace, workspace_bytes, status, as_stream(stream), 0);
}
