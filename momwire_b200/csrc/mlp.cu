// Learned Sommerfeld surrogate (sm_100a): a 5 -> 128 -> 128 -> 128 -> 128
// -> 8 MLP with GELU that predicts the four remainder surfaces
// (I_rho^V, I_z^V, I_rho^H, I_phi^H; eqs 156-159 of the NEC-2 theory
// manual) of a Sommerfeld ground from normalised (rho, z+z', |eps|, arg eps,
// f).  The reference has no surrogate: it tabulates the surfaces by
// quadrature on an (R1, theta) grid per (eps, r1) bucket
// (_sommerfeld.py:648-813); the quadrature of somm.cu makes the training
// data and stays the fallback.
//
// Numerics: weights are BF16 (FP32 master copies for Adam), every product
// accumulates in FP32, GELU is the exact erf form in FP32.
//
// Training (hand-written SIMT kernels; an offline, once-per-model cost):
//   forward   per layer Z = X W^T + b, A = gelu(Z) (tiled FP32 GEMM with
//             BF16 weights converted on load), Z and A kept for backward;
//   loss      mean squared error over the 8 outputs;
//   backward  dZ = dA gelu'(Z), dW = dZ^T X, db = sum dZ, dX = dZ W;
//   Adam      bias-corrected moments, FP32 master weights re-rounded to BF16.
//
// Inference (tcgen05): one CTA evaluates 128 rows per tile.  Weights live in
// shared memory as K-major BF16 UMMA tiles; each layer is M=128 x N=128 x
// K=16-steps kind::f16 MMAs into a 128-column TMEM accumulator; the four
// warps read their TMEM lane quadrant, add bias, apply GELU and write the
// next layer's activations back to shared memory split as BF16 hi + lo
// (x = hi + lo, two MMAs per K step), which keeps ~16 significant bits of
// each activation against BF16's 8.  Every wait is bounded.
#include <cuda_bf16.h>

#include <cmath>
#include <cstdint>

#include "common.cuh"
#include "somm_proj.cuh"
#include "tc_common.cuh"

namespace mw {

constexpr int MLP_IN = 5, MLP_H = 128, MLP_OUT = 8, MLP_NL = 5;
__host__ __device__ constexpr int mlp_in_dim(int l) { return l == 0 ? MLP_IN : MLP_H; }
__host__ __device__ constexpr int mlp_out_dim(int l) { return l == MLP_NL - 1 ? MLP_OUT : MLP_H; }
__host__ __device__ constexpr int mlp_w_off(int l) {
    int o = 0;
    for (int i = 0; i < l; ++i) o += mlp_in_dim(i) * mlp_out_dim(i) + mlp_out_dim(i);
    return o;
}
__host__ __device__ constexpr int mlp_b_off(int l) { return mlp_w_off(l) + mlp_in_dim(l) * mlp_out_dim(l); }
constexpr int MLP_PARAMS = mlp_w_off(MLP_NL);  // 51,336

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_grad(float x) {
    const float cdf = 0.5f * (1.0f + erff(x * 0.70710678118654752f));
    const float pdf = 0.39894228040143268f * expf(-0.5f * x * x);
    return cdf + x * pdf;
}

// ---------------------------------------------------------------- training
// C (M x N) = A (M x K) B (K x N) [+ bias per column] [accumulate], element
// (i, k) of A at A[i*sai + k*sak], (k, j) of B at B[k*sbk + j*sbj]; B may be
// BF16 (weights).  64 x 64 tiles, 256 threads, 4 x 4 outputs per thread.
template <bool B_BF16>
__global__ void __launch_bounds__(256) mlp_gemm_kernel(int M, int N, int K, const float* __restrict__ A, int64_t sai,
                                                       int64_t sak, const void* __restrict__ Bv, int64_t sbk,
                                                       int64_t sbj, const float* __restrict__ bias,
                                                       float* __restrict__ C, int64_t ldc, int accumulate) {
    __shared__ float sA[16][64 + 4];
    __shared__ float sB[16][64 + 4];
    const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
    const int i0 = blockIdx.y * 64, j0 = blockIdx.x * 64;
    float acc[4][4] = {};
    for (int k0 = 0; k0 < K; k0 += 16) {
        for (int q = threadIdx.x; q < 16 * 64; q += 256) {
            const int kk = q / 64, r = q % 64;
            const int i = i0 + r, k = k0 + kk, j = j0 + r;
            sA[kk][r] = (i < M && k < K) ? A[i * sai + k * sak] : 0.f;
            float bval = 0.f;
            if (k < K && j < N) {
                if (B_BF16)
                    bval = __bfloat162float(reinterpret_cast<const __nv_bfloat16*>(Bv)[k * sbk + j * sbj]);
                else
                    bval = reinterpret_cast<const float*>(Bv)[k * sbk + j * sbj];
            }
            sB[kk][r] = bval;
        }
        __syncthreads();
#pragma unroll
        for (int kk = 0; kk < 16; ++kk) {
            float a[4], b[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                a[u] = sA[kk][ty * 4 + u];
                b[u] = sB[kk][tx * 4 + u];
            }
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[u][v] = fmaf(a[u], b[v], acc[u][v]);
        }
        __syncthreads();
    }
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) {
            const int i = i0 + ty * 4 + u, j = j0 + tx * 4 + v;
            if (i < M && j < N) {
                float val = acc[u][v] + (bias ? bias[j] : 0.f);
                if (accumulate) val += C[(int64_t)i * ldc + j];
                C[(int64_t)i * ldc + j] = val;
            }
        }
}

__global__ void gelu_fwd_kernel(const float* __restrict__ Z, float* __restrict__ A, int64_t n) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        A[q] = gelu(Z[q]);
}

__global__ void gelu_bwd_kernel(const float* __restrict__ Z, float* __restrict__ dA, int64_t n) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x)
        dA[q] *= gelu_grad(Z[q]);
}

// dOut = 2 (out - t) / (B * 8); loss += sum (out - t)^2 / (B * 8)
__global__ void mse_kernel(const float* __restrict__ out, const float* __restrict__ t, float* __restrict__ dout,
                           int64_t n, float inv_n, float* loss) {
    float s = 0.f;
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < n; q += (int64_t)gridDim.x * blockDim.x) {
        const float e = out[q] - t[q];
        dout[q] = 2.f * e * inv_n;
        s += e * e;
    }
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) atomicAdd(loss, s * inv_n);
}

// db[j] = sum_i dZ[i][j]
__global__ void colsum_kernel(const float* __restrict__ dZ, int M, int N, float* __restrict__ db) {
    const int j = blockIdx.x;
    float s = 0.f;
    for (int i = threadIdx.x; i < M; i += blockDim.x) s += dZ[(int64_t)i * N + j];
    __shared__ float red[32];
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        s = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.f;
        for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
        if (threadIdx.x == 0) db[j] = s;
    }
}

__global__ void adam_kernel(int n, float* __restrict__ p, __nv_bfloat16* __restrict__ pb, const float* __restrict__ g,
                            float* __restrict__ m, float* __restrict__ v, float lr, float b1, float b2, float eps,
                            float c1, float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi * c1) / (sqrtf(vi * c2) + eps);
        p[i] = pi;
        pb[i] = __float2bfloat16_rn(pi);
    }
}

// rows idx[i] of src (width w) -> row i of dst
__global__ void gather_rows_kernel(int n, int w, const float* __restrict__ src, const int64_t* __restrict__ idx,
                                   float* __restrict__ dst) {
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < n * w; q += gridDim.x * blockDim.x) {
        const int i = q / w, c = q - i * w;
        dst[q] = src[idx[i] * w + c];
    }
}

__global__ void to_bf16_kernel(int n, const float* __restrict__ p, __nv_bfloat16* __restrict__ pb) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        pb[i] = __float2bfloat16_rn(p[i]);
}

// training workspace: Z_l, A_l (B x 128 each, l < 4), out / dout (B x 8),
// two dA buffers (B x 128), gradient (MLP_PARAMS)
static size_t train_ws_floats(int B) {
    return (size_t)B * MLP_H * 8 + (size_t)B * MLP_OUT * 2 + (size_t)B * MLP_H * 2 + MLP_PARAMS +
           (size_t)B * (MLP_IN + MLP_OUT) + 64;
}

struct TrainWs {
    float *Z[4], *A[4], *out, *dout, *d0, *d1, *grad, *xg, *tg;
};

static TrainWs train_ws(void* ws, int B) {
    float* w = static_cast<float*>(ws);
    TrainWs t;
    for (int l = 0; l < 4; ++l) {
        t.Z[l] = w;
        w += (size_t)B * MLP_H;
        t.A[l] = w;
        w += (size_t)B * MLP_H;
    }
    t.out = w;
    w += (size_t)B * MLP_OUT;
    t.dout = w;
    w += (size_t)B * MLP_OUT;
    t.d0 = w;
    w += (size_t)B * MLP_H;
    t.d1 = w;
    w += (size_t)B * MLP_H;
    t.grad = w;
    w += MLP_PARAMS;
    t.xg = w;
    w += (size_t)B * MLP_IN;
    t.tg = w;
    return t;
}

static void gemm(int M, int N, int K, const float* A, int64_t sai, int64_t sak, const void* B, bool b_bf16,
                 int64_t sbk, int64_t sbj, const float* bias, float* C, int64_t ldc, bool acc, cudaStream_t st) {
    dim3 grid((N + 63) / 64, (M + 63) / 64);
    if (b_bf16)
        mlp_gemm_kernel<true><<<grid, 256, 0, st>>>(M, N, K, A, sai, sak, B, sbk, sbj, bias, C, ldc, acc);
    else
        mlp_gemm_kernel<false><<<grid, 256, 0, st>>>(M, N, K, A, sai, sak, B, sbk, sbj, bias, C, ldc, acc);
    count_launch();
}

// forward over B rows: fills t.Z / t.A / t.out
static void forward_train(const float* X, int B, const __nv_bfloat16* pb, const float* pf, TrainWs& t,
                          cudaStream_t st) {
    const float* in = X;
    for (int l = 0; l < MLP_NL; ++l) {
        const int K = mlp_in_dim(l), N = mlp_out_dim(l);
        float* Z = l < 4 ? t.Z[l] : t.out;
        // Z = in (B x K) W^T (K x N): W is N x K row-major -> (k, j) at W[j*K + k]
        gemm(B, N, K, in, K, 1, pb + mlp_w_off(l), true, 1, K, pf + mlp_b_off(l), Z, N, false, st);
        if (l < 4) {
            const int64_t n = (int64_t)B * N;
            gelu_fwd_kernel<<<(unsigned)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096), 256, 0, st>>>(Z, t.A[l], n);
            count_launch();
            in = t.A[l];
        }
    }
}

// backward from t.dout: gradient of every parameter into t.grad
static void backward_train(const float* X, int B, const __nv_bfloat16* pb, TrainWs& t, cudaStream_t st) {
    float* dcur = t.dout;  // dZ of layer l (B x N_l)
    float* bufs[2] = {t.d0, t.d1};
    for (int l = MLP_NL - 1; l >= 0; --l) {
        const int K = mlp_in_dim(l), N = mlp_out_dim(l);
        const float* in = l == 0 ? X : t.A[l - 1];
        // dW (N x K) = dZ^T (N x B) in (B x K)
        gemm(N, K, B, dcur, 1, N, in, false, K, 1, nullptr, t.grad + mlp_w_off(l), K, false, st);
        colsum_kernel<<<N, 256, 0, st>>>(dcur, B, N, t.grad + mlp_b_off(l));
        count_launch();
        if (l == 0) break;
        // dA_{l-1} (B x K) = dZ (B x N) W (N x K)
        float* dprev = bufs[l & 1];
        gemm(B, K, N, dcur, N, 1, pb + mlp_w_off(l), true, K, 1, nullptr, dprev, K, false, st);
        const int64_t n = (int64_t)B * K;
        gelu_bwd_kernel<<<(unsigned)((n + 255) / 256 < 4096 ? (n + 255) / 256 : 4096), 256, 0, st>>>(t.Z[l - 1], dprev,
                                                                                                    n);
        count_launch();
        dcur = dprev;
    }
}

// ---------------------------------------------------------- tc inference
constexpr int MI_ROWS = 128;
constexpr int MI_THREADS = 128;
constexpr int MI_K0 = 16;                                 // padded input width
constexpr int MI_W0_BYTES = MLP_H * MI_K0 * 2;            // 4 KB
constexpr int MI_WH_BYTES = MLP_H * MLP_H * 2;            // 32 KB
constexpr int MI_N4 = 16;                                 // padded output width
constexpr int MI_W4_BYTES = MI_N4 * MLP_H * 2;            // 4 KB
constexpr int MI_ACT_BYTES = MI_ROWS * MLP_H * 2;         // 32 KB per plane
constexpr int MI_OFF_W0 = 0;
constexpr int MI_OFF_WH = MI_OFF_W0 + MI_W0_BYTES;
constexpr int MI_OFF_W4 = MI_OFF_WH + 3 * MI_WH_BYTES;
constexpr int MI_OFF_HI = MI_OFF_W4 + MI_W4_BYTES;
constexpr int MI_OFF_LO = MI_OFF_HI + MI_ACT_BYTES;
constexpr int MI_OFF_BIAS = MI_OFF_LO + MI_ACT_BYTES;
constexpr int MI_SMEM = MI_OFF_BIAS + (4 * MLP_H + MI_N4) * 4;  // ~170 KB

// byte offset of element (row, k) in a K-major no-swizzle tile with R rows:
// [k / 8][row][8 x bf16]
__host__ __device__ __forceinline__ uint32_t kmaj_off(int row, int k, int R) {
    return (uint32_t)((k >> 3) * R * 16 + row * 16 + (k & 7) * 2);
}

struct MlpTc {
    uint8_t* sm;
    uint32_t tmem;
    uint64_t* bar;
    uint32_t phase;
};

// Stage weights (BF16, N x K row-major in pb) as K-major UMMA tiles, and the
// biases, into shared memory.
__device__ void mlp_tc_stage(uint8_t* sm, const __nv_bfloat16* __restrict__ pb, const float* __restrict__ pf) {
    const int tid = threadIdx.x;
    for (int q = tid; q < MLP_H * MI_K0; q += blockDim.x) {
        const int n = q / MI_K0, k = q % MI_K0;
        const __nv_bfloat16 v = k < MLP_IN ? pb[mlp_w_off(0) + n * MLP_IN + k] : __float2bfloat16_rn(0.f);
        *reinterpret_cast<__nv_bfloat16*>(sm + MI_OFF_W0 + kmaj_off(n, k, MLP_H)) = v;
    }
    for (int l = 1; l <= 3; ++l)
        for (int q = tid; q < MLP_H * MLP_H; q += blockDim.x) {
            const int n = q / MLP_H, k = q % MLP_H;
            *reinterpret_cast<__nv_bfloat16*>(sm + MI_OFF_WH + (l - 1) * MI_WH_BYTES + kmaj_off(n, k, MLP_H)) =
                pb[mlp_w_off(l) + n * MLP_H + k];
        }
    for (int q = tid; q < MI_N4 * MLP_H; q += blockDim.x) {
        const int n = q / MLP_H, k = q % MLP_H;
        const __nv_bfloat16 v = n < MLP_OUT ? pb[mlp_w_off(4) + n * MLP_H + k] : __float2bfloat16_rn(0.f);
        *reinterpret_cast<__nv_bfloat16*>(sm + MI_OFF_W4 + kmaj_off(n, k, MI_N4)) = v;
    }
    float* bias = reinterpret_cast<float*>(sm + MI_OFF_BIAS);
    for (int q = tid; q < 4 * MLP_H + MI_N4; q += blockDim.x) {
        const int l = q / MLP_H, j = q % MLP_H;
        float v = 0.f;
        if (l < 4)
            v = pf[mlp_b_off(l) + j];
        else if (j < MLP_OUT)
            v = pf[mlp_b_off(4) + j];
        bias[q] = v;
    }
}

// write 8 consecutive activations (k0..k0+7) of `row` as hi / lo BF16
__device__ __forceinline__ void put8(uint8_t* sm, int row, int k0, const float* x) {
    __align__(16) __nv_bfloat16 hi[8], lo[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        hi[i] = __float2bfloat16_rn(x[i]);
        lo[i] = __float2bfloat16_rn(x[i] - __bfloat162float(hi[i]));
    }
    *reinterpret_cast<uint4*>(sm + MI_OFF_HI + kmaj_off(row, k0, MI_ROWS)) = *reinterpret_cast<uint4*>(hi);
    *reinterpret_cast<uint4*>(sm + MI_OFF_LO + kmaj_off(row, k0, MI_ROWS)) = *reinterpret_cast<uint4*>(lo);
}

// One layer: D (TMEM) = A (hi + lo) W^T over K (multiple of 16); thread 0
// issues, every thread waits for completion.  Returns false on a timeout.
__device__ __forceinline__ bool mlp_tc_layer(MlpTc& c, int K, int N, uint32_t w_off, int* err) {
    fence_proxy_async_smem();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x == 0) {
        const uint32_t idesc = idesc_bf16(MI_ROWS, N);
        const uint32_t a_hi = smem_u32(c.sm + MI_OFF_HI), a_lo = smem_u32(c.sm + MI_OFF_LO);
        const uint32_t w = smem_u32(c.sm + w_off);
        for (int ks = 0; ks < K / 16; ++ks) {
            // one MMA step covers two 16-byte K chunks
            const uint64_t da_hi = umma_desc(a_hi + ks * 2 * MI_ROWS * 16, MI_ROWS * 16, 128);
            const uint64_t da_lo = umma_desc(a_lo + ks * 2 * MI_ROWS * 16, MI_ROWS * 16, 128);
            const uint64_t db = umma_desc(w + ks * 2 * N * 16, N * 16, 128);
            mma_bf16(c.tmem, da_hi, db, idesc, ks > 0 ? 1u : 0u);
            mma_bf16(c.tmem, da_lo, db, idesc, 1u);
        }
        mma_commit(c.bar);
    }
    // a block-wide vote keeps the control flow uniform even if the waits
    // of different threads were to end differently
    const bool ok = __syncthreads_and(mbar_wait(c.bar, c.phase, err) ? 1 : 0) != 0;
    c.phase ^= 1;
    tc_fence_after();
    return ok;
}

// Evaluate the tile whose layer-0 inputs (5 features per row, rows in the
// thread order) are `x`: returns this thread's 8 outputs in y.
__device__ bool mlp_tc_tile(MlpTc& c, const float x[MLP_IN], float y[MLP_OUT], int* err) {
    const int row = threadIdx.x;
    const float* bias = reinterpret_cast<const float*>(c.sm + MI_OFF_BIAS);
    {
        float v[8] = {x[0], x[1], x[2], x[3], x[4], 0.f, 0.f, 0.f};
        const float z[8] = {0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f, 0.f};
        put8(c.sm, row, 0, v);
        put8(c.sm, row, 8, z);
    }
    if (!mlp_tc_layer(c, MI_K0, MLP_H, MI_OFF_W0, err)) return false;
    const uint32_t trow = c.tmem + ((uint32_t)((threadIdx.x >> 5) * 32) << 16);
    for (int l = 1; l <= 4; ++l) {
        // epilogue of layer l-1: bias + GELU -> activations
        for (int c0 = 0; c0 < MLP_H; c0 += 16) {
            float v[16];
            tmem_ld16(trow + c0, v);
#pragma unroll
            for (int i = 0; i < 16; ++i) v[i] = gelu(v[i] + bias[(l - 1) * MLP_H + c0 + i]);
            put8(c.sm, row, c0, v);
            put8(c.sm, row, c0 + 8, v + 8);
        }
        const bool ok = l < 4 ? mlp_tc_layer(c, MLP_H, MLP_H, MI_OFF_WH + (l - 1) * MI_WH_BYTES, err)
                              : mlp_tc_layer(c, MLP_H, MI_N4, MI_OFF_W4, err);
        if (!ok) return false;
    }
    float v[16];
    tmem_ld16(trow, v);
#pragma unroll
    for (int i = 0; i < MLP_OUT; ++i) y[i] = v[i] + bias[4 * MLP_H + i];
    tc_fence_before();
    return true;
}

__device__ void mlp_tc_begin(MlpTc& c, uint8_t* sm, uint64_t* bar, uint32_t* tmem_slot) {
    c.sm = sm;
    c.bar = bar;
    c.phase = 0;
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (threadIdx.x < 32) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                     "r"(128)
                     : "memory");
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    c.tmem = *tmem_slot;
}

__device__ void mlp_tc_end(MlpTc& c) {
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (threadIdx.x < 32)
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(c.tmem), "r"(128) : "memory");
}

// rows of X (n x 5 features) -> Y (n x 8); persistent CTAs over 128-row tiles
__global__ void __launch_bounds__(MI_THREADS, 1) mlp_infer_tc_kernel(int64_t n, const float* __restrict__ X,
                                                                     const __nv_bfloat16* __restrict__ pb,
                                                                     const float* __restrict__ pf,
                                                                     float* __restrict__ Y, int* err) {
    extern __shared__ __align__(1024) uint8_t mi_smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_slot;
    mlp_tc_stage(mi_smem, pb, pf);
    MlpTc c;
    mlp_tc_begin(c, mi_smem, &bar, &tmem_slot);
    const int64_t tiles = (n + MI_ROWS - 1) / MI_ROWS;
    for (int64_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const int64_t r = t * MI_ROWS + threadIdx.x;
        float x[MLP_IN], y[MLP_OUT];
#pragma unroll
        for (int i = 0; i < MLP_IN; ++i) x[i] = r < n ? X[r * MLP_IN + i] : 0.f;
        if (!mlp_tc_tile(c, x, y, err)) break;
        if (r < n)
#pragma unroll
            for (int i = 0; i < MLP_OUT; ++i) Y[r * MLP_OUT + i] = y[i];
    }
    mlp_tc_end(c);
}

// ------------------------------------------- surrogate remainder block Q
// Q[m, n] = sum over node pairs f_m(q) F(q, r) f_n(r), F the projected
// remainder field with the four surfaces predicted by the MLP.  Persistent
// CTAs walk the (row tile, column tile) pairs of the fill's basis tiling;
// per tile pair the node pairs go through the tensor-core MLP 128 at a time,
// and each thread adds its pair's field, weighted by the basis values at the
// two nodes, into a shared 16 x 16 tile of Q.
constexpr int SQ_MAX_NQ = 8;
constexpr int SQ_MAX_NODES = MW_MAX_TILE_SEG * SQ_MAX_NQ;  // 192

struct SqArgs {
    mw_segments seg;
    mw_basis basis;
    const __nv_bfloat16* pb;
    const float* pf;
    float fe2, fe3, fe4;      // per-structure features (|eps|, arg eps, f)
    double inv_lambda;        // 1 / wavelength
    double vscale;            // SCALE (omega mu) / (omega0 mu0)
    double tiny;              // rho below which the azimuth degenerates
    double gz, k;
    int nq;
    double tq[SQ_MAX_NQ], wq[SQ_MAX_NQ];
    double* Z;
    int64_t ldz;
    float* Z32;
    int64_t ldz32;
    int* err;
};

struct SqNode {
    double x, y, z;
    double f[3];  // basis values x Gauss weight at this node, per wing slot
    int m[3];     // local basis index of each slot (-1: none)
};

template <int D>
__device__ void sq_stage_nodes(const SqArgs& A, int tile, int ns, SqNode* nodes, double* tang) {
    constexpr int NM = D + 1;
    const int nq = A.nq;
    const int SMAX = A.basis.max_tile_seg, TB = A.basis.max_tile_basis;
    const int nb = A.basis.tile_nb[tile], fb = A.basis.tile_first[tile];
    for (int q = threadIdx.x; q < ns * nq; q += blockDim.x) {
        const int li = q / nq, iq = q - li * nq;
        const int s = A.basis.tile_seg[(size_t)tile * SMAX + li];
        const double* l = A.seg.seg_l + 3 * s;
        const double* r = A.seg.seg_r + 3 * s;
        const double dx = r[0] - l[0], dy = r[1] - l[1], dz = r[2] - l[2];
        const double L = sqrt(dx * dx + dy * dy + dz * dz);
        const double t = A.tq[iq];
        SqNode nd;
        nd.x = l[0] + t * dx;
        nd.y = l[1] + t * dy;
        nd.z = l[2] + t * dz;
        double wpow[NM];
        double wp = L * A.wq[iq];
        const double u = L * t;
        for (int p = 0; p < NM; ++p) {
            wpow[p] = wp;
            wp *= u;
        }
        int slot = 0;
        for (int i = 0; i < 3; ++i) {
            nd.m[i] = -1;
            nd.f[i] = 0.0;
        }
        for (int mi = 0; mi < nb && slot < 3; ++mi)
            for (int a = 0; a < NM; ++a)
                if (A.basis.loc[(size_t)(fb + mi) * NM + a] == li && slot < 3) {
                    const double* C = A.basis.polys + ((size_t)(fb + mi) * NM + a) * NM;
                    double v = 0.0;
                    for (int p = 0; p < NM; ++p) v += C[p] * wpow[p];
                    nd.m[slot] = mi;
                    nd.f[slot] = v;
                    ++slot;
                }
        nodes[q] = nd;
    }
    for (int i = threadIdx.x; i < ns; i += blockDim.x) {
        const int s = A.basis.tile_seg[(size_t)tile * SMAX + i];
        for (int c = 0; c < 3; ++c) tang[3 * i + c] = A.seg.tangent[3 * s + c];
    }
    (void)TB;
}

template <int D>
__global__ void __launch_bounds__(MI_THREADS, 1) somm_q_mlp_kernel(SqArgs A) {
    extern __shared__ __align__(1024) uint8_t sq_smem[];
    __shared__ __align__(8) uint64_t bar;
    __shared__ uint32_t tmem_slot;
    SqNode* nodes_r = reinterpret_cast<SqNode*>(sq_smem + MI_SMEM);
    SqNode* nodes_c = nodes_r + SQ_MAX_NODES;
    double* tang_r = reinterpret_cast<double*>(nodes_c + SQ_MAX_NODES);
    double* tang_c = tang_r + 3 * MW_MAX_TILE_SEG;
    double* Qs = tang_c + 3 * MW_MAX_TILE_SEG;  // MW_MAX_TILE_BASIS^2 complex
    mlp_tc_stage(sq_smem, A.pb, A.pf);
    MlpTc c;
    mlp_tc_begin(c, sq_smem, &bar, &tmem_slot);
    const int nt = A.basis.n_tile;
    const int TB = A.basis.max_tile_basis;
    const int nq = A.nq;
    bool alive = true;
    for (int64_t tp = blockIdx.x; tp < (int64_t)nt * nt && alive; tp += gridDim.x) {
        const int tr = (int)(tp / nt), tc = (int)(tp - (int64_t)tr * nt);
        const int ns_r = A.basis.tile_ns[tr], ns_c = A.basis.tile_ns[tc];
        __syncthreads();  // previous tile's readers are done with the staging
        sq_stage_nodes<D>(A, tr, ns_r, nodes_r, tang_r);
        sq_stage_nodes<D>(A, tc, ns_c, nodes_c, tang_c);
        for (int i = threadIdx.x; i < TB * TB * 2; i += blockDim.x) Qs[i] = 0.0;
        __syncthreads();
        const int nr = ns_r * nq, ncn = ns_c * nq;
        const int npair = nr * ncn;
        for (int p0 = 0; p0 < npair; p0 += MI_ROWS) {
            const int p = p0 + threadIdx.x;
            const bool valid = p < npair;
            const int ir = valid ? p / ncn : 0, ic = valid ? p - ir * ncn : 0;
            const SqNode& o = nodes_r[ir];
            const SqNode& sn = nodes_c[ic];
            const PairGeom g = pair_geom(A.gz, o.x, o.y, o.z, sn.x, sn.y, sn.z);
            float x[MLP_IN], y[MLP_OUT];
            const double r1w = fmin(g.r1 * A.inv_lambda, 4.0);
            x[0] = (float)(2.0 * sqrt(r1w / 4.0) - 1.0);
            x[1] = (float)(4.0 * g.theta / kPi - 1.0);
            x[2] = A.fe2;
            x[3] = A.fe3;
            x[4] = A.fe4;
            if (!mlp_tc_tile(c, x, y, A.err)) {
                alive = false;
                break;
            }
            if (valid) {
                cd surf[4];
#pragma unroll
                for (int s = 0; s < 4; ++s) surf[s] = cd{(double)y[2 * s], (double)y[2 * s + 1]};
                const int li = ir / nq, lj = ic / nq;
                const double* to = tang_r + 3 * li;
                const double* tsv = tang_c + 3 * lj;
                const SrcTangent ts = split_tangent(tsv[0], tsv[1], tsv[2]);
                const cd F = project_surfaces(g, surf, A.k, A.vscale, A.tiny, to[0], to[1], to[2], ts);
#pragma unroll
                for (int a = 0; a < 3; ++a) {
                    const int mi = o.m[a];
                    if (mi < 0) continue;
#pragma unroll
                    for (int b = 0; b < 3; ++b) {
                        const int ni = sn.m[b];
                        if (ni < 0) continue;
                        const double w = o.f[a] * sn.f[b];
                        atomicAdd(&Qs[2 * (mi * TB + ni)], w * F.re);
                        atomicAdd(&Qs[2 * (mi * TB + ni) + 1], w * F.im);
                    }
                }
            }
        }
        __syncthreads();
        const int nb_r = A.basis.tile_nb[tr], nb_c = A.basis.tile_nb[tc];
        const int fb_r = A.basis.tile_first[tr], fb_c = A.basis.tile_first[tc];
        for (int q = threadIdx.x; q < nb_r * nb_c; q += blockDim.x) {
            const int mi = q % nb_r, ni = q / nb_r;
            const int64_t m = fb_r + mi, n = fb_c + ni;
            double* zp = A.Z + 2 * (m + n * A.ldz);
            const double zr = zp[0] - Qs[2 * (mi * TB + ni)], zi = zp[1] - Qs[2 * (mi * TB + ni) + 1];
            zp[0] = zr;
            zp[1] = zi;
            if (A.Z32) {
                float* z32 = A.Z32 + 2 * (m + n * A.ldz32);
                z32[0] = (float)zr;
                z32[1] = (float)zi;
            }
        }
    }
    mlp_tc_end(c);
}

constexpr size_t SQ_SMEM = MI_SMEM + 2 * SQ_MAX_NODES * sizeof(SqNode) + 6 * MW_MAX_TILE_SEG * sizeof(double) +
                           2 * MW_MAX_TILE_BASIS * MW_MAX_TILE_BASIS * sizeof(double);

}  // namespace mw

using namespace mw;

extern "C" int32_t mw_mlp_param_count(void) { return MLP_PARAMS; }

extern "C" size_t mw_mlp_train_workspace_size(int32_t batch) { return train_ws_floats(batch) * sizeof(float); }

extern "C" mw_status mw_mlp_to_bf16(const float* params, void* params_bf16, void* stream) {
    MW_REQUIRE(params && params_bf16, "NULL argument");
    cudaStream_t st = as_stream(stream);
    to_bf16_kernel<<<64, 256, 0, st>>>(MLP_PARAMS, params, reinterpret_cast<__nv_bfloat16*>(params_bf16));
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

extern "C" mw_status mw_mlp_forward(int32_t n, const float* X, const void* params_bf16, const float* params,
                                    float* Y, void* workspace, size_t workspace_bytes, void* stream) {
    MW_REQUIRE(n >= 1 && X && params_bf16 && params && Y && workspace, "bad arguments");
    MW_REQUIRE(workspace_bytes >= train_ws_floats(n) * sizeof(float), "workspace too small");
    cudaStream_t st = as_stream(stream);
    TrainWs t = train_ws(workspace, n);
    forward_train(X, n, reinterpret_cast<const __nv_bfloat16*>(params_bf16), params, t, st);
    MW_CHECK_CUDA(cudaMemcpyAsync(Y, t.out, sizeof(float) * n * MLP_OUT, cudaMemcpyDeviceToDevice, st));
    MW_CHECK_CUDA(cudaGetLastError());
    return MW_OK;
}

extern "C" mw_status mw_mlp_grad(int32_t n, const float* X, const float* T, const void* params_bf16,
                                 const float* params, float* grad, float* loss, void* workspace,
                                 size_t workspace_bytes, void* stream) {
    MW_REQUIRE(n >= 1 && X && T && params_bf16 && params && grad && loss && workspace, "bad arguments");
    MW_REQUIRE(workspace_bytes >= train_ws_floats(n) * sizeof(float), "workspace too small");
    cudaStream_t st = as_stream(stream);
    TrainWs t = train_ws(workspace, n);
    const __nv_bfloat16* pb = reinterpret_cast<const __nv_bfloat16*>(params_bf16);
    forward_train(X, n, pb, params, t, st);
    MW_CHECK_CUDA(cudaMemsetAsync(loss, 0, sizeof(float), st));
    const int64_t no = (int64_t)n * MLP_OUT;
    mse_kernel<<<(unsigned)((no + 255) / 256 < 1024 ? (no + 255) / 256 : 1024), 256, 0, st>>>(
        t.out, T, t.dout, no, 1.0f / (float)no, loss);
    count_launch();
    backward_train(X, n, pb, t, st);
    MW_CHECK_CUDA(cudaMemcpyAsync(grad, t.grad, sizeof(float) * MLP_PARAMS, cudaMemcpyDeviceToDevice, st));
    MW_CHECK_CUDA(cudaGetLastError());
    return MW_OK;
}

extern "C" mw_status mw_mlp_train_step(int32_t n, const float* X, const float* T, const int64_t* rows,
                                       float* params, void* params_bf16, float* adam_m, float* adam_v, int32_t step,
                                       float lr, float beta1, float beta2, float eps, float* loss, void* workspace,
                                       size_t workspace_bytes, void* stream) {
    MW_REQUIRE(n >= 1 && X && T && params && params_bf16 && adam_m && adam_v && loss && workspace, "bad arguments");
    MW_REQUIRE(step >= 1, "Adam step counts from 1");
    MW_REQUIRE(workspace_bytes >= train_ws_floats(n) * sizeof(float), "workspace too small");
    cudaStream_t st = as_stream(stream);
    TrainWs t = train_ws(workspace, n);
    if (rows) {
        // the batch is rows[0..n) of the full training set
        gather_rows_kernel<<<256, 256, 0, st>>>(n, MLP_IN, X, rows, t.xg);
        gather_rows_kernel<<<256, 256, 0, st>>>(n, MLP_OUT, T, rows, t.tg);
        count_launch(2);
        X = t.xg;
        T = t.tg;
    }
    __nv_bfloat16* pb = reinterpret_cast<__nv_bfloat16*>(params_bf16);
    forward_train(X, n, pb, params, t, st);
    const int64_t no = (int64_t)n * MLP_OUT;
    mse_kernel<<<(unsigned)((no + 255) / 256 < 1024 ? (no + 255) / 256 : 1024), 256, 0, st>>>(
        t.out, T, t.dout, no, 1.0f / (float)no, loss);
    count_launch();
    backward_train(X, n, pb, t, st);
    const float c1 = 1.f / (1.f - powf(beta1, (float)step)), c2 = 1.f / (1.f - powf(beta2, (float)step));
    adam_kernel<<<64, 256, 0, st>>>(MLP_PARAMS, params, pb, t.grad, adam_m, adam_v, lr, beta1, beta2, eps, c1, c2);
    count_launch();
    MW_CHECK_CUDA(cudaGetLastError());
    return MW_OK;
}

extern "C" mw_status mw_mlp_infer(int64_t n, const float* X, const void* params_bf16, const float* params, float* Y,
                                  int32_t* err, void* stream) {
    MW_REQUIRE(n >= 1 && X && params_bf16 && params && Y && err, "bad arguments");
    cudaStream_t st = as_stream(stream);
    static bool attr = false;
    if (!attr) {
        MW_CHECK_CUDA(cudaFuncSetAttribute(mlp_infer_tc_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, MI_SMEM));
        attr = true;
    }
    int dev = 0, sms = 148;
    MW_CHECK_CUDA(cudaGetDevice(&dev));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t tiles = (n + MI_ROWS - 1) / MI_ROWS;
    const int grid = (int)(tiles < sms ? tiles : sms);
    mlp_infer_tc_kernel<<<grid, MI_THREADS, MI_SMEM, st>>>(n, X, reinterpret_cast<const __nv_bfloat16*>(params_bf16),
                                                           params, Y, err);
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

extern "C" mw_status mw_somm_remainder_q_mlp(const mw_segments* seg, const mw_basis* basis, const void* params_bf16,
                                             const float* params, const float* struct_features,
                                             double wavelength, double value_scale, int32_t n_qp, double ground_z,
                                             double k, double* Z, int64_t ldz, float* Z32, int64_t ldz32,
                                             int32_t* err, void* stream) {
    MW_REQUIRE(seg && basis && params_bf16 && params && struct_features && Z && err, "NULL argument");
    MW_REQUIRE(basis->degree == 1 || basis->degree == 2, "degree must be 1 or 2");
    MW_REQUIRE(n_qp >= 1 && n_qp <= SQ_MAX_NQ, "n_qp_sommerfeld must be in [1, %d]", SQ_MAX_NQ);
    MW_REQUIRE(basis->max_tile_seg >= 1 && basis->max_tile_seg <= MW_MAX_TILE_SEG &&
                   basis->max_tile_basis >= 1 && basis->max_tile_basis <= MW_MAX_TILE_BASIS && basis->n_tile >= 1,
               "bad basis tiling");
    MW_REQUIRE(wavelength > 0.0, "wavelength must be positive");
    cudaStream_t st = as_stream(stream);
    SqArgs A{};
    A.seg = *seg;
    A.basis = *basis;
    A.pb = reinterpret_cast<const __nv_bfloat16*>(params_bf16);
    A.pf = params;
    A.fe2 = struct_features[0];
    A.fe3 = struct_features[1];
    A.fe4 = struct_features[2];
    A.inv_lambda = 1.0 / wavelength;
    A.vscale = value_scale;
    A.tiny = 1e-12 * 4.0 * wavelength;  // the grid path's 1e-12 r1_max at a 4-wavelength grid
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
    A.err = err;
    int dev = 0, sms = 148;
    MW_CHECK_CUDA(cudaGetDevice(&dev));
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int64_t pairs = (int64_t)basis->n_tile * basis->n_tile;
    const int grid = (int)(pairs < sms ? pairs : sms);
    ProfileScope ps(PC_SOMM_Q, st);
    if (basis->degree == 1) {
        MW_CHECK_CUDA(cudaFuncSetAttribute(somm_q_mlp_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)SQ_SMEM));
        somm_q_mlp_kernel<1><<<grid, MI_THREADS, SQ_SMEM, st>>>(A);
    } else {
        MW_CHECK_CUDA(cudaFuncSetAttribute(somm_q_mlp_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)SQ_SMEM));
        somm_q_mlp_kernel<2><<<grid, MI_THREADS, SQ_SMEM, st>>>(A);
    }
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}
