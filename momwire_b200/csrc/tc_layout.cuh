// Packed operand layout of the tensor-core complex update (cgemm_tc.cu),
// shared with the kernels that write operands in it directly.
//
// The complex update C -= A B runs as the real GEMM
//     C_real (2m x n) -= Ahat (2m x 2k) * Breal (2k x n)
// with Ahat holding each complex a as [[re, -im], [im, re]] and Breal the
// re / im of B interleaved down each column.  Every fp32 operand is split
// x = hi + lo (hi = tf32(x)) into two planes.  A plane is stored as the
// shared-memory image of K-major, no-swizzle UMMA tiles:
//   Ahat: [m block of TC_M real rows][K stage of TC_KS][16-byte chunk][row][4]
//   Breal^T: [n block of TC_N columns][K stage][16-byte chunk][column][4]
// so one stage of one block is a contiguous bulk copy.
#pragma once

#include <cstdint>

namespace mw {

#ifndef MW_TC_KS
#define MW_TC_KS 16
#endif
constexpr int TC_M = 128;                     // real rows per tile
constexpr int TC_N = 256;                     // columns per tile
constexpr int TC_KS = MW_TC_KS;               // real K per stage (a multiple of 8)
constexpr int TC_CHUNKS = TC_KS / 4;          // 16-byte K chunks per stage
constexpr int TC_A_BYTES = TC_M * TC_KS * 4;  // per plane and stage
constexpr int TC_B_BYTES = TC_N * TC_KS * 4;

// K stages of a complex inner dimension k (real K = 2k).
__host__ __device__ __forceinline__ int tc_n_ks(int64_t k) { return (int)((2 * k + TC_KS - 1) / TC_KS); }

__device__ __forceinline__ float tf32_hi(float x) {
    uint32_t r;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(r) : "f"(x));
    return __uint_as_float(r);
}

__device__ __forceinline__ void tc_split_store(float* hi, float* lo, int64_t q, float4 v) {
    float4 h, l;
    h.x = tf32_hi(v.x); l.x = v.x - h.x;
    h.y = tf32_hi(v.y); l.y = v.y - h.y;
    h.z = tf32_hi(v.z); l.z = v.z - h.z;
    h.w = tf32_hi(v.w); l.w = v.w - h.w;
    reinterpret_cast<float4*>(hi)[q] = h;
    reinterpret_cast<float4*>(lo)[q] = l;
}

// Ahat elements (rho, kap4 .. kap4 + 3), kap4 a multiple of 4, as hi / lo.
__device__ __forceinline__ void tc_store_a4(float* hi, float* lo, int n_ks, int64_t rho, int64_t kap4, float4 v) {
    const int64_t q = (((rho / TC_M) * n_ks + kap4 / TC_KS) * TC_CHUNKS + (kap4 % TC_KS) / 4) * TC_M + rho % TC_M;
    tc_split_store(hi, lo, q, v);
}

// Breal^T elements (column j, kap4 .. kap4 + 3) as hi / lo.
__device__ __forceinline__ void tc_store_b4(float* hi, float* lo, int n_ks, int64_t j, int64_t kap4, float4 v) {
    const int64_t q = (((j / TC_N) * n_ks + kap4 / TC_KS) * TC_CHUNKS + (kap4 % TC_KS) / 4) * TC_N + j % TC_N;
    tc_split_store(hi, lo, q, v);
}

// The four planes of a packed update (each a device pointer to floats).
struct TcPlanes {
    float* a_hi;
    float* a_lo;
    float* b_hi;
    float* b_lo;
};

}  // namespace mw
