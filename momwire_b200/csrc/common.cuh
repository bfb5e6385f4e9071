// Shared device/host helpers for the momwire_b200 kernels (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/momwire_b200.h"

namespace mw {

// ---------------------------------------------------------------- complex
struct cd {
    double re, im;
};
struct cf {
    float re, im;
};

__host__ __device__ __forceinline__ cd cmk(double r, double i) { return cd{r, i}; }
__host__ __device__ __forceinline__ cd operator+(cd a, cd b) { return cd{a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ cd operator-(cd a, cd b) { return cd{a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ cd operator*(cd a, cd b) {
    return cd{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__host__ __device__ __forceinline__ cd operator*(double s, cd a) { return cd{s * a.re, s * a.im}; }
__host__ __device__ __forceinline__ cd cdiv(cd a, cd b) {
    // Smith's algorithm: avoids overflow/underflow of |b|^2.
    if (fabs(b.re) >= fabs(b.im)) {
        double r = b.im / b.re, den = b.re + b.im * r;
        return cd{(a.re + a.im * r) / den, (a.im - a.re * r) / den};
    } else {
        double r = b.re / b.im, den = b.re * r + b.im;
        return cd{(a.re * r + a.im) / den, (a.im * r - a.re) / den};
    }
}
__host__ __device__ __forceinline__ cf operator+(cf a, cf b) { return cf{a.re + b.re, a.im + b.im}; }
__host__ __device__ __forceinline__ cf operator-(cf a, cf b) { return cf{a.re - b.re, a.im - b.im}; }
__host__ __device__ __forceinline__ cf operator*(cf a, cf b) {
    return cf{a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
}
__host__ __device__ __forceinline__ cf cdiv(cf a, cf b) {
    if (fabsf(b.re) >= fabsf(b.im)) {
        float r = b.im / b.re, den = b.re + b.im * r;
        return cf{(a.re + a.im * r) / den, (a.im - a.re * r) / den};
    } else {
        float r = b.re / b.im, den = b.re * r + b.im;
        return cf{(a.re * r + a.im) / den, (a.im * r - a.re) / den};
    }
}
__host__ __device__ __forceinline__ double cabs1(cd z) { return fabs(z.re) + fabs(z.im); }
__host__ __device__ __forceinline__ double cabs1(cf z) { return (double)fabsf(z.re) + (double)fabsf(z.im); }
template <class T> __host__ __device__ __forceinline__ T cone();
template <> __host__ __device__ __forceinline__ cd cone<cd>() { return cd{1.0, 0.0}; }
template <> __host__ __device__ __forceinline__ cf cone<cf>() { return cf{1.0f, 0.0f}; }

// Principal square root (branch cut on the negative real axis; Im >= 0
// except that -0 imaginary input maps to the lower half, like numpy).
__host__ __device__ __forceinline__ cd csqrt_p(cd z) {
    double x = z.re, y = z.im;
    if (x == 0.0 && y == 0.0) return cd{0.0, y};
    double r = hypot(x, y);
    if (x >= 0.0) {
        double t = sqrt(0.5 * (r + x));
        return cd{t, y / (2.0 * t)};
    } else {
        double t = sqrt(0.5 * (r - x));
        return cd{fabs(y) / (2.0 * t), copysign(t, y)};
    }
}

constexpr double kPi = 3.14159265358979323846;
constexpr double kInv4Pi = 0.079577471545947667884;  // 1/(4 pi)

// ------------------------------------------------------------ error state
void set_error(const char* fmt, ...);
mw_status cuda_status(cudaError_t e, const char* what);

#define MW_CHECK_CUDA(call)                                           \
    do {                                                              \
        cudaError_t _e = (call);                                      \
        if (_e != cudaSuccess) return ::mw::cuda_status(_e, #call);   \
    } while (0)

#define MW_REQUIRE(cond, ...)                                         \
    do {                                                              \
        if (!(cond)) {                                                \
            ::mw::set_error(__VA_ARGS__);                             \
            return MW_ERR_INVALID;                                    \
        }                                                             \
    } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// Host-side count of kernels this library has launched (mw_launch_count).
void count_launch(int64_t n = 1);

// Optional per-kernel-class timing (mw_profile_*): while enabled, a scope
// records a CUDA event pair around the launches it encloses on `stream` and
// carries the launch's algorithmic flop and byte counts.
enum ProfileClass {
    PC_TABLE = 0,
    PC_FILL = 1,
    PC_FILL_IMAGE = 2,
    PC_PANEL = 3,
    PC_LASWP = 4,
    PC_TRSM = 5,
    PC_ZGEMM = 6,
    PC_CGEMM_TC = 7,
    PC_REFINE = 8,
    PC_MISC = 9,
    PC_SOMM_GRID = 10,
    PC_SOMM_Q = 11,
    PC_FACTOR = 12,  // whole factorisations (wall, enclosing the classes above)
    PC_SOLVE = 13,   // whole triangular solves with many right-hand sides (wall)
    PC_L21 = 14,     // static-pivot panels: the rows below the diagonal block
    PC_COUNT = 15
};

struct ProfileScope {
    ProfileScope(int cls, cudaStream_t st, double flops = 0.0, double bytes = 0.0);
    ~ProfileScope();
    int cls_;
    cudaStream_t st_;
    double flops_, bytes_;
    void* rec_;
};

// Gauss-Legendre nodes/weights on [0,1] for n <= 32, computed on the host
// by Newton iteration on P_n (cached).  Returns pointers to host arrays.
void gauss_legendre01(int n, const double** t, const double** w);

}  // namespace mw
