// Bounded device-wide waits shared by the factorisation kernels and the
// wait self-test (sm_100a).  Every wait gives up after a spin limit, records
// MW_ERR_TIMEOUT in a device error word and returns false, so a kernel that
// waits for a peer that never arrives ends instead of hanging the GPU.
#pragma once

#include "common.cuh"

namespace mw {

// Spins of the grid barrier's arrival poll before it gives up.
constexpr long long kGridSpinLimit = 1ll << 26;

struct PanelWs {
    unsigned int counter;    // grid barrier arrivals
    int err;                 // device status (MW_ERR_TIMEOUT)
    unsigned int lmax_bits;  // static-pivot panels: largest |L21| (float bits; +inf when singular)
    int spare;
};

__device__ __forceinline__ unsigned int ld_acquire(const unsigned int* p) {
    unsigned int v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Bounded grid barrier: every CTA adds one arrival and waits until
// `target` arrivals are counted.  Returns false (for every thread of the
// CTA) when the wait gave up -- after `spin_limit` polls, recording
// MW_ERR_TIMEOUT -- or when another CTA already had.
static __device__ __noinline__ bool grid_sync_bounded(PanelWs* ws, unsigned int target,
                                                      long long spin_limit = kGridSpinLimit) {
    __shared__ int s_ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        // the release add publishes every write the CTA made before the
        // __syncthreads above (cumulativity); the acquire loads order the
        // reads that follow the barrier
        asm volatile("red.release.gpu.global.add.u32 [%0], 1;" ::"l"(&ws->counter) : "memory");
        int ok = 1;
        long long spins = 0;
        while (ld_acquire(&ws->counter) < target) {
            if ((++spins & 255) == 0) {
                if (*(volatile int*)&ws->err) { ok = 0; break; }
                if (spins > spin_limit) {
                    atomicExch(&ws->err, MW_ERR_TIMEOUT);
                    ok = 0;
                    break;
                }
            }
        }
        s_ok = ok;
    }
    __syncthreads();
    return s_ok != 0;
}

}  // namespace mw
