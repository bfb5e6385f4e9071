// mw_selftest_wait_timeout: makes one of the library's bounded device waits
// run out on purpose, with a short spin limit, so that a test can check
// that the wait ends, records MW_ERR_TIMEOUT and leaves the context usable.
// The waits are the production helpers themselves (waits.cuh, tc_common.cuh);
// only the limit is shortened and the awaited event never comes:
//   which = 0: the grid barrier of the complex128 LU panel, two CTAs waiting
//              for three arrivals;
//   which = 1: the mbarrier wait of the tensor-core kernels, one thread
//              waiting on a barrier that nobody arrives at.
#include "common.cuh"
#include "tc_common.cuh"
#include "waits.cuh"

namespace mw {
namespace {

__global__ void grid_wait_selftest_kernel(PanelWs* ws, long long limit) {
    // gridDim.x CTAs can never make gridDim.x + 1 arrivals
    grid_sync_bounded(ws, gridDim.x + 1u, limit);
}

__global__ void mbar_wait_selftest_kernel(int* err, long long limit) {
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) mbar_wait(&bar, 0, err, limit);
    __syncthreads();
}

}  // namespace
}  // namespace mw

extern "C" mw_status mw_selftest_wait_timeout(int32_t which, int64_t spin_limit, void* workspace, void* stream) {
    using namespace mw;
    MW_REQUIRE(which == 0 || which == 1, "which must be 0 (grid barrier) or 1 (mbarrier), got %d", which);
    MW_REQUIRE(spin_limit >= 256 && spin_limit <= (int64_t(1) << 24),
               "spin_limit must lie in [256, 2^24] (got %lld)", (long long)spin_limit);
    MW_REQUIRE(workspace != nullptr, "NULL workspace");
    cudaStream_t st = as_stream(stream);
    PanelWs* ws = static_cast<PanelWs*>(workspace);
    MW_CHECK_CUDA(cudaMemsetAsync(ws, 0, sizeof(PanelWs), st));
    if (which == 0)
        grid_wait_selftest_kernel<<<2, 32, 0, st>>>(ws, spin_limit);
    else
        mbar_wait_selftest_kernel<<<1, 32, 0, st>>>(&ws->err, spin_limit);
    count_launch();
    MW_CHECK_CUDA(cudaGetLastError());
    int err = 0;
    MW_CHECK_CUDA(cudaMemcpyAsync(&err, &ws->err, sizeof(int), cudaMemcpyDeviceToHost, st));
    MW_CHECK_CUDA(cudaStreamSynchronize(st));
    if (err != 0) {
        set_error("bounded %s wait gave up after %lld polls (self-test)", which == 0 ? "grid barrier" : "mbarrier",
                  (long long)spin_limit);
        return err;
    }
    return MW_OK;
}
