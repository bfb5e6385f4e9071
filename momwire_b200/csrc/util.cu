// Small device utilities of the solve pipeline (sm_100a).
#include "common.cuh"

namespace mw {

// out[rows[q] + cols[q] * ld] += vals[q] (complex128); duplicates add up.
__global__ void scatter_add_c128_kernel(int64_t nnz, const int64_t* __restrict__ rows,
                                        const int64_t* __restrict__ cols, const double2* __restrict__ vals,
                                        double* __restrict__ out, int64_t ld) {
    for (int64_t q = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; q < nnz; q += (int64_t)gridDim.x * blockDim.x) {
        const int64_t o = 2 * (rows[q] + cols[q] * ld);
        atomicAdd(out + o, vals[q].x);
        atomicAdd(out + o + 1, vals[q].y);
    }
}

}  // namespace mw

using namespace mw;

extern "C" mw_status mw_scatter_c128(int64_t ld, int64_t ncols, int64_t nnz, const int64_t* rows,
                                     const int64_t* cols, const double* vals, double* out, void* stream) {
    MW_REQUIRE(ld >= 0 && ncols >= 0 && nnz >= 0, "sizes must be >= 0");
    MW_REQUIRE(out != nullptr || ld * ncols == 0, "NULL output");
    cudaStream_t st = as_stream(stream);
    if (ld * ncols > 0) MW_CHECK_CUDA(cudaMemsetAsync(out, 0, sizeof(double) * 2 * ld * ncols, st));
    if (nnz == 0) return MW_OK;
    MW_REQUIRE(rows && cols && vals, "NULL entries");
    const int64_t blocks = (nnz + 255) / 256;
    scatter_add_c128_kernel<<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0, st>>>(
        nnz, rows, cols, reinterpret_cast<const double2*>(vals), out, ld);
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}
