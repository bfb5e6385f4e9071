// mw_fill_z_noalloc: the impedance fill for callers that cannot allocate
// device memory.
//
// mw_fill_z needs a scratch buffer between its two stages -- the same-edge
// Toeplitz table that mw_same_edge_table writes and the fill kernel reads --
// and expects the caller to have allocated it.  Some hosts of this library
// cannot do that: a plugin whose host process owns every device allocation
// through its own pool and hands the plugin only the input and output
// buffers, or a foreign-language binding that has no way to reach
// cudaMalloc.  For them this file keeps the table in a fixed-size array of
// device memory that exists from the moment the library is loaded, so the
// call itself allocates nothing.
//
// Limits and sharing rules:
//   * capacity: kNoallocTableDoubles doubles (4.5 MiB), i.e. 32768 table
//     rows at degree 2 (73728 at degree 1); the number of rows a structure
//     needs is the sum over its straight edges of 2*n_segments - 1, and a
//     larger structure is rejected with MW_ERR_WORKSPACE;
//   * every GPU that loads the library holds this array until the process
//     exits;
//   * all calls share the one array: two calls whose work overlaps on the
//     GPU (different streams, or different host threads on one device) race
//     on it, so serialise them;
//   * every call resolves the array's device address on the current device
//     (cudaGetSymbolAddress) unless the stream is being captured, when the
//     address remembered from the last uncaptured call on that device is
//     used; make one call on each device before any stream capture.  A
//     cudaDeviceReset, or a context other than the device's primary one,
//     gets a fresh address on the next uncaptured call;
//   * nothing needs to start at zero: every call overwrites the rows it
//     reads.
#include <mutex>

#include "common.cuh"

namespace {

constexpr size_t kNoallocTableDoubles = size_t(32768) * 9 * 2;

__device__ __align__(256) double g_noalloc_table[kNoallocTableDoubles];

constexpr int kMaxDevices = 64;
std::mutex g_noalloc_mu;
double* g_noalloc_ptr[kMaxDevices] = {};

// Device address of the array on the current device.  Host code cannot use
// the symbol's name as a device pointer, so the runtime is asked for it on
// every call (cheap) -- a cached address could outlive its context after a
// device reset.  While `stream` is capturing, the runtime may not be queried
// in ways that break the capture, so the address remembered from the last
// uncaptured call on this device is used.
mw_status noalloc_table_ptr(void* stream, double** out) {
    int dev = 0;
    MW_CHECK_CUDA(cudaGetDevice(&dev));
    MW_REQUIRE(dev >= 0 && dev < kMaxDevices, "device ordinal %d out of range", dev);
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    MW_CHECK_CUDA(cudaStreamIsCapturing(static_cast<cudaStream_t>(stream), &cap));
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    if (cap == cudaStreamCaptureStatusNone) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_table);
        if (e != cudaSuccess) return mw::cuda_status(e, "cudaGetSymbolAddress(g_noalloc_table)");
        g_noalloc_ptr[dev] = static_cast<double*>(p);
    }
    MW_REQUIRE(g_noalloc_ptr[dev] != nullptr,
               "mw_fill_z_noalloc: the first call on device %d was made during stream capture; make one call "
               "before capturing", dev);
    *out = g_noalloc_ptr[dev];
    return MW_OK;
}

}  // namespace

extern "C" size_t mw_fill_z_noalloc_capacity(int32_t degree) {
    if (degree != 1 && degree != 2) return 0;
    size_t per_row = (size_t)(degree + 1) * (degree + 1) * 2;
    return kNoallocTableDoubles / per_row;
}

extern "C" mw_status mw_fill_z_noalloc(const mw_segments* seg, const mw_basis* basis, const mw_edges* edges,
                                       const mw_freq* freq, int32_t n_qp, int32_t extended_kernel, double* Z,
                                       int64_t ldz, void* stream) {
    MW_REQUIRE(seg && basis && edges && freq && Z, "NULL argument");
    MW_REQUIRE(basis->degree == 1 || basis->degree == 2, "degree must be 1 or 2 (got %d)", basis->degree);
    size_t cap = mw_fill_z_noalloc_capacity(basis->degree);
    if (edges->table_rows < 0 || (size_t)edges->table_rows > cap) {
        mw::set_error("same-edge table needs %lld rows but the built-in scratch holds %zu at degree %d "
                      "(sum over edges of 2*n-1); use mw_same_edge_table + mw_fill_z with a caller buffer",
                      (long long)edges->table_rows, cap, basis->degree);
        return MW_ERR_WORKSPACE;
    }
    double* table = nullptr;
    mw_status s = noalloc_table_ptr(stream, &table);
    if (s != MW_OK) return s;
    s = mw_same_edge_table(edges, basis->degree, n_qp, extended_kernel, freq->k, table, stream);
    if (s != MW_OK) return s;
    return mw_fill_z(seg, basis, table, edges, freq, n_qp, Z, ldz, nullptr, 0, stream);
}
