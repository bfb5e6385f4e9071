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

// Z[b][rows[q] + cols[q] * ldz] += zw[b][wire[q]] * vals[q] for unique
// (row, col) entries (no two threads touch one element), and the complex64
// mirror, when given, takes the rounded new value.  Entries outside the
// n x n matrix or naming a wire outside [0, n_wires) are skipped and counted.
__global__ void add_loading_kernel(int64_t n, int batch, int64_t nnz, const int64_t* __restrict__ rows,
                                   const int64_t* __restrict__ cols, const double* __restrict__ vals,
                                   const int32_t* __restrict__ wire, const double2* __restrict__ zw, int n_wires,
                                   double2* __restrict__ Z, int64_t ldz, int64_t sz, float2* __restrict__ Z32,
                                   int64_t ld32, int64_t s32, int32_t* __restrict__ bad) {
    const int64_t total = nnz * (int64_t)batch;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total;
         t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t b = t / nnz, q = t - b * nnz;
        const int64_t r = rows[q], c = cols[q];
        const int w = wire[q];
        if (r < 0 || r >= n || c < 0 || c >= n || w < 0 || w >= n_wires) {
            if (bad) atomicAdd(bad, 1);
            continue;
        }
        const double2 z = zw[b * n_wires + w];
        const double v = vals[q];
        double2* p = Z + b * sz + r + c * ldz;
        double2 cur = *p;
        cur.x += z.x * v;
        cur.y += z.y * v;
        *p = cur;
        if (Z32) Z32[b * s32 + r + c * ld32] = make_float2((float)cur.x, (float)cur.y);
    }
}

// Pad each of `count` matrices (column-major, order nb, the leading n x n
// block already filled) to [[Z, 0], [0, I]]: rows n..nb-1 of the first n
// columns and all of columns n..nb-1 are written, the diagonal with 1.
__global__ void pad_identity_kernel(int64_t n, int64_t nb, double2* __restrict__ Z, int64_t ldz, int64_t sz,
                                    float2* __restrict__ Z32, int64_t ld32, int64_t s32) {
    const int64_t col = blockIdx.x, b = blockIdx.y;
    const int64_t r0 = col < n ? n : 0;
    double2* z = Z + b * sz + col * ldz;
    float2* z32 = Z32 ? Z32 + b * s32 + col * ld32 : nullptr;
    for (int64_t r = r0 + threadIdx.x; r < nb; r += blockDim.x) {
        const double v = (r == col) ? 1.0 : 0.0;
        z[r] = make_double2(v, 0.0);
        if (z32) z32[r] = make_float2((float)v, 0.f);
    }
}

// Y (n_out x ncols, column-major) = S X for S sparse in CSR (n_out rows;
// row r's entries at [row_ptr[r], row_ptr[r+1]) in order: deterministic
// sums) and X dense column-major.  One thread per output, rows fastest.
__global__ void csr_mm_c128_kernel(int64_t n_out, int64_t ncols, const int64_t* __restrict__ row_ptr,
                                   const int64_t* __restrict__ col_idx, const double2* __restrict__ vals,
                                   const double2* __restrict__ X, int64_t ldx, double2* __restrict__ Y, int64_t ldy) {
    const int64_t total = n_out * ncols;
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int64_t j = t / n_out, r = t - j * n_out;
        const double2* x = X + j * ldx;
        double re = 0.0, im = 0.0;
        for (int64_t q = row_ptr[r]; q < row_ptr[r + 1]; ++q) {
            const double2 v = vals[q], a = x[col_idx[q]];
            re = fma(v.x, a.x, re);
            re = fma(-v.y, a.y, re);
            im = fma(v.x, a.y, im);
            im = fma(v.y, a.x, im);
        }
        Y[r + j * ldy] = make_double2(re, im);
    }
}

}  // namespace mw

using namespace mw;

extern "C" mw_status mw_csr_mm_c128(int64_t n_out, int64_t ncols, const int64_t* row_ptr, const int64_t* col_idx,
                                    const double* vals, const double* X, int64_t ldx, double* Y, int64_t ldy,
                                    void* stream) {
    MW_REQUIRE(n_out >= 0 && ncols >= 0, "sizes must be >= 0");
    MW_REQUIRE(ldy >= n_out, "ldy < n_out");
    if (n_out == 0 || ncols == 0) return MW_OK;
    MW_REQUIRE(row_ptr && Y && X, "NULL argument");
    cudaStream_t st = as_stream(stream);
    const int64_t total = n_out * ncols;
    const int64_t blocks = (total + 255) / 256;
    {
        ProfileScope ps(PC_ZGEMM, st);
        csr_mm_c128_kernel<<<(unsigned)(blocks < 8192 ? blocks : 8192), 256, 0, st>>>(
            n_out, ncols, row_ptr, col_idx, reinterpret_cast<const double2*>(vals), reinterpret_cast<const double2*>(X),
            ldx, reinterpret_cast<double2*>(Y), ldy);
    }
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

extern "C" mw_status mw_pad_identity(int64_t n, int64_t nb, int32_t count, double* Z, int64_t ldz, int64_t z_stride,
                                     float* Z32, int64_t ld32, int64_t z32_stride, void* stream) {
    MW_REQUIRE(n >= 0 && nb >= n && count >= 0 && count <= 65535, "bad sizes");
    MW_REQUIRE(ldz >= nb && (Z32 == nullptr || ld32 >= nb), "leading dimension smaller than nb");
    MW_REQUIRE(count <= 1 || (z_stride >= ldz * nb && (Z32 == nullptr || z32_stride >= ld32 * nb)),
               "batch stride smaller than one matrix");
    if (nb == n || count == 0) return MW_OK;
    MW_REQUIRE(Z != nullptr, "NULL Z");
    MW_REQUIRE(nb <= 0x7fffffff, "nb too large");
    cudaStream_t st = as_stream(stream);
    pad_identity_kernel<<<dim3((unsigned)nb, (unsigned)count), 128, 0, st>>>(
        n, nb, reinterpret_cast<double2*>(Z), ldz, z_stride, reinterpret_cast<float2*>(Z32), ld32, z32_stride);
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

extern "C" mw_status mw_add_loading(int64_t n, int32_t batch, int64_t nnz, const int64_t* rows, const int64_t* cols,
                                    const double* vals, const int32_t* wire, const double* zw, int32_t n_wires,
                                    double* Z, int64_t ldz, int64_t z_stride, float* Z32, int64_t ld32,
                                    int64_t z32_stride, int32_t* bad, void* stream) {
    MW_REQUIRE(n >= 0 && nnz >= 0 && batch >= 0 && n_wires >= 0, "sizes must be >= 0");
    MW_REQUIRE(ldz >= n && (Z32 == nullptr || ld32 >= n), "leading dimension smaller than n");
    MW_REQUIRE(batch <= 1 || (z_stride >= ldz * n && (Z32 == nullptr || z32_stride >= ld32 * n)),
               "batch stride smaller than one matrix");
    if (nnz == 0 || batch == 0 || n == 0) return MW_OK;
    MW_REQUIRE(rows && cols && vals && wire && zw && Z, "NULL argument");
    MW_REQUIRE(n_wires > 0, "entries need at least one wire");
    cudaStream_t st = as_stream(stream);
    const int64_t total = nnz * (int64_t)batch;
    const int64_t blocks = (total + 255) / 256;
    add_loading_kernel<<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0, st>>>(
        n, batch, nnz, rows, cols, vals, wire, reinterpret_cast<const double2*>(zw), n_wires,
        reinterpret_cast<double2*>(Z), ldz, z_stride, reinterpret_cast<float2*>(Z32), ld32, z32_stride, bad);
    MW_CHECK_CUDA(cudaGetLastError());
    count_launch();
    return MW_OK;
}

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
