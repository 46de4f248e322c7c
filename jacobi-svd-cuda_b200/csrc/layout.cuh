// Layout kernels shared by the sweep engines (sm_100a): tiled 32 x 32
// transposes between the caller's row-major matrices and the column-major
// working copies, and V = I.  The reference's tiled transpose is
// src/kernels.cu:246-275; its identity kernel is src/kernels.cu:387-399.
// Defined in an anonymous namespace: each translation unit that includes this
// header gets its own copy of the kernels.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>

namespace jsvd {
namespace {

constexpr int kTile = 32;
constexpr int kTileRows = 8;

// row-major src (rows x cols) -> column-major dst (leading dimension ldd).
__global__ void __launch_bounds__(kTile *kTileRows)
    rowmajor_to_colmajor_kernel(const double *__restrict__ src, int rows, int cols, double *__restrict__ dst,
                                long ldd)
{
    __shared__ double tile[kTile][kTile + 1];
    const int c0 = blockIdx.x * kTile, r0 = blockIdx.y * kTile;
    for (int k = threadIdx.y; k < kTile; k += kTileRows) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if (r < rows && c < cols) tile[k][threadIdx.x] = src[(size_t)r * cols + c];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < kTile; k += kTileRows) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (r < rows && c < cols) dst[(size_t)c * ldd + r] = tile[threadIdx.x][k];
    }
}

// rowmajor_to_colmajor_kernel over all rows: row tiles run along grid.y
// (at most 65535 blocks), so taller inputs take one launch per 65535 * 32 rows,
// each on the sub-matrix starting at that row (src advanced by whole rows, dst
// by the same number of rows within each column).  One launch, with exactly
// the plain arguments, up to 2,097,120 rows.
constexpr int kTransposeMaxRows = 65535 * kTile;  // rows one launch covers

// Launches launch_rowmajor_to_colmajor makes for `rows` rows.
inline int rowmajor_to_colmajor_launches(int rows)
{
    return rows <= 0 ? 0 : 1 + (rows - 1) / kTransposeMaxRows;
}

inline cudaError_t launch_rowmajor_to_colmajor(const double *src, int rows, int cols, double *dst, long ldd,
                                               cudaStream_t stream)
{
    constexpr int kMaxRows = kTransposeMaxRows;
    const dim3 block(kTile, kTileRows);
    for (long long r0 = 0; r0 < rows; r0 += kMaxRows) {
        const int rr = (int)std::min<long long>(kMaxRows, rows - r0);
        const dim3 grid((cols + kTile - 1) / kTile, (rr + kTile - 1) / kTile);
        rowmajor_to_colmajor_kernel<<<grid, block, 0, stream>>>(src + (size_t)r0 * cols, rr, cols, dst + r0, ldd);
        const cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// column-major src (rows x cols, leading dimension lds) -> row-major dst.
// With sigma != nullptr each column is divided by sigma[c], or zeroed when
// sigma[c] <= eps (src/kernels.cu:622-627).
__global__ void __launch_bounds__(kTile *kTileRows)
    colmajor_to_rowmajor_kernel(const double *__restrict__ src, long lds, int rows, int cols,
                                double *__restrict__ dst, const double *__restrict__ sigma, double eps)
{
    __shared__ double tile[kTile][kTile + 1];
    const int r0 = blockIdx.x * kTile, c0 = blockIdx.y * kTile;
    for (int k = threadIdx.y; k < kTile; k += kTileRows) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (r < rows && c < cols) tile[k][threadIdx.x] = src[(size_t)c * lds + r];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < kTile; k += kTileRows) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if (r < rows && c < cols) {
            double val = tile[threadIdx.x][k];
            if (sigma != nullptr) {
                const double sg = sigma[c];
                val = (sg > eps) ? (val / sg) : 0.0;
            }
            dst[(size_t)r * cols + c] = val;
        }
    }
}

__global__ void identity_colmajor_kernel(double *__restrict__ v, int n, long ldv)
{
    const size_t total = (size_t)n * ldv;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x) {
        const size_t col = idx / ldv, row = idx % ldv;
        v[idx] = (row == col) ? 1.0 : 0.0;
    }
}

}  // namespace
}  // namespace jsvd
