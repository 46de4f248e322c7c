// Layout kernels shared by the sweep engines (sm_100a): tiled 32 x 32
// transposes between the caller's row-major matrices and the column-major
// working copies, and V = I.  The reference's tiled transpose is
// src/kernels.cu:246-275; its identity kernel is src/kernels.cu:387-399.
// Defined in an anonymous namespace: each translation unit that includes this
// header gets its own copy of the kernels.
#pragma once

#include <cuda_runtime.h>

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
