// Host interface of the blocked FP64 sweep (csrc/blocked.cu).
#pragma once

#include <cuda_runtime.h>

namespace jsvd {

struct BlockedStats {
    unsigned long long solves = 0, sweeps = 0, block_rounds = 0;
    double sweep_ms = 0.0;
};

BlockedStats &blocked_stats();

// Blocked one-sided Jacobi on row-major d_a (rows x n, rows >= n); outputs as
// the plain path (row-major U and V, unsorted sigma; any may be null).
int blocked_solve(const double *d_a, int rows, int n, double eps, int max_sweeps, double *d_u, double *d_sigma,
                  double *d_v, int *sweeps, cudaStream_t st);

}  // namespace jsvd
