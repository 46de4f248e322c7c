// One-sided block-pair Jacobi sweep engine (see blockpair.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

namespace jsvd {

struct BpStats {
    unsigned long long solves = 0, sweeps = 0, round_launches = 0;
    double round_ms = 0.0;
};
BpStats &bp_stats();

// True when an m x n problem (m >= n) fits a block-pair variant (m <= 4096).
bool bp_supported(size_t m, size_t n);

// Forces the block width and threads per CTA of later plans (0 = built-in).
void bp_set_variant(int block_cols, int threads);

// Drops the calling thread's cached block-pair plans.
void bp_release_thread_plans();

// Block-pair solve of row-major d_a (m x n) on stream st; outputs as the plain
// path's (row-major U and V, sigma unsorted), each may be null.
int bp_solve(const double *d_a, size_t m, size_t n, double eps, int max_sweeps, double *d_u, double *d_sigma,
             double *d_v, int *sweeps, cudaStream_t st);

}  // namespace jsvd
