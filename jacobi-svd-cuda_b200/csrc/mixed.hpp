// Blocked mixed-precision one-sided Jacobi (mixed.cu): internal interface.
#pragma once

#include <cuda_runtime.h>

#include "jsvd.h"

namespace jsvd {

// Blocked one-sided Jacobi of X (rows x cols, row-major, device, rows >= cols):
// a tensor-core phase (3xTF32 block Grams and block rotations on tcgen05, FP64
// block eigen-solves), re-orthogonalisation of its V in FP64, X' = X V', then
// FP64 blocked refinement sweeps (DMMA) until no pair rotates.  u (rows x
// cols), sigma (cols), v (cols x cols) row-major; any may be null.
int mixed_solve(const double *x, int rows, int cols, const jsvd_config &c, const jsvd_mixed_options &o, double *u,
                double *sigma, double *v, int *sweeps, cudaStream_t st);

// Counts one solve of the mixed path (and a fallback to the plain sweep).
void mixed_note_solve(double qr_ms, bool fallback);

// Drops the calling thread's cached mixed-path workspaces.
void mixed_release_thread_cache();

// The calling thread's options (jsvd_mixed_set_options).
const jsvd_mixed_options &mixed_options();

// Wait-limit check of the tensor-core kernels' mbarrier wait: one thread
// initialises an mbarrier and waits on its first phase with limit_ns;
// `arrive` makes it arrive first (the wait then completes at once).  On
// expiry kDevWaitTimeout is written to *status.
int mixed_wait_limit_check(long long limit_ns, bool arrive, int *status, cudaStream_t st);

// Smallest column count the blocked engine takes (narrower inputs go to the
// plain sweep).
constexpr int kMixedMinCols = 128;

}  // namespace jsvd
