// Host-side interface of the batched solver (csrc/batched.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <vector>

#include "jsvd.h"

namespace jsvd {

// One matrix of a batch; offsets are element offsets into the packed buffers.
struct BatchDesc {
    int m, n;
    long long a_off, s_off, v_off, u_off;
};

struct BatchRequest {
    int count = 0;
    const int *rows = nullptr;
    const int *cols = nullptr;
    const long long *a_offsets = nullptr;  // element offsets of each A in `a`
    const void *a = nullptr;               // device, row-major, FP32 or FP64
    int a_is_f32 = 0;
    double eps = 1e-9;
    int max_sweeps = 128;
    double *sigma = nullptr;  // device, packed n per matrix (input order)
    double *v = nullptr;      // device, packed n*n row-major, or null
    double *u = nullptr;      // device, packed m*n row-major, or null
    int *sweeps = nullptr;    // host, per matrix, or null
    const jsvd_batch_tuning *tuning = nullptr;  // one entry per class, or null
};

struct BatchStats {
    unsigned long long calls = 0, launches = 0, matrices = 0, sweeps = 0;
    double kernel_ms = 0.0;
    unsigned long long class_count[5] = {};
    double class_ms[5] = {};
};

BatchStats &batch_stats();
int batch_solve(const BatchRequest &req, cudaStream_t stream);

// Sweep-granular batching (the serving core's small requests).  A member's
// state, A (m x n) and V (n x n), FP64 column-major, lives in device memory
// between steps.
struct StepDesc {
    int m, n;
    double *a, *v;        // state
    const double *in;     // row-major FP64 input for the first step, else null
    double *s_out, *v_out, *u_out;  // outputs written by batch_finish (u_out null: none)
};

// Device descriptors and flags reused from step to step (one per thread).
struct StepScratch {
    StepDesc *d_descs = nullptr;  // 2 * cap
    int *d_rot = nullptr, *h_rot = nullptr;
    int cap = 0;
    int ensure(int count);
    ~StepScratch();
};

// Whether an m x n member can take part (A and the round scratch fit one
// CTA's shared memory).
bool step_fits(int m, int n, size_t *smem_cap = nullptr);
// One sweep of every member of `descs` (one CTA each); rotated[i] = 1 when
// member i's sweep rotated a pair (0: converged).  Synchronises `st`.
int batch_step(const std::vector<StepDesc> &descs, double eps, int *rotated, StepScratch &sc, cudaStream_t st);
// sigma, V and U of retired members into `out` (asynchronous on `st`).
int batch_finish(const std::vector<StepDesc> &descs, double eps, StepScratch &sc, cudaStream_t st);

}  // namespace jsvd
