// Host-side interface of the batched solver (csrc/batched.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>

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

}  // namespace jsvd
