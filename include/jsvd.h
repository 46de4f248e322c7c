/*
 * jsvd.h - C ABI of the B200 (sm_100a) one-sided Jacobi SVD.
 *
 * Plain pointers and sizes only.  Every entry point returns a status code
 * (JSVD_OK on success); the message of the last failure on the calling thread
 * is available from jsvd_last_error().  The C++ headers kernels.hpp,
 * pipeline.hpp and io.hpp in this directory are implemented on top of this
 * ABI and turn the status codes back into the exception types of
 * kleedaisuki/jacobi-svd-cuda.
 *
 * Matrices are row-major FP64 unless a function says otherwise, as in the
 * reference (include/kernels.hpp:249-280).
 */
#ifndef JSVD_H
#define JSVD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes --------------------------------------------------------- */
#define JSVD_OK 0
#define JSVD_ERR_INVALID_ARGUMENT 1 /* std::invalid_argument in the reference            */
#define JSVD_ERR_CUDA 2             /* jacobi::svd::CudaError (kernels.hpp:65-73)          */
#define JSVD_ERR_OVERFLOW 3         /* std::overflow_error (size arithmetic)               */
#define JSVD_ERR_RUNTIME 4          /* std::runtime_error (device wait limit, I/O, ...)    */
#define JSVD_ERR_BUDGET 5           /* request larger than the serving memory budget     */

/* Layout-transpose policy, include/kernels.hpp:13-29.  Accepted and validated;
 * the sweep always runs on a column-major working copy, so the arithmetic does
 * not depend on it. */
#define JSVD_LAYOUT_AUTO 0
#define JSVD_LAYOUT_FORCE_ENABLE 1
#define JSVD_LAYOUT_FORCE_DISABLE 2

/* Mirrors jacobi::svd::JacobiSvdConfig, include/kernels.hpp:78-124. */
typedef struct jsvd_config {
    double epsilon;                             /* relative convergence tolerance (> 0)   */
    int max_sweeps;                             /* > 0                                     */
    int threads_per_block;                      /* reduction width T of the dot products   */
    int layout_transpose_mode;                  /* JSVD_LAYOUT_*                           */
    int layout_transpose_min_columns;           /* > 0                                     */
    size_t layout_transpose_min_elements;       /* > 0                                     */
    int layout_transpose_auto_tune;             /* bool                                    */
    int layout_transpose_benchmark_repetitions; /* > 0                                     */
    int layout_transpose_benchmark_sweeps;      /* > 0                                     */
} jsvd_config;

/* Mirrors jacobi::svd::LayoutTransposeAutoTuneReport, include/kernels.hpp:34-60. */
typedef struct jsvd_autotune_report {
    int executed;
    int recommended_min_columns;
    size_t recommended_min_elements;
    double estimated_best_speedup;
    size_t sample_count;
} jsvd_autotune_report;

/* Fills *cfg with the reference's defaults (eps 1e-9, 128 sweeps, T = 256, ...). */
void jsvd_config_default(jsvd_config *cfg);

/* Message of the last failure on this thread (NUL-terminated, truncated to
 * len).  Returns the status code of that failure (JSVD_OK if none). */
int jsvd_last_error(char *buf, size_t len);

/* Library version string. */
const char *jsvd_version(void);

/* FMA placement code of the plain path's rotation (p form | q form << 2);
 * tests hand it to the oracle. */
int jsvd_plain_arith_variant(void);

/*
 * Plain one-sided Jacobi SVD of one matrix, host buffers, synchronous.
 * Replaces jacobi::svd::one_sided_jacobi_svd (include/kernels.hpp:295-298,
 * src/kernels.cu:1066-1076): same validation and messages, same arithmetic
 * and cyclic round-robin order, U (m x n), sigma (n, unsorted) and V (n x n)
 * row-major.  u, sigma or v may be NULL to skip that output.  *sweeps gets
 * the executed sweep count (== max_sweeps when it did not converge).
 */
int jsvd_plain_svd(const double *a, size_t rows, size_t columns, const jsvd_config *cfg, double *u,
                   double *sigma, double *v, int *sweeps);

/*
 * Same as jsvd_plain_svd on device buffers, ordered on `stream`
 * (a cudaStream_t; NULL selects the library's per-thread stream).  Returns
 * after the solve has finished on the device.
 */
int jsvd_plain_svd_device(const double *d_a, size_t rows, size_t columns, const jsvd_config *cfg, double *d_u,
                          double *d_sigma, double *d_v, int *sweeps, void *stream);

/*
 * Allocation-free variant of jsvd_plain_svd_device.  It has no counterpart in
 * the reference: it exists for callers that cannot call cudaMalloc once they
 * are running (a framework that reserved the device for its own pool,
 * latency-critical code that cannot afford the device synchronisation of
 * cudaMalloc/cudaFree, plugin hosts that forbid device allocation).
 * It allocates nothing: the caller passes device buffers for A, U, sigma and
 * V (U, sigma, V may be NULL), work runs on `stream` as given (NULL = the
 * legacy default stream), and the working copies live in one fixed 16 MiB
 * device array inside the library, so rows*columns + columns*columns +
 * columns + 1 must not exceed 2097152 (larger requests fail with
 * JSVD_ERR_INVALID_ARGUMENT).  That array is held by every GPU that loads the
 * library until exit and is shared by all calls: calls that overlap on the GPU
 * race and must be serialised by the caller.  The first call on a device looks
 * up the array's device address; make it before any stream capture begins.
 * Results are bit-identical to jsvd_plain_svd_device.
 */
int jsvd_plain_svd_noalloc(const double *d_a, size_t rows, size_t columns, const jsvd_config *cfg, double *d_u,
                           double *d_sigma, double *d_v, int *sweeps, void *stream);

/*
 * Replaces jacobi::svd::auto_tune_layout_transpose_threshold
 * (include/kernels.hpp:306-307, src/kernels.cu:1078-1126): scans
 * n in {8,12,16,24,32,48,64,96}, m = 2n, on the reference's deterministic
 * benchmark matrix and times the solve with the layout forced on and off.
 */
int jsvd_auto_tune_layout(const jsvd_config *cfg, jsvd_autotune_report *report);

/* Cumulative counters of the plain path on the calling thread.  round_ms and
 * vpass_ms are device times of the round kernels and of the deferred V pass,
 * taken by event-record nodes inside each replayed sweep graph. */
typedef struct jsvd_plain_stats {
    unsigned long long solves;
    unsigned long long sweeps;
    unsigned long long round_launches;
    unsigned long long vpass_launches;
    unsigned long long other_launches; /* layout, identity, sigma, U and V kernels */
    double round_ms;
    double vpass_ms;
} jsvd_plain_stats;

void jsvd_plain_stats_get(jsvd_plain_stats *out);
void jsvd_plain_stats_reset(void);

/* Releases the calling thread's cached device workspaces and graphs. */
void jsvd_release_thread_cache(void);

#ifdef __cplusplus
}
#endif

#endif /* JSVD_H */
