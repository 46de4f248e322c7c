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
 * columns + 1 must not exceed 2097152 and rows 2097120 (larger requests fail
 * with JSVD_ERR_INVALID_ARGUMENT).  The array is committed on a device when
 * the library's module is loaded there; CUDA loads modules lazily by default,
 * so that happens on the first call on each device: a caller that reserves
 * the rest of the device afterwards makes one warm-up call per device first
 * (or sets CUDA_MODULE_LOADING=EAGER).  It then stays until the process
 * exits.  The array is shared by all calls and keeps the last call's
 * contents: calls that overlap on the GPU race and must be serialised by the
 * caller.  The first call on a device, and again the first call after the
 * device's context is replaced (cudaDeviceReset), looks up the array's device
 * address.  Each sweep waits on the host for a device-to-host copy, so the
 * entry cannot be used while its stream is being captured into a graph.
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
    unsigned long long gram_checks; /* Gram convergence tests (QR-preconditioned path) */
} jsvd_plain_stats;

void jsvd_plain_stats_get(jsvd_plain_stats *out);

/* How the plain path launches a sweep (process-wide, read when a plan is
 * created): 0 = one kernel per round, replayed from a CUDA graph, each CTA
 * reducing its pair's dot products and deriving the angle once, in one warp
 * (default); 1 = one persistent cooperative kernel per sweep whose CTAs
 * synchronise with their neighbours through per-CTA round counters (bounded
 * waits); 2 = as 0 with programmatic dependent launch, each round scheduled
 * while the previous one drains; 3 = as 0 with every warp reducing and
 * deriving the angle itself (one barrier fewer, eight times the FP64 work).
 * All give bit-identical results.  Measured per 512-row round on B200: mode 0
 * 2.6 us, mode 3 2.9 us, mode 2 3.9 us, mode 1 6.9 us. */
void jsvd_plain_set_sweep_mode(int mode);
int jsvd_plain_get_sweep_mode(void);

/* Forces (1) or releases (0) the in-place global-memory form of the plain
 * path's deferred V pass for plans created afterwards.  That form is used by
 * itself for more than 25600 columns, where a row of V does not fit a CTA's
 * shared memory; results are the same bytes either way.  Process-wide; for
 * tests. */
void jsvd_plain_set_vpass_in_global(int enable);
void jsvd_plain_stats_reset(void);

/*
 * The round-robin pair schedule the kernels follow (reference
 * src/kernels.cu:637-678): for n columns, rounds = n_e - 1 (n_e = n rounded
 * up to even; no rounds for n = 1) of n/2 pairs each, written round-major as
 * (p, q) int pairs.  form 0: the table the plain path uploads; form 1: the
 * closed form that the kernels deriving their own pairs evaluate.  *needed
 * (optional) receives 2 * rounds * (n/2); out may be NULL to query it.
 * 1 <= n <= 65536.  No CUDA call.
 */
int jsvd_round_robin_schedule(int n, int form, int *out, size_t capacity, size_t *needed);

/* ---- validation -------------------------------------------------------------
 * The reference's validation metrics of one result
 * (tex/sections/03-gpu-parallel-reduction.tex:30-40), computed on the host. */
typedef struct jsvd_residual_report {
    double rho_a;     /* ||A - U S V^T||_F / max(1, ||A||_F); -1 when a or u is NULL */
    double rho_u;     /* ||U^T U - I||_F over the columns with sigma > 0; -1 when u is NULL */
    double rho_v;     /* ||V^T V - I||_F */
    double sigma_max; /* largest sigma */
} jsvd_residual_report;

/* a (optional) rows x columns, u (optional) rows x columns, v columns x
 * columns, all row-major host buffers as jsvd_plain_svd returns them; sigma
 * the columns singular values.  Uses the host's threads; no CUDA call. */
int jsvd_residuals(const double *a, const double *u, const double *sigma, const double *v, size_t rows,
                   size_t columns, jsvd_residual_report *out);

/* ---- batched solver ---------------------------------------------------------
 * Many independent matrices in one persistent launch per size class.  The
 * reference solves them one call at a time from a host thread pool
 * (src/pipeline.cpp:799-807 -> one_sided_jacobi_svd); this replaces that loop
 * for matrices that are all resident on the device.  Arithmetic per matrix is
 * the plain path's (T = 256 reduction order), so each result is bit-identical
 * to jsvd_plain_svd on the FP64-promoted input. */

/* Launch shape of one size class.  An entry of three zeros keeps the
 * built-in shape of its class; otherwise threads or ctas_per_sm 0 keeps that
 * built-in value and max_ctas 0 means no cap. */
typedef struct jsvd_batch_tuning {
    int threads;     /* threads per CTA (multiple of 32, <= 512) */
    int ctas_per_sm; /* persistent CTAs per SM */
    int max_ctas;    /* upper bound on the class's grid (bounds the L2 working set of the global classes) */
} jsvd_batch_tuning;

/* The built-in shapes (5 entries), compiled in from the table that
 * jsvd_batch_autotune's generator writes.  No CUDA call. */
void jsvd_batch_builtin_tuning(jsvd_batch_tuning *out);

/*
 * count matrices; matrix i is rows[i] x cols[i] (rows >= cols >= 1), row-major
 * at element offset a_offsets[i] of d_a (FP32 when a_is_f32, else FP64).
 * Outputs are packed in input order: d_sigma gets cols[i] values per matrix,
 * d_v (optional) cols[i]^2 row-major, d_u (optional) rows[i]*cols[i]
 * row-major; sweeps (host, optional) the sweep count of each matrix.  cfg's
 * epsilon and max_sweeps apply (threads_per_block must be 256).  tuning may
 * be NULL or point to 5 entries, one per size class: A and V in <= 48 KiB,
 * <= 100 KiB, <= ~226 KiB of shared memory; A alone in shared memory; A and V
 * in global memory.
 * Synchronous on `stream` (NULL = library stream, ordered after the legacy
 * default stream).
 */
int jsvd_batch_svd_device(int count, const int *rows, const int *cols, const long long *a_offsets, const void *d_a,
                          int a_is_f32, const jsvd_config *cfg, double *d_sigma, double *d_v, double *d_u,
                          int *sweeps, const jsvd_batch_tuning *tuning, void *stream);

/* Size classes whose members are solved by a thread-block cluster (2, 4 or 8
 * CTAs, the smallest whose distributed shared memory holds A and V with at
 * least two column pairs per CTA) instead of by one CTA: bit c = class c,
 * classes 2, 3 and 4 only (default: the compiled-in tuning table's choice,
 * JSVD_BATCH_CLUSTER_CLASSES, which batch_autotune.py measures: 3 and 4).  A member that fits no cluster
 * stays with its class's own kernel, which is also the only one the class's
 * tuning entry shapes.  Results are the same bytes either way.
 * Process-wide; *previous (optional) gets the old mask. */
int jsvd_batch_set_cluster_classes(int mask, int *previous);

/* Result of jsvd_batch_autotune, per size class. */
typedef struct jsvd_batch_autotune_report {
    jsvd_batch_tuning best[5];    /* chosen shape (the built-in one unless another is > 2% faster) */
    jsvd_batch_tuning builtin[5]; /* the built-in shape */
    double best_ms[5];            /* device ms of the class's sample under best (min over reps) */
    double builtin_ms[5];         /* the same under the built-in shape */
    int members[5];               /* matrices of the batch in the class */
    int sampled[5];               /* matrices timed */
    int candidates[5];            /* shapes timed, the built-in one included */
} jsvd_batch_autotune_report;

/*
 * Launch-shape autotuner of the batched solver.  Takes the same batch
 * description as jsvd_batch_svd_device (the outputs go to buffers of its own)
 * and, for every size class with members, times the built-in shape and each
 * candidate shape (threads 128/256/512 x CTAs per SM as shared memory allows;
 * for the classes that take a whole SM, threads x grid cap none/0.75/0.5 of the
 * SMs) on up to `sample` of the class's matrices (0 = all; evenly spaced over
 * the work order), L2 flushed before each of `reps` runs (0 = 2), minimum kept.
 * Every shape must give the same sigma bytes and sweep counts as the built-in
 * one, else JSVD_ERR_RUNTIME.  want_u / want_v: compute U / V as the timed
 * workload does.  Synchronous on `stream` (NULL = library stream).  The
 * batch statistics are left as they were.
 */
int jsvd_batch_autotune(int count, const int *rows, const int *cols, const long long *a_offsets, const void *d_a,
                        int a_is_f32, const jsvd_config *cfg, int sample, int reps, int want_u, int want_v,
                        jsvd_batch_autotune_report *report, void *stream);

/*
 * One-sided block-pair Jacobi on device buffers (same arguments and outputs as
 * jsvd_plain_svd_device).  No single reference function corresponds: it
 * replaces the cyclic sweep loop of run_one_sided_jacobi_svd_internal
 * (src/kernels.cu:889-981) with an outer sweep over pairs of column blocks
 * (B = 2, 4 or 8 columns), each block pair solved by one CTA with a full
 * inner cyclic sweep over its 2B columns held in registers; V takes the
 * product of a block pair's rotations once.  Rotation test, angle formula and
 * stopping rule (an outer sweep without rotation) are the reference's; the
 * ordering is not, so results agree with the plain path to working accuracy,
 * not bit for bit.  Up to 4096 rows; taller inputs run the plain path.
 */
int jsvd_blockpair_svd_device(const double *d_a, size_t rows, size_t columns, const jsvd_config *cfg, double *d_u,
                              double *d_sigma, double *d_v, int *sweeps, void *stream);

/* The same on host buffers (copies in and out on the library's stream). */
int jsvd_blockpair_svd(const double *a, size_t rows, size_t columns, const jsvd_config *cfg, double *u, double *sigma,
                       double *v, int *sweeps);

/* Forces the block width (2, 4, 8) and threads per CTA (128, 256, 512) of
 * block-pair plans created afterwards; 0 keeps the built-in choice for that
 * parameter.  Process-wide; for tuning and tests. */
void jsvd_blockpair_set_variant(int block_columns, int threads);

/* Cumulative counters of the block-pair engine on the calling thread. */
typedef struct jsvd_blockpair_stats {
    unsigned long long solves;
    unsigned long long sweeps;          /* outer sweeps */
    unsigned long long round_launches;  /* outer-round kernels */
    double round_ms;                    /* device time of the outer sweeps */
} jsvd_blockpair_stats;
void jsvd_blockpair_stats_get(jsvd_blockpair_stats *out);
void jsvd_blockpair_stats_reset(void);

/* Engine of the Jacobi stage inside jsvd_precond_svd*: 0 = block-pair sweep
 * where it applies, else plain; 1 = the plain sweep (default, faster on B200
 * for the shapes measured).  Process-wide. */
void jsvd_precond_set_inner(int engine);

/* 1 (default): inside jsvd_precond_svd*, when epsilon >= 1e-12 and a sweep
 * of the plain Jacobi stage rotates fewer than 1/8 of its pairs, every pair is
 * tested on the Gram matrix of the columns (one lower-triangle GEMM); when none would
 * rotate, the final sweep (which would rotate nothing) is not run but is
 * still counted in `sweeps`.  Below 1e-12 the GEMM's own rounding of the
 * off-diagonal entries is too close to epsilon for the test to succeed.
 * 0: always run that sweep.  Process-wide. */
void jsvd_precond_set_gram_stop(int enable);

/* Cumulative counters of the batched solver on the calling thread. */
typedef struct jsvd_batch_stats {
    unsigned long long calls;
    unsigned long long launches;
    unsigned long long matrices;
    unsigned long long sweeps;
    double kernel_ms; /* device time of the persistent launches (events) */
    unsigned long long class_count[5]; /* matrices per size class */
    double class_ms[5];                /* device time of each class's launch */
} jsvd_batch_stats;

void jsvd_batch_stats_get(jsvd_batch_stats *out);
void jsvd_batch_stats_reset(void);

/* ---- QR-preconditioned path -------------------------------------------------
 * The fast path for tall and ill-conditioned matrices (no counterpart in the
 * reference, which always sweeps A directly): A = Q R by shifted CholeskyQR3,
 * one-sided Jacobi (the plain sweep) on X = R^T, then V_A = normalised columns
 * of the rotated X, U_A = Q V_x.  Same inputs, outputs and validation as
 * jsvd_plain_svd / jsvd_plain_svd_device; sigma is unsorted; *sweeps is the
 * sweep count on X.  Falls back to the plain path if a Cholesky pivot is not
 * positive.  Results agree with the plain path to working accuracy
 * (normwise sigma error ~1e-14, orthogonality ~1e-13), not bit for bit. */
int jsvd_precond_svd(const double *a, size_t rows, size_t columns, const jsvd_config *cfg, double *u,
                     double *sigma, double *v, int *sweeps);
int jsvd_precond_svd_device(const double *d_a, size_t rows, size_t columns, const jsvd_config *cfg, double *d_u,
                            double *d_sigma, double *d_v, int *sweeps, void *stream);

/* Blocked FP64 one-sided Jacobi (no counterpart in the reference): column
 * blocks of 32, block pairs in the round-robin order, per pair a panel Gram,
 * a two-sided Jacobi solve of the 64 x 64 Gram and the panel update P <- P W.
 * Same arguments and outputs as jsvd_plain_svd_device; accurate to working
 * precision, not bit-identical to the plain path.  Below 64 columns (fewer
 * than two blocks) it runs the plain sweep. */
int jsvd_blocked_svd_device(const double *d_a, size_t rows, size_t columns, const jsvd_config *cfg, double *d_u,
                            double *d_sigma, double *d_v, int *sweeps, void *stream);

/* The same on host buffers (copies in and out on the library's stream). */
int jsvd_blocked_svd(const double *a, size_t rows, size_t columns, const jsvd_config *cfg, double *u, double *sigma,
                     double *v, int *sweeps);

typedef struct jsvd_blocked_stats {
    unsigned long long solves, sweeps, block_rounds;
    double sweep_ms; /* device time of the sweeps (events) */
} jsvd_blocked_stats;

void jsvd_blocked_stats_get(jsvd_blocked_stats *out);
void jsvd_blocked_stats_reset(void);

typedef struct jsvd_precond_stats {
    unsigned long long solves, fallbacks;
    double qr_ms, jacobi_ms, u_ms; /* device time per phase (events) */
} jsvd_precond_stats;

void jsvd_precond_stats_get(jsvd_precond_stats *out);
void jsvd_precond_stats_reset(void);

/* ---- blocked mixed-precision path -------------------------------------------
 * No counterpart in the reference, whose only sweep is the scalar column-pair
 * loop of src/kernels.cu:889-981.  A is first QR-preconditioned as in
 * jsvd_precond_svd (A = Q R, R^T = Q1 P, X = P^T).  X's columns are grouped in
 * blocks of 32 and the blocks paired in the round-robin order.  For each block
 * pair, the 64 x 64 Gram G = [X_i X_j]^T [X_i X_j] is eigen-solved in FP64
 * (cyclic two-sided Jacobi, G = W L W^T) and the pair is rotated,
 * [X_i X_j] <- [X_i X_j] W, likewise V.
 *   1. Tensor-core phase: Grams and rotations are tcgen05 GEMMs in 3xTF32
 *      (each FP32 operand split into a TF32 head and tail) with FP32
 *      accumulation, operands brought in by TMA; X and V are held as TF32
 *      head/tail pairs.
 *   2. V of phase 1 is made orthogonal in FP64 (Newton-Schulz polar
 *      iteration), X' = X V' (FP64).
 *   3. FP64 refinement: the same blocked sweeps in FP64 (DMMA GEMMs) on X'
 *      until no pair rotates (threshold max(epsilon, 4 sqrt(m) 2^-53)).
 * Same arguments, outputs and validation as jsvd_precond_svd; sigma unsorted;
 * *sweeps = phase-1 sweeps + refinement sweeps.  Inputs with fewer than 128
 * columns run the QR-preconditioned plain path.  Accurate to working
 * precision (normwise), not bit-identical to the plain path. */
typedef struct jsvd_mixed_options {
    int precondition;   /* 1 (default): blocked sweeps on X = P^T after the two QRs; 0: on A   */
    int tc_max_sweeps;  /* tensor-core sweeps at most; 0 = FP64 blocked sweeps only; -1 (default) =
                           automatic (the built-in tuning table, by column count)              */
    double tc_tol;      /* phase 1 ends when no pair's |g_pq| / sqrt(g_pp g_qq) exceeds this    */
    int inner_sweeps;   /* two-sided sweeps per 64 x 64 block eigen-solve; 0 (default) =
                           automatic (the built-in tuning table)                               */
    int refine;         /* refinement: 0 = blocked FP64 sweeps (default), 1 = plain scalar sweep */
    int f64_max_sweeps; /* cap on refinement sweeps; 0 = the config's max_sweeps                  */
    int gram_splits;    /* row splits of each block-pair Gram; 0 = automatic (the table's value,
                           else enough CTAs to cover the GPU twice)                           */
    int sort;           /* 1 (default): each block eigen-solve gives the larger eigenvalues to the
                           lower-numbered block (decreasing column norms, de Rijk's ordering)   */
} jsvd_mixed_options;

void jsvd_mixed_options_default(jsvd_mixed_options *o);
/* The mixed path's built-in tuning table (csrc/mixed_tuning_table.h, made by
 * jacobi-svd-cuda_b200/mixed_autotune.py on a B200): entry i is out[4i..4i+3]
 * = {largest column count it covers (0 = any), tc_max_sweeps, inner_sweeps,
 * gram_splits (0 = automatic)}; the first covering entry resolves a solve's
 * automatic options.  Writes at most `capacity` entries (out may be NULL)
 * and returns the number of entries.  No counterpart in the reference (its
 * only tuner is auto_tune_layout_transpose_threshold, src/kernels.cu:1078-1126,
 * which this table's role extends to the blocked path). */
int jsvd_mixed_builtin_tuning(int *out, int capacity);
/* Options of later jsvd_mixed_svd* calls on the calling thread (NULL: defaults). */
void jsvd_mixed_set_options(const jsvd_mixed_options *o);

int jsvd_mixed_svd(const double *a, size_t rows, size_t columns, const jsvd_config *cfg, double *u, double *sigma,
                   double *v, int *sweeps);
int jsvd_mixed_svd_device(const double *d_a, size_t rows, size_t columns, const jsvd_config *cfg, double *d_u,
                          double *d_sigma, double *d_v, int *sweeps, void *stream);

/* Cumulative counters of the mixed path on the calling thread. */
typedef struct jsvd_mixed_stats {
    unsigned long long solves, tc_sweeps, f64_sweeps, block_rounds, fallbacks;
    double qr_ms, tc_ms, orth_ms, refine_ms, out_ms; /* device time per phase (events)           */
    double last_tc_offdiag;   /* largest scaled off-diagonal Gram entry, last phase-1 sweep      */
    double last_f64_offdiag;  /* the same for the last refinement sweep                           */
    int last_tc_sweeps, last_f64_sweeps;
    unsigned long long tc_gram_launches, tc_rot_launches, f64_gram_launches, f64_rot_launches, evd_launches;
    unsigned long long tc_discarded; /* solves whose phase-1 V did not orthogonalise (FP64 sweeps from X) */
    /* device time of the Gram, eigen-solve and rotation kernels of sampled
     * block rounds (rounds 0 and rounds/2 of every sweep; events around each
     * launch), per phase, and the number of sampled rounds */
    double tc_gram_ms, tc_evd_ms, tc_rot_ms, f64_gram_ms, f64_evd_ms, f64_rot_ms;
    unsigned long long tc_sampled_rounds, f64_sampled_rounds;
    /* block pairs rotated in the sampled rounds (each rotation kernel moves
     * (rows_pad + cols_pad) x 64 elements of X and V per rotated pair) */
    unsigned long long tc_sampled_pairs, f64_sampled_pairs;
    int rows_pad, cols_pad, block_pairs; /* working shape of the last sweep */
} jsvd_mixed_stats;

void jsvd_mixed_stats_get(jsvd_mixed_stats *out);
void jsvd_mixed_stats_reset(void);

/* Sweeps of the calling thread's last mixed solve, in order: phase (1 tensor
 * core, 3 FP64 refinement), the largest scaled off-diagonal Gram entry the
 * sweep saw, and the block pairs it rotated.  Fills at most `capacity`
 * entries (any pointer may be NULL) and returns the number of sweeps
 * recorded (at most 64). */
int jsvd_mixed_sweep_history(int *phase, double *offdiag, unsigned long long *rotated, int capacity);

/* Kernel-level test hook of the mixed path: one block round (`round`) of its
 * kernels on X (rows x cols, column-major FP64, device, both multiples of
 * 128).  kind 0: tensor-core Gram of each block pair -> gw (pairs x 64 x 64,
 * column-major FP64); 1: FP64 Gram -> gw; 2: tensor-core rotation
 * X_pair <- X_pair W_pair with W read from gw, in place; 3: FP64 rotation. */
int jsvd_mixed_test_round(int kind, double *d_x, int rows, int cols, int round, double *d_gw);

/* Failure-detection check of the bounded device waits: one wait with a
 * limit of limit_ms (1..2000) on something nothing completes during the
 * launch.  which 0: the persistent sweep's acquire-load wait on another CTA's
 * round flag; 1: the tensor-core kernels' mbarrier wait.  preset != 0 sets
 * the flag (arrives on the barrier) first, so the wait ends at once.  On
 * expiry the kernel writes status 2 (wait timeout) and returns, the context
 * stays usable, and the call returns JSVD_ERR_RUNTIME with a last-error
 * message, as a sweep stopped at its limit does.  *device_status and
 * *elapsed_ms (launch time) may be NULL. */
int jsvd_test_wait_limit(int which, int limit_ms, int preset, int *device_status, double *elapsed_ms);

/* FP64 GEMM of the library (DMMA tensor cores), for tests and tools:
 * C = alpha op(A) op(B) + beta C, column-major device buffers, op 'N' or 'T';
 * lower != 0 writes only C's lower triangle.  Synchronous on the calling
 * thread's library stream. */
int jsvd_dgemm_device(char op_a, char op_b, int m, int n, int k, double alpha, const double *a, long lda,
                      const double *b, long ldb, double beta, double *c, long ldc, int lower);

/* ---- serving loop -----------------------------------------------------------
 * Continuous batching of SVD requests on the current device.  Replaces the
 * reference's thread-pool dispatch of one_sided_jacobi_svd per testcase
 * (src/pipeline.cpp:234-394, 754-863): requests are admitted against a
 * device-memory budget.  Small ones (A's FP64 copy fits a CTA's shared
 * memory) are batched at sweep granularity: each admitted request keeps A and
 * V on the device, every step runs one sweep of all active requests, the
 * converged ones retire after it and queued ones join before the next step.
 * Large ones run concurrently on worker streams.  Results do not depend on
 * what else is in flight (every path keeps the plain arithmetic). */

typedef struct jsvd_server jsvd_server;

typedef struct jsvd_server_options {
    size_t device_budget_bytes; /* admission budget (0 = 40 GiB)                    */
    int small_workers;          /* sweep-stepping workers, each with its own active
                                   set and stream (0 = 2)                           */
    int large_workers;          /* concurrent large solves, one stream each (0 = 4) */
    int max_batch;              /* active small requests per worker (0 = 4096)      */
    jsvd_config cfg;            /* epsilon, max_sweeps, threads_per_block           */
    int large_path;             /* 0 = plain sweep, 1 = QR-preconditioned, 2 = mixed  */
} jsvd_server_options;

typedef struct jsvd_server_stats {
    unsigned long long submitted, completed, failed;
    unsigned long long batches;          /* sweep steps of the small-request workers */
    unsigned long long batched_requests, large_solves;
    double p50_ms, p99_ms, mean_ms; /* submit-to-completion latency */
    size_t peak_device_bytes, device_bytes_in_use;
} jsvd_server_stats;

void jsvd_server_options_default(jsvd_server_options *opt);
int jsvd_server_create(const jsvd_server_options *opt, jsvd_server **out);
/* Copies A (row-major m x n, m >= n) and queues it; JSVD_ERR_BUDGET when its
 * footprint exceeds the whole budget. */
int jsvd_server_submit(jsvd_server *s, const double *a, size_t rows, size_t columns, int want_u, uint64_t *ticket);
/* Blocks until the request is done and copies its results (row-major U if
 * requested at submit, sigma, row-major V); each ticket can be collected once. */
int jsvd_server_wait(jsvd_server *s, uint64_t ticket, double *u, double *sigma, double *v, int *sweeps,
                     double *latency_ms);
/* Non-blocking: *done = 1 when the request has finished (a following
 * jsvd_server_wait returns without blocking), else 0.  JSVD_ERR_INVALID_ARGUMENT
 * for a ticket that is unknown, already collected, or being waited on. */
int jsvd_server_poll(jsvd_server *s, uint64_t ticket, int *done);
int jsvd_server_get_stats(jsvd_server *s, jsvd_server_stats *out);
/* Stops the workers (requests being solved finish first).  Requests still
 * queued fail with JSVD_ERR_RUNTIME, which wakes threads waiting on them;
 * returns once no thread is inside jsvd_server_wait.  No call on s after. */
void jsvd_server_destroy(jsvd_server *s);

/* Measured FP64 FMA throughput of the current device in TFLOP/s (eight
 * independent FMA chains per thread, best of 5 launches): the roofline
 * denominator of the FP64-bound kernels. */
int jsvd_probe_fp64_tflops(double *tflops);

/* Releases the calling thread's cached device workspaces and graphs. */
void jsvd_release_thread_cache(void);

#ifdef __cplusplus
}
#endif

#endif /* JSVD_H */
