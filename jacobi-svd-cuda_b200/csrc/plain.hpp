// Host-side plan of the plain FP64 sweep: device workspace for one shape and
// the captured sweep graph.  Plans are cached per thread (see abi.cu), so a
// caller that solves many matrices of one shape pays for allocation and
// graph instantiation once.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <memory>

#include "jsvd.h"

namespace jsvd {

// The deferred V pass keeps R >= 1 whole rows of V in one CTA's shared memory,
// at most this many bytes; longer rows (more than 25600 columns) are rotated
// in place in global memory, one row per CTA.
constexpr size_t kVpassSmemCap = 200 * 1024;

// Forces the in-place global-memory form of the V pass for plans created
// afterwards (process-wide; part of the plan cache key).  For tests.
bool vpass_global_forced();
void set_vpass_global_forced(bool on);

struct PlainPlan {
    int device = -1;
    cudaStream_t stream = nullptr;  // allocation / release stream (the creating thread's)
    size_t m = 0, n = 0;
    int T = 256;
    double eps = 0.0;
    long lda = 0, ldv = 0;
    int rounds = 0, npairs = 0;
    int vpass_rows = 1, vpass_smem = 0, vpass_threads = 256;
    bool vpass_staged = true;          // rows of V staged in shared memory (else rotated in global memory)
    bool vpass_global_forced = false;  // created under set_vpass_global_forced(true)
    size_t bytes = 0;

    double *a_w = nullptr;      // column-major working copy of A (m x n)
    double *v_w = nullptr;      // column-major V (n x n)
    double *sigma_w = nullptr;  // sigma when the caller does not want it
    int2 *pairs = nullptr;      // rounds x npairs schedule
    double2 *cs = nullptr;      // (c, s) of every pair of even sweeps
    double2 *cs2 = nullptr;     // (c, s) of every pair of odd sweeps
    unsigned *counter = nullptr;  // [0] rotations in the sweep, [1] device status
    int *flags = nullptr;         // persistent sweep: rounds completed per CTA
    bool persistent = false;      // one cooperative launch per sweep
    int slots_per_cta = 1, sweep_grid = 0;
    int mode = 0;         // sweep_mode() at creation
    bool use_pdl = false;     // programmatic dependent launch between rounds
    bool angle_once = false;  // rounds reduce and derive the angle in one warp
    unsigned long long uses = 0;
    bool sweep_exec_capturing = false;
    // staging for host-buffer calls
    double *d_in = nullptr, *d_u = nullptr, *d_sigma = nullptr, *d_v = nullptr;
    // convergence test on the Gram matrix (run option gram_stop), made on first use
    double *gram = nullptr;            // n x n, lower triangle
    unsigned *gram_count = nullptr;    // pairs that would rotate
    unsigned *h_gram_count = nullptr;  // pinned

    cudaGraphExec_t sweep_exec = nullptr;   // rounds of even sweeps
    cudaGraphExec_t sweep_exec2 = nullptr;  // rounds of odd sweeps
    cudaStream_t vstream = nullptr;         // the deferred V passes
    cudaEvent_t ev_rounds_done[2] = {}, ev_vpass_done[2] = {}, ev_v0[2] = {}, ev_v1[2] = {};
    // Event-record nodes inside the sweep graph: before the first round,
    // after the last round, after the V pass (live kernel timing).
    cudaEvent_t ev_round_begin = nullptr, ev_round_end = nullptr;

    PlainPlan() = default;
    ~PlainPlan();
    PlainPlan(const PlainPlan &) = delete;
    PlainPlan &operator=(const PlainPlan &) = delete;

    static int create(int dev, size_t m, size_t n, int T, double eps, cudaStream_t stream,
                      std::unique_ptr<PlainPlan> &out);
    int ensure_host_staging();
    int enqueue_rounds(cudaStream_t st, int parity);
    int enqueue_vpass(cudaStream_t st, int parity);
    int enqueue_persistent(cudaStream_t st, int parity, int g0);
    int capture_rounds(cudaStream_t st, int parity);
    // Runs the whole solve on device buffers; outputs may be null.  With
    // gram_stop and eps >= 1e-12, a sweep that rotated few pairs is followed
    // by a test of every pair on G = A^T A (one lower-triangle GEMM): when no pair would
    // rotate, the next sweep would change nothing and is not run (it is
    // counted in `sweeps`).  The
    // dot products then come from the GEMM, not the reference's reduction
    // tree, so results equal the default's only to working accuracy; the
    // bit-exact drop-in never sets it.
    int run(const double *d_a, double *out_u, double *out_sigma, double *out_v, int max_sweeps, int *sweeps,
            cudaStream_t stream, bool gram_stop = false);
    int gram_converged(cudaStream_t stream, bool &converged);
};

// Cumulative per-thread counters of the plain path (jsvd_plain_stats).
struct PlainStats {
    unsigned long long solves = 0, sweeps = 0, round_launches = 0, vpass_launches = 0, other_launches = 0;
    unsigned long long gram_checks = 0;  // Gram convergence tests (run option gram_stop)
    double round_ms = 0.0, vpass_ms = 0.0;
};
PlainStats &plain_stats();

// Process-wide choice of how a sweep is launched: 0 = one kernel per round,
// replayed from a CUDA graph, each CTA reducing the dot products and deriving
// the angle in one warp (the default), 1 = one persistent cooperative kernel
// per sweep, 2 = as 0 with programmatic dependent launch between rounds, 3 = as
// 0 with every warp deriving the angle itself (one barrier fewer).  Plans
// record the mode they were created with.
int sweep_mode();
void set_sweep_mode(int mode);

// The plain device-buffer solve (jsvd_plain_svd_device) with the run option
// gram_stop (see PlainPlan::run); for paths held to a tolerance.
int plain_device_solve(const double *d_a, size_t rows, size_t cols, const jsvd_config *cfg, double *d_u,
                       double *d_sigma, double *d_v, int *sweeps, cudaStream_t stream, bool gram_stop);

// Per-thread plan cache and stream.
int acquire_plain_plan(size_t m, size_t n, int T, double eps, cudaStream_t stream, PlainPlan **plan);
cudaStream_t thread_stream(int device);

// The stream a device-buffer entry point runs on: the caller's when it passed
// one, else the calling thread's library stream on the current device, made to
// wait (on the device, without blocking the host) for all work queued so far on
// the legacy default stream, where the caller's buffers were produced.
int entry_stream(void *caller_stream, cudaStream_t *out);

}  // namespace jsvd
