// QR-preconditioned one-sided Jacobi SVD (sm_100a): the fast path for tall
// and for ill-conditioned matrices.
//
//   1. A = Q R by shifted CholeskyQR3 (Fukaya, Kannan, Nakatsukasa, Yamamoto,
//      Yanagisawa, SIAM J. Sci. Comput. 2020): one Cholesky QR pass on
//      A^T A + s I, s = 11 (m n + n (n + 1)) u ||A||_F^2, then two plain passes
//      (CholeskyQR2).  Stable for kappa(A) up to about 1/u; Q orthogonal to
//      working precision.
//   2. One-sided Jacobi on X = R^T (n x n) with the plain sweep (same
//      arithmetic, same round-robin order).  For ill-conditioned A the columns
//      of R^T are graded and the sweep count drops (Drmac and Veselic, SIAM J.
//      Matrix Anal. Appl. 29, 2008); for tall A every round also moves m/n
//      times fewer bytes.
//   3. X V_x = U_x Sigma  =>  A = Q R = Q V_x Sigma U_x^T, so
//      V_A = U_x (normalised columns of the rotated X), U_A = Q V_x, Sigma_A =
//      Sigma_x (unsorted, in X's column order).
// Gram products and triangular updates run on this library's FP64 tensor-core
// GEMM (dgemm.cu); the Cholesky diagonal blocks, the triangular row solves,
// the shift and the layout kernels are written here.  If a Cholesky pivot is
// not positive the solve falls back to the plain path on A.
#include <cuda_runtime.h>

#include <atomic>

#include <algorithm>
#include <memory>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "blockpair.hpp"
#include "dgemm.hpp"
#include "internal.hpp"
#include "jsvd.h"
#include "layout.cuh"
#include "mixed.hpp"
#include "plain.hpp"

namespace jsvd {
namespace {

constexpr int kNb = 64;  // Cholesky / triangular block size

#define JSVD_GEMM_TRY(EXPR)                       \
    do {                                          \
        const int gemm_rc_ = (EXPR);              \
        if (gemm_rc_ != JSVD_OK) return gemm_rc_; \
    } while (0)

// row-major (rows x cols) -> column-major (ld = rows), one launch (the n x n
// factor; the m x n input goes through launch_rowmajor_to_colmajor)
__global__ void __launch_bounds__(kTile *kTileRows)
    pc_to_colmajor(const double *__restrict__ src, int rows, int cols, double *__restrict__ dst)
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
        if (r < rows && c < cols) dst[(size_t)c * rows + r] = tile[threadIdx.x][k];
    }
}

// G_ii += s with s = 11 (m n + n (n + 1)) u trace(G)   (one CTA)
__global__ void __launch_bounds__(256) pc_shift_diagonal(double *__restrict__ G, int n, int m)
{
    __shared__ double red[256];
    double acc = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) acc += G[(size_t)i * n + i];
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    const double u = 1.1102230246251565e-16;  // 2^-53
    const double shift = 11.0 * ((double)m * n + (double)n * (n + 1)) * u * red[0];
    for (int i = threadIdx.x; i < n; i += blockDim.x) G[(size_t)i * n + i] += shift;
}

// Cholesky of the kb x kb diagonal block at (k0, k0) of the lower triangle of
// G (column-major, ld = n) into the same block of Lm, and the inverse of that
// factor into Linv (column-major, ld = kNb).  The block is padded to kNb x kNb
// with the identity.
//
// The factor is computed as G = L D L^T (L unit lower): each column costs one
// reciprocal of its pivot on the serial chain, and the square roots are taken
// afterwards, all at once (Cholesky factor L sqrt(D), inverse
// D^{-1/2} L^{-1}, where L^{-1} needs no division).  Panels of kPanel columns:
//   factorisation: warp 0 factors the panel's columns (right-looking inside
//     the panel, __syncwarp between columns; each lane owns two rows and reads
//     the pivot column's panel entries before they are rescaled), then all
//     threads apply the panel's update to the trailing triangle,
//     a[i][k] -= sum_j L(i,j) d_j L(k,j);
//   inverse of L: block forward substitution of [L | I], kPanel rows at a
//     time: thread c solves column c through the panel's unit triangle, then
//     all threads subtract the panel's contribution from the rows below.
// A form with a square root and a reciprocal per column measured about 60 us
// per block on B200 (ncu), set by that serial chain of 64 pivots.
// status <- 1 on a pivot that is not positive and finite.
constexpr int kPanel = 8;
constexpr int kDiagThreads = 256;
constexpr size_t kDiagSmem = sizeof(double) * 2 * kNb * (kNb + 1);

__global__ void __launch_bounds__(kDiagThreads) pc_chol_inv_diag(const double *__restrict__ G,
                                                                 double *__restrict__ Lm, int n, int k0, int kb,
                                                                 double *__restrict__ Linv, int *__restrict__ status)
{
    extern __shared__ double dsm[];
    __shared__ double dvec[kNb];  // pivots d_i
    __shared__ double sq[kNb];    // sqrt(d_i)
    __shared__ double isq[kNb];   // 1 / sqrt(d_i)
    double(*a)[kNb + 1] = reinterpret_cast<double(*)[kNb + 1]>(dsm);
    double(*x)[kNb + 1] = reinterpret_cast<double(*)[kNb + 1]>(dsm + kNb * (kNb + 1));
    const int t = threadIdx.x;
    {
        // all of a thread's loads in flight before its stores
        constexpr int kPer = kNb * kNb / kDiagThreads;
        double g[kPer];
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int e = t + u * kDiagThreads;
            const int i = e % kNb, k = e / kNb;  // consecutive threads read consecutive rows of column k
            g[u] = (i < kb && k < kb) ? (i >= k ? G[(size_t)(k0 + k) * n + k0 + i] : 0.0) : (i == k ? 1.0 : 0.0);
        }
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int e = t + u * kDiagThreads;
            const int i = e % kNb, k = e / kNb;
            a[i][k] = g[u];
            x[i][k] = (i == k) ? 1.0 : 0.0;
        }
    }
    __syncthreads();
    // ---- G = L D L^T ----
    for (int c0 = 0; c0 < kNb; c0 += kPanel) {
        if (t < 32) {
            const int lane = t;
            for (int j = 0; j < kPanel; ++j) {
                const int cj = c0 + j;
                const double d0 = a[cj][cj];
                const bool ok = d0 > 0.0 && d0 < INFINITY;
                const double d = ok ? d0 : 1.0;
                // 1 / d by Newton's iteration r <- r (2 - d r) from the
                // single-precision reciprocal (2^-23 -> 2^-46 -> rounding),
                // by division outside the single-precision range
                double rd;
                if (d > 1.0e-30 && d < 1.0e30) {
                    rd = (double)__frcp_rn((float)d);
                    rd = rd * fma(-d, rd, 2.0);
                    rd = rd * fma(-d, rd, 2.0);
                } else {
                    rd = 1.0 / d;
                }
                if (lane == 0) {
                    if (!ok) atomicExch(status, 1);
                    dvec[cj] = d;
                }
                double colk[kPanel];  // a[k][cj] = L(k,cj) d_cj of the panel rows below cj
#pragma unroll
                for (int kk = 0; kk < kPanel; ++kk) colk[kk] = (kk > j) ? a[c0 + kk][cj] : 0.0;
                __syncwarp();
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const int i = c0 + lane + 32 * h;
                    if (i >= kNb || i <= cj) continue;
                    const double lij = a[i][cj] * rd;
                    a[i][cj] = lij;
#pragma unroll
                    for (int kk = 0; kk < kPanel; ++kk) {
                        const int k = c0 + kk;
                        if (kk > j && k <= i) a[i][k] = fma(-lij, colk[kk], a[i][k]);
                    }
                }
                __syncwarp();
            }
        }
        __syncthreads();
        const int base = c0 + kPanel, w = kNb - base;
        for (int e = t; e < w * w; e += kDiagThreads) {
            const int i = base + e / w, k = base + e % w;
            if (k > i) continue;
            double acc = a[i][k];
#pragma unroll
            for (int jj = 0; jj < kPanel; ++jj) acc = fma(-a[i][c0 + jj], a[k][c0 + jj] * dvec[c0 + jj], acc);
            a[i][k] = acc;
        }
        __syncthreads();
    }
    if (t < kNb) {
        sq[t] = sqrt(dvec[t]);
        isq[t] = 1.0 / sq[t];
    }
    // ---- L^{-1}: forward substitution of [L | I] (unit diagonal) ----
    for (int r0 = 0; r0 < kNb; r0 += kPanel) {
        const int cols = r0 + kPanel;  // columns 0 .. cols-1 can be non-zero in these rows
        if (t < cols) {
            const int c = t;
#pragma unroll
            for (int r = 0; r < kPanel; ++r) {
                const int i = r0 + r;
                double val = x[i][c];
#pragma unroll
                for (int rr = 0; rr < r; ++rr) val = fma(-a[i][r0 + rr], x[r0 + rr][c], val);
                x[i][c] = val;
            }
        }
        __syncthreads();
        const int below = kNb - cols;
        for (int e = t; e < below * cols; e += kDiagThreads) {
            const int i = cols + e / cols, c = e % cols;
            double acc = x[i][c];
#pragma unroll
            for (int r = 0; r < kPanel; ++r) acc = fma(-a[i][r0 + r], x[r0 + r][c], acc);
            x[i][c] = acc;
        }
        __syncthreads();
    }
    // Cholesky factor L sqrt(D) and its inverse D^{-1/2} L^{-1}
    for (int e = t; e < kb * kb; e += kDiagThreads) {
        const int i = e % kb, k = e / kb;
        if (i >= k) Lm[(size_t)(k0 + k) * n + k0 + i] = (i == k) ? sq[i] : a[i][k] * sq[k];
    }
    for (int e = t; e < kNb * kNb; e += kDiagThreads) {
        const int i = e % kNb, k = e / kNb;
        Linv[i + (size_t)k * kNb] = (i < kb && k < kb && k <= i) ? x[i][k] * isq[i] : 0.0;
    }
}

// R (upper, column-major n x n) = L^T with zeros below the diagonal.
__global__ void pc_lower_to_upper(const double *__restrict__ L, double *__restrict__ R, int n)
{
    const size_t total = (size_t)n * n;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const size_t i = e % n, j = e / n;  // R(i, j)
        R[e] = (i <= j) ? L[i * n + j] : 0.0;
    }
}

// One Cholesky QR pass: G = Q^T Q (+ shift), G = L L^T (blocked,
// right-looking; diagonal blocks factored and inverted by pc_chol_inv_diag,
// panels L21 = G21 L11^{-T} and trailing updates as GEMMs), then
// Qout = Q L^{-T} by a blocked right-looking solve (Qout_J = Q_J Linv_J^T,
// Q_{>J} -= Qout_J L_{>J,J}^T; Q is overwritten) and R = L^T.
int chol_qr_pass(cudaStream_t st, double *Q, double *Qout, int m, int n, double *G, double *Lm, double *Linv,
                 double *R, bool shift, int *d_status)
{
    JSVD_GEMM_TRY(dgemm(st, 'T', 'N', n, n, m, 1.0, Q, m, Q, m, 0.0, G, n, 1));
    if (shift) {
        pc_shift_diagonal<<<1, 256, 0, st>>>(G, n, m);
        JSVD_CUDA_TRY(cudaGetLastError());
    }
    for (int k0 = 0, blk = 0; k0 < n; k0 += kNb, ++blk) {
        const int kb = std::min(kNb, n - k0);
        double *li = Linv + (size_t)blk * kNb * kNb;
        pc_chol_inv_diag<<<1, kDiagThreads, kDiagSmem, st>>>(G, Lm, n, k0, kb, li, d_status);
        JSVD_CUDA_TRY(cudaGetLastError());
        const int rest = n - k0 - kb;
        if (rest > 0) {
            // L21 = G21 L11^{-T}
            JSVD_GEMM_TRY(dgemm(st, 'N', 'T', rest, kb, kb, 1.0, G + (size_t)k0 * n + k0 + kb, n, li, kNb, 0.0,
                                Lm + (size_t)k0 * n + k0 + kb, n));
            // G22 -= L21 L21^T (lower)
            JSVD_GEMM_TRY(dgemm(st, 'N', 'T', rest, rest, kb, -1.0, Lm + (size_t)k0 * n + k0 + kb, n,
                                Lm + (size_t)k0 * n + k0 + kb, n, 1.0, G + (size_t)(k0 + kb) * n + k0 + kb, n, 1));
        }
    }
    for (int j0 = 0, blk = 0; j0 < n; j0 += kNb, ++blk) {
        const int kb = std::min(kNb, n - j0);
        const double *li = Linv + (size_t)blk * kNb * kNb;
        JSVD_GEMM_TRY(
            dgemm(st, 'N', 'T', m, kb, kb, 1.0, Q + (size_t)j0 * m, m, li, kNb, 0.0, Qout + (size_t)j0 * m, m));
        const int rest = n - j0 - kb;
        if (rest > 0)
            JSVD_GEMM_TRY(dgemm(st, 'N', 'T', m, rest, kb, -1.0, Qout + (size_t)j0 * m, m, Lm + (size_t)j0 * n + j0 + kb,
                                n, 1.0, Q + (size_t)(j0 + kb) * m, m));
    }
    pc_lower_to_upper<<<std::min<size_t>(1184, ((size_t)n * n + 255) / 256), 256, 0, st>>>(Lm, R, n);
    JSVD_CUDA_TRY(cudaGetLastError());
    return JSVD_OK;
}

std::atomic<int> g_inner{1};
std::atomic<int> g_gram_stop{1};

// The Jacobi stage on X (row-major cols x cols): the plain sweep (default) or,
// when selected, the block-pair engine where it applies.  The plain sweep
// measured faster on B200 for the 1024-column factor of a 4096 x 1024 input
// (4.0 us per round, 1023 rounds per sweep, against 18 us per block-pair outer
// round, 255 per sweep).
// Engine 2 is the blocked mixed-precision sweep (mixed.cu), used by
// jsvd_mixed_svd*.
constexpr int kEngineMixed = 2;

int inner_jacobi(const double *x, size_t cols, const jsvd_config &c, double *u, double *sigma, double *v, int *sweeps,
                 cudaStream_t st, int engine)
{
    if (engine == kEngineMixed && cols >= (size_t)kMixedMinCols)
        return mixed_solve(x, (int)cols, (int)cols, c, mixed_options(), u, sigma, v, sweeps, st);
    if (engine == 0 && bp_supported(cols, cols))
        return bp_solve(x, cols, cols, c.epsilon, c.max_sweeps, u, sigma, v, sweeps, st);
    // The last, rotation-free sweep is replaced by a test of every pair on the
    // Gram matrix (this path is held to a tolerance, not to the bits).
    return plain_device_solve(x, cols, cols, &c, u, sigma, v, sweeps, st, g_gram_stop.load() != 0);
}

struct PrecondStats {
    unsigned long long solves = 0, fallbacks = 0;
    double qr_ms = 0.0, jacobi_ms = 0.0, u_ms = 0.0;
    int last_sweeps = 0;
};

PrecondStats &precond_stats()
{
    thread_local PrecondStats s;
    return s;
}

// Per-thread cached resources of the QR stage for one shape: the workspace,
// a stream for allocation and graph capture, and the two shifted CholeskyQR3
// stages captured as graphs on the plan's second use.  The stage is ~500 small
// launches whose enqueueing, not their device time, set its duration.
struct PcPlan {
    int device = -1;
    size_t m = 0, n = 0;
    double *ws = nullptr;
    cudaStream_t own = nullptr;
    cudaGraphExec_t qr1 = nullptr, qr2 = nullptr;
    bool no_graph = false;  // a capture failed: launch directly from then on
    unsigned long long uses = 0;
    ~PcPlan()
    {
        if (qr1) cudaGraphExecDestroy(qr1);
        if (qr2) cudaGraphExecDestroy(qr2);
        if (own) {
            if (ws) cudaFreeAsync(ws, own);
            cudaStreamSynchronize(own);
            cudaStreamDestroy(own);
        }
    }
};

constexpr size_t kPcMaxPlanBytes = size_t(2) << 30;  // larger shapes allocate per call, no graphs
constexpr size_t kPcMaxPlans = 2;

std::vector<std::unique_ptr<PcPlan>> &pc_plans()
{
    thread_local std::vector<std::unique_ptr<PcPlan>> plans;
    return plans;
}

// The cached plan for (device, m, n), created on first use; nullptr (and
// JSVD_OK) when the shape's workspace is above kPcMaxPlanBytes.
int acquire_pc_plan(int dev, size_t m, size_t n, size_t ws_doubles, PcPlan **out)
{
    *out = nullptr;
    if (sizeof(double) * ws_doubles > kPcMaxPlanBytes) return JSVD_OK;
    auto &plans = pc_plans();
    for (size_t i = 0; i < plans.size(); ++i) {
        if (plans[i]->device == dev && plans[i]->m == m && plans[i]->n == n) {
            std::rotate(plans.begin(), plans.begin() + i, plans.begin() + i + 1);
            *out = plans.front().get();
            return JSVD_OK;
        }
    }
    auto p = std::make_unique<PcPlan>();
    p->device = dev;
    p->m = m;
    p->n = n;
    {
        const cudaError_t e = cudaStreamCreateWithFlags(&p->own, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            p->own = nullptr;
            return cuda_failure(e, "cudaStreamCreateWithFlags", __FILE__, __LINE__);
        }
    }
    JSVD_CUDA_TRY(cudaMallocAsync((void **)&p->ws, sizeof(double) * ws_doubles, p->own));
    JSVD_CUDA_TRY(cudaStreamSynchronize(p->own));
    JSVD_CUDA_TRY(cudaFuncSetAttribute(pc_chol_inv_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDiagSmem));
    plans.insert(plans.begin(), std::move(p));
    while (plans.size() > kPcMaxPlans) plans.pop_back();
    *out = plans.front().get();
    return JSVD_OK;
}

int precond_impl(const double *d_a, size_t rows, size_t cols, const jsvd_config &c, double *d_u, double *d_sigma,
                 double *d_v, int *sweeps, cudaStream_t st, int engine)
{
    const int m = (int)rows, n = (int)cols;
    int dev = 0;
    JSVD_CUDA_TRY(cudaGetDevice(&dev));
    const size_t mn = (size_t)m * n, nn = (size_t)n * n;
    // workspace: Qa, Qb (m x n) | G | Lm | R1 | R2 | R3 | T | Vx | Ux | Sa | Sb | P1 (n x n)
    //            | Linv (blocks x 64 x 64) | sigma | status
    const int nblk = (n + kNb - 1) / kNb;
    const size_t ws_doubles = 2 * mn + 11 * nn + (size_t)nblk * kNb * kNb + n + 1;
    PcPlan *plan = nullptr;
    int rc = acquire_pc_plan(dev, rows, cols, ws_doubles, &plan);
    if (rc != JSVD_OK) return rc;
    JSVD_CUDA_TRY(cudaFuncSetAttribute(pc_chol_inv_diag, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDiagSmem));
    double *ws = plan ? plan->ws : nullptr;
    if (!plan) JSVD_CUDA_TRY(cudaMallocAsync((void **)&ws, sizeof(double) * ws_doubles, st));
    double *Qa = ws, *Qb = Qa + mn, *G = Qb + mn, *Lm = G + nn, *R1 = Lm + nn, *R2 = R1 + nn, *R3 = R2 + nn,
           *Tm = R3 + nn, *Vx = Tm + nn, *Ux = Vx + nn, *Sa = Ux + nn, *Sb = Sa + nn, *P1 = Sb + nn,
           *Linv = P1 + nn, *sg = Linv + (size_t)nblk * kNb * kNb;
    int *d_status = reinterpret_cast<int *>(sg + n);
    double *Q = Qb;   // after three passes (Qa -> Qb -> Qa -> Qb) the factor is in Qb
    double *Q1 = Sb;  // likewise for the second factorisation (Sa -> Sb -> Sa -> Sb)
    cudaEvent_t e0, e1, e2, e3;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    cudaEventCreate(&e3);
    bool cleaned = false;
    auto cleanup = [&]() {
        if (cleaned) return;
        cleaned = true;
        if (!plan) cudaFreeAsync(ws, st);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaEventDestroy(e2);
        cudaEventDestroy(e3);
    };
    // every return below, the early ones of the status macros included, releases them
    ScopeExit guard([&] { cleanup(); });
    // Shifted CholeskyQR3 of Xa (rows x n, column-major, overwritten): the
    // orthonormal factor ends in Xb, R = R3 R2 R1 in Ra (upper, column-major);
    // Rb, Rc are scratch.
    auto scqr3 = [&](cudaStream_t s2, double *Xa, double *Xb, int rows, double *Ra, double *Rb, double *Rc) -> int {
        int r = chol_qr_pass(s2, Xa, Xb, rows, n, G, Lm, Linv, Ra, true, d_status);
        if (r == JSVD_OK) r = chol_qr_pass(s2, Xb, Xa, rows, n, G, Lm, Linv, Rb, false, d_status);
        if (r == JSVD_OK) r = chol_qr_pass(s2, Xa, Xb, rows, n, G, Lm, Linv, Rc, false, d_status);
        if (r != JSVD_OK) return r;
        JSVD_GEMM_TRY(dgemm(s2, 'N', 'N', n, n, n, 1.0, Rb, n, Ra, n, 0.0, Tm, n));
        JSVD_GEMM_TRY(dgemm(s2, 'N', 'N', n, n, n, 1.0, Rc, n, Tm, n, 0.0, Ra, n));
        return JSVD_OK;
    };
    // Runs a QR stage: directly, or (a plan on its second use onwards) as a
    // graph captured once on the plan's own stream and replayed on st.
    auto run_stage = [&](cudaGraphExec_t *exec, auto &&enqueue) -> int {
        if (plan && !plan->no_graph && *exec == nullptr && plan->uses >= 1) {
            cudaGraph_t graph = nullptr;
            int r = JSVD_OK;
            cudaError_t ce = cudaStreamBeginCapture(plan->own, cudaStreamCaptureModeThreadLocal);
            if (ce == cudaSuccess) {
                r = enqueue(plan->own);
                ce = cudaStreamEndCapture(plan->own, &graph);
            }
            if (r == JSVD_OK && ce == cudaSuccess && graph != nullptr) {
                if (cudaGraphInstantiate(exec, graph, 0) != cudaSuccess) *exec = nullptr;
            }
            if (graph) cudaGraphDestroy(graph);
            if (*exec == nullptr) {
                plan->no_graph = true;  // launch directly from now on
                cudaGetLastError();
                set_last_error(JSVD_OK, "");
            }
        }
        if (plan && *exec != nullptr) {
            JSVD_CUDA_TRY(cudaGraphLaunch(*exec, st));
            return JSVD_OK;
        }
        return enqueue(st);
    };
    auto read_status = [&](int *out) -> int {
        JSVD_CUDA_TRY(cudaMemcpyAsync(out, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
        JSVD_CUDA_TRY(cudaStreamSynchronize(st));
        return JSVD_OK;
    };
    cudaEventRecord(e0, st);
    JSVD_CUDA_TRY(cudaMemsetAsync(d_status, 0, sizeof(int), st));
    JSVD_CUDA_TRY(launch_rowmajor_to_colmajor(d_a, m, n, Qa, m, st));
    // A = Q R
    rc = run_stage(plan ? &plan->qr1 : nullptr,
                   [&](cudaStream_t s2) { return scqr3(s2, Qa, Qb, m, R1, R2, R3); });
    int status = 0;
    if (rc == JSVD_OK) rc = read_status(&status);
    if (rc != JSVD_OK) {
        cleanup();
        return rc;
    }
    PrecondStats &ps = precond_stats();
    if (status != 0) {
        // Gram not positive definite in floating point: plain path on A.
        cudaEventRecord(e1, st);
        cleanup();
        ps.fallbacks += 1;
        if (engine == kEngineMixed) mixed_note_solve(0.0, true);
        return jsvd_plain_svd_device(d_a, rows, cols, &c, d_u, d_sigma, d_v, sweeps, st);
    }
    // R^T = Q1 P (P upper): R1's column-major buffer read as row-major is R^T.
    rc = run_stage(plan ? &plan->qr2 : nullptr, [&](cudaStream_t s2) -> int {
        pc_to_colmajor<<<dim3((n + kTile - 1) / kTile, (n + kTile - 1) / kTile), dim3(kTile, kTileRows), 0, s2>>>(
            R1, n, n, Sa);
        JSVD_CUDA_TRY(cudaGetLastError());
        return scqr3(s2, Sa, Sb, n, P1, R2, R3);
    });
    int status2 = 0;
    if (rc == JSVD_OK) rc = read_status(&status2);
    if (rc != JSVD_OK) {
        cleanup();
        return rc;
    }
    cudaEventRecord(e1, st);
    double *sout = d_sigma ? d_sigma : sg;
    if (status2 == 0) {
        // A = Q R = Q P^T Q1^T.  Jacobi on X = P^T (P1's column-major buffer read
        // as row-major): X = Ux S Vx^T, so U_A = Q Ux and V_A = Q1 Vx.
        rc = inner_jacobi(P1, cols, c, d_u ? Ux : nullptr, sout, d_v ? Vx : nullptr, sweeps, st, engine);
        if (rc != JSVD_OK) {
            cleanup();
            return rc;
        }
        cudaEventRecord(e2, st);
        // Row-major U_A (m x n) is column-major U_A^T = Ux^T Q^T; Ux's row-major
        // buffer is Ux^T column-major.  The same for V_A^T = Vx^T Q1^T.
        if (d_u)
            JSVD_GEMM_TRY(dgemm(st, 'N', 'T', n, m, n, 1.0, Ux, n, Q, m, 0.0, d_u, n));
        if (d_v)
            JSVD_GEMM_TRY(dgemm(st, 'N', 'T', n, n, n, 1.0, Vx, n, Q1, n, 0.0, d_v, n));
    } else {
        // Second factorisation failed: Jacobi on X = R^T, A = Q X^T =
        // (Q Vx) S Ux^T, so U_A = Q Vx and V_A = Ux.
        ps.fallbacks += 1;
        double *vout = d_v ? d_v : Ux;
        rc = inner_jacobi(R1, cols, c, vout, sout, Vx, sweeps, st, engine);
        if (rc != JSVD_OK) {
            cleanup();
            return rc;
        }
        cudaEventRecord(e2, st);
        if (d_u)
            JSVD_GEMM_TRY(dgemm(st, 'N', 'T', n, m, n, 1.0, Vx, n, Q, m, 0.0, d_u, n));
    }
    cudaEventRecord(e3, st);
    JSVD_CUDA_TRY(cudaStreamSynchronize(st));
    float a = 0, b = 0, d = 0;
    cudaEventElapsedTime(&a, e0, e1);
    cudaEventElapsedTime(&b, e1, e2);
    cudaEventElapsedTime(&d, e2, e3);
    ps.solves += 1;
    ps.qr_ms += a;
    ps.jacobi_ms += b;
    ps.u_ms += d;
    ps.last_sweeps = sweeps ? *sweeps : 0;
    if (engine == kEngineMixed) mixed_note_solve(a, status2 != 0);
    if (plan) plan->uses += 1;
    cleanup();
    return JSVD_OK;
}

}  // namespace
}  // namespace jsvd

using namespace jsvd;

extern "C" int jsvd_precond_svd_device(const double *d_a, size_t rows, size_t columns, const jsvd_config *cfg,
                                       double *d_u, double *d_sigma, double *d_v, int *sweeps, void *stream)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        jsvd_config def;
        const jsvd_config &c = config_or_default(cfg, def);
        int rc = validate_plain_request(d_a, rows, columns, c);
        if (rc != JSVD_OK) return rc;
        cudaStream_t st = nullptr;
        if (const int e = entry_stream(stream, &st); e != JSVD_OK) return e;
        if (columns == 1) return jsvd_plain_svd_device(d_a, rows, columns, &c, d_u, d_sigma, d_v, sweeps, st);
        return precond_impl(d_a, rows, columns, c, d_u, d_sigma, d_v, sweeps, st, g_inner.load());
    });
}

extern "C" int jsvd_precond_svd(const double *a, size_t rows, size_t columns, const jsvd_config *cfg, double *u,
                                double *sigma, double *v, int *sweeps)
{
    return c_entry([&]() -> int {
        return host_buffer_solve(jsvd_precond_svd_device, a, rows, columns, cfg, u, sigma, v, sweeps);
    });
}

namespace jsvd {
void pc_release_thread_plans() { pc_plans().clear(); }
}  // namespace jsvd

extern "C" int jsvd_mixed_svd_device(const double *d_a, size_t rows, size_t columns, const jsvd_config *cfg,
                                     double *d_u, double *d_sigma, double *d_v, int *sweeps, void *stream)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        jsvd_config def;
        const jsvd_config &c = config_or_default(cfg, def);
        int rc = validate_plain_request(d_a, rows, columns, c);
        if (rc != JSVD_OK) return rc;
        cudaStream_t st = nullptr;
        if (const int e = entry_stream(stream, &st); e != JSVD_OK) return e;
        if (columns == 1) return jsvd_plain_svd_device(d_a, rows, columns, &c, d_u, d_sigma, d_v, sweeps, st);
        const jsvd_mixed_options &o = mixed_options();
        if (!o.precondition && columns >= (size_t)kMixedMinCols) {
            // the blocked sweeps directly on A (row tiles of 32 along the
            // transpose grid's y dimension bound the rows)
            if (rows > (size_t)65535 * 32)
                return invalid_argument("jsvd_mixed_svd: too many rows for the unpreconditioned blocked sweep.");
            rc = mixed_solve(d_a, (int)rows, (int)columns, c, o, d_u, d_sigma, d_v, sweeps, st);
            if (rc == JSVD_OK) mixed_note_solve(0.0, false);
            return rc;
        }
        return precond_impl(d_a, rows, columns, c, d_u, d_sigma, d_v, sweeps, st, kEngineMixed);
    });
}

extern "C" int jsvd_mixed_svd(const double *a, size_t rows, size_t columns, const jsvd_config *cfg, double *u,
                              double *sigma, double *v, int *sweeps)
{
    return c_entry([&]() -> int {
        return host_buffer_solve(jsvd_mixed_svd_device, a, rows, columns, cfg, u, sigma, v, sweeps);
    });
}

extern "C" void jsvd_precond_set_inner(int engine) { g_inner.store(engine == 0 ? 0 : 1); }

extern "C" void jsvd_precond_set_gram_stop(int enable) { g_gram_stop.store(enable ? 1 : 0); }

extern "C" void jsvd_precond_stats_get(jsvd_precond_stats *out)
{
    if (!out) return;
    const PrecondStats &s = precond_stats();
    out->solves = s.solves;
    out->fallbacks = s.fallbacks;
    out->qr_ms = s.qr_ms;
    out->jacobi_ms = s.jacobi_ms;
    out->u_ms = s.u_ms;
}

extern "C" void jsvd_precond_stats_reset(void) { precond_stats() = PrecondStats{}; }
