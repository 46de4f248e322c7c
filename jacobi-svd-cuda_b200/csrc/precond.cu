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
// Gram products and triangular updates are plain DGEMM/DSYRK calls (cuBLAS);
// the Cholesky diagonal blocks, the triangular row solves, the shift and the
// layout kernels are written here.  If a Cholesky pivot is not positive the
// solve falls back to the plain path on A.
#include <cublas_v2.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "internal.hpp"
#include "jsvd.h"
#include "plain.hpp"

namespace jsvd {
namespace {

constexpr int kNb = 64;  // Cholesky / triangular block size

const char *cublas_name(cublasStatus_t s)
{
    switch (s) {
    case CUBLAS_STATUS_SUCCESS: return "CUBLAS_STATUS_SUCCESS";
    case CUBLAS_STATUS_NOT_INITIALIZED: return "CUBLAS_STATUS_NOT_INITIALIZED";
    case CUBLAS_STATUS_ALLOC_FAILED: return "CUBLAS_STATUS_ALLOC_FAILED";
    case CUBLAS_STATUS_INVALID_VALUE: return "CUBLAS_STATUS_INVALID_VALUE";
    case CUBLAS_STATUS_EXECUTION_FAILED: return "CUBLAS_STATUS_EXECUTION_FAILED";
    default: return "CUBLAS error";
    }
}

int cublas_failure(cublasStatus_t s, const char *expr, const char *file, int line)
{
    set_last_error(JSVD_ERR_CUDA, std::string("cuBLAS call failed: ") + expr + " @ " + file + ":" +
                                      std::to_string(line) + ", status=" + cublas_name(s));
    return JSVD_ERR_CUDA;
}

#define JSVD_CUBLAS_TRY(EXPR)                                                              \
    do {                                                                                   \
        cublasStatus_t st_ = (EXPR);                                                       \
        if (st_ != CUBLAS_STATUS_SUCCESS) return cublas_failure(st_, #EXPR, __FILE__, __LINE__); \
    } while (0)

constexpr int kTile = 32, kTileRows = 8;

// row-major (rows x cols) -> column-major (ld = rows)
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

// In-place Cholesky of the kb x kb diagonal block at (k0, k0) of the lower
// triangle of G (column-major, ld = n), one CTA; status <- 1 on a pivot that
// is not positive and finite.
__global__ void __launch_bounds__(256) pc_chol_diag(double *__restrict__ G, int n, int k0, int kb,
                                                    int *__restrict__ status)
{
    __shared__ double a[kNb][kNb + 1];
    const int tid = threadIdx.x;
    for (int e = tid; e < kb * kb; e += blockDim.x) {
        const int i = e % kb, j = e / kb;
        a[i][j] = (i >= j) ? G[(size_t)(k0 + j) * n + k0 + i] : 0.0;
    }
    __syncthreads();
    for (int j = 0; j < kb; ++j) {
        const double d = a[j][j];
        const bool ok = d > 0.0 && d < INFINITY;
        const double r = ok ? sqrt(d) : 1.0;
        __syncthreads();
        if (tid == 0) {
            a[j][j] = r;
            if (!ok) atomicExch(status, 1);
        }
        for (int i = j + 1 + tid; i < kb; i += blockDim.x) a[i][j] /= r;
        __syncthreads();
        // trailing update of the lower triangle
        const int t = kb - j - 1;
        for (int e = tid; e < t * t; e += blockDim.x) {
            const int i = j + 1 + e % t, k = j + 1 + e / t;
            if (i >= k) a[i][k] = fma(-a[i][j], a[k][j], a[i][k]);
        }
        __syncthreads();
    }
    for (int e = tid; e < kb * kb; e += blockDim.x) {
        const int i = e % kb, j = e / kb;
        if (i >= j) G[(size_t)(k0 + j) * n + k0 + i] = a[i][j];
    }
}

// Forward substitution on rows: for every row r of B (column-major, ld = ldb,
// columns [c0, c0 + kb)), solve x L^T = b with L the kb x kb lower block at
// (l0, l0) of Lm (column-major, ld = ldl):  x_j = (b_j - sum_{l<j} x_l L_jl) / L_jj.
// Dynamic shared memory: the block of L, then the solved x of each thread.
constexpr int kTrsmThreads = 64;
constexpr size_t kTrsmSmem = sizeof(double) * (kNb * (kNb + 1) + kNb * kTrsmThreads);

__global__ void __launch_bounds__(kTrsmThreads) pc_trsm_rows(double *__restrict__ B, long ldb, int rows, int c0,
                                                             const double *__restrict__ Lm, long ldl, int l0, int kb)
{
    extern __shared__ double dsm[];
    double(*L)[kNb + 1] = reinterpret_cast<double(*)[kNb + 1]>(dsm);
    double(*xs)[kTrsmThreads] = reinterpret_cast<double(*)[kTrsmThreads]>(dsm + kNb * (kNb + 1));
    for (int e = threadIdx.x; e < kb * kb; e += blockDim.x) {
        const int i = e % kb, j = e / kb;
        L[i][j] = (i >= j) ? Lm[(size_t)(l0 + j) * ldl + l0 + i] : 0.0;
    }
    __syncthreads();
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= rows) return;
    for (int j = 0; j < kb; ++j) {
        double acc = B[(size_t)(c0 + j) * ldb + r];
        for (int l = 0; l < j; ++l) acc = fma(-xs[l][threadIdx.x], L[j][l], acc);
        const double x = acc / L[j][j];
        xs[j][threadIdx.x] = x;
        B[(size_t)(c0 + j) * ldb + r] = x;
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

struct CublasHandle {
    cublasHandle_t h = nullptr;
    int device = -1;
    ~CublasHandle()
    {
        if (h) cublasDestroy(h);
    }
};

int thread_cublas(int dev, cudaStream_t st, cublasHandle_t *out)
{
    thread_local CublasHandle ch;
    if (ch.h == nullptr || ch.device != dev) {
        if (ch.h) cublasDestroy(ch.h);
        ch.h = nullptr;
        JSVD_CUBLAS_TRY(cublasCreate(&ch.h));
        ch.device = dev;
    }
    JSVD_CUBLAS_TRY(cublasSetStream(ch.h, st));
    *out = ch.h;
    return JSVD_OK;
}

// One Cholesky QR pass on Q (m x n column-major, in place): G = Q^T Q (+ shift),
// G = L L^T, Q <- Q L^{-T}, R = L^T.  G is n x n scratch.
int chol_qr_pass(cublasHandle_t hb, cudaStream_t st, double *Q, int m, int n, double *G, double *R, bool shift,
                 int *d_status)
{
    const double one = 1.0, zero = 0.0, mone = -1.0;
    JSVD_CUDA_TRY(cudaFuncSetAttribute(pc_trsm_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsmSmem));
    JSVD_CUBLAS_TRY(cublasDsyrk(hb, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_T, n, m, &one, Q, m, &zero, G, n));
    if (shift) {
        pc_shift_diagonal<<<1, 256, 0, st>>>(G, n, m);
        JSVD_CUDA_TRY(cudaGetLastError());
    }
    // Blocked right-looking Cholesky (lower).
    for (int k0 = 0; k0 < n; k0 += kNb) {
        const int kb = std::min(kNb, n - k0);
        pc_chol_diag<<<1, 256, 0, st>>>(G, n, k0, kb, d_status);
        JSVD_CUDA_TRY(cudaGetLastError());
        const int rest = n - k0 - kb;
        if (rest > 0) {
            // L21 = G21 L11^{-T}: rows of G below the block, columns [k0, k0+kb)
            pc_trsm_rows<<<(rest + kTrsmThreads - 1) / kTrsmThreads, kTrsmThreads, kTrsmSmem, st>>>(
                G + (k0 + kb), n, rest, k0, G, n, k0, kb);
            JSVD_CUDA_TRY(cudaGetLastError());
            // G22 -= L21 L21^T (lower)
            JSVD_CUBLAS_TRY(cublasDsyrk(hb, CUBLAS_FILL_MODE_LOWER, CUBLAS_OP_N, rest, kb, &mone,
                                        G + (size_t)k0 * n + (k0 + kb), n, &one,
                                        G + (size_t)(k0 + kb) * n + (k0 + kb), n));
        }
    }
    // Q <- Q L^{-T}: blocked right-looking over column blocks.
    for (int j0 = 0; j0 < n; j0 += kNb) {
        const int kb = std::min(kNb, n - j0);
        pc_trsm_rows<<<(m + kTrsmThreads - 1) / kTrsmThreads, kTrsmThreads, kTrsmSmem, st>>>(Q, m, m, j0, G, n,
                                                                                              j0, kb);
        JSVD_CUDA_TRY(cudaGetLastError());
        const int rest = n - j0 - kb;
        if (rest > 0) {
            // Q[:, j0+kb:] -= Q[:, j0:j0+kb] * L[j0+kb:, j0:j0+kb]^T
            JSVD_CUBLAS_TRY(cublasDgemm(hb, CUBLAS_OP_N, CUBLAS_OP_T, m, rest, kb, &mone, Q + (size_t)j0 * m, m,
                                        G + (size_t)j0 * n + (j0 + kb), n, &one, Q + (size_t)(j0 + kb) * m, m));
        }
    }
    pc_lower_to_upper<<<std::min<size_t>(1184, ((size_t)n * n + 255) / 256), 256, 0, st>>>(G, R, n);
    JSVD_CUDA_TRY(cudaGetLastError());
    return JSVD_OK;
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

int precond_impl(const double *d_a, size_t rows, size_t cols, const jsvd_config &c, double *d_u, double *d_sigma,
                 double *d_v, int *sweeps, cudaStream_t st)
{
    const int m = (int)rows, n = (int)cols;
    int dev = 0;
    JSVD_CUDA_TRY(cudaGetDevice(&dev));
    cublasHandle_t hb = nullptr;
    int rc = thread_cublas(dev, st, &hb);
    if (rc != JSVD_OK) return rc;
    const size_t mn = (size_t)m * n, nn = (size_t)n * n;
    // workspace: Q (m x n) | G | R1 | R2 | R3 | T | Vx (n x n each) | Ux (if the caller skips V) | sigma | status
    double *ws = nullptr;
    const size_t ws_doubles = mn + 7 * nn + n + 1;
    JSVD_CUDA_TRY(cudaMallocAsync((void **)&ws, sizeof(double) * ws_doubles, st));
    double *Q = ws, *G = Q + mn, *R1 = G + nn, *R2 = R1 + nn, *R3 = R2 + nn, *Tm = R3 + nn, *Vx = Tm + nn,
           *Ux = Vx + nn, *sg = Ux + nn;
    int *d_status = reinterpret_cast<int *>(sg + n);
    cudaEvent_t e0, e1, e2, e3;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    cudaEventCreate(&e3);
    auto cleanup = [&]() {
        cudaFreeAsync(ws, st);
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
        cudaEventDestroy(e2);
        cudaEventDestroy(e3);
    };
    cudaEventRecord(e0, st);
    JSVD_CUDA_TRY(cudaMemsetAsync(d_status, 0, sizeof(int), st));
    pc_to_colmajor<<<dim3((n + kTile - 1) / kTile, (m + kTile - 1) / kTile), dim3(kTile, kTileRows), 0, st>>>(
        d_a, m, n, Q);
    JSVD_CUDA_TRY(cudaGetLastError());
    rc = chol_qr_pass(hb, st, Q, m, n, G, R1, true, d_status);
    if (rc == JSVD_OK) rc = chol_qr_pass(hb, st, Q, m, n, G, R2, false, d_status);
    if (rc == JSVD_OK) rc = chol_qr_pass(hb, st, Q, m, n, G, R3, false, d_status);
    if (rc != JSVD_OK) {
        cleanup();
        return rc;
    }
    const double one = 1.0, zero = 0.0;
    // R = R3 R2 R1  (upper)
    JSVD_CUBLAS_TRY(cublasDgemm(hb, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, R2, n, R1, n, &zero, Tm, n));
    JSVD_CUBLAS_TRY(cublasDgemm(hb, CUBLAS_OP_N, CUBLAS_OP_N, n, n, n, &one, R3, n, Tm, n, &zero, R1, n));
    int status = 0;
    JSVD_CUDA_TRY(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    JSVD_CUDA_TRY(cudaStreamSynchronize(st));
    cudaEventRecord(e1, st);
    PrecondStats &ps = precond_stats();
    if (status != 0) {
        // Gram not positive definite in floating point: plain path on A.
        cleanup();
        ps.fallbacks += 1;
        return jsvd_plain_svd_device(d_a, rows, cols, &c, d_u, d_sigma, d_v, sweeps, st);
    }
    // Jacobi on X = R^T: R's column-major buffer read as row-major is R^T.
    double *vout = d_v ? d_v : Ux;  // V_A = U_x
    double *sout = d_sigma ? d_sigma : sg;
    rc = jsvd_plain_svd_device(R1, cols, cols, &c, vout, sout, Vx, sweeps, st);
    if (rc != JSVD_OK) {
        cleanup();
        return rc;
    }
    cudaEventRecord(e2, st);
    if (d_u) {
        // U_A (row-major m x n) = Q V_x; as column-major it is (Q V_x)^T = V_x^T Q^T,
        // and V_x's row-major buffer is V_x^T column-major.
        JSVD_CUBLAS_TRY(cublasDgemm(hb, CUBLAS_OP_N, CUBLAS_OP_T, n, m, n, &one, Vx, n, Q, m, &zero, d_u, n));
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
    cleanup();
    return JSVD_OK;
}

}  // namespace
}  // namespace jsvd

using namespace jsvd;

extern "C" int jsvd_precond_svd_device(const double *d_a, size_t rows, size_t columns, const jsvd_config *cfg,
                                       double *d_u, double *d_sigma, double *d_v, int *sweeps, void *stream)
{
    set_last_error(JSVD_OK, "");
    jsvd_config def;
    jsvd_config_default(&def);
    const jsvd_config &c = cfg ? *cfg : def;
    int rc = validate_plain_request(d_a, rows, columns, c);
    if (rc != JSVD_OK) return rc;
    int dev = 0;
    JSVD_CUDA_TRY(cudaGetDevice(&dev));
    cudaStream_t st = (cudaStream_t)stream;
    if (st == nullptr) {
        st = thread_stream(dev);
        if (st == nullptr) return cuda_failure(cudaGetLastError(), "cudaStreamCreateWithFlags", __FILE__, __LINE__);
        JSVD_CUDA_TRY(cudaStreamSynchronize(cudaStreamLegacy));
    }
    if (columns == 1) return jsvd_plain_svd_device(d_a, rows, columns, &c, d_u, d_sigma, d_v, sweeps, st);
    return precond_impl(d_a, rows, columns, c, d_u, d_sigma, d_v, sweeps, st);
}

extern "C" int jsvd_precond_svd(const double *a, size_t rows, size_t columns, const jsvd_config *cfg, double *u,
                                double *sigma, double *v, int *sweeps)
{
    set_last_error(JSVD_OK, "");
    jsvd_config def;
    jsvd_config_default(&def);
    const jsvd_config &c = cfg ? *cfg : def;
    int rc = validate_plain_request(a, rows, columns, c);
    if (rc != JSVD_OK) return rc;
    int dev = 0;
    JSVD_CUDA_TRY(cudaGetDevice(&dev));
    cudaStream_t st = thread_stream(dev);
    if (st == nullptr) return cuda_failure(cudaGetLastError(), "cudaStreamCreateWithFlags", __FILE__, __LINE__);
    const size_t mn = rows * columns, nn = columns * columns;
    double *d = nullptr;
    JSVD_CUDA_TRY(cudaMallocAsync((void **)&d, sizeof(double) * (2 * mn + nn + columns), st));
    double *da = d, *du = d + mn, *dv = du + mn, *ds = dv + nn;
    JSVD_CUDA_TRY(cudaMemcpyAsync(da, a, sizeof(double) * mn, cudaMemcpyHostToDevice, st));
    rc = jsvd_precond_svd_device(da, rows, columns, &c, u ? du : nullptr, ds, v ? dv : nullptr, sweeps, st);
    if (rc == JSVD_OK) {
        if (u) JSVD_CUDA_TRY(cudaMemcpyAsync(u, du, sizeof(double) * mn, cudaMemcpyDeviceToHost, st));
        if (sigma) JSVD_CUDA_TRY(cudaMemcpyAsync(sigma, ds, sizeof(double) * columns, cudaMemcpyDeviceToHost, st));
        if (v) JSVD_CUDA_TRY(cudaMemcpyAsync(v, dv, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    }
    cudaFreeAsync(d, st);
    JSVD_CUDA_TRY(cudaStreamSynchronize(st));
    return rc;
}

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
