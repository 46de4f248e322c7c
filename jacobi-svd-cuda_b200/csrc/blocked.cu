// Blocked one-sided Jacobi SVD in FP64 (sm_100a).
//
// Columns are grouped into blocks of b; a sweep pairs the blocks with the same
// fixed-head circle schedule the plain path uses for columns (reference
// src/kernels.cu:637-678, applied to blocks).  For a block pair (I, J) with
// panel P = [X_I X_J] (w = |I| + |J| <= 2b columns):
//   1. Gram   G = P^T P, split over row chunks (one CTA per chunk, partial
//              Grams summed in a fixed order -> deterministic);
//   2. solve  if some column pair of P fails the reference's orthogonality test
//              |g_pq| <= eps sqrt(g_pp g_qq), a cyclic two-sided Jacobi on G in
//              shared memory accumulates the orthogonal W (at most kInnerSweeps
//              inner sweeps; the outer sweeps finish the job);
//   3. apply  P <- P W and V_(I,J) <- V_(I,J) W, row chunk by row chunk, in
//              place.
// The sweep stops when no panel needed a rotation.  All arithmetic is FP64, so
// the convergence test is the plain path's and the result is accurate to
// working precision (normwise); it is not bit-identical to the plain path.
// A block round is three launches instead of b column rounds; a sweep has
// about n/b block rounds instead of n column rounds.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "blocked.hpp"
#include "internal.hpp"
#include "jsvd.h"
#include "plain.hpp"

namespace jsvd {
namespace {

constexpr int kB = 32;          // columns per block
constexpr int kW = 2 * kB;      // panel width
constexpr int kRC = 128;        // rows per chunk (Gram and apply)
constexpr int kInnerSweeps = 2; // two-sided sweeps per panel solve
constexpr int kThreads = 256;

// Block pair k of block round r (closed-form fixed-head circle over nb blocks).
__device__ __forceinline__ int2 block_pair(int nb, int r, int k)
{
    const int ne = nb + (nb & 1);
    const int L = ne - 1;
    int i = k;
    if (nb & 1) {
        const int j = 1 + ((nb - 1 + r) % L);
        const int slot = j < ne / 2 ? j : ne - 1 - j;
        if (i >= slot) i += 1;
    }
    const int i2 = ne - 1 - i;
    const int p = i == 0 ? 0 : 1 + ((i - 1 - r) % L + L) % L;
    const int q = 1 + ((i2 - 1 - r) % L + L) % L;
    return make_int2(p, q);
}

struct Panel {
    int c0, w0, c1, w1;  // first column and width of each block
    __device__ __forceinline__ int col(int j) const { return j < w0 ? c0 + j : c1 + (j - w0); }
    __device__ __forceinline__ int width() const { return w0 + w1; }
};

__device__ __forceinline__ Panel make_panel(int n, int nb, int r, int k)
{
    const int2 ij = block_pair(nb, r, k);
    Panel p;
    p.c0 = ij.x * kB;
    p.w0 = min(kB, n - p.c0);
    p.c1 = ij.y * kB;
    p.w1 = min(kB, n - p.c1);
    return p;
}

// 1. Partial Grams: blockIdx.x = block pair, blockIdx.y = row chunk of X.
constexpr size_t kGramSmem = sizeof(double) * kRC * (kW + 1);
constexpr size_t kSolveSmem = sizeof(double) * 2 * kW * (kW + 1);
constexpr size_t kApplySmem = sizeof(double) * (kRC + kW) * (kW + 1);

__global__ void __launch_bounds__(kThreads) blk_gram(const double *__restrict__ X, int rows, int n, int nb, int round,
                                                     double *__restrict__ partial)
{
    extern __shared__ double dsm[];
    double(*T)[kW + 1] = reinterpret_cast<double(*)[kW + 1]>(dsm);
    const Panel pn = make_panel(n, nb, round, blockIdx.x);
    const int w = pn.width();
    const int r0 = blockIdx.y * kRC;
    const int rc = min(kRC, rows - r0);
    for (int e = threadIdx.x; e < kRC * kW; e += blockDim.x) {
        const int j = e / kRC, i = e - j * kRC;  // consecutive threads walk down a column
        T[i][j] = (i < rc && j < w) ? X[(size_t)pn.col(j) * rows + r0 + i] : 0.0;
    }
    __syncthreads();
    // thread -> 4 x 4 tile of the 64 x 64 Gram
    const int ti = (threadIdx.x >> 4) * 4, tj = (threadIdx.x & 15) * 4;
    double acc[4][4] = {};
    for (int i = 0; i < rc; ++i) {
        double a[4], b[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            a[u] = T[i][ti + u];
            b[u] = T[i][tj + u];
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] = fma(a[u], b[v], acc[u][v]);
    }
    double *out = partial + ((size_t)blockIdx.x * gridDim.y + blockIdx.y) * kW * kW;
#pragma unroll
    for (int u = 0; u < 4; ++u)
#pragma unroll
        for (int v = 0; v < 4; ++v) out[(ti + u) * kW + tj + v] = acc[u][v];
}

// 2. Panel solve: one CTA per block pair.
__global__ void __launch_bounds__(1024) blk_solve(const double *__restrict__ partial, int chunks, int n, int nb,
                                                  int round, double eps, double *__restrict__ Wout,
                                                  int *__restrict__ flags, unsigned *__restrict__ counter)
{
    extern __shared__ double dsm[];
    double(*G)[kW + 1] = reinterpret_cast<double(*)[kW + 1]>(dsm);
    double(*Wm)[kW + 1] = reinterpret_cast<double(*)[kW + 1]>(dsm + kW * (kW + 1));
    __shared__ double cs[kW / 2][2];
    __shared__ int any;
    const Panel pn = make_panel(n, nb, round, blockIdx.x);
    const int w = pn.width();
    const int tid = threadIdx.x;
    for (int e = tid; e < kW * kW; e += blockDim.x) {
        const int i = e / kW, j = e - i * kW;
        double s = 0.0;
        for (int c = 0; c < chunks; ++c) s += partial[((size_t)blockIdx.x * chunks + c) * kW * kW + e];
        G[i][j] = s;
        Wm[i][j] = (i == j) ? 1.0 : 0.0;
    }
    if (tid == 0) any = 0;
    __syncthreads();
    // any column pair of the panel above the threshold?
    for (int e = tid; e < w * w; e += blockDim.x) {
        const int i = e / w, j = e - i * w;
        if (i < j) {
            const double pq = G[i][j];
            if (fabs(pq) > eps * sqrt(fmax(G[i][i], 0.0) * fmax(G[j][j], 0.0)) && fabs(pq) > 1.0e-300) any = 1;
        }
    }
    __syncthreads();
    if (!any) {
        if (tid == 0) flags[blockIdx.x] = 0;
        return;
    }
    // cyclic two-sided Jacobi on G (size w, even-padded), W accumulates J's
    const int we = w + (w & 1);
    const int L = we - 1;
    for (int sw = 0; sw < kInnerSweeps; ++sw) {
        for (int r = 0; r < L; ++r) {
            if (tid < we / 2) {
                const int i = tid, i2 = we - 1 - tid;
                const int p = i == 0 ? 0 : 1 + ((i - 1 - r) % L + L) % L;
                const int q = 1 + ((i2 - 1 - r) % L + L) % L;
                double c = 1.0, s = 0.0;
                if (p < w && q < w) {
                    const double a = G[p][p], d = G[q][q], o = G[p][q];
                    if (fabs(o) > eps * sqrt(fmax(a, 0.0) * fmax(d, 0.0)) && fabs(o) > 1.0e-300) {
                        const double tau = (d - a) / (2.0 * o);
                        const double t = (tau >= 0.0) ? 1.0 / (tau + sqrt(fma(tau, tau, 1.0)))
                                                      : -1.0 / (-tau + sqrt(fma(tau, tau, 1.0)));
                        c = 1.0 / sqrt(fma(t, t, 1.0));
                        s = t * c;
                    }
                }
                cs[tid][0] = c;
                cs[tid][1] = s;
            }
            __syncthreads();
            // columns: G <- G J, W <- W J   (items: row x pair)
            for (int e = tid; e < we * (we / 2); e += blockDim.x) {
                const int row = e / (we / 2), k = e - row * (we / 2);
                const double c = cs[k][0], s = cs[k][1];
                if (s == 0.0) continue;
                const int i2 = we - 1 - k;
                const int p = k == 0 ? 0 : 1 + ((k - 1 - r) % L + L) % L;
                const int q = 1 + ((i2 - 1 - r) % L + L) % L;
                const double gp = G[row][p], gq = G[row][q];
                G[row][p] = fma(c, gp, -(s * gq));
                G[row][q] = fma(s, gp, c * gq);
                const double wp = Wm[row][p], wq = Wm[row][q];
                Wm[row][p] = fma(c, wp, -(s * wq));
                Wm[row][q] = fma(s, wp, c * wq);
            }
            __syncthreads();
            // rows: G <- J^T G
            for (int e = tid; e < we * (we / 2); e += blockDim.x) {
                const int col = e / (we / 2), k = e - col * (we / 2);
                const double c = cs[k][0], s = cs[k][1];
                if (s == 0.0) continue;
                const int i2 = we - 1 - k;
                const int p = k == 0 ? 0 : 1 + ((k - 1 - r) % L + L) % L;
                const int q = 1 + ((i2 - 1 - r) % L + L) % L;
                const double gp = G[p][col], gq = G[q][col];
                G[p][col] = fma(c, gp, -(s * gq));
                G[q][col] = fma(s, gp, c * gq);
            }
            __syncthreads();
        }
    }
    double *wo = Wout + (size_t)blockIdx.x * kW * kW;
    for (int e = tid; e < kW * kW; e += blockDim.x) wo[e] = Wm[e / kW][e % kW];
    if (tid == 0) {
        flags[blockIdx.x] = 1;
        atomicAdd(counter, 1u);
    }
}

// 3. Apply: blockIdx.x = block pair, blockIdx.y = row chunk over X's rows then
// V's rows.  P_chunk <- P_chunk W in place.
__global__ void __launch_bounds__(kThreads) blk_apply(double *__restrict__ X, int rows, double *__restrict__ V, int n,
                                                      int nb, int round, int x_chunks,
                                                      const double *__restrict__ Win,
                                                      const int *__restrict__ flags)
{
    if (flags[blockIdx.x] == 0) return;
    extern __shared__ double dsm[];
    double(*T)[kW + 1] = reinterpret_cast<double(*)[kW + 1]>(dsm);
    double(*Ws)[kW + 1] = reinterpret_cast<double(*)[kW + 1]>(dsm + kRC * (kW + 1));
    const Panel pn = make_panel(n, nb, round, blockIdx.x);
    const int w = pn.width();
    const bool onX = (int)blockIdx.y < x_chunks;
    double *M = onX ? X : V;
    const int ld = onX ? rows : n;
    const int r0 = (onX ? blockIdx.y : blockIdx.y - x_chunks) * kRC;
    const int rc = min(kRC, ld - r0);
    const double *wi = Win + (size_t)blockIdx.x * kW * kW;
    for (int e = threadIdx.x; e < kW * kW; e += blockDim.x) Ws[e / kW][e % kW] = wi[e];
    for (int e = threadIdx.x; e < kRC * kW; e += blockDim.x) {
        const int j = e / kRC, i = e - j * kRC;
        T[i][j] = (i < rc && j < w) ? M[(size_t)pn.col(j) * ld + r0 + i] : 0.0;
    }
    __syncthreads();
    // thread -> rows {ti + 32u}, columns tj..tj+7  (32 outputs)
    const int ti = threadIdx.x & 31, tj = (threadIdx.x >> 5) * 8;
    double acc[4][8] = {};
    for (int k = 0; k < w; ++k) {
        double b[8];
#pragma unroll
        for (int v = 0; v < 8; ++v) b[v] = Ws[k][tj + v];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const double a = T[ti + 32 * u][k];
#pragma unroll
            for (int v = 0; v < 8; ++v) acc[u][v] = fma(a, b[v], acc[u][v]);
        }
    }
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int i = ti + 32 * u;
        if (i >= rc) continue;
#pragma unroll
        for (int v = 0; v < 8; ++v) {
            const int j = tj + v;
            if (j < w) M[(size_t)pn.col(j) * ld + r0 + i] = acc[u][v];
        }
    }
}

constexpr int kTile = 32, kTileRows = 8;

__global__ void __launch_bounds__(kTile *kTileRows)
    blk_to_colmajor(const double *__restrict__ src, int rows, int cols, double *__restrict__ dst)
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

// column-major -> row-major, optionally dividing column c by sigma[c]
// (zero when sigma[c] <= eps).
__global__ void __launch_bounds__(kTile *kTileRows)
    blk_to_rowmajor(const double *__restrict__ src, int rows, int cols, double *__restrict__ dst,
                    const double *__restrict__ sigma, double eps)
{
    __shared__ double tile[kTile][kTile + 1];
    const int r0 = blockIdx.x * kTile, c0 = blockIdx.y * kTile;
    for (int k = threadIdx.y; k < kTile; k += kTileRows) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (r < rows && c < cols) tile[k][threadIdx.x] = src[(size_t)c * rows + r];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < kTile; k += kTileRows) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if (r < rows && c < cols) {
            double val = tile[threadIdx.x][k];
            if (sigma != nullptr) {
                const double sg = sigma[c];
                val = (sg > eps) ? (val / sg) : 0.0;
            }
            dst[(size_t)r * cols + c] = val;
        }
    }
}

__global__ void blk_identity(double *__restrict__ v, int n)
{
    const size_t total = (size_t)n * n;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x)
        v[e] = (e / n == e % n) ? 1.0 : 0.0;
}

// sigma_j = ||x_j|| (sequential sum per column, one warp per column)
__global__ void blk_sigma(const double *__restrict__ X, int rows, int n, double *__restrict__ sigma)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double *x = X + (size_t)warp * rows;
    double acc = 0.0;
    for (int i = lane; i < rows; i += 32) acc = fma(x[i], x[i], acc);
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) sigma[warp] = sqrt(acc);
}

}  // namespace

BlockedStats &blocked_stats()
{
    thread_local BlockedStats s;
    return s;
}

int blocked_solve(const double *d_a, int rows, int n, double eps, int max_sweeps, double *d_u, double *d_sigma,
                  double *d_v, int *sweeps, cudaStream_t st)
{
    JSVD_CUDA_TRY(cudaFuncSetAttribute(blk_gram, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGramSmem));
    JSVD_CUDA_TRY(cudaFuncSetAttribute(blk_solve, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSolveSmem));
    JSVD_CUDA_TRY(cudaFuncSetAttribute(blk_apply, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kApplySmem));
    const int nb = (n + kB - 1) / kB;
    const int nbe = nb + (nb & 1);
    const int rounds = nb >= 2 ? nbe - 1 : 0;
    const int npairs = nb / 2;
    const int xc = (rows + kRC - 1) / kRC, vc = (n + kRC - 1) / kRC;
    const size_t mn = (size_t)rows * n, nn = (size_t)n * n;
    const size_t part = (size_t)std::max(1, npairs) * xc * kW * kW;
    const size_t wbytes = (size_t)std::max(1, npairs) * kW * kW;
    double *ws = nullptr;
    const size_t doubles = mn + nn + n + part + wbytes;
    JSVD_CUDA_TRY(cudaMallocAsync((void **)&ws, sizeof(double) * doubles + sizeof(int) * (npairs + 2), st));
    ScopeExit free_ws([&] { cudaFreeAsync(ws, st); });
    double *X = ws, *V = X + mn, *sg = V + nn, *partial = sg + n, *W = partial + part;
    int *flags = reinterpret_cast<int *>(W + wbytes);
    unsigned *counter = reinterpret_cast<unsigned *>(flags + npairs + 1);
    const dim3 tb(kTile, kTileRows);
    blk_to_colmajor<<<dim3((n + kTile - 1) / kTile, (rows + kTile - 1) / kTile), tb, 0, st>>>(d_a, rows, n, X);
    blk_identity<<<std::min<size_t>(1184, (nn + 255) / 256), 256, 0, st>>>(V, n);
    JSVD_CUDA_TRY(cudaGetLastError());
    BlockedStats &bs = blocked_stats();
    int executed = 1;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    ScopeExit destroy_events([&] {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    });
    cudaEventRecord(e0, st);
    if (rounds > 0) {
        for (int s = 0; s < max_sweeps; ++s) {
            JSVD_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned), st));
            for (int r = 0; r < rounds; ++r) {
                blk_gram<<<dim3(npairs, xc), kThreads, kGramSmem, st>>>(X, rows, n, nb, r, partial);
                blk_solve<<<npairs, 1024, kSolveSmem, st>>>(partial, xc, n, nb, r, eps, W, flags, counter);
                blk_apply<<<dim3(npairs, xc + vc), kThreads, kApplySmem, st>>>(X, rows, V, n, nb, r, xc, W,
                                                                               flags);
            }
            JSVD_CUDA_TRY(cudaGetLastError());
            unsigned rotated = 0;
            JSVD_CUDA_TRY(cudaMemcpyAsync(&rotated, counter, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
            JSVD_CUDA_TRY(cudaStreamSynchronize(st));
            executed = s + 1;
            bs.block_rounds += (unsigned long long)rounds;
            if (rotated == 0) break;
        }
    }
    cudaEventRecord(e1, st);
    double *sig = d_sigma ? d_sigma : sg;
    blk_sigma<<<(n * 32 + 255) / 256, 256, 0, st>>>(X, rows, n, sig);
    if (d_u)
        blk_to_rowmajor<<<dim3((rows + kTile - 1) / kTile, (n + kTile - 1) / kTile), tb, 0, st>>>(X, rows, n, d_u,
                                                                                             sig, eps);
    if (d_v)
        blk_to_rowmajor<<<dim3((n + kTile - 1) / kTile, (n + kTile - 1) / kTile), tb, 0, st>>>(V, n, n, d_v,
                                                                                           nullptr, 0.0);
    JSVD_CUDA_TRY(cudaGetLastError());
    JSVD_CUDA_TRY(cudaStreamSynchronize(st));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    bs.solves += 1;
    bs.sweeps += (unsigned long long)executed;
    bs.sweep_ms += ms;
    if (sweeps) *sweeps = executed;
    return JSVD_OK;
}

}  // namespace jsvd

using namespace jsvd;

extern "C" int jsvd_blocked_svd_device(const double *d_a, size_t rows, size_t columns, const jsvd_config *cfg,
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
        // Fewer than two blocks: there is no block pair to rotate; the plain sweep
        // handles it.  So does it for inputs taller than this engine's grids
        // allow (row tiles of 32 along grid.y, at most 65535 blocks).
        if (columns < 2 * (size_t)kB || rows > (size_t)65535 * 32)
            return jsvd_plain_svd_device(d_a, rows, columns, &c, d_u, d_sigma, d_v, sweeps, st);
        return blocked_solve(d_a, (int)rows, (int)columns, c.epsilon, c.max_sweeps, d_u, d_sigma, d_v, sweeps, st);
    });
}

extern "C" int jsvd_blocked_svd(const double *a, size_t rows, size_t columns, const jsvd_config *cfg, double *u,
                                double *sigma, double *v, int *sweeps)
{
    return c_entry([&]() -> int {
        return host_buffer_solve(jsvd_blocked_svd_device, a, rows, columns, cfg, u, sigma, v, sweeps);
    });
}

extern "C" void jsvd_blocked_stats_get(jsvd_blocked_stats *out)
{
    if (!out) return;
    const BlockedStats &s = blocked_stats();
    out->solves = s.solves;
    out->sweeps = s.sweeps;
    out->block_rounds = s.block_rounds;
    out->sweep_ms = s.sweep_ms;
}

extern "C" void jsvd_blocked_stats_reset(void) { blocked_stats() = BlockedStats{}; }
