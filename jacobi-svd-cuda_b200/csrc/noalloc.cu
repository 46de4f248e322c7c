// Plain one-sided Jacobi SVD that allocates no memory: jsvd_plain_svd_noalloc.
//
// Who needs it: callers that must not call cudaMalloc/cudaFree once they are
// running - applications whose framework reserved the whole device for its
// own memory pool up front (a late cudaMalloc then fails or fragments it),
// latency-critical services where cudaMalloc/cudaFree would synchronise the
// device and stall unrelated streams, and plugin hosts that forbid device
// allocation after start-up.  The regular entry points allocate a cached
// workspace (plans, staging buffers, a pinned counter, a per-thread stream);
// this one uses only the caller's buffers and the fixed scratch array below.
//
// Scratch: one file-scope device array of kNoAllocScratchDoubles doubles
// (16 MiB).  It is part of the module, so every GPU that loads the library
// holds it until the process exits.  Layout per call:
//   [ A working copy m*n | V n*n | sigma n | rotation counter ]
// which caps a call at m*n + n*n + n + 1 <= kNoAllocScratchDoubles
// (e.g. 1024 x 1023, or 2048 x 600).  Every call shares the array and leaves
// its contents behind; everything that must start at zero is cleared by the
// call itself.  Calls whose work overlaps on the GPU (two host threads, or two
// streams, at the same time) race on the array and corrupt each other's
// results: serialise them.
//
// Host code cannot use the array's name as a device address (it names a host
// shadow).  The first call on each device (more precisely, in each CUDA
// context: after cudaDeviceReset the device gets a new primary context and the
// module, with the array, is loaded again, possibly at another address) looks
// the address up with cudaGetSymbolAddress while that device is current and
// caches it together with the context's process-unique ID; later calls in the
// same context reuse it, a call in a new context looks it up again.
//
// Memory is committed when the module is loaded.  CUDA loads modules lazily by
// default (CUDA_MODULE_LOADING=LAZY since 12.2), so on each device the array is
// committed by the first call, not when the library is loaded: a caller that
// reserves the rest of the device afterwards must make one warm-up call per
// device first (or run with CUDA_MODULE_LOADING=EAGER).
//
// Each sweep reads its rotation count back with a device-to-host copy and
// waits for it on the host, so the entry cannot be used while its stream is
// being captured into a CUDA graph.
//
// The arithmetic is the plain path's: same reduction order, same rotation,
// same cyclic round-robin order; V is rotated inside the round kernel (no
// (c, s) table), so results are bit-identical to jsvd_plain_svd_device.
#include <cuda.h>
#include <cuda_runtime.h>

#include <mutex>

#include "common.cuh"
#include "internal.hpp"
#include "jsvd.h"

namespace jsvd {
namespace {

constexpr size_t kNoAllocScratchDoubles = size_t(2) << 20;  // 16 MiB
constexpr int kNoAllocMaxDevices = 64;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

struct ScratchAddress {
    unsigned long long context_id = 0;  // 0: not looked up yet
    double *ptr = nullptr;
};

std::mutex g_noalloc_mutex;
ScratchAddress g_noalloc_addr[kNoAllocMaxDevices];

using CtxGetCurrentFn = CUresult (*)(CUcontext *);
using CtxGetIdFn = CUresult (*)(CUcontext, unsigned long long *);

// Process-unique ID of the current CUDA context (driver entry points fetched
// through the runtime, so the library needs no link against libcuda).
int current_context_id(unsigned long long *id)
{
    static CtxGetCurrentFn get_current = nullptr;
    static CtxGetIdFn get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q{};
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<CtxGetCurrentFn>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<CtxGetIdFn>(p);
    });
    if (!get_current || !get_id) {
        set_last_error(JSVD_ERR_CUDA, "cuCtxGetCurrent/cuCtxGetId are not available from the CUDA driver.");
        return JSVD_ERR_CUDA;
    }
    CUcontext ctx = nullptr;
    if (get_current(&ctx) != CUDA_SUCCESS || ctx == nullptr || get_id(ctx, id) != CUDA_SUCCESS) {
        set_last_error(JSVD_ERR_CUDA, "jsvd_plain_svd_noalloc: no current CUDA context on the device.");
        return JSVD_ERR_CUDA;
    }
    return JSVD_OK;
}

// Device address of the scratch array on the current device: looked up once
// per device and context (the caller has made `dev` current and initialised
// its primary context).
int noalloc_scratch(int dev, double **out)
{
    if (dev < 0 || dev >= kNoAllocMaxDevices) return invalid_argument("Device ordinal out of range.");
    unsigned long long ctx_id = 0;
    if (int rc = current_context_id(&ctx_id); rc != JSVD_OK) return rc;
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    ScratchAddress &slot = g_noalloc_addr[dev];
    if (slot.context_id != ctx_id || slot.ptr == nullptr) {
        double *ptr = nullptr;
        JSVD_CUDA_TRY(cudaGetSymbolAddress((void **)&ptr, g_noalloc_scratch));
        slot.ptr = ptr;
        slot.context_id = ctx_id;
    }
    *out = slot.ptr;
    return JSVD_OK;
}

constexpr int kTile = 32, kTileRows = 8;

__global__ void __launch_bounds__(kTile *kTileRows)
    na_to_colmajor(const double *__restrict__ src, int rows, int cols, double *__restrict__ dst)
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

__global__ void __launch_bounds__(kTile *kTileRows)
    na_to_rowmajor(const double *__restrict__ src, int rows, int cols, double *__restrict__ dst,
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

__global__ void na_identity(double *__restrict__ v, int n)
{
    const size_t total = (size_t)n * n;
    for (size_t idx = blockIdx.x * (size_t)blockDim.x + threadIdx.x; idx < total;
         idx += (size_t)gridDim.x * blockDim.x)
        v[idx] = (idx / n == idx % n) ? 1.0 : 0.0;
}

template <int T>
__device__ __forceinline__ void na_tree3(double &pp, double &qq, double &pq, double *red)
{
    if constexpr (T == 32) {
        pp = warp_tree1(pp);
        qq = warp_tree1(qq);
        pq = warp_tree1(pq);
    } else {
        constexpr int W = T / 32;
        const int t = threadIdx.x;
        red[t] = pp;
        red[T + t] = qq;
        red[2 * T + t] = pq;
        __syncthreads();
        if (t < 32) {
            double y[W];
#pragma unroll
            for (int w = 0; w < W; ++w) y[w] = red[w * 32 + t];
            pp = warp_tree<W>(y);
#pragma unroll
            for (int w = 0; w < W; ++w) y[w] = red[T + w * 32 + t];
            qq = warp_tree<W>(y);
#pragma unroll
            for (int w = 0; w < W; ++w) y[w] = red[2 * T + w * 32 + t];
            pq = warp_tree<W>(y);
        }
    }
}

// Round kernel of this entry point: pair from the closed-form schedule, dot
// products in the reference's T-lane order, rotation of the A columns and of
// the V columns (column-major V, n rows) in the same launch.
template <int T>
__global__ void __launch_bounds__(T) na_round_kernel(double *__restrict__ a, int m, double *__restrict__ v, int n,
                                                      int round, double eps, unsigned *__restrict__ counter)
{
    __shared__ double red[T == 32 ? 1 : 3 * T];
    __shared__ double2 rot;
    const int t = threadIdx.x;
    const int2 pq_idx = round_robin_pair(n, round, blockIdx.x);
    double *__restrict__ ap = a + (size_t)pq_idx.x * m;
    double *__restrict__ aq = a + (size_t)pq_idx.y * m;
    double spp = 0.0, sqq = 0.0, spq = 0.0;
    for (int r = t; r < m; r += T) {
        const double x = ap[r], y = aq[r];
        spp = fma(x, x, spp);
        sqq = fma(y, y, sqq);
        spq = fma(x, y, spq);
    }
    na_tree3<T>(spp, sqq, spq, red);
    if (t == 0) {
        double c, s;
        if (rotation_params(spp, sqq, spq, eps, c, s)) atomicAdd(counter, 1u);
        rot = make_double2(c, s);
    }
    __syncthreads();
    const double c = rot.x, s = rot.y;
    if (c == 0.0) return;
    for (int r = t; r < m; r += T) {
        const double x = ap[r], y = aq[r];
        ap[r] = rot_p(c, s, x, y);
        aq[r] = rot_q(c, s, x, y);
    }
    double *__restrict__ vp = v + (size_t)pq_idx.x * n;
    double *__restrict__ vq = v + (size_t)pq_idx.y * n;
    for (int r = t; r < n; r += T) {
        const double x = vp[r], y = vq[r];
        vp[r] = rot_p(c, s, x, y);
        vq[r] = rot_q(c, s, x, y);
    }
}

template <int T>
__global__ void __launch_bounds__(T) na_sigma_kernel(const double *__restrict__ a, int m, double *__restrict__ sigma)
{
    __shared__ double red[T == 32 ? 1 : T];
    const int t = threadIdx.x;
    const double *__restrict__ col = a + (size_t)blockIdx.x * m;
    double acc = 0.0;
    for (int r = t; r < m; r += T) acc = fma(col[r], col[r], acc);
    if constexpr (T == 32) {
        acc = warp_tree1(acc);
    } else {
        constexpr int W = T / 32;
        red[t] = acc;
        __syncthreads();
        if (t < 32) {
            double y[W];
#pragma unroll
            for (int w = 0; w < W; ++w) y[w] = red[w * 32 + t];
            acc = warp_tree<W>(y);
        }
    }
    if (t == 0) sigma[blockIdx.x] = sqrt(fmax(acc, 0.0));
}

template <int T>
int na_solve(const double *d_a, int m, int n, double eps, int max_sweeps, double *d_u, double *d_sigma, double *d_v,
             int *sweeps, cudaStream_t stream, double *scratch)
{
    double *a_w = scratch;
    double *v_w = a_w + (size_t)m * n;
    double *sig_w = v_w + (size_t)n * n;
    unsigned *counter = reinterpret_cast<unsigned *>(sig_w + n);
    const dim3 tb(kTile, kTileRows);
    na_to_colmajor<<<dim3((n + kTile - 1) / kTile, (m + kTile - 1) / kTile), tb, 0, stream>>>(d_a, m, n, a_w);
    JSVD_CUDA_TRY(cudaGetLastError());
    na_identity<<<(unsigned)(((size_t)n * n + 255) / 256 < 1184 ? ((size_t)n * n + 255) / 256 : 1184), 256, 0,
                  stream>>>(v_w, n);
    JSVD_CUDA_TRY(cudaGetLastError());
    const int ne = n + (n & 1);
    const int rounds = n >= 2 ? ne - 1 : 0;
    const int npairs = n / 2;
    int executed = 1;
    if (rounds > 0) {
        for (int sweep = 0; sweep < max_sweeps; ++sweep) {
            JSVD_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned), stream));
            for (int r = 0; r < rounds; ++r)
                na_round_kernel<T><<<npairs, T, 0, stream>>>(a_w, m, v_w, n, r, eps, counter);
            JSVD_CUDA_TRY(cudaGetLastError());
            unsigned rotated = 0;
            JSVD_CUDA_TRY(cudaMemcpyAsync(&rotated, counter, sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
            JSVD_CUDA_TRY(cudaStreamSynchronize(stream));
            executed = sweep + 1;
            if (rotated == 0) break;
        }
    }
    double *sig = d_sigma ? d_sigma : sig_w;
    na_sigma_kernel<T><<<n, T, 0, stream>>>(a_w, m, sig);
    JSVD_CUDA_TRY(cudaGetLastError());
    if (d_u) {
        na_to_rowmajor<<<dim3((m + kTile - 1) / kTile, (n + kTile - 1) / kTile), tb, 0, stream>>>(a_w, m, n, d_u,
                                                                                              sig, eps);
        JSVD_CUDA_TRY(cudaGetLastError());
    }
    if (d_v) {
        na_to_rowmajor<<<dim3((n + kTile - 1) / kTile, (n + kTile - 1) / kTile), tb, 0, stream>>>(v_w, n, n, d_v,
                                                                                              nullptr, 0.0);
        JSVD_CUDA_TRY(cudaGetLastError());
    }
    JSVD_CUDA_TRY(cudaStreamSynchronize(stream));
    if (sweeps) *sweeps = executed;
    return JSVD_OK;
}

}  // namespace
}  // namespace jsvd

using namespace jsvd;

extern "C" int jsvd_plain_svd_noalloc(const double *d_a, size_t rows, size_t columns, const jsvd_config *cfg,
                                      double *d_u, double *d_sigma, double *d_v, int *sweeps, void *stream)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        jsvd_config def;
        const jsvd_config &c = config_or_default(cfg, def);
        int rc = validate_plain_request(d_a, rows, columns, c);
        if (rc != JSVD_OK) return rc;
        const size_t need = rows * columns + columns * columns + columns + 1;
        if (rows > kNoAllocScratchDoubles || need > kNoAllocScratchDoubles)
            return invalid_argument(
                "jsvd_plain_svd_noalloc: rows*columns + columns*columns + columns + 1 exceeds the fixed scratch of "
                "2097152 doubles (16 MiB).");
        // its input transpose runs one launch with row tiles of 32 along grid.y
        if (rows > (size_t)65535 * 32)
            return invalid_argument("jsvd_plain_svd_noalloc: at most 2097120 rows.");
        int dev = 0;
        JSVD_CUDA_TRY(cudaGetDevice(&dev));
        // since CUDA 12 this also initialises the device's primary context, so
        // the context ID below exists on the very first call
        JSVD_CUDA_TRY(cudaSetDevice(dev));
        double *scratch = nullptr;
        rc = noalloc_scratch(dev, &scratch);
        if (rc != JSVD_OK) return rc;
        cudaStream_t st = (cudaStream_t)stream;
        const int m = (int)rows, n = (int)columns;
        switch (reduction_lanes(c.threads_per_block)) {
        case 32: return na_solve<32>(d_a, m, n, c.epsilon, c.max_sweeps, d_u, d_sigma, d_v, sweeps, st, scratch);
        case 64: return na_solve<64>(d_a, m, n, c.epsilon, c.max_sweeps, d_u, d_sigma, d_v, sweeps, st, scratch);
        case 128: return na_solve<128>(d_a, m, n, c.epsilon, c.max_sweeps, d_u, d_sigma, d_v, sweeps, st, scratch);
        case 256: return na_solve<256>(d_a, m, n, c.epsilon, c.max_sweeps, d_u, d_sigma, d_v, sweeps, st, scratch);
        case 512: return na_solve<512>(d_a, m, n, c.epsilon, c.max_sweeps, d_u, d_sigma, d_v, sweeps, st, scratch);
        default: return na_solve<1024>(d_a, m, n, c.epsilon, c.max_sweeps, d_u, d_sigma, d_v, sweeps, st, scratch);
        }
    });
}
