// One-sided block-pair Jacobi sweep (FP64, sm_100a).
//
// The columns are split into blocks of B.  An outer sweep pairs every block
// with every other block once (fixed-head circle over the blocks, one kernel
// launch per outer round); one CTA takes one block pair, i.e. 2B columns, and
// runs a full inner cyclic sweep over them (2B - 1 inner rounds of B pairs,
// the same fixed-head circle on the 2B local columns) before it writes them
// back.  Pairs of columns from different blocks meet once per outer sweep and
// pairs inside a block once per block pair, so an outer sweep is a cyclic
// sweep with extra inner work; the algorithm stops after the first outer sweep
// in which no pair rotates, with the reference's rotation test (src/kernels.cu
// :485-521: |a_pq| > eps sqrt(a_pp a_qq) and |a_pq| > 1e-300) and its
// Rutishauser angle.  The ordering differs from the reference's cyclic
// round robin, so the results are not bit-identical to it; they are one-sided
// Jacobi results to working accuracy (checked against the oracle within a
// tolerance in the tests).
//
// Why this shape on B200: a scalar cyclic sweep of an n-column matrix is
// n - 1 dependent rounds, each a kernel that moves every column through L2 and
// waits on a reduction and a square-root/division chain.  Here one launch does
// 2B - 1 rounds for its columns with the columns in registers: thread t holds
// rows t, t + NT, ... of all 2B columns, so the rotation of round r and the dot
// products of round r + 1 touch only the thread's own registers and an inner
// round needs two barriers (partial sums published, angles published).  The
// angle of a pair is computed once, by one thread, and the 2B x 2B product of
// the inner rotations is applied to V's 2B columns once per block pair.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <memory>
#include <vector>

#include "blockpair.hpp"
#include "common.cuh"
#include "internal.hpp"
#include "layout.cuh"
#include "plain.hpp"

namespace jsvd {
namespace {

// Fixed-head circle on C (even) positions: pair k of round r is
// (pos_k, pos_{C-1-k}); position 0 stays, positions 1..C-1 rotate by one per
// round (src/kernels.cu:637-678 builds the same sequence with a host table).
__host__ __device__ constexpr int circle_at(int C, int r, int pos)
{
    return pos == 0 ? 0 : 1 + ((pos - 1 - r) % (C - 1) + (C - 1)) % (C - 1);
}

// One outer round: CTA b takes block pair bpairs[b] = (I, J), columns
// I*B .. I*B+B-1 and J*B .. J*B+B-1 of x (column-major m x n, ld m); columns at
// or beyond n (the last block's tail, the dummy block of an odd block count)
// are absent and never rotate.  v is column-major n x n.  counter[0] counts the
// CTAs in which some pair rotated.  Requires m <= RPT * NT and n <= m.
template <int B, int RPT, int NT>
__global__ void __launch_bounds__(NT) bp_round_kernel(double *__restrict__ x, int m, int n, double *__restrict__ v,
                                                      const int2 *__restrict__ bpairs, double eps,
                                                      unsigned *__restrict__ counter)
{
    constexpr int C = 2 * B;
    constexpr int NW = NT / 32;
    static_assert(NT % 32 == 0 && NT <= 1024, "whole warps");
    __shared__ double red[NW][3 * B];
    __shared__ double2 cs[B];
    __shared__ double w[C][C];  // w[j][i] = T(i, j); A_new = A_old T over the 2B columns
    __shared__ int any;
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    const int2 blk = bpairs[blockIdx.x];
    int gcol[C];
    unsigned vmask = 0;
#pragma unroll
    for (int c = 0; c < C; ++c) {
        gcol[c] = c < B ? blk.x * B + c : blk.y * B + (c - B);
        if (gcol[c] < n) vmask |= 1u << c;
    }
    double xa[C][RPT];
#pragma unroll
    for (int c = 0; c < C; ++c) {
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
            const int row = t + i * NT;
            xa[c][i] = (((vmask >> c) & 1u) && row < m) ? x[(size_t)gcol[c] * m + row] : 0.0;
        }
    }
    for (int e = t; e < C * C; e += NT) w[e / C][e % C] = (e / C == e % C) ? 1.0 : 0.0;
    if (t == 0) any = 0;
    __syncthreads();
    // xa[pos] holds the local column at circle position pos: in round r that
    // is circle_at(C, r, pos), and the pairs of every round are the fixed
    // positions (k, C - 1 - k).  After a round the registers shift as the
    // circle does (position j takes j - 1, position 1 takes C - 1), so the
    // round is a real loop with compile-time register indices (a fully
    // unrolled sweep overflowed the instruction cache); after the C - 1 rounds
    // position c holds local column c again.
#pragma unroll 1
    for (int r = 0; r < C - 1; ++r) {
        double part[3 * B];
#pragma unroll
        for (int k = 0; k < B; ++k) {
            double spp = 0.0, sqq = 0.0, spq = 0.0;
#pragma unroll
            for (int i = 0; i < RPT; ++i) {
                spp = fma(xa[k][i], xa[k][i], spp);
                sqq = fma(xa[C - 1 - k][i], xa[C - 1 - k][i], sqq);
                spq = fma(xa[k][i], xa[C - 1 - k][i], spq);
            }
            part[3 * k] = spp;
            part[3 * k + 1] = sqq;
            part[3 * k + 2] = spq;
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
#pragma unroll
            for (int e = 0; e < 3 * B; ++e) part[e] += __shfl_down_sync(0xffffffffu, part[e], off);
        }
        if (lane == 0) {
#pragma unroll
            for (int e = 0; e < 3 * B; ++e) red[warp][e] = part[e];
        }
        __syncthreads();
        if (t < B) {
            // One thread per pair: totals in warp order, angle, transform.
            const int p = circle_at(C, r, t), q = circle_at(C, r, C - 1 - t);
            double pp = 0.0, qq = 0.0, pq = 0.0;
#pragma unroll
            for (int wv = 0; wv < NW; ++wv) {
                pp += red[wv][3 * t];
                qq += red[wv][3 * t + 1];
                pq += red[wv][3 * t + 2];
            }
            double c = 0.0, s = 0.0;
            if (((vmask >> p) & 1u) && ((vmask >> q) & 1u) && rotation_params(pp, qq, pq, eps, c, s)) {
                any = 1;
#pragma unroll
                for (int i = 0; i < C; ++i) {
                    const double a = w[p][i], b = w[q][i];
                    w[p][i] = rot_p(c, s, a, b);
                    w[q][i] = rot_q(c, s, a, b);
                }
            } else {
                c = 0.0;  // c == 0 marks a pair that does not rotate
            }
            cs[t] = make_double2(c, s);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < B; ++k) {
            const double2 g = cs[k];
            if (g.x != 0.0) {
#pragma unroll
                for (int i = 0; i < RPT; ++i) {
                    const double a = xa[k][i], b = xa[C - 1 - k][i];
                    xa[k][i] = rot_p(g.x, g.y, a, b);
                    xa[C - 1 - k][i] = rot_q(g.x, g.y, a, b);
                }
            }
        }
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
            const double last = xa[C - 1][i];
#pragma unroll
            for (int j = C - 1; j >= 2; --j) xa[j][i] = xa[j - 1][i];
            xa[1][i] = last;
        }
    }
    // `any` and w were last written before the final barrier of the loop.
    if (!any) return;  // no pair rotated: columns and V unchanged
#pragma unroll
    for (int c = 0; c < C; ++c) {
        if (!((vmask >> c) & 1u)) continue;
#pragma unroll
        for (int i = 0; i < RPT; ++i) {
            const int row = t + i * NT;
            if (row < m) x[(size_t)gcol[c] * m + row] = xa[c][i];
        }
    }
    // V(:, cols) <- V(:, cols) T, one row of V per thread and step.
#pragma unroll 1
    for (int i = 0; i < RPT; ++i) {
        const int row = t + i * NT;
        if (row >= n) break;
        double vv[C];
#pragma unroll
        for (int c = 0; c < C; ++c) vv[c] = ((vmask >> c) & 1u) ? v[(size_t)gcol[c] * n + row] : 0.0;
#pragma unroll
        for (int j = 0; j < C; ++j) {
            if (!((vmask >> j) & 1u)) continue;
            double acc = 0.0;
#pragma unroll
            for (int c = 0; c < C; ++c) acc = fma(vv[c], w[j][c], acc);
            v[(size_t)gcol[j] * n + row] = acc;
        }
    }
    if (t == 0) atomicAdd(counter, 1u);
}

// sigma_j = ||x_j|| (one warp per column).
__global__ void bp_sigma_kernel(const double *__restrict__ x, int m, int n, double *__restrict__ sigma)
{
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double *col = x + (size_t)warp * m;
    double acc = 0.0;
    for (int r = lane; r < m; r += 32) acc = fma(col[r], col[r], acc);
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) sigma[warp] = sqrt(fmax(acc, 0.0));
}

using BpFn = void (*)(double *, int, int, double *, const int2 *, double, unsigned *);

struct Variant {
    int B, rpt, threads;
    BpFn fn;
};

// Instantiated shapes: (B, rows per thread, threads).  Few threads with many
// rows each: the block-wide reduction of the 3B dot products (warp shuffles,
// then one partial per warp) is the fixed cost of an inner round and grows
// with the number of warps, while the per-row work is a handful of FMAs.
const Variant kVariants[] = {
    {4, 1, 128, bp_round_kernel<4, 1, 128>},   {4, 2, 128, bp_round_kernel<4, 2, 128>},
    {4, 4, 128, bp_round_kernel<4, 4, 128>},   {4, 8, 128, bp_round_kernel<4, 8, 128>},
    {4, 8, 256, bp_round_kernel<4, 8, 256>},   {2, 8, 128, bp_round_kernel<2, 8, 128>},
    {2, 16, 128, bp_round_kernel<2, 16, 128>}, {2, 16, 256, bp_round_kernel<2, 16, 256>},
    {8, 4, 128, bp_round_kernel<8, 4, 128>},
    {2, 2, 512, bp_round_kernel<2, 2, 512>},
};

std::atomic<int> g_force_b{0}, g_force_threads{0};

// The variant for m rows: the forced (B, threads) if one is set and fits,
// else the built-in choice; nullptr when m is too tall for any.
const Variant *pick_variant(size_t m)
{
    const int fb = g_force_b.load(), ft = g_force_threads.load();
    const Variant *best = nullptr;
    if (fb > 0 || ft > 0) {
        for (const Variant &v : kVariants) {
            if ((fb > 0 && v.B != fb) || (ft > 0 && v.threads != ft)) continue;
            if ((size_t)v.rpt * v.threads < m) continue;
            if (best == nullptr || v.rpt < best->rpt) best = &v;  // fewest rows per thread that fit
        }
        if (best) return best;
    }
    auto find = [](int B, int rpt, int threads) -> const Variant * {
        for (const Variant &v : kVariants)
            if (v.B == B && v.rpt == rpt && v.threads == threads) return &v;
        return nullptr;
    };
    if (m <= 128) return find(4, 1, 128);
    if (m <= 256) return find(4, 2, 128);
    if (m <= 512) return find(4, 4, 128);
    if (m <= 1024) return find(4, 8, 128);
    if (m <= 2048) return find(4, 8, 256);
    if (m <= 4096) return find(2, 16, 256);
    return nullptr;
}

struct BpPlan {
    int device = -1;
    size_t m = 0, n = 0;
    const Variant *var = nullptr;
    int nblocks = 0, rounds = 0, npairs = 0;
    double *xw = nullptr, *vw = nullptr, *sig = nullptr;
    int2 *bpairs = nullptr;
    unsigned *counter = nullptr;
    unsigned *h_counter = nullptr;  // pinned
    cudaStream_t alloc_stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    unsigned long long uses = 0;
    size_t bytes = 0;

    ~BpPlan()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        if (h_counter) cudaFreeHost(h_counter);
        if (alloc_stream) {
            if (xw) cudaFreeAsync(xw, alloc_stream);
            if (bpairs) cudaFreeAsync(bpairs, alloc_stream);
            cudaStreamSynchronize(alloc_stream);
            cudaStreamDestroy(alloc_stream);
        }
    }

    int enqueue_rounds(cudaStream_t st)
    {
        for (int r = 0; r < rounds; ++r)
            var->fn<<<npairs, var->threads, 0, st>>>(xw, (int)m, (int)n, vw, bpairs + (size_t)r * npairs, eps_,
                                                     counter);
        JSVD_CUDA_TRY(cudaGetLastError());
        return JSVD_OK;
    }
    double eps_ = 0.0;
};

BpStats &bp_stats_ref()
{
    thread_local BpStats s;
    return s;
}

struct BpCache {
    std::vector<std::unique_ptr<BpPlan>> plans;
};

BpCache &bp_cache()
{
    thread_local BpCache c;
    return c;
}

constexpr size_t kMaxPlans = 4;

int create_plan(int dev, size_t m, size_t n, const Variant *var, std::unique_ptr<BpPlan> &out)
{
    auto plan = std::make_unique<BpPlan>();
    plan->device = dev;
    plan->m = m;
    plan->n = n;
    plan->var = var;
    // The plan owns its allocation stream: plans are cached per thread and may
    // outlive the library's per-thread streams at thread exit.  Every solve
    // synchronises before it returns, so no work of a plan is in flight when
    // it is released.
    {
        const cudaError_t e = cudaStreamCreateWithFlags(&plan->alloc_stream, cudaStreamNonBlocking);
        if (e != cudaSuccess) {
            plan->alloc_stream = nullptr;
            return cuda_failure(e, "cudaStreamCreateWithFlags", __FILE__, __LINE__);
        }
    }
    const int B = var->B;
    plan->nblocks = (int)((n + B - 1) / B);
    const int nbe = plan->nblocks + (plan->nblocks & 1);
    plan->rounds = nbe - 1;
    plan->npairs = nbe / 2;
    std::vector<int2> tab((size_t)plan->rounds * plan->npairs);
    for (int r = 0; r < plan->rounds; ++r)
        for (int k = 0; k < plan->npairs; ++k)
            tab[(size_t)r * plan->npairs + k] = make_int2(circle_at(nbe, r, k), circle_at(nbe, r, nbe - 1 - k));
    // one allocation: x (m n) | v (n n) | sigma (n) | counter
    const size_t doubles = m * n + n * n + n + 1;
    plan->bytes = sizeof(double) * doubles + sizeof(int2) * tab.size();
    JSVD_CUDA_TRY(cudaMallocAsync((void **)&plan->xw, sizeof(double) * doubles, plan->alloc_stream));
    plan->vw = plan->xw + m * n;
    plan->sig = plan->vw + n * n;
    plan->counter = reinterpret_cast<unsigned *>(plan->sig + n);
    JSVD_CUDA_TRY(cudaMallocAsync((void **)&plan->bpairs, sizeof(int2) * tab.size(), plan->alloc_stream));
    JSVD_CUDA_TRY(cudaMemcpyAsync(plan->bpairs, tab.data(), sizeof(int2) * tab.size(), cudaMemcpyHostToDevice,
                                  plan->alloc_stream));
    JSVD_CUDA_TRY(cudaMallocHost((void **)&plan->h_counter, sizeof(unsigned)));
    JSVD_CUDA_TRY(cudaEventCreate(&plan->e0));
    JSVD_CUDA_TRY(cudaEventCreate(&plan->e1));
    JSVD_CUDA_TRY(cudaStreamSynchronize(plan->alloc_stream));
    out = std::move(plan);
    return JSVD_OK;
}

int acquire_plan(size_t m, size_t n, double eps, BpPlan **out)
{
    int dev = 0;
    JSVD_CUDA_TRY(cudaGetDevice(&dev));
    const Variant *var = pick_variant(m);
    if (var == nullptr) return invalid_argument("The block-pair sweep supports at most 4096 rows.");
    auto &plans = bp_cache().plans;
    for (size_t i = 0; i < plans.size(); ++i) {
        BpPlan *p = plans[i].get();
        if (p->device == dev && p->m == m && p->n == n && p->var == var && p->eps_ == eps) {
            std::rotate(plans.begin(), plans.begin() + i, plans.begin() + i + 1);  // most recent first
            *out = plans.front().get();
            return JSVD_OK;
        }
    }
    std::unique_ptr<BpPlan> plan;
    int rc = create_plan(dev, m, n, var, plan);
    if (rc != JSVD_OK) return rc;
    plan->eps_ = eps;  // baked into the captured sweep graph
    plans.insert(plans.begin(), std::move(plan));
    while (plans.size() > kMaxPlans) plans.pop_back();
    *out = plans.front().get();
    return JSVD_OK;
}

// Captures one outer sweep (all outer rounds) into a graph; done on a plan's
// second use, as one-off shapes are not worth the instantiation.
int capture(BpPlan *p, cudaStream_t st)
{
    cudaGraph_t graph = nullptr;
    JSVD_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int rc = p->enqueue_rounds(st);
    cudaError_t cap = cudaStreamEndCapture(st, &graph);
    if (rc != JSVD_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (cap != cudaSuccess) return cuda_failure(cap, "cudaStreamEndCapture", __FILE__, __LINE__);
    cudaError_t inst = cudaGraphInstantiate(&p->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (inst != cudaSuccess) return cuda_failure(inst, "cudaGraphInstantiate", __FILE__, __LINE__);
    return JSVD_OK;
}

}  // namespace

BpStats &bp_stats() { return bp_stats_ref(); }

bool bp_supported(size_t m, size_t n) { return n >= 2 && m >= n && pick_variant(m) != nullptr; }

void bp_set_variant(int block_cols, int threads)
{
    g_force_b.store(block_cols > 0 ? block_cols : 0);
    g_force_threads.store(threads > 0 ? threads : 0);
}

void bp_release_thread_plans() { bp_cache().plans.clear(); }

int bp_solve(const double *d_a, size_t m, size_t n, double eps, int max_sweeps, double *d_u, double *d_sigma,
             double *d_v, int *sweeps, cudaStream_t st)
{
    BpPlan *p = nullptr;
    int rc = acquire_plan(m, n, eps, &p);
    if (rc != JSVD_OK) return rc;
    if (p->uses == 1 && p->exec == nullptr) {
        rc = capture(p, st);
        if (rc != JSVD_OK) return rc;
    }
    const int im = (int)m, in = (int)n;
    dim3 tb(kTile, kTileRows);
    rowmajor_to_colmajor_kernel<<<dim3((in + kTile - 1) / kTile, (im + kTile - 1) / kTile), tb, 0, st>>>(d_a, im, in,
                                                                                                      p->xw, im);
    identity_colmajor_kernel<<<std::min<size_t>(1184, (n * n + 255) / 256), 256, 0, st>>>(p->vw, in, in);
    JSVD_CUDA_TRY(cudaGetLastError());
    BpStats &stt = bp_stats_ref();
    int executed = 0;
    for (int s = 0; s < max_sweeps; ++s) {
        JSVD_CUDA_TRY(cudaMemsetAsync(p->counter, 0, sizeof(unsigned), st));
        JSVD_CUDA_TRY(cudaEventRecord(p->e0, st));
        if (p->exec) {
            JSVD_CUDA_TRY(cudaGraphLaunch(p->exec, st));
        } else {
            rc = p->enqueue_rounds(st);
            if (rc != JSVD_OK) return rc;
        }
        JSVD_CUDA_TRY(cudaEventRecord(p->e1, st));
        JSVD_CUDA_TRY(cudaMemcpyAsync(p->h_counter, p->counter, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
        JSVD_CUDA_TRY(cudaStreamSynchronize(st));
        executed = s + 1;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, p->e0, p->e1) == cudaSuccess) stt.round_ms += ms;
        stt.round_launches += (unsigned long long)p->rounds;
        if (*p->h_counter == 0) break;
    }
    double *sig = d_sigma ? d_sigma : p->sig;
    bp_sigma_kernel<<<(in * 32 + 255) / 256, 256, 0, st>>>(p->xw, im, in, sig);
    if (d_u)
        colmajor_to_rowmajor_kernel<<<dim3((im + kTile - 1) / kTile, (in + kTile - 1) / kTile), tb, 0, st>>>(
            p->xw, im, im, in, d_u, sig, eps);
    if (d_v)
        colmajor_to_rowmajor_kernel<<<dim3((in + kTile - 1) / kTile, (in + kTile - 1) / kTile), tb, 0, st>>>(
            p->vw, in, in, in, d_v, nullptr, 0.0);
    JSVD_CUDA_TRY(cudaGetLastError());
    p->uses += 1;
    stt.solves += 1;
    stt.sweeps += (unsigned long long)executed;
    if (sweeps) *sweeps = executed;
    return JSVD_OK;
}

}  // namespace jsvd

using namespace jsvd;

extern "C" int jsvd_blockpair_svd_device(const double *d_a, size_t rows, size_t columns, const jsvd_config *cfg,
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
        if (!bp_supported(rows, columns))
            return jsvd_plain_svd_device(d_a, rows, columns, &c, d_u, d_sigma, d_v, sweeps, st);
        rc = bp_solve(d_a, rows, columns, c.epsilon, c.max_sweeps, d_u, d_sigma, d_v, sweeps, st);
        if (rc != JSVD_OK) return rc;
        JSVD_CUDA_TRY(cudaStreamSynchronize(st));
        return JSVD_OK;
    });
}

extern "C" int jsvd_blockpair_svd(const double *a, size_t rows, size_t columns, const jsvd_config *cfg, double *u,
                                  double *sigma, double *v, int *sweeps)
{
    return c_entry([&]() -> int {
        return host_buffer_solve(jsvd_blockpair_svd_device, a, rows, columns, cfg, u, sigma, v, sweeps);
    });
}

extern "C" void jsvd_blockpair_set_variant(int block_columns, int threads) { bp_set_variant(block_columns, threads); }

extern "C" void jsvd_blockpair_stats_get(jsvd_blockpair_stats *out)
{
    if (!out) return;
    const BpStats &s = bp_stats_ref();
    out->solves = s.solves;
    out->sweeps = s.sweeps;
    out->round_launches = s.round_launches;
    out->round_ms = s.round_ms;
}

extern "C" void jsvd_blockpair_stats_reset(void) { bp_stats_ref() = BpStats{}; }
