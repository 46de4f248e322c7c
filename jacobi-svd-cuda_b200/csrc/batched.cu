// Batched one-sided Jacobi SVD: thousands of independent small matrices,
// one persistent launch per size class, largest class first (sm_100a).
//
// Each CTA pulls matrix indices from a device work queue (one atomic counter
// per class; matrices sorted by work, largest first) and solves the whole
// matrix before taking the next one.  Where the FP64 working copies live
// depends on the class:
//   class 0-2: A and V in shared memory (<= 48 KiB, <= 100 KiB, <= ~226 KiB)
//   class 3  : A in shared memory, V in a per-CTA slice of global memory
//   class 4  : A and V in global memory (L2-resident per-CTA slices), the
//              leading columns of A that fit in shared memory kept there
// By default the members of classes 3 and 4 are instead solved by a
// thread-block cluster each (batch_cluster_kernel: A and V in the cluster's
// distributed shared memory; see the section "cluster classes"); a member no
// cluster holds stays with its class's kernel.
// Launch shapes per class (threads, CTAs per SM, grid cap) come from the
// compiled-in table batch_tuning_table.h, which batch_autotune.py writes from
// jsvd_batch_autotune (defined at the end of this file).
// Each round runs in three phases separated by __syncthreads:
//   1. one warp per pair: the three dot products, reduced in the reference's
//      order (T = 256 virtual lanes; lane l holds virtual lanes l + 32j, then
//      the halving tree) - so every matrix is bit-identical to the plain path
//      and to the oracle on the same (FP64-promoted) input;
//   2. one thread per pair: the rotation angle (the long sqrt/div chain runs
//      for all pairs of the round in parallel instead of serially per warp);
//   3. one warp per pair: rotation of the A and V columns.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <numeric>
#include <vector>

#include "batch_tuning_table.h"
#include "batched.hpp"
#include "common.cuh"
#include "internal.hpp"
#include "plain.hpp"

namespace jsvd {
namespace {

constexpr int kLanes = 256;      // reduction width T (reference default)
constexpr int kW = kLanes / 32;  // virtual lanes per physical lane
constexpr int kClasses = 5;

// Reference-order dot products of columns x, y (length m) by one warp; the
// totals are valid in lane 0.
__device__ __forceinline__ void warp_pair_stats(const double *x, const double *y, int m, int lane, double &pp,
                                                double &qq, double &pq)
{
    double app[kW], aqq[kW], apq[kW];
#pragma unroll
    for (int j = 0; j < kW; ++j) app[j] = aqq[j] = apq[j] = 0.0;
    for (int base = 0; base < m; base += kLanes) {
#pragma unroll
        for (int j = 0; j < kW; ++j) {
            const int r = base + 32 * j + lane;
            if (r < m) {
                const double a = x[r], b = y[r];
                app[j] = fma(a, a, app[j]);
                aqq[j] = fma(b, b, aqq[j]);
                apq[j] = fma(a, b, apq[j]);
            }
        }
    }
    pp = warp_tree<kW>(app);
    qq = warp_tree<kW>(aqq);
    pq = warp_tree<kW>(apq);
}

// Rotation of one column pair of A (length m) and of V (length n) by one
// warp.  Each 256-row chunk of all four columns is loaded into registers
// before any store: with the working copies in global memory a load -> rotate
// -> store loop pays one L2 round trip per 32 rows, because the compiler cannot
// move a load past a store to a possibly aliasing column.
__device__ __forceinline__ void warp_rotate(double *x, double *y, int m, double *vx, double *vy, int n, int lane,
                                            double c, double s)
{
    const int len = m > n ? m : n;
    for (int base = 0; base < len; base += kLanes) {
        double xa[kW], ya[kW], xv[kW], yv[kW];
#pragma unroll
        for (int j = 0; j < kW; ++j) {
            const int r = base + 32 * j + lane;
            if (r < m) {
                xa[j] = x[r];
                ya[j] = y[r];
            }
            if (r < n) {
                xv[j] = vx[r];
                yv[j] = vy[r];
            }
        }
#pragma unroll
        for (int j = 0; j < kW; ++j) {
            const int r = base + 32 * j + lane;
            if (r < m) {
                x[r] = rot_p(c, s, xa[j], ya[j]);
                y[r] = rot_q(c, s, xa[j], ya[j]);
            }
            if (r < n) {
                vx[r] = rot_p(c, s, xv[j], yv[j]);
                vy[r] = rot_q(c, s, xv[j], yv[j]);
            }
        }
    }
}

__device__ __forceinline__ double warp_norm2(const double *x, int m, int lane)
{
    double acc[kW];
#pragma unroll
    for (int j = 0; j < kW; ++j) acc[j] = 0.0;
    for (int base = 0; base < m; base += kLanes) {
#pragma unroll
        for (int j = 0; j < kW; ++j) {
            const int r = base + 32 * j + lane;
            if (r < m) acc[j] = fma(x[r], x[r], acc[j]);
        }
    }
    return __shfl_sync(0xffffffffu, warp_tree<kW>(acc), 0);
}

// Per-round scratch (pair statistics and angles): `half` is n/2 rounded up to
// an even count so the double2 angle array starts on a 16-byte boundary.
__host__ __device__ constexpr int round_half(int n) { return (n / 2 + 2) & ~1; }
__host__ __device__ constexpr size_t round_scratch_doubles(int n) { return (size_t)5 * round_half(n); }

// One sweep (every round of the circle) of an m x n member whose columns
// colA(c) and V live wherever the caller keeps them, by the whole CTA; true
// when some pair rotated.  s_rot must be 0 on entry and is 0 again on return.
// The same phases and operations as one sweep of batch_kernel (which keeps
// its own copy of the loop: sharing it raised that kernel's register spills).
template <class ColA>
__device__ __forceinline__ bool batch_sweep(ColA colA, double *V, int m, int n, double eps, double *st_pp,
                                            double *st_qq, double *st_pq, double2 *st_cs, int &s_rot)
{
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int ne = n + (n & 1);
    const int rounds = n >= 2 ? ne - 1 : 0;
    const int npairs = n / 2;
    for (int r = 0; r < rounds; ++r) {
        // phase 1: dot products, one warp per pair
        for (int k = warp; k < npairs; k += nwarps) {
            const int2 pq = round_robin_pair(n, r, k);
            double pp, qq, pqv;
            warp_pair_stats(colA(pq.x), colA(pq.y), m, lane, pp, qq, pqv);
            if (lane == 0) {
                st_pp[k] = pp;
                st_qq[k] = qq;
                st_pq[k] = pqv;
            }
        }
        __syncthreads();
        // phase 2: angles, one thread per pair
        for (int k = threadIdx.x; k < npairs; k += blockDim.x) {
            double c, s;
            if (rotation_params(st_pp[k], st_qq[k], st_pq[k], eps, c, s)) s_rot = 1;
            st_cs[k] = make_double2(c, s);
        }
        __syncthreads();
        // phase 3: rotations, one warp per pair
        for (int k = warp; k < npairs; k += nwarps) {
            const double2 g = st_cs[k];
            if (g.x == 0.0) continue;
            const int2 pq = round_robin_pair(n, r, k);
            warp_rotate(colA(pq.x), colA(pq.y), m, V + (size_t)pq.x * n, V + (size_t)pq.y * n, n, lane, g.x, g.y);
        }
        __syncthreads();
    }
    const bool any = s_rot != 0;
    __syncthreads();  // every thread has read the flag before it is reset
    if (threadIdx.x == 0) s_rot = 0;
    return any;
}

template <bool kAShared, bool kVShared>
__global__ void __launch_bounds__(512) batch_kernel(const BatchDesc *__restrict__ descs, int count,
                                                    int *__restrict__ next, const void *__restrict__ a_all,
                                                    int a_is_f32, double eps, int max_sweeps,
                                                    double *__restrict__ sigma_all, double *__restrict__ v_all,
                                                    double *__restrict__ u_all, int *__restrict__ sweeps_all,
                                                    double *__restrict__ workspace, size_t ws_stride,
                                                    int smem_doubles)
{
    // A and V in global memory: the leading columns of A that fit the shared
    // memory left over live there instead (a pair reads its columns from
    // whichever space holds them).
    constexpr bool kHybrid = !kAShared && !kVShared;
    extern __shared__ double smem[];
    __shared__ int s_idx;
    __shared__ int s_rot;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    double *gws = workspace + (size_t)blockIdx.x * ws_stride;
    for (;;) {
        if (threadIdx.x == 0) s_idx = atomicAdd(next, 1);
        __syncthreads();
        const int idx = s_idx;
        if (idx >= count) return;
        const BatchDesc d = descs[idx];
        const int m = d.m, n = d.n;
        const int half = round_half(n);
        // smem layout: [round scratch 5*half][A if shared][V if shared]
        double *st_pp = smem, *st_qq = smem + half, *st_pq = smem + 2 * half;
        double2 *st_cs = reinterpret_cast<double2 *>(smem + 3 * half);  // 2*half doubles, 16-byte aligned
        double *sm_rest = smem + round_scratch_doubles(n);
        double *A = kAShared ? sm_rest : gws;
        double *V = kVShared ? (kAShared ? sm_rest + (size_t)m * n : gws + (size_t)m * n)
                             : (kAShared ? gws : gws + (size_t)m * n);
        // columns 0 .. ks-1 of A in shared memory, ks .. n-1 in the global slice
        const int ks = kHybrid ? max(0, min(n, (smem_doubles - (int)round_scratch_doubles(n)) / m)) : 0;
        auto colA = [&](int c) -> double * {
            if constexpr (kHybrid) return c < ks ? sm_rest + (size_t)c * m : gws + (size_t)(c - ks) * m;
            else return A + (size_t)c * m;
        };
        const size_t mn = (size_t)m * n;
        if (a_is_f32) {
            const float *src = reinterpret_cast<const float *>(a_all) + d.a_off;
            for (size_t e = threadIdx.x; e < mn; e += blockDim.x) {
                const size_t r = e / n, c = e - r * n;
                colA((int)c)[r] = (double)src[e];
            }
        } else {
            const double *src = reinterpret_cast<const double *>(a_all) + d.a_off;
            for (size_t e = threadIdx.x; e < mn; e += blockDim.x) {
                const size_t r = e / n, c = e - r * n;
                colA((int)c)[r] = src[e];
            }
        }
        for (size_t e = threadIdx.x; e < (size_t)n * n; e += blockDim.x) V[e] = (e / n == e % n) ? 1.0 : 0.0;
        if (threadIdx.x == 0) s_rot = 0;
        __syncthreads();
        const int ne = n + (n & 1);
        const int rounds = n >= 2 ? ne - 1 : 0;
        const int npairs = n / 2;
        int sweeps = 1;
        if (rounds > 0) {
            for (int sw = 0; sw < max_sweeps; ++sw) {
                for (int r = 0; r < rounds; ++r) {
                    // phase 1: dot products, one warp per pair
                    for (int k = warp; k < npairs; k += nwarps) {
                        const int2 pq = round_robin_pair(n, r, k);
                        double pp, qq, pqv;
                        warp_pair_stats(colA(pq.x), colA(pq.y), m, lane, pp, qq, pqv);
                        if (lane == 0) {
                            st_pp[k] = pp;
                            st_qq[k] = qq;
                            st_pq[k] = pqv;
                        }
                    }
                    __syncthreads();
                    // phase 2: angles, one thread per pair
                    for (int k = threadIdx.x; k < npairs; k += blockDim.x) {
                        double c, s;
                        if (rotation_params(st_pp[k], st_qq[k], st_pq[k], eps, c, s)) s_rot = 1;
                        st_cs[k] = make_double2(c, s);
                    }
                    __syncthreads();
                    // phase 3: rotations, one warp per pair
                    for (int k = warp; k < npairs; k += nwarps) {
                        const double2 g = st_cs[k];
                        if (g.x == 0.0) continue;
                        const int2 pq = round_robin_pair(n, r, k);
                        warp_rotate(colA(pq.x), colA(pq.y), m, V + (size_t)pq.x * n,
                                    V + (size_t)pq.y * n, n, lane, g.x, g.y);
                    }
                    __syncthreads();
                }
                const bool any = s_rot != 0;
                __syncthreads();  // every thread has read the flag before it is reset
                if (threadIdx.x == 0) s_rot = 0;
                sweeps = sw + 1;
                if (!any) break;
            }
        }
        // sigma, U (optional), V (row-major)
        double *sg = sigma_all + d.s_off;
        for (int c = warp; c < n; c += nwarps) {
            const double *x = colA(c);
            const double sc = sqrt(fmax(warp_norm2(x, m, lane), 0.0));
            if (lane == 0) sg[c] = sc;
            if (u_all != nullptr) {
                double *u = u_all + d.u_off;
                for (int i = lane; i < m; i += 32) u[(size_t)i * n + c] = (sc > eps) ? (x[i] / sc) : 0.0;
            }
        }
        if (v_all != nullptr) {
            double *vo = v_all + d.v_off;
            for (size_t e = threadIdx.x; e < (size_t)n * n; e += blockDim.x) {
                const size_t r = e / n, c = e - r * n;
                vo[e] = V[c * n + r];
            }
        }
        if (sweeps_all != nullptr && threadIdx.x == 0) sweeps_all[idx] = sweeps;
        __syncthreads();  // the working copies are reused by the next matrix
    }
}

// One sweep step of the sweep-granular batch (serving core): CTA i runs one
// sweep of member i, whose state (A and V, FP64, column-major) stays in
// global memory between steps.  On its first step (in != null) a member
// starts from its row-major FP64 input with V = I, as batch_kernel does.  A
// is worked on in shared memory, and V too when kVShared (else in place in
// the state).  rotated[i] = 1 when some pair of the sweep rotated: a member
// whose sweep did not rotate has converged, exactly where batch_kernel's
// loop over sweeps stops.
template <bool kVShared>
__global__ void __launch_bounds__(256, 2) batch_step_kernel(const StepDesc *__restrict__ descs, double eps,
                                                            int *__restrict__ rotated)
{
    extern __shared__ double smem[];
    __shared__ int s_rot;
    const StepDesc d = descs[blockIdx.x];
    const int m = d.m, n = d.n;
    const int half = round_half(n);
    double *st_pp = smem, *st_qq = smem + half, *st_pq = smem + 2 * half;
    double2 *st_cs = reinterpret_cast<double2 *>(smem + 3 * half);
    double *A = smem + round_scratch_doubles(n);
    double *gA = d.a, *gV = d.v;
    double *V = kVShared ? A + (size_t)m * n : gV;
    const size_t mn = (size_t)m * n, nn = (size_t)n * n;
    if (d.in != nullptr) {
        const double *src = d.in;
        for (size_t e = threadIdx.x; e < mn; e += blockDim.x) {
            const size_t r = e / n, c = e - r * n;
            A[c * m + r] = src[e];
        }
        for (size_t e = threadIdx.x; e < nn; e += blockDim.x) V[e] = (e / n == e % n) ? 1.0 : 0.0;
    } else {
        for (size_t e = threadIdx.x; e < mn; e += blockDim.x) A[e] = gA[e];
        if (kVShared)
            for (size_t e = threadIdx.x; e < nn; e += blockDim.x) V[e] = gV[e];
    }
    if (threadIdx.x == 0) s_rot = 0;
    __syncthreads();
    bool any = false;
    if (n >= 2) any = batch_sweep([&](int c) { return A + (size_t)c * m; }, V, m, n, eps, st_pp, st_qq, st_pq, st_cs, s_rot);
    for (size_t e = threadIdx.x; e < mn; e += blockDim.x) gA[e] = A[e];
    if (kVShared)
        for (size_t e = threadIdx.x; e < nn; e += blockDim.x) gV[e] = V[e];
    if (threadIdx.x == 0) rotated[blockIdx.x] = any ? 1 : 0;
}

// Outputs of retired members of the sweep-granular batch: sigma, V
// (row-major) and optionally U (row-major) from the state, with
// batch_kernel's formulas (CTA i: member i).
__global__ void __launch_bounds__(256) batch_finish_kernel(const StepDesc *__restrict__ descs, double eps)
{
    const StepDesc d = descs[blockIdx.x];
    const int m = d.m, n = d.n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const double *gA = d.a, *gV = d.v;
    double *sg = d.s_out;
    for (int c = warp; c < n; c += nwarps) {
        const double *x = gA + (size_t)c * m;
        const double sc = sqrt(fmax(warp_norm2(x, m, lane), 0.0));
        if (lane == 0) sg[c] = sc;
        if (d.u_out != nullptr) {
            double *u = d.u_out;
            for (int i = lane; i < m; i += 32) u[(size_t)i * n + c] = (sc > eps) ? (x[i] / sc) : 0.0;
        }
    }
    double *vo = d.v_out;
    for (size_t e = threadIdx.x; e < (size_t)n * n; e += blockDim.x) {
        const size_t r = e / n, c = e - r * n;
        vo[e] = gV[c * n + r];
    }
}

// ---- cluster classes ----------------------------------------------------------
// A member whose A and V do not fit one CTA's shared memory is solved by a
// cluster of C CTAs (C = 2, 4, 8) with A and V spread over the cluster's
// distributed shared memory, laid out as the round-robin circle itself.
// CTA i owns the contiguous pair slots [k0, k1) of the circle (slot k =
// positions k and ne-1-k, the pair (top, bottom)) and one warp works a slot.
// Between rounds the top row moves one slot right and the bottom row one slot
// left (position 0 stays; ne-1 goes to 1, half-1 to half), so inside a CTA no
// column moves at all: the top slots live in a ring of S+1 column buffers
// indexed (j - g) mod (S+1) at round g, the bottom slots in a ring indexed
// (j + g) mod (S+1), and the spare buffer of each ring receives the one
// column that arrives for round g+1.  Per round a CTA sends two columns: its
// last top column to the right neighbour's spare top buffer and its first
// bottom column to the left neighbour's spare bottom buffer (both written
// straight from the rotation's registers over distributed shared memory; the
// two end CTAs send one of them to themselves).  One cluster barrier per
// round.  A buffer holds a column of A (m) followed by the same column of V
// (n), rotated together.  Pair arithmetic is batch_kernel's (warp-per-pair
// dot products in the T = 256 order, Rutishauser angle, rot_p / rot_q), so
// every member stays bit-identical to the plain path.

constexpr int kClusterThreads = 512;
constexpr int kClusterSlotsPerWarp = 4;  // a CTA holds at most 4 * 16 pair slots

__host__ __device__ constexpr int cluster_slots_max(int n, int C) { return ((n + (n & 1)) / 2 + C - 1) / C; }

// Column buffer length: A's m rows, then V's n rows, padded to whole warps
// (the padding rows are rotated and moved like the others and never read).
__host__ __device__ constexpr int cluster_ld(int m, int n) { return (m + n + 31) & ~31; }

// Shared memory of one CTA: column 0's fixed buffer and two rings.
__host__ __device__ constexpr size_t cluster_smem_bytes(int m, int n, int C)
{
    return sizeof(double) * (size_t)(2 * cluster_slots_max(n, C) + 3) * (size_t)cluster_ld(m, n);
}

__device__ __forceinline__ int pmod(int a, int b)
{
    const int r = a % b;
    return r < 0 ? r + b : r;
}

// Address of this CTA's shared-memory location `p` in the shared memory of
// CTA `rank` of the cluster (a shared::cluster address).
__device__ __forceinline__ uint32_t cluster_addr(const void *p, int rank)
{
    uint32_t out;
    const uint32_t a = static_cast<uint32_t>(__cvta_generic_to_shared(p));
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(out) : "r"(a), "r"(rank));
    return out;
}

__device__ __forceinline__ void st_cluster(uint32_t addr, double v)
{
    asm volatile("st.shared::cluster.f64 [%0], %1;" ::"r"(addr), "d"(v) : "memory");
}

// Rotation of a column pair held in this CTA's buffers (x, y: ld rows, a
// multiple of 32), written to (xo, yo): shared::cluster addresses of the same
// buffers or of a neighbour's.  Every 256-row chunk is loaded before it is
// stored, so in-place use is safe.  c = 0: the columns are only moved.
__device__ __forceinline__ void warp_rotate_cl(const double *x, const double *y, uint32_t xo, uint32_t yo, int ld,
                                               int lane, double c, double s, bool rotate)
{
    int r0 = 0;
    for (; r0 + kLanes <= ld; r0 += kLanes) {
        double xa[kW], ya[kW];
#pragma unroll
        for (int j = 0; j < kW; ++j) {
            xa[j] = x[r0 + 32 * j + lane];
            ya[j] = y[r0 + 32 * j + lane];
        }
#pragma unroll
        for (int j = 0; j < kW; ++j) {
            const uint32_t off = 8u * (uint32_t)(r0 + 32 * j + lane);
            st_cluster(xo + off, rotate ? rot_p(c, s, xa[j], ya[j]) : xa[j]);
            st_cluster(yo + off, rotate ? rot_q(c, s, xa[j], ya[j]) : ya[j]);
        }
    }
    for (; r0 < ld; r0 += 32) {
        const double xv = x[r0 + lane], yv = y[r0 + lane];
        const uint32_t off = 8u * (uint32_t)(r0 + lane);
        st_cluster(xo + off, rotate ? rot_p(c, s, xv, yv) : xv);
        st_cluster(yo + off, rotate ? rot_q(c, s, xv, yv) : yv);
    }
}

// Moves one column (ld rows) to a shared::cluster address.
__device__ __forceinline__ void warp_move_cl(const double *x, uint32_t xo, int ld, int lane)
{
    for (int r = lane; r < ld; r += 32) st_cluster(xo + 8u * (uint32_t)r, x[r]);
}

template <int C>
__global__ void __launch_bounds__(kClusterThreads, 1)
    batch_cluster_kernel(const BatchDesc *__restrict__ descs, int count, int *__restrict__ next,
                         const void *__restrict__ a_all, int a_is_f32, double eps, int max_sweeps,
                         double *__restrict__ sigma_all, double *__restrict__ v_all, double *__restrict__ u_all,
                         int *__restrict__ sweeps_all)
{
    namespace cg = cooperative_groups;
    extern __shared__ double smem[];
    __shared__ int s_idx;
    __shared__ int s_rot;
    __shared__ unsigned long long s_stamp;  // rank 0's copy: last (member, sweep) stamp that rotated
    cg::cluster_group cluster = cg::this_cluster();
    const int rank = (int)cluster.block_rank();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const int *idx0 = cluster.map_shared_rank(&s_idx, 0);
    unsigned long long *stamp0 = cluster.map_shared_rank(&s_stamp, 0);
    // shared::cluster addresses of the start of the dynamic shared memory:
    // this CTA's own and its neighbours' (same layout in every CTA)
    const uint32_t sm_self = cluster_addr(smem, rank);
    const uint32_t sm_right = cluster_addr(smem, rank < C - 1 ? rank + 1 : rank);
    const uint32_t sm_left = cluster_addr(smem, rank > 0 ? rank - 1 : rank);
    if (threadIdx.x == 0) {
        s_rot = 0;
        s_stamp = 0;
    }
    for (;;) {
        if (rank == 0 && threadIdx.x == 0) s_idx = atomicAdd(next, 1);
        cluster.sync();  // (the first one also orders the initialisation above)
        const int idx = *(volatile const int *)idx0;
        // every CTA has read the index and finished the previous member's
        // outputs before any CTA writes into another's buffers or exits
        cluster.sync();
        if (idx >= count) return;
        const BatchDesc d = descs[idx];
        const int m = d.m, n = d.n;
        const int ne = n + (n & 1), half = ne / 2, L = ne - 1;
        const int rounds = n >= 2 ? L : 0;
        const int ld = cluster_ld(m, n);
        const int smax = cluster_slots_max(n, C);
        const int k0 = rank * half / C, k1 = (rank + 1) * half / C, S = k1 - k0;  // S >= 2 (host: half >= 2C)
        // buffers (offsets in doubles): column 0's fixed one (CTA 0 only), the
        // top ring, the bottom ring
        const int top_off = ld, bot_off = (smax + 2) * ld;
        const int jt0 = rank == 0 ? 1 : 0;  // first top slot that moves
        const int rt = S - jt0 + 1, rb = S + 1;
        const int s_right = rank < C - 1 ? (rank + 2) * half / C - k1 : 0;
        const int s_left = rank > 0 ? k0 - (rank - 1) * half / C : 0;
        // top slot j is in top buffer (j - jt0 - g) mod rt at round g, bottom
        // slot j in bottom buffer (j + g) mod rb
        auto top_at = [&](int j, int g) { return (rank == 0 && j == 0) ? 0 : top_off + pmod(j - jt0 - g, rt) * ld; };
        auto bot_at = [&](int j, int g) { return bot_off + pmod(j + g, rb) * ld; };
        // round 0: position p holds column p; V = I
        const int ncl = 2 * S;
        for (int e = threadIdx.x; e < m * ncl; e += blockDim.x) {
            const int row = e / ncl, cc = e - row * ncl;
            const int j = cc < S ? cc : cc - S;
            const int col = cc < S ? k0 + j : ne - 1 - (k0 + j);
            if (col >= n) continue;  // the dummy column of an odd n
            const size_t src = (size_t)d.a_off + (size_t)row * n + col;
            smem[(cc < S ? top_at(j, 0) : bot_at(j, 0)) + row] =
                a_is_f32 ? (double)reinterpret_cast<const float *>(a_all)[src]
                         : reinterpret_cast<const double *>(a_all)[src];
        }
        for (int e = threadIdx.x; e < n * ncl; e += blockDim.x) {
            const int row = e / ncl, cc = e - row * ncl;
            const int j = cc < S ? cc : cc - S;
            const int col = cc < S ? k0 + j : ne - 1 - (k0 + j);
            if (col >= n) continue;
            smem[(cc < S ? top_at(j, 0) : bot_at(j, 0)) + m + row] = row == col ? 1.0 : 0.0;
        }
        __syncthreads();
        // This warp's slots j = warp + t * nwarps, tracked from round to round:
        // the circle values at their two positions (n = the dummy) and their
        // ring buffers.  Position values fall by one per round (1 -> L).
        int pv[kClusterSlotsPerWarp], qv[kClusterSlotsPerWarp], tb[kClusterSlotsPerWarp], bb[kClusterSlotsPerWarp];
#pragma unroll
        for (int t = 0; t < kClusterSlotsPerWarp; ++t) {
            const int j = warp + t * nwarps, k = k0 + j;
            pv[t] = k;
            qv[t] = ne - 1 - k;
            tb[t] = (rank == 0 && j == 0) ? -1 : j - jt0;
            bb[t] = j;
        }
        // ring buffers that receive this CTA's outgoing columns in round g:
        // the right neighbour's spare top buffer (the last CTA: its own spare
        // bottom one) and the left neighbour's spare bottom buffer (CTA 0: its
        // own spare top one)
        int o_top = rank < C - 1 ? s_right : S;
        int o_bot = rank > 0 ? s_left : rt - 1;
        int g = 0, sweeps = 1;
        if (rounds > 0) {
            for (int sw = 0; sw < max_sweeps; ++sw) {
                for (int r = 0; r < rounds; ++r, ++g) {
#pragma unroll
                    for (int t = 0; t < kClusterSlotsPerWarp; ++t) {
                        const int j = warp + t * nwarps;
                        if (j < S) {
                            const int xo = tb[t] < 0 ? 0 : top_off + tb[t] * ld;
                            const int yo = bot_off + bb[t] * ld;
                            const double *xt = smem + xo;
                            const double *xb = smem + yo;
                            const uint32_t dt = j == S - 1
                                                    ? (rank < C - 1 ? sm_right + 8u * (uint32_t)(top_off + o_top * ld)
                                                                    : sm_self + 8u * (uint32_t)(bot_off + o_top * ld))
                                                    : sm_self + 8u * (uint32_t)xo;
                            const uint32_t db = j == 0
                                                    ? (rank > 0 ? sm_left + 8u * (uint32_t)(bot_off + o_bot * ld)
                                                                : sm_self + 8u * (uint32_t)(top_off + o_bot * ld))
                                                    : sm_self + 8u * (uint32_t)yo;
                            const bool real = pv[t] != n && qv[t] != n;
                            double c = 0.0, s = 0.0;
                            if (real) {
                                double pp, qq, pqv;
                                warp_pair_stats(xt, xb, m, lane, pp, qq, pqv);
                                if (lane == 0 && rotation_params(pp, qq, pqv, eps, c, s)) s_rot = 1;
                                c = __shfl_sync(0xffffffffu, c, 0);
                                s = __shfl_sync(0xffffffffu, s, 0);
                            }
                            if (c != 0.0) {
                                warp_rotate_cl(xt, xb, dt, db, ld, lane, c, s, true);
                            } else {  // no rotation (or the dummy's slot): the columns only move
                                if (j == S - 1 && pv[t] != n) warp_move_cl(xt, dt, ld, lane);
                                if (j == 0 && qv[t] != n) warp_move_cl(xb, db, ld, lane);
                            }
                            if (pv[t] != 0) pv[t] = pv[t] == 1 ? L : pv[t] - 1;
                            qv[t] = qv[t] == 1 ? L : qv[t] - 1;
                            if (tb[t] >= 0) tb[t] = tb[t] == 0 ? rt - 1 : tb[t] - 1;
                            bb[t] = bb[t] == rb - 1 ? 0 : bb[t] + 1;
                        }
                    }
                    if (rank < C - 1) o_top = o_top == 0 ? s_right : o_top - 1;
                    else o_top = o_top == rb - 1 ? 0 : o_top + 1;
                    if (rank > 0) o_bot = o_bot == s_left ? 0 : o_bot + 1;
                    else o_bot = o_bot == 0 ? rt - 1 : o_bot - 1;
                    cluster.sync();
                }
                // sweep test over the cluster: a CTA that rotated raises rank 0's stamp
                const unsigned long long stamp = (unsigned long long)idx * (unsigned)(max_sweeps + 1) + sw + 1;
                if (threadIdx.x == 0) {
                    if (s_rot) atomicMax(stamp0, stamp);
                    s_rot = 0;
                }
                cluster.sync();
                const bool any = *(volatile const unsigned long long *)stamp0 == stamp;
                sweeps = sw + 1;
                if (!any) break;
            }
        }
        // every sweep is a whole turn of the circle: position p holds column p again
        double *sg = sigma_all + d.s_off;
        for (int cc = warp; cc < ncl; cc += nwarps) {
            const int j = cc < S ? cc : cc - S;
            const int col = cc < S ? k0 + j : ne - 1 - (k0 + j);
            if (col >= n) continue;
            const double *x = smem + (cc < S ? top_at(j, g) : bot_at(j, g));
            const double sc = sqrt(fmax(warp_norm2(x, m, lane), 0.0));
            if (lane == 0) sg[col] = sc;
            if (u_all != nullptr) {
                double *u = u_all + d.u_off;
                for (int i = lane; i < m; i += 32) u[(size_t)i * n + col] = (sc > eps) ? (x[i] / sc) : 0.0;
            }
            if (v_all != nullptr) {
                double *vo = v_all + d.v_off;
                for (int i = lane; i < n; i += 32) vo[(size_t)i * n + col] = x[m + i];
            }
        }
        if (rank == 0 && threadIdx.x == 0 && sweeps_all != nullptr) sweeps_all[idx] = sweeps;
    }
}

using ClusterFn = void (*)(const BatchDesc *, int, int *, const void *, int, double, int, double *, double *, double *,
                           int *);

ClusterFn cluster_fn(int C)
{
    return C == 2 ? batch_cluster_kernel<2> : (C == 4 ? batch_cluster_kernel<4> : batch_cluster_kernel<8>);
}

// Size classes whose members go to clusters where one fits (bit c = class c;
// classes 2-4 only), initially the compiled-in tuning table's choice.
// Process-wide.
#ifndef JSVD_BATCH_CLUSTER_CLASSES
#define JSVD_BATCH_CLUSTER_CLASSES ((1 << 3) | (1 << 4))
#endif
std::atomic<int> g_cluster_mask{JSVD_BATCH_CLUSTER_CLASSES};  // the tuning table's choice
int batch_cluster_mask() { return g_cluster_mask.load(std::memory_order_relaxed); }

// Smallest cluster (2, 4, 8 CTAs) whose shared memory holds an m x n member
// with at least two and at most 64 pair slots per CTA; 0 when none does.
int cluster_size_for(int m, int n, size_t smem_cap)
{
    const int half = (n + (n & 1)) / 2;
    for (int C : {2, 4, 8})
        if (half >= 2 * C && cluster_slots_max(n, C) <= kClusterSlotsPerWarp * (kClusterThreads / 32) &&
            cluster_smem_bytes(m, n, C) <= smem_cap)
            return C;
    return 0;
}

using BatchFn = void (*)(const BatchDesc *, int, int *, const void *, int, double, int, double *, double *,
                         double *, int *, double *, size_t, int);

// Per-thread timing events: whole call and one pair per size class.
struct ThreadEvents {
    cudaEvent_t t0 = nullptr, t1 = nullptr;
    cudaEvent_t c0[kClasses] = {}, c1[kClasses] = {};
    int device = -1;
    ~ThreadEvents()
    {
        for (int c = 0; c < kClasses; ++c) {
            if (c0[c]) cudaEventDestroy(c0[c]);
            if (c1[c]) cudaEventDestroy(c1[c]);
        }
        if (t0) cudaEventDestroy(t0);
        if (t1) cudaEventDestroy(t1);
    }
};

int thread_events(int dev, ThreadEvents **out)
{
    thread_local ThreadEvents ts;
    if (ts.device != dev) {
        if (ts.device >= 0) return invalid_argument("The batched solver is bound to the first device it ran on.");
        for (int c = 0; c < kClasses; ++c) {
            JSVD_CUDA_TRY(cudaEventCreate(&ts.c0[c]));
            JSVD_CUDA_TRY(cudaEventCreate(&ts.c1[c]));
        }
        JSVD_CUDA_TRY(cudaEventCreate(&ts.t0));
        JSVD_CUDA_TRY(cudaEventCreate(&ts.t1));
        ts.device = dev;
    }
    *out = &ts;
    return JSVD_OK;
}

constexpr jsvd_batch_tuning kBuiltinTuning[kClasses] = JSVD_BATCH_TUNING_TABLE;

// Where each class keeps its working copies (see the file comment).
constexpr bool class_a_shared(int c) { return c <= 3; }
constexpr bool class_v_shared(int c) { return c <= 2; }

// Largest dynamic shared memory a batch CTA asks for: the opt-in limit less
// 1 KiB for the static variables.
int batch_smem_cap(int dev, size_t *cap)
{
    int smem_optin = 0;
    JSVD_CUDA_TRY(cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    *cap = (size_t)std::min(smem_optin, 227 * 1024) - 1024;
    return JSVD_OK;
}

// Size class of an m x n member and the shared-memory bytes it needs there.
int member_class(int m, int n, size_t smem_cap, size_t *smem_need)
{
    const size_t scratch = sizeof(double) * round_scratch_doubles(n);
    const size_t a_bytes = sizeof(double) * (size_t)m * n, v_bytes = sizeof(double) * (size_t)n * n;
    int c;
    if (scratch + a_bytes + v_bytes <= 48 * 1024) c = 0;
    else if (scratch + a_bytes + v_bytes <= 100 * 1024) c = 1;
    else if (scratch + a_bytes + v_bytes <= smem_cap) c = 2;
    else if (scratch + a_bytes <= smem_cap) c = 3;
    else c = 4;
    if (smem_need)
        *smem_need = scratch + (class_a_shared(c) ? a_bytes : 0) + (class_v_shared(c) ? v_bytes : 0);
    return c;
}

// Work of one member per sweep, ~ n^2 (m + n): the queue order inside a class.
double member_work(int m, int n) { return (double)n * n * (m + n); }

// Argument checks shared by the solver and the autotuner.
int check_batch_args(int count, const int *rows, const int *cols, const long long *a_offsets, const void *d_a,
                     bool sigma_missing, const jsvd_config &c)
{
    if (count < 0) return invalid_argument("count must be non-negative.");
    if (count > 0 && (rows == nullptr || cols == nullptr || a_offsets == nullptr || d_a == nullptr || sigma_missing))
        return invalid_argument("Batch buffers must not be null.");
    if (!(c.epsilon > 0.0)) return invalid_argument("epsilon must be positive.");
    if (c.max_sweeps <= 0) return invalid_argument("max_sweeps must be positive.");
    if (reduction_lanes(c.threads_per_block) != 256)
        return invalid_argument("The batched solver reduces with threads_per_block = 256.");
    return JSVD_OK;
}

}  // namespace

BatchStats &batch_stats()
{
    thread_local BatchStats s;
    return s;
}

int batch_solve(const BatchRequest &req, cudaStream_t stream)
{
    const int count = req.count;
    if (count <= 0) return JSVD_OK;
    int dev = 0;
    JSVD_CUDA_TRY(cudaGetDevice(&dev));
    int sms = 0;
    JSVD_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    size_t smem_cap = 0;
    int rc = batch_smem_cap(dev, &smem_cap);
    if (rc != JSVD_OK) return rc;
    ThreadEvents *ts = nullptr;
    rc = thread_events(dev, &ts);
    if (rc != JSVD_OK) return rc;

    struct Class {
        int threads;
        int ctas_per_sm;
        bool a_shared, v_shared;
        BatchFn fn;
    };
    Class classes[kClasses];
    int max_ctas[kClasses] = {};
    for (int c = 0; c < kClasses; ++c) {
        classes[c].threads = kBuiltinTuning[c].threads;
        classes[c].ctas_per_sm = kBuiltinTuning[c].ctas_per_sm;
        classes[c].a_shared = class_a_shared(c);
        classes[c].v_shared = class_v_shared(c);
        classes[c].fn = c <= 2 ? batch_kernel<true, true>
                               : (c == 3 ? batch_kernel<true, false> : batch_kernel<false, false>);
        max_ctas[c] = kBuiltinTuning[c].max_ctas;
    }
    if (req.tuning != nullptr) {
        for (int c = 0; c < kClasses; ++c) {
            const jsvd_batch_tuning &t = req.tuning[c];
            if (t.threads < 0 || t.threads > 512 || t.threads % 32 != 0 || t.ctas_per_sm < 0 || t.max_ctas < 0)
                return invalid_argument("Batch tuning: threads must be a multiple of 32 up to 512, counts >= 0.");
            if (t.threads > 0) classes[c].threads = t.threads;
            if (t.ctas_per_sm > 0) classes[c].ctas_per_sm = t.ctas_per_sm;
            if (t.threads > 0 || t.ctas_per_sm > 0 || t.max_ctas > 0) max_ctas[c] = t.max_ctas;
        }
    }
    std::vector<std::vector<int>> members(kClasses);
    std::vector<BatchDesc> all(count);
    std::vector<size_t> need_smem(count);
    size_t s_off = 0, v_off = 0, u_off = 0;
    for (int i = 0; i < count; ++i) {
        BatchDesc d;
        d.m = req.rows[i];
        d.n = req.cols[i];
        if (d.m <= 0 || d.n <= 0 || d.m < d.n)
            return invalid_argument("Batch matrix shape must satisfy rows >= columns > 0.");
        if (dims_out_of_range((size_t)d.m, (size_t)d.n)) {
            set_last_error(JSVD_ERR_OVERFLOW, "Matrix dimensions exceed the supported range.");
            return JSVD_ERR_OVERFLOW;
        }
        d.a_off = req.a_offsets[i];
        d.s_off = (long long)s_off;
        d.v_off = (long long)v_off;
        d.u_off = (long long)u_off;
        s_off += d.n;
        v_off += (size_t)d.n * d.n;
        u_off += (size_t)d.m * d.n;
        all[i] = d;
        members[member_class(d.m, d.n, smem_cap, &need_smem[i])].push_back(i);
    }
    // Launch groups in launch order: per class, largest first, the members
    // solved by clusters of 8, 4 and 2 CTAs (classes whose bit is set in the
    // cluster mask), then the rest by the class's own kernel.  Largest work
    // first inside each group (tail balance of the work queue).
    struct Group {
        int cls, csize, first, count;
        size_t smem, gws;
        int grid;
    };
    auto work = [&](int i) { return member_work(all[i].m, all[i].n); };
    const int mask = batch_cluster_mask();
    std::vector<Group> groups;
    std::vector<BatchDesc> ordered;
    ordered.reserve(count);
    std::vector<int> order_index;
    order_index.reserve(count);
    for (int c = kClasses - 1; c >= 0; --c) {
        std::sort(members[c].begin(), members[c].end(), [&](int x, int y) { return work(x) > work(y); });
        std::vector<int> sub[4];  // own kernel, clusters of 2, 4, 8
        for (int i : members[c]) {
            const int C = ((mask >> c) & 1) ? cluster_size_for(all[i].m, all[i].n, smem_cap) : 0;
            sub[C == 0 ? 0 : (C == 2 ? 1 : (C == 4 ? 2 : 3))].push_back(i);
        }
        for (int s : {3, 2, 1, 0}) {
            if (sub[s].empty()) continue;
            Group g{c, s == 0 ? 0 : (1 << s), (int)ordered.size(), (int)sub[s].size(), 0, 0, 0};
            for (int i : sub[s]) {
                ordered.push_back(all[i]);
                order_index.push_back(i);
                if (g.csize > 0) {
                    g.smem = std::max(g.smem, cluster_smem_bytes(all[i].m, all[i].n, g.csize));
                } else {
                    g.smem = std::max(g.smem, need_smem[i]);
                    size_t w = 0;
                    if (!classes[c].a_shared) w += (size_t)all[i].m * all[i].n;
                    if (!classes[c].v_shared) w += (size_t)all[i].n * all[i].n;
                    g.gws = std::max(g.gws, w);
                }
            }
            groups.push_back(g);
        }
    }
    std::vector<size_t> gws_base(groups.size(), 0);
    size_t gws_total = 0;
    for (size_t k = 0; k < groups.size(); ++k) {
        Group &g = groups[k];
        if (g.csize > 0) {
            JSVD_CUDA_TRY(cudaFuncSetAttribute(cluster_fn(g.csize), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem_cap));
            cudaLaunchConfig_t lc = {};
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = (unsigned)g.csize;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            lc.gridDim = dim3((unsigned)g.csize);
            lc.blockDim = dim3(kClusterThreads);
            lc.dynamicSmemBytes = g.smem;
            lc.attrs = at;
            lc.numAttrs = 1;
            int clusters = 0;
            JSVD_CUDA_TRY(cudaOccupancyMaxActiveClusters(&clusters, cluster_fn(g.csize), &lc));
            if (clusters <= 0) {
                set_last_error(JSVD_ERR_RUNTIME, "No cluster of the batched solver fits the device.");
                return JSVD_ERR_RUNTIME;
            }
            g.grid = std::min(g.count, clusters) * g.csize;
        } else {
            const Class &cl = classes[g.cls];
            g.grid = std::min(g.count, sms * cl.ctas_per_sm);
            if (max_ctas[g.cls] > 0) g.grid = std::min(g.grid, max_ctas[g.cls]);
            gws_base[k] = gws_total;
            gws_total += g.gws * (size_t)g.grid;
        }
    }

    BatchDesc *d_desc = nullptr;
    int *d_next = nullptr, *d_sweeps = nullptr;
    double *d_ws = nullptr;
    ScopeExit free_buffers([&] {  // stream-ordered, on every return path
        if (d_desc) cudaFreeAsync(d_desc, stream);
        if (d_next) cudaFreeAsync(d_next, stream);
        if (d_sweeps) cudaFreeAsync(d_sweeps, stream);
        if (d_ws) cudaFreeAsync(d_ws, stream);
    });
    const size_t ngroups = std::max<size_t>(groups.size(), 1);
    JSVD_CUDA_TRY(cudaMallocAsync(&d_desc, sizeof(BatchDesc) * ordered.size(), stream));
    JSVD_CUDA_TRY(cudaMallocAsync(&d_next, sizeof(int) * ngroups, stream));
    JSVD_CUDA_TRY(cudaMallocAsync(&d_sweeps, sizeof(int) * (size_t)count, stream));
    if (gws_total > 0) JSVD_CUDA_TRY(cudaMallocAsync(&d_ws, sizeof(double) * gws_total, stream));
    JSVD_CUDA_TRY(cudaMemcpyAsync(d_desc, ordered.data(), sizeof(BatchDesc) * ordered.size(), cudaMemcpyHostToDevice,
                                  stream));
    JSVD_CUDA_TRY(cudaMemsetAsync(d_next, 0, sizeof(int) * ngroups, stream));
    for (BatchFn fn : {(BatchFn)batch_kernel<true, true>, (BatchFn)batch_kernel<true, false>,
                       (BatchFn)batch_kernel<false, false>})
        JSVD_CUDA_TRY(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_cap));
    JSVD_CUDA_TRY(cudaEventRecord(ts->t0, stream));
    int launches = 0;
    std::vector<int> class_count(kClasses, 0);
    for (size_t k = 0; k < groups.size(); ++k) {
        const Group &g = groups[k];
        const int c = g.cls;
        // The classes run one after another on one stream: persistent CTAs of
        // a class hold their SMs until its queue drains, and concurrent classes
        // starved each other (a 512-thread CTA of the global class fills an
        // SM's register file).
        if (k == 0 || groups[k - 1].cls != c) JSVD_CUDA_TRY(cudaEventRecord(ts->c0[c], stream));
        class_count[c] += g.count;
        if (g.csize > 0) {
            cudaLaunchConfig_t lc = {};
            cudaLaunchAttribute at[1];
            at[0].id = cudaLaunchAttributeClusterDimension;
            at[0].val.clusterDim.x = (unsigned)g.csize;
            at[0].val.clusterDim.y = 1;
            at[0].val.clusterDim.z = 1;
            lc.gridDim = dim3((unsigned)g.grid);
            lc.blockDim = dim3(kClusterThreads);
            lc.dynamicSmemBytes = g.smem;
            lc.stream = stream;
            lc.attrs = at;
            lc.numAttrs = 1;
            JSVD_CUDA_TRY(cudaLaunchKernelEx(&lc, cluster_fn(g.csize), (const BatchDesc *)(d_desc + g.first), g.count,
                                             d_next + k, req.a, req.a_is_f32, req.eps, req.max_sweeps, req.sigma,
                                             req.v, req.u, d_sweeps + g.first));
        } else {
            const Class &cl = classes[c];
            // The global class keeps leading columns of A in the shared memory left over.
            const size_t dyn = (!cl.a_shared && !cl.v_shared) ? (smem_cap & ~(size_t)7) : g.smem;
            cl.fn<<<g.grid, cl.threads, dyn, stream>>>(d_desc + g.first, g.count, d_next + k, req.a, req.a_is_f32,
                                                       req.eps, req.max_sweeps, req.sigma, req.v, req.u,
                                                       d_sweeps + g.first, d_ws + gws_base[k], g.gws,
                                                       (int)(dyn / sizeof(double)));
            JSVD_CUDA_TRY(cudaGetLastError());
        }
        if (k + 1 == groups.size() || groups[k + 1].cls != c) JSVD_CUDA_TRY(cudaEventRecord(ts->c1[c], stream));
        ++launches;
    }
    JSVD_CUDA_TRY(cudaEventRecord(ts->t1, stream));
    std::vector<int> h_sweeps(count);
    JSVD_CUDA_TRY(cudaMemcpyAsync(h_sweeps.data(), d_sweeps, sizeof(int) * count, cudaMemcpyDeviceToHost, stream));
    JSVD_CUDA_TRY(cudaStreamSynchronize(stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, ts->t0, ts->t1);
    BatchStats &st = batch_stats();
    st.calls += 1;
    st.launches += (unsigned long long)launches;
    st.kernel_ms += ms;
    unsigned long long total_sweeps = 0;
    for (int p = 0; p < count; ++p) {
        total_sweeps += (unsigned long long)h_sweeps[p];
        if (req.sweeps) req.sweeps[order_index[p]] = h_sweeps[p];
    }
    st.sweeps += total_sweeps;
    st.matrices += (unsigned long long)count;
    for (int c = 0; c < kClasses; ++c) {
        st.class_count[c] += (unsigned long long)class_count[c];
        float cms = 0.f;
        if (class_count[c] > 0 && cudaEventElapsedTime(&cms, ts->c0[c], ts->c1[c]) == cudaSuccess)
            st.class_ms[c] += cms;
    }
    return JSVD_OK;
}

}  // namespace jsvd

using namespace jsvd;

namespace jsvd {

size_t step_smem(int m, int n, bool v_shared)
{
    return sizeof(double) * (round_scratch_doubles(n) + (size_t)m * n + (v_shared ? (size_t)n * n : 0));
}

bool step_fits(int m, int n, size_t *smem_cap_out)
{
    int dev = 0;
    size_t cap = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || batch_smem_cap(dev, &cap) != JSVD_OK) return false;
    if (smem_cap_out) *smem_cap_out = cap;
    return step_smem(m, n, false) <= cap;
}

int StepScratch::ensure(int count)
{
    if (count <= cap) return JSVD_OK;
    if (d_descs) cudaFree(d_descs);
    if (d_rot) cudaFree(d_rot);
    if (h_rot) cudaFreeHost(h_rot);
    d_descs = nullptr;
    d_rot = nullptr;
    h_rot = nullptr;
    cap = 0;
    const int c = std::max(count, 256);
    JSVD_CUDA_TRY(cudaMalloc((void **)&d_descs, sizeof(StepDesc) * 2 * c));
    JSVD_CUDA_TRY(cudaMalloc((void **)&d_rot, sizeof(int) * c));
    JSVD_CUDA_TRY(cudaMallocHost((void **)&h_rot, sizeof(int) * c));
    cap = c;
    return JSVD_OK;
}

StepScratch::~StepScratch()
{
    if (d_descs) cudaFree(d_descs);
    if (d_rot) cudaFree(d_rot);
    if (h_rot) cudaFreeHost(h_rot);
}

int batch_step(const std::vector<StepDesc> &descs, double eps, int *rotated, StepScratch &sc, cudaStream_t st)
{
    const int count = (int)descs.size();
    if (count == 0) return JSVD_OK;
    int dev = 0;
    size_t cap = 0;
    JSVD_CUDA_TRY(cudaGetDevice(&dev));
    if (int rc = batch_smem_cap(dev, &cap); rc != JSVD_OK) return rc;
    if (int rc = sc.ensure(count); rc != JSVD_OK) return rc;
    // members whose V fits beside A in shared memory first, the others after
    std::vector<int> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_partition(order.begin(), order.end(),
                          [&](int i) { return step_smem(descs[i].m, descs[i].n, true) <= cap; });
    std::vector<StepDesc> sorted(count);
    size_t smem_vs = 0, smem_vg = 0;
    int n_vs = 0;
    for (int i = 0; i < count; ++i) {
        const StepDesc &d = descs[order[i]];
        sorted[i] = d;
        if (step_smem(d.m, d.n, true) <= cap) {
            smem_vs = std::max(smem_vs, step_smem(d.m, d.n, true));
            ++n_vs;
        } else {
            if (step_smem(d.m, d.n, false) > cap) return invalid_argument("A step member does not fit shared memory.");
            smem_vg = std::max(smem_vg, step_smem(d.m, d.n, false));
        }
    }
    JSVD_CUDA_TRY(cudaMemcpyAsync(sc.d_descs, sorted.data(), sizeof(StepDesc) * count, cudaMemcpyHostToDevice, st));
    static thread_local unsigned long long attr_done = 0;
    if (dev < 64 && !(attr_done & (1ull << dev))) {
        JSVD_CUDA_TRY(cudaFuncSetAttribute(batch_step_kernel<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)cap));
        JSVD_CUDA_TRY(cudaFuncSetAttribute(batch_step_kernel<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           (int)cap));
        attr_done |= 1ull << dev;
    }
    if (n_vs > 0) batch_step_kernel<true><<<n_vs, 256, smem_vs, st>>>(sc.d_descs, eps, sc.d_rot);
    if (count > n_vs)
        batch_step_kernel<false><<<count - n_vs, 256, smem_vg, st>>>(sc.d_descs + n_vs, eps, sc.d_rot + n_vs);
    JSVD_CUDA_TRY(cudaGetLastError());
    JSVD_CUDA_TRY(cudaMemcpyAsync(sc.h_rot, sc.d_rot, sizeof(int) * count, cudaMemcpyDeviceToHost, st));
    JSVD_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < count; ++i) rotated[order[i]] = sc.h_rot[i];
    return JSVD_OK;
}

int batch_finish(const std::vector<StepDesc> &descs, double eps, StepScratch &sc, cudaStream_t st)
{
    const int count = (int)descs.size();
    if (count == 0) return JSVD_OK;
    if (int rc = sc.ensure(count); rc != JSVD_OK) return rc;
    StepDesc *d2 = sc.d_descs + sc.cap;  // the second half: the step's descriptors may still be read
    JSVD_CUDA_TRY(cudaMemcpyAsync(d2, descs.data(), sizeof(StepDesc) * count, cudaMemcpyHostToDevice, st));
    batch_finish_kernel<<<count, 256, 0, st>>>(d2, eps);
    JSVD_CUDA_TRY(cudaGetLastError());
    return JSVD_OK;
}

}  // namespace jsvd

using namespace jsvd;

extern "C" int jsvd_batch_svd_device(int count, const int *rows, const int *cols, const long long *a_offsets,
                                     const void *d_a, int a_is_f32, const jsvd_config *cfg, double *d_sigma,
                                     double *d_v, double *d_u, int *sweeps, const jsvd_batch_tuning *tuning,
                                     void *stream)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        jsvd_config def;
        const jsvd_config &c = config_or_default(cfg, def);
        const int bad = check_batch_args(count, rows, cols, a_offsets, d_a, d_sigma == nullptr, c);
        if (bad != JSVD_OK) return bad;
        if (count == 0) return JSVD_OK;  // nothing to solve, no CUDA call
        cudaStream_t st = nullptr;
        if (const int e = entry_stream(stream, &st); e != JSVD_OK) return e;
        BatchRequest req;
        req.count = count;
        req.rows = rows;
        req.cols = cols;
        req.a_offsets = a_offsets;
        req.a = d_a;
        req.a_is_f32 = a_is_f32;
        req.eps = c.epsilon;
        req.max_sweeps = c.max_sweeps;
        req.sigma = d_sigma;
        req.v = d_v;
        req.u = d_u;
        req.sweeps = sweeps;
        req.tuning = tuning;
        return batch_solve(req, st);
    });
}

extern "C" void jsvd_batch_stats_get(jsvd_batch_stats *out)
{
    if (!out) return;
    const BatchStats &s = batch_stats();
    out->calls = s.calls;
    out->launches = s.launches;
    out->matrices = s.matrices;
    out->sweeps = s.sweeps;
    out->kernel_ms = s.kernel_ms;
    for (int c = 0; c < 5; ++c) {
        out->class_count[c] = s.class_count[c];
        out->class_ms[c] = s.class_ms[c];
    }
}

extern "C" void jsvd_batch_stats_reset(void) { batch_stats() = BatchStats{}; }

extern "C" int jsvd_batch_set_cluster_classes(int mask, int *previous)
{
    if (mask & ~((1 << 2) | (1 << 3) | (1 << 4)))
        return invalid_argument("Only size classes 2, 3 and 4 can be solved by clusters.");
    const int old = g_cluster_mask.exchange(mask);
    if (previous) *previous = old;
    return JSVD_OK;
}

extern "C" void jsvd_batch_builtin_tuning(jsvd_batch_tuning *out)
{
    if (!out) return;
    for (int c = 0; c < kClasses; ++c) out[c] = kBuiltinTuning[c];
}

namespace jsvd {
namespace {

// Candidate launch shapes of class c whose largest sampled member needs
// smem_need bytes of shared memory.  Classes 0-2: threads x persistent CTAs
// per SM, as many CTAs as the SM's shared memory and 2048 threads allow.
// Classes 3-4 take a whole SM's shared memory per CTA: threads x grid cap
// (the cap bounds the per-CTA global-memory slices that compete for L2).
std::vector<jsvd_batch_tuning> batch_candidates(int c, size_t smem_need, int sms, size_t smem_per_sm)
{
    std::vector<jsvd_batch_tuning> out;
    for (int t : {128, 256, 512}) {
        if (c <= 2) {
            for (int k : {1, 2, 4, 8})
                if (t * k <= 2048 && (size_t)k * (smem_need + 1024) <= smem_per_sm) out.push_back({t, k, 0});
        } else {
            for (int cap : {0, (3 * sms) / 4, sms / 2}) out.push_back({t, 1, cap});
        }
    }
    return out;
}

bool same_shape(const jsvd_batch_tuning &x, const jsvd_batch_tuning &y)
{
    return x.threads == y.threads && x.ctas_per_sm == y.ctas_per_sm && x.max_ctas == y.max_ctas;
}

}  // namespace
}  // namespace jsvd

extern "C" int jsvd_batch_autotune(int count, const int *rows, const int *cols, const long long *a_offsets,
                                   const void *d_a, int a_is_f32, const jsvd_config *cfg, int sample, int reps,
                                   int want_u, int want_v, jsvd_batch_autotune_report *report, void *stream)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        jsvd_config def;
        const jsvd_config &c = config_or_default(cfg, def);
        if (report == nullptr) return invalid_argument("Autotune report must not be null.");
        const int bad = check_batch_args(count, rows, cols, a_offsets, d_a, false, c);
        if (bad != JSVD_OK) return bad;
        *report = jsvd_batch_autotune_report{};
        for (int k = 0; k < kClasses; ++k) report->builtin[k] = kBuiltinTuning[k];
        if (count == 0) return JSVD_OK;
        if (reps <= 0) reps = 2;
        cudaStream_t st = nullptr;
        if (const int e = entry_stream(stream, &st); e != JSVD_OK) return e;
        int dev = 0;
        JSVD_CUDA_TRY(cudaGetDevice(&dev));
        int sms = 0, smem_per_sm = 0;
        JSVD_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        JSVD_CUDA_TRY(cudaDeviceGetAttribute(&smem_per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
        size_t smem_cap = 0;
        int rc = batch_smem_cap(dev, &smem_cap);
        if (rc != JSVD_OK) return rc;

        std::vector<std::vector<int>> members(kClasses);
        for (int i = 0; i < count; ++i) {
            if (rows[i] <= 0 || cols[i] <= 0 || rows[i] < cols[i])
                return invalid_argument("Batch matrix shape must satisfy rows >= columns > 0.");
            if (dims_out_of_range((size_t)rows[i], (size_t)cols[i])) {
                set_last_error(JSVD_ERR_OVERFLOW, "Matrix dimensions exceed the supported range.");
                return JSVD_ERR_OVERFLOW;
            }
            members[member_class(rows[i], cols[i], smem_cap, nullptr)].push_back(i);
        }

        // Flush buffer (larger than L2) and output buffers sized for the largest sample.
        const size_t flush_bytes = (size_t)256 << 20;
        std::vector<std::vector<int>> picked(kClasses);
        size_t max_s = 0, max_v = 0, max_u = 0;
        for (int k = 0; k < kClasses; ++k) {
            auto &mem = members[k];
            std::sort(mem.begin(), mem.end(),
                      [&](int x, int y) { return member_work(rows[x], cols[x]) > member_work(rows[y], cols[y]); });
            const size_t cnt = mem.size();
            const size_t s = (sample > 0 && (size_t)sample < cnt) ? (size_t)sample : cnt;
            size_t ns = 0, nv = 0, nu = 0;
            for (size_t j = 0; j < s; ++j) {  // evenly spaced over the work order
                const int i = mem[j * cnt / s];
                picked[k].push_back(i);
                ns += (size_t)cols[i];
                nv += (size_t)cols[i] * cols[i];
                nu += (size_t)rows[i] * cols[i];
            }
            max_s = std::max(max_s, ns);
            max_v = std::max(max_v, nv);
            max_u = std::max(max_u, nu);
            report->members[k] = (int)cnt;
            report->sampled[k] = (int)s;
        }
        void *d_flush = nullptr;
        double *d_sigma = nullptr, *d_v = nullptr, *d_u = nullptr;
        // The autotuner's own solves are not counted in the batch statistics.
        // Buffers and statistics are restored on every path, a C++ exception's
        // included.
        const BatchStats saved = batch_stats();
        ScopeExit restore([&] {
            if (d_flush) cudaFreeAsync(d_flush, st);
            if (d_sigma) cudaFreeAsync(d_sigma, st);
            if (d_v) cudaFreeAsync(d_v, st);
            if (d_u) cudaFreeAsync(d_u, st);
            cudaStreamSynchronize(st);
            batch_stats() = saved;
        });
        if (cudaMallocAsync(&d_flush, flush_bytes, st) != cudaSuccess ||
            cudaMallocAsync((void **)&d_sigma, sizeof(double) * std::max<size_t>(max_s, 1), st) != cudaSuccess ||
            (want_v &&
             cudaMallocAsync((void **)&d_v, sizeof(double) * std::max<size_t>(max_v, 1), st) != cudaSuccess) ||
            (want_u && cudaMallocAsync((void **)&d_u, sizeof(double) * std::max<size_t>(max_u, 1), st) != cudaSuccess))
            return cuda_failure(cudaGetLastError(), "cudaMallocAsync", __FILE__, __LINE__);

        for (int k = 0; k < kClasses; ++k) {
            const auto &pk = picked[k];
            if (pk.empty()) continue;
            const int s = (int)pk.size();
            std::vector<int> r_s(s), c_s(s), sw(s), sw_ref(s);
            std::vector<long long> off_s(s);
            size_t need = 0, nsig = 0;
            for (int j = 0; j < s; ++j) {
                r_s[j] = rows[pk[j]];
                c_s[j] = cols[pk[j]];
                off_s[j] = a_offsets[pk[j]];
                size_t nj = 0;
                member_class(r_s[j], c_s[j], smem_cap, &nj);
                need = std::max(need, nj);
                nsig += (size_t)c_s[j];
            }
            std::vector<double> sig(nsig), sig_ref(nsig);
            // the built-in shape first: it is the yardstick and the bitwise reference
            std::vector<jsvd_batch_tuning> cands{kBuiltinTuning[k]};
            for (const auto &t : batch_candidates(k, need, sms, (size_t)smem_per_sm))
                if (!same_shape(t, kBuiltinTuning[k])) cands.push_back(t);
            report->candidates[k] = (int)cands.size();
            double best_ms = -1.0;
            jsvd_batch_tuning best = kBuiltinTuning[k];
            for (size_t ci = 0; ci < cands.size(); ++ci) {
                jsvd_batch_tuning tun[kClasses] = {};
                tun[k] = cands[ci];
                BatchRequest req;
                req.count = s;
                req.rows = r_s.data();
                req.cols = c_s.data();
                req.a_offsets = off_s.data();
                req.a = d_a;
                req.a_is_f32 = a_is_f32;
                req.eps = c.epsilon;
                req.max_sweeps = c.max_sweeps;
                req.sigma = d_sigma;
                req.v = d_v;
                req.u = d_u;
                req.sweeps = sw.data();
                req.tuning = tun;
                double ms = -1.0;
                for (int r = 0; r < reps; ++r) {
                    if (cudaMemsetAsync(d_flush, r & 0xff, flush_bytes, st) != cudaSuccess)
                        return cuda_failure(cudaGetLastError(), "cudaMemsetAsync", __FILE__, __LINE__);
                    const double before = batch_stats().class_ms[k];
                    rc = batch_solve(req, st);
                    if (rc != JSVD_OK) return rc;
                    const double t = batch_stats().class_ms[k] - before;
                    ms = ms < 0.0 ? t : std::min(ms, t);
                }
                if (cudaMemcpyAsync(sig.data(), d_sigma, sizeof(double) * nsig, cudaMemcpyDeviceToHost, st) !=
                        cudaSuccess ||
                    cudaStreamSynchronize(st) != cudaSuccess)
                    return cuda_failure(cudaGetLastError(), "cudaMemcpyAsync", __FILE__, __LINE__);
                if (ci == 0) {
                    sig_ref = sig;
                    sw_ref = sw;
                    report->builtin_ms[k] = ms;
                } else if (std::memcmp(sig.data(), sig_ref.data(), sizeof(double) * nsig) != 0 || sw != sw_ref) {
                    set_last_error(JSVD_ERR_RUNTIME, "Batch launch shapes disagree on sigma or sweep counts.");
                    return JSVD_ERR_RUNTIME;
                }
                if (best_ms < 0.0 || ms < best_ms) {
                    best_ms = ms;
                    best = cands[ci];
                }
            }
            // a shape replaces the built-in one only when it is more than 2% faster
            if (best_ms > 0.98 * report->builtin_ms[k]) {
                best = kBuiltinTuning[k];
                best_ms = report->builtin_ms[k];
            }
            report->best[k] = best;
            report->best_ms[k] = best_ms;
        }
        return JSVD_OK;
    });
}
