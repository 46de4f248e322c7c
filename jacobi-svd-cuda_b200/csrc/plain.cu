// Plain FP64 one-sided Jacobi SVD for sm_100a: the drop-in for
// jacobi::svd::one_sided_jacobi_svd (kleedaisuki/jacobi-svd-cuda
// src/kernels.cu:844-1004, 1066-1076).
//
// Same arithmetic and cyclic round-robin order as the reference; different
// execution:
//   * A lives in a column-major working copy (lda = m), so every pair reads two
//     contiguous columns with fully coalesced accesses.
//   * One fused kernel per round: Gram dot products (fma chains over T virtual
//     lanes + the reference's halving tree, warp shuffles for the in-warp
//     levels), Rutishauser angle in registers, rotation of the register-held
//     column tiles written back in place.  The reference needs three launches
//     and three blocking host transfers per round.
//   * V never sits on the round-to-round critical path.  Each round records
//     its (c, s); after a sweep that rotated, one row-parallel pass applies the
//     whole sweep to V, rows held in shared memory (rotated in place in global
//     memory when a row is longer than the shared-memory cap), on a second
//     stream while the next sweep's rounds run (the angle tables alternate
//     between sweeps).
//     The pass is kept as narrow as it can be while it still ends inside
//     those rounds, so that it takes few of their registers.  Per element the
//     sequence of rotations is the reference's, so V is bit-identical.
//   * The n-1 round kernels of a sweep are launched directly the first time a
//     plan (device, m, n, T, eps, sweep mode) is used and captured into a CUDA
//     graph when the plan is reused; the host reads one rotation counter per
//     sweep.
//   * Plan workspaces use stream-ordered allocation, so creating or evicting a
//     plan never synchronises the whole device.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "dgemm.hpp"
#include "internal.hpp"
#include "layout.cuh"
#include "mixed.hpp"
#include "plain.hpp"

namespace jsvd {
namespace {

// Block-wide reference tree over T lanes for three quantities.  Every warp
// reads all T partial sums and reduces them in the reference's order itself,
// so every thread ends with the totals after a single barrier (no second
// barrier to broadcast a result computed by one thread).  `red` holds 3*T
// doubles.
template <int T>
__device__ __forceinline__ void block_tree3_all(double &pp, double &qq, double &pq, double *red)
{
    if constexpr (T == 32) {
        pp = __shfl_sync(0xffffffffu, warp_tree1(pp), 0);
        qq = __shfl_sync(0xffffffffu, warp_tree1(qq), 0);
        pq = __shfl_sync(0xffffffffu, warp_tree1(pq), 0);
    } else {
        constexpr int W = T / 32;
        const int t = threadIdx.x, lane = t & 31;
        red[t] = pp;
        red[T + t] = qq;
        red[2 * T + t] = pq;
        __syncthreads();
        double y[W];
#pragma unroll
        for (int w = 0; w < W; ++w) y[w] = red[w * 32 + lane];
        pp = __shfl_sync(0xffffffffu, warp_tree<W>(y), 0);
#pragma unroll
        for (int w = 0; w < W; ++w) y[w] = red[T + w * 32 + lane];
        qq = __shfl_sync(0xffffffffu, warp_tree<W>(y), 0);
#pragma unroll
        for (int w = 0; w < W; ++w) y[w] = red[2 * T + w * 32 + lane];
        pq = __shfl_sync(0xffffffffu, warp_tree<W>(y), 0);
    }
}

// The same totals and angle computed once: the partial sums go to shared
// memory, warp 0 reduces them in the reference's order and lane 0 derives
// (c, s), which the other threads read after a second barrier.  The
// arithmetic is block_tree3_all's followed by rotation_params, so the result
// is bit-identical; the FP64 pipe does the reduction trees and the
// square-root/division chain of the angle once per CTA instead of once per warp.
template <int T>
__device__ __forceinline__ bool block_angle_once(double pp, double qq, double pq, double *red, double2 *cs_sh,
                                                 double eps, double &c, double &s)
{
    if constexpr (T == 32) {
        pp = warp_tree1(pp);
        qq = warp_tree1(qq);
        pq = warp_tree1(pq);
        double cc = 0.0, ss = 0.0;
        if (threadIdx.x == 0) {
            rotation_params(pp, qq, pq, eps, cc, ss);
        }
        c = __shfl_sync(0xffffffffu, cc, 0);
        s = __shfl_sync(0xffffffffu, ss, 0);
    } else {
        constexpr int W = T / 32;
        const int t = threadIdx.x, lane = t & 31;
        red[t] = pp;
        red[T + t] = qq;
        red[2 * T + t] = pq;
        __syncthreads();
        if (t < 32) {
            double y[W];
#pragma unroll
            for (int w = 0; w < W; ++w) y[w] = red[w * 32 + lane];
            pp = warp_tree<W>(y);
#pragma unroll
            for (int w = 0; w < W; ++w) y[w] = red[T + w * 32 + lane];
            qq = warp_tree<W>(y);
#pragma unroll
            for (int w = 0; w < W; ++w) y[w] = red[2 * T + w * 32 + lane];
            pq = warp_tree<W>(y);
            if (lane == 0) {
                double cc, ss;
                rotation_params(pp, qq, pq, eps, cc, ss);
                *cs_sh = make_double2(cc, ss);
            }
        }
        __syncthreads();
        const double2 g = *cs_sh;
        c = g.x;
        s = g.y;
    }
    return c != 0.0;  // rotation_params gives c > 0 for a rotation, c = 0 otherwise
}

// One round of the sweep: blockIdx.x = pair slot.  T threads = T virtual
// lanes; thread t owns rows t + k*T.  K > 0: the K row-tiles of both columns
// stay in registers between the dot products and the rotation.  K == 0: the
// columns are streamed twice (m > K_max * T).
template <int T, int K, bool kOnce>
__global__ void __launch_bounds__(T) plain_round_kernel(double *__restrict__ a, long lda, int m,
                                                         const int2 *__restrict__ pairs,
                                                         double2 *__restrict__ cs, double eps,
                                                         unsigned *__restrict__ counter)
{
    __shared__ double red[T == 32 ? 1 : 3 * T];
    __shared__ double2 cs_sh;
    const int t = threadIdx.x;
    // Programmatic dependent launch: the next round may be scheduled now; its
    // CTAs stop at pdl_wait() until this grid has completed and its stores
    // are visible.
    pdl_launch_dependents();
    const int2 pq_idx = pairs[blockIdx.x];  // written once per plan
    double *__restrict__ ap = a + (size_t)pq_idx.x * lda;
    double *__restrict__ aq = a + (size_t)pq_idx.y * lda;
    pdl_wait();  // the previous round's columns and counter

    double spp = 0.0, sqq = 0.0, spq = 0.0;
    double xp[K > 0 ? K : 1], xq[K > 0 ? K : 1];
    if constexpr (K > 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int r = t + k * T;
            xp[k] = (r < m) ? ap[r] : 0.0;
            xq[k] = (r < m) ? aq[r] : 0.0;
        }
#pragma unroll
        for (int k = 0; k < K; ++k) {
            if (t + k * T < m) {
                spp = fma(xp[k], xp[k], spp);
                sqq = fma(xq[k], xq[k], sqq);
                spq = fma(xp[k], xq[k], spq);
            }
        }
    } else {
        for (int r = t; r < m; r += T) {
            const double x = ap[r], y = aq[r];
            spp = fma(x, x, spp);
            sqq = fma(y, y, sqq);
            spq = fma(x, y, spq);
        }
    }
    double c, s;
    bool rotates;
    if constexpr (kOnce) {
        rotates = block_angle_once<T>(spp, sqq, spq, red, &cs_sh, eps, c, s);
    } else {
        block_tree3_all<T>(spp, sqq, spq, red);
        // every thread derives the same angle from the same totals
        rotates = rotation_params(spp, sqq, spq, eps, c, s);
    }
    if (t == 0) {
        cs[blockIdx.x] = make_double2(c, s);
        if (rotates) atomicAdd(counter, 1u);
    }
    if (!rotates) return;  // no rotation: columns unchanged
    if constexpr (K > 0) {
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const int r = t + k * T;
            if (r < m) {
                ap[r] = rot_p(c, s, xp[k], xq[k]);
                aq[r] = rot_q(c, s, xp[k], xq[k]);
            }
        }
    } else {
        for (int r = t; r < m; r += T) {
            const double x = ap[r], y = aq[r];
            ap[r] = rot_p(c, s, x, y);
            aq[r] = rot_q(c, s, x, y);
        }
    }
}

// Counts the pairs p > q of the lower triangle of G (column-major, ld n) that
// pass the reference's rotation test (src/kernels.cu:503-505):
// |g_pq| > eps sqrt(max(g_pp, 0) max(g_qq, 0)) and |g_pq| > 1e-300.
__global__ void gram_offdiag_count(const double *__restrict__ G, int n, double eps, unsigned *__restrict__ count)
{
    unsigned local = 0;
    const size_t total = (size_t)n * n;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int q = (int)(e / n), p = (int)(e - (size_t)q * n);
        if (p <= q) continue;
        const double g = G[e];
        const double rhs = eps * sqrt(fmax(G[(size_t)p * n + p], 0.0) * fmax(G[(size_t)q * n + q], 0.0));
        if (fabs(g) > rhs && fabs(g) > 1.0e-300) ++local;
    }
    for (int off = 16; off > 0; off >>= 1) local += __shfl_down_sync(0xffffffffu, local, off);
    if ((threadIdx.x & 31) == 0 && local) atomicAdd(count, local);
}

// Deferred V update: applies every rotation of one sweep to R rows of V
// (R in {1, 2, 4, 8}, a template parameter so the row loop unrolls).
// V is column-major (element (row, col) at col*ldv + row); the CTA stages its
// R rows row by row in shared memory, sv[rr*n + col], so the round-to-round
// dependency never leaves the SM and the 32 lanes of a warp, which rotate 32
// unrelated column pairs, spread over the banks instead of all starting at the
// same bank (which a column-by-column staging with R = 8 would cause).
// Thread k owns pair slot k of every round; the (c, s) of the next round is
// loaded while the current one is applied.
// kStaged = false (R = 1) is the form for V rows too long for shared memory:
// the CTA rotates its row of V in place in global memory; the pairs of a
// round are disjoint and the barrier between rounds makes each round's global
// stores visible to the block, so the sequence of rotations per element, and
// so the result, is the same.
constexpr int kVpassSlots = 8;  // prefetched pair slots per thread and round

template <int R, bool kStaged>
__global__ void __launch_bounds__(512) plain_vpass_kernel(double *__restrict__ v, long ldv, int n,
                                                          const double2 *__restrict__ cs, int rounds, int npairs)
{
    extern __shared__ double sv[];
    const int r0 = blockIdx.x * R;
    const int rows = min(R, n - r0);
    const int total = n * R;
    // element (h, col) of this CTA's rows of V
    auto elem = [&](int h, int col) -> double & {
        if constexpr (kStaged) return sv[h * n + col];
        else return v[(size_t)col * ldv + r0 + h];
    };
    if constexpr (kStaged) {
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            const int col = idx / R, rr = idx - col * R;
            sv[rr * n + col] = (rr < rows) ? v[(size_t)col * ldv + r0 + rr] : 0.0;
        }
        __syncthreads();
    }
    // Thread k0 owns pair slots k0, k0 + blockDim.x, ...: the (c, s) of its
    // first kVpassSlots slots for round r + 1 are loaded while round r is
    // applied, so a round waits on one L2 round trip, not one per slot (the
    // loads cannot move past the shared-memory stores of the previous slot).
    // Slots beyond those (more than kVpassSlots * blockDim.x pairs) are read
    // when used.
    const int k0 = threadIdx.x;
    const int nb = blockDim.x;
    double2 g_next[kVpassSlots];
#pragma unroll
    for (int j = 0; j < kVpassSlots; ++j) {
        const int k = k0 + j * nb;
        g_next[j] = (k < npairs) ? cs[k] : make_double2(0.0, 0.0);
    }
    for (int r = 0; r < rounds; ++r) {
        double2 g_cur[kVpassSlots];
#pragma unroll
        for (int j = 0; j < kVpassSlots; ++j) g_cur[j] = g_next[j];
        if (r + 1 < rounds) {
#pragma unroll
            for (int j = 0; j < kVpassSlots; ++j) {
                const int k = k0 + j * nb;
                if (k < npairs) g_next[j] = cs[(size_t)(r + 1) * npairs + k];
            }
        }
#pragma unroll
        for (int j = 0; j < kVpassSlots; ++j) {
            const int k = k0 + j * nb;
            const double2 g = g_cur[j];
            if (k < npairs && g.x != 0.0) {
                const int2 pq = round_robin_pair(n, r, k);
                double x[R], y[R];
#pragma unroll
                for (int h = 0; h < R; ++h) {
                    x[h] = elem(h, pq.x);
                    y[h] = elem(h, pq.y);
                }
#pragma unroll
                for (int h = 0; h < R; ++h) {
                    elem(h, pq.x) = rot_p(g.x, g.y, x[h], y[h]);
                    elem(h, pq.y) = rot_q(g.x, g.y, x[h], y[h]);
                }
            }
        }
        for (int k = k0 + kVpassSlots * nb; k < npairs; k += nb) {
            const double2 g = cs[(size_t)r * npairs + k];
            if (g.x != 0.0) {
                const int2 pq = round_robin_pair(n, r, k);
                double x[R], y[R];
#pragma unroll
                for (int h = 0; h < R; ++h) {
                    x[h] = elem(h, pq.x);
                    y[h] = elem(h, pq.y);
                }
#pragma unroll
                for (int h = 0; h < R; ++h) {
                    elem(h, pq.x) = rot_p(g.x, g.y, x[h], y[h]);
                    elem(h, pq.y) = rot_q(g.x, g.y, x[h], y[h]);
                }
            }
        }
        __syncthreads();
    }
    if constexpr (kStaged) {
        for (int idx = threadIdx.x; idx < total; idx += blockDim.x) {
            const int col = idx / R, rr = idx - col * R;
            if (rr < rows) v[(size_t)col * ldv + r0 + rr] = sv[rr * n + col];
        }
    }
}

// sigma_j = sqrt(max(||a_j||^2, 0)) with the reference's T-lane order
// (src/kernels.cu:586-629).
template <int T>
__global__ void __launch_bounds__(T) plain_sigma_kernel(const double *__restrict__ a, long lda, int m,
                                                        double *__restrict__ sigma)
{
    __shared__ double red[T == 32 ? 1 : T];
    const int t = threadIdx.x;
    const double *__restrict__ col = a + (size_t)blockIdx.x * lda;
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

// ---- persistent sweep ---------------------------------------------------------
// One launch per sweep instead of one per round.  CTA c owns the contiguous
// pair slots [c*S, c*S + S) of the circle (slot k = positions k and ne-1-k) and
// runs every round of the sweep; a slot's two columns in round r+1 come only
// from slots k-1 (0 for k <= 1), k and k+1 (k for the last slot) of round r,
// so CTAs synchronise point to point: after a round a CTA publishes the number
// of rounds it has completed (flags[c], release at GPU scope) and before a
// round it waits (acquire) for the CTAs owning its slots' sources.  All CTAs
// are co-resident (cooperative launch).  Waits are bounded: after
// kSpinLimitNs the CTA records kDevWaitTimeout in *status and returns.
// Column loads and stores bypass L1 (other SMs write the columns).  The
// arithmetic of a pair is the round kernel's, so results are bit-identical.

constexpr long long kSpinLimitNs = 2000000000LL;  // 2 s

__device__ __forceinline__ int ld_acquire_gpu(const int *p)
{
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(int *p, int v)
{
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

__device__ __forceinline__ long long global_ns()
{
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// Waits until the CTAs lo and hi (and CTA 0 when need0) have completed g
// rounds (acquire loads of their flags); false after limit_ns.
__device__ __forceinline__ bool wait_for_rounds(const int *flags, int lo, int hi, bool need0, int g,
                                                long long limit_ns)
{
    const long long t0 = global_ns();
    for (;;) {
        const int f1 = ld_acquire_gpu(flags + lo);
        const int f2 = ld_acquire_gpu(flags + hi);
        const int f3 = ld_acquire_gpu(flags + 0);
        if (f1 >= g && f2 >= g && (!need0 || f3 >= g)) return true;
        if (global_ns() - t0 > limit_ns) return false;
    }
}

// Wait-limit check: thread 0 waits, as a persistent-sweep CTA does, for
// flags[0] to reach round 1, with a short limit; on expiry it records
// kDevWaitTimeout like the sweep.  Nothing sets the flag during the launch.
__global__ void wait_limit_check_kernel(const int *flags, long long limit_ns, int *status)
{
    if (threadIdx.x == 0 && !wait_for_rounds(flags, 0, 0, false, 1, limit_ns)) atomicExch(status, (int)kDevWaitTimeout);
}

template <int T, int K>
__global__ void __launch_bounds__(T) plain_sweep_persistent(double *__restrict__ a, long lda, int m, int n,
                                                             int rounds, int slots_per_cta, double2 *__restrict__ cs,
                                                             int npairs, double eps, unsigned *__restrict__ counter,
                                                             int *__restrict__ flags, int g0,
                                                             int *__restrict__ status)
{
    __shared__ double red[T == 32 ? 1 : 3 * T];
    __shared__ int s_ok;
    const int t = threadIdx.x;
    const int ne = n + (n & 1), half = ne / 2, L = ne - 1;
    const int k_lo = blockIdx.x * slots_per_cta;
    const int k_hi = min(half, k_lo + slots_per_cta);
    // CTAs owning the sources of this CTA's slots (besides itself)
    const int dep_lo = (k_lo <= 1 ? 0 : k_lo - 1) / slots_per_cta;
    const int dep_hi = (k_hi - 1 < half - 1 ? k_hi : k_hi - 1) / slots_per_cta;
    for (int r = 0; r < rounds; ++r) {
        const int g = g0 + r;
        if (r > 0) {
            if (t == 0) s_ok = wait_for_rounds(flags, dep_lo, dep_hi, k_lo == 1, g, kSpinLimitNs) ? 1 : 0;
            if (t == 0 && !s_ok) atomicExch(status, (int)kDevWaitTimeout);
            __syncthreads();
            if (!s_ok) return;
        }
        // position of the dummy column (odd n) in this round and its slot
        int dummy_slot = -1;
        if (n & 1) {
            const int j = 1 + ((n - 1 + r) % L);
            dummy_slot = j < half ? j : ne - 1 - j;
        }
        for (int k = k_lo; k < k_hi; ++k) {
            if (k == dummy_slot) continue;
            const int p = circle_col(n, L, r, k), q = circle_col(n, L, r, ne - 1 - k);
            const int pair = (dummy_slot >= 0 && k > dummy_slot) ? k - 1 : k;
            double *__restrict__ ap = a + (size_t)p * lda;
            double *__restrict__ aq = a + (size_t)q * lda;
            double spp = 0.0, sqq = 0.0, spq = 0.0;
            double xp[K > 0 ? K : 1], xq[K > 0 ? K : 1];
            if constexpr (K > 0) {
#pragma unroll
                for (int kk = 0; kk < K; ++kk) {
                    const int row = t + kk * T;
                    xp[kk] = (row < m) ? __ldcg(ap + row) : 0.0;
                    xq[kk] = (row < m) ? __ldcg(aq + row) : 0.0;
                }
#pragma unroll
                for (int kk = 0; kk < K; ++kk) {
                    if (t + kk * T < m) {
                        spp = fma(xp[kk], xp[kk], spp);
                        sqq = fma(xq[kk], xq[kk], sqq);
                        spq = fma(xp[kk], xq[kk], spq);
                    }
                }
            } else {
                for (int row = t; row < m; row += T) {
                    const double x = __ldcg(ap + row), y = __ldcg(aq + row);
                    spp = fma(x, x, spp);
                    sqq = fma(y, y, sqq);
                    spq = fma(x, y, spq);
                }
            }
            block_tree3_all<T>(spp, sqq, spq, red);
            double c, s;
            const bool rotates = rotation_params(spp, sqq, spq, eps, c, s);
            if (t == 0) {
                cs[(size_t)r * npairs + pair] = make_double2(c, s);
                if (rotates) atomicAdd(counter, 1u);
            }
            if (rotates) {
                if constexpr (K > 0) {
#pragma unroll
                    for (int kk = 0; kk < K; ++kk) {
                        const int row = t + kk * T;
                        if (row < m) {
                            __stcg(ap + row, rot_p(c, s, xp[kk], xq[kk]));
                            __stcg(aq + row, rot_q(c, s, xp[kk], xq[kk]));
                        }
                    }
                } else {
                    for (int row = t; row < m; row += T) {
                        const double x = __ldcg(ap + row), y = __ldcg(aq + row);
                        __stcg(ap + row, rot_p(c, s, x, y));
                        __stcg(aq + row, rot_q(c, s, x, y));
                    }
                }
            }
            __syncthreads();  // red[] is reused by the next slot
        }
        // bar.sync above orders the CTA's column stores before thread 0's
        // release, which is cumulative at GPU scope.
        if (t == 0) st_release_gpu(flags + blockIdx.x, g + 1);
    }
}

using SweepFn = void (*)(double *, long, int, int, int, int, double2 *, int, double, unsigned *, int *, int, int *);

template <int T>
SweepFn pick_sweep_t(int m)
{
    constexpr int kmax = T <= 256 ? 16 : (T == 512 ? 8 : 4);
    if (m <= 1 * T) return plain_sweep_persistent<T, 1>;
    if (m <= 2 * T) return plain_sweep_persistent<T, 2>;
    if (m <= 4 * T) return plain_sweep_persistent<T, 4>;
    if (kmax >= 8 && m <= 8 * T) return plain_sweep_persistent<T, (kmax >= 8 ? 8 : 4)>;
    if (kmax >= 16 && m <= 16 * T) return plain_sweep_persistent<T, (kmax >= 16 ? 16 : 4)>;
    return plain_sweep_persistent<T, 0>;
}

SweepFn pick_sweep(int T, int m)
{
    switch (T) {
    case 32: return pick_sweep_t<32>(m);
    case 64: return pick_sweep_t<64>(m);
    case 128: return pick_sweep_t<128>(m);
    case 256: return pick_sweep_t<256>(m);
    case 512: return pick_sweep_t<512>(m);
    default: return pick_sweep_t<1024>(m);
    }
}

using RoundFn = void (*)(double *, long, int, const int2 *, double2 *, double, unsigned *);
using SigmaFn = void (*)(const double *, long, int, double *);
using VpassFn = void (*)(double *, long, int, const double2 *, int, int);

VpassFn pick_vpass(int R, bool staged)
{
    if (!staged) return plain_vpass_kernel<1, false>;
    switch (R) {
    case 1: return plain_vpass_kernel<1, true>;
    case 2: return plain_vpass_kernel<2, true>;
    case 4: return plain_vpass_kernel<4, true>;
    default: return plain_vpass_kernel<8, true>;
    }
}

template <int T, bool kOnce>
RoundFn pick_round_t(int m)
{
    // K rows per thread stay in registers between the dot products and the
    // rotation; K = 0 streams the columns twice (taller than K_max * T).
    constexpr int kmax = T <= 128 ? 16 : (T == 256 ? 32 : (T == 512 ? 8 : 4));
    if (m <= 1 * T) return plain_round_kernel<T, 1, kOnce>;
    if (m <= 2 * T) return plain_round_kernel<T, 2, kOnce>;
    if (m <= 4 * T) return plain_round_kernel<T, 4, kOnce>;
    if (kmax >= 8 && m <= 8 * T) return plain_round_kernel<T, (kmax >= 8 ? 8 : 4), kOnce>;
    if (kmax >= 16 && m <= 16 * T) return plain_round_kernel<T, (kmax >= 16 ? 16 : 4), kOnce>;
    if (kmax >= 32 && m <= 32 * T) return plain_round_kernel<T, (kmax >= 32 ? 32 : 4), kOnce>;
    return plain_round_kernel<T, 0, kOnce>;
}

template <bool kOnce>
RoundFn pick_round_o(int T, int m)
{
    switch (T) {
    case 32: return pick_round_t<32, kOnce>(m);
    case 64: return pick_round_t<64, kOnce>(m);
    case 128: return pick_round_t<128, kOnce>(m);
    case 256: return pick_round_t<256, kOnce>(m);
    case 512: return pick_round_t<512, kOnce>(m);
    default: return pick_round_t<1024, kOnce>(m);
    }
}

RoundFn pick_round(int T, int m, bool once) { return once ? pick_round_o<true>(T, m) : pick_round_o<false>(T, m); }

SigmaFn pick_sigma(int T)
{
    switch (T) {
    case 32: return plain_sigma_kernel<32>;
    case 64: return plain_sigma_kernel<64>;
    case 128: return plain_sigma_kernel<128>;
    case 256: return plain_sigma_kernel<256>;
    case 512: return plain_sigma_kernel<512>;
    default: return plain_sigma_kernel<1024>;
    }
}

// Round-robin schedule, identical to src/kernels.cu:637-678 (fixed head,
// dummy column for odd n, pair i = (circle[i], circle[ne-1-i])).  Every round
// has the same number of real pairs, floor(n/2).
void build_schedule(int n, std::vector<int2> &pairs, int &rounds, int &npairs)
{
    pairs.clear();
    if (n < 2) {
        rounds = 0;
        npairs = 0;
        return;
    }
    const int ne = (n % 2) ? n + 1 : n;
    std::vector<int> circle(ne, -1);
    for (int i = 0; i < n; ++i) circle[i] = i;
    rounds = ne - 1;
    npairs = n / 2;
    pairs.reserve((size_t)rounds * npairs);
    for (int r = 0; r < rounds; ++r) {
        for (int i = 0; i < ne / 2; ++i) {
            const int lhs = circle[i], rhs = circle[ne - 1 - i];
            if (lhs >= 0 && rhs >= 0) pairs.push_back(make_int2(lhs, rhs));
        }
        const int last = circle[ne - 1];
        for (int i = ne - 1; i > 1; --i) circle[i] = circle[i - 1];
        circle[1] = last;
    }
}

}  // namespace

namespace {
std::atomic<int> g_sweep_mode{0};
std::atomic<int> g_vpass_global{0};
}  // namespace

bool vpass_global_forced() { return g_vpass_global.load() != 0; }
void set_vpass_global_forced(bool on) { g_vpass_global.store(on ? 1 : 0); }

int sweep_mode() { return g_sweep_mode.load(); }
void set_sweep_mode(int mode) { g_sweep_mode.store(mode >= 0 && mode <= 3 ? mode : 0); }

PlainStats &plain_stats()
{
    thread_local PlainStats stats;
    return stats;
}

PlainPlan::~PlainPlan()
{
    int prev = -1;
    cudaGetDevice(&prev);
    if (device >= 0) cudaSetDevice(device);
    if (sweep_exec) cudaGraphExecDestroy(sweep_exec);
    for (cudaEvent_t e : {ev_round_begin, ev_round_end})
        if (e) cudaEventDestroy(e);
    // Stream-ordered release: no device-wide synchronisation, so evicting a
    // plan does not stall work on other streams.
    if (vstream) {
        cudaStreamSynchronize(vstream);
        cudaStreamDestroy(vstream);
    }
    for (cudaGraphExec_t g : {sweep_exec2})
        if (g) cudaGraphExecDestroy(g);
    for (int p = 0; p < 2; ++p)
        for (cudaEvent_t e : {ev_rounds_done[p], ev_vpass_done[p], ev_v0[p], ev_v1[p]})
            if (e) cudaEventDestroy(e);
    for (void *p : {(void *)a_w, (void *)v_w, (void *)pairs, (void *)cs, (void *)cs2, (void *)counter, (void *)flags,
                    (void *)d_in, (void *)d_u, (void *)d_sigma, (void *)d_v, (void *)sigma_w, (void *)gram,
                    (void *)gram_count})
        if (p) cudaFreeAsync(p, stream);
    if (h_gram_count) cudaFreeHost(h_gram_count);
    if (prev >= 0) cudaSetDevice(prev);
}

int PlainPlan::create(int dev, size_t m_, size_t n_, int T_, double eps_, cudaStream_t stream,
                      std::unique_ptr<PlainPlan> &out)
{
    auto plan = std::make_unique<PlainPlan>();
    plan->device = dev;
    plan->stream = stream;
    plan->m = m_;
    plan->n = n_;
    plan->T = T_;
    plan->eps = eps_;
    plan->lda = (long)m_;
    plan->ldv = (long)n_;
    std::vector<int2> host_pairs;
    build_schedule((int)n_, host_pairs, plan->rounds, plan->npairs);
    JSVD_CUDA_TRY(cudaMallocAsync((void **)&plan->a_w, sizeof(double) * m_ * n_, stream));
    JSVD_CUDA_TRY(cudaMallocAsync((void **)&plan->v_w, sizeof(double) * n_ * n_, stream));
    JSVD_CUDA_TRY(cudaMallocAsync((void **)&plan->sigma_w, sizeof(double) * n_, stream));
    JSVD_CUDA_TRY(cudaMallocAsync((void **)&plan->counter, 2 * sizeof(unsigned), stream));  // rotations, status
    if (plan->rounds > 0) {
        const size_t np = (size_t)plan->rounds * plan->npairs;
        JSVD_CUDA_TRY(cudaMallocAsync((void **)&plan->pairs, sizeof(int2) * np, stream));
        JSVD_CUDA_TRY(cudaMallocAsync((void **)&plan->cs, sizeof(double2) * np, stream));
        JSVD_CUDA_TRY(cudaMallocAsync((void **)&plan->cs2, sizeof(double2) * np, stream));
        JSVD_CUDA_TRY(cudaStreamCreateWithFlags(&plan->vstream, cudaStreamNonBlocking));
        for (int p = 0; p < 2; ++p) {
            JSVD_CUDA_TRY(cudaEventCreateWithFlags(&plan->ev_rounds_done[p], cudaEventDisableTiming));
            JSVD_CUDA_TRY(cudaEventCreateWithFlags(&plan->ev_vpass_done[p], cudaEventDisableTiming));
            JSVD_CUDA_TRY(cudaEventCreate(&plan->ev_v0[p]));
            JSVD_CUDA_TRY(cudaEventCreate(&plan->ev_v1[p]));
        }
        JSVD_CUDA_TRY(cudaMemcpyAsync(plan->pairs, host_pairs.data(), sizeof(int2) * np, cudaMemcpyHostToDevice,
                                      stream));
        // host_pairs dies at return: the copy must have consumed it.
        JSVD_CUDA_TRY(cudaStreamSynchronize(stream));
        // V pass geometry: R rows of V per CTA (R in {1,2,4,8}), about n/128 so
        // the grid covers the SMs, capped by 200 KB of shared memory.
        // Rows of more than kVpassSmemCap bytes (n > 25600), or the forced
        // global form: one row per CTA, rotated in place in global memory.
        const size_t smem_cap = kVpassSmemCap;
        plan->vpass_global_forced = jsvd::vpass_global_forced();
        plan->vpass_staged = !plan->vpass_global_forced && sizeof(double) * n_ <= smem_cap;
        const int rmax = (int)std::max<size_t>(1, smem_cap / (sizeof(double) * n_));
        int R = 1;
        while (plan->vpass_staged && R * 2 <= 8 && R * 2 <= rmax && (size_t)(R * 2) * 128 <= n_) R *= 2;
        plan->vpass_rows = R;
        plan->vpass_smem = plan->vpass_staged ? (int)(sizeof(double) * n_ * R) : 0;
        plan->vpass_threads = std::min(512, std::max(32, (plan->npairs + 31) / 32 * 32));
        // The attribute is per function and process-wide: always raise it to the
        // fixed cap, never to this plan's size, or a plan created concurrently
        // on another thread could lower it under a larger plan's launch.
        if (plan->vpass_staged)
            JSVD_CUDA_TRY(cudaFuncSetAttribute(pick_vpass(R, true), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               (int)smem_cap));
        JSVD_CUDA_TRY(cudaEventCreate(&plan->ev_round_begin));
        JSVD_CUDA_TRY(cudaEventCreate(&plan->ev_round_end));
        // Persistent sweep when the whole grid can be co-resident.
        int coop = 0, sms = 0, per_sm = 0;
        JSVD_CUDA_TRY(cudaDeviceGetAttribute(&coop, cudaDevAttrCooperativeLaunch, dev));
        JSVD_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        SweepFn sfn = pick_sweep(T_, (int)m_);
        JSVD_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sfn, T_, 0));
        const int half = (int)((n_ + (n_ & 1)) / 2);
        if (coop && per_sm > 0 && sweep_mode() == 1) {
            const int max_ctas = per_sm * sms;
            plan->slots_per_cta = (half + max_ctas - 1) / max_ctas;
            plan->sweep_grid = (half + plan->slots_per_cta - 1) / plan->slots_per_cta;
            JSVD_CUDA_TRY(cudaMallocAsync((void **)&plan->flags, sizeof(int) * (plan->sweep_grid + 1), stream));
            plan->persistent = true;
        }
    }
    plan->bytes = sizeof(double) * (m_ * n_ + n_ * n_ + n_) +
                  (sizeof(int2) + 2 * sizeof(double2)) * (size_t)plan->rounds * plan->npairs;
    // The allocations become usable on any stream once this one has drained.
    JSVD_CUDA_TRY(cudaStreamSynchronize(stream));
    out = std::move(plan);
    return JSVD_OK;
}

// Enqueues the round kernels of one sweep on `st`, writing their angles into
// the (c, s) table of `parity`, bracketed by the plan's timing events.  Used
// for direct launches and for capture.
int PlainPlan::enqueue_rounds(cudaStream_t st, int parity)
{
    RoundFn round_fn = pick_round(T, (int)m, angle_once);
    double2 *tab = parity ? cs2 : cs;
    JSVD_CUDA_TRY(cudaEventRecordWithFlags(ev_round_begin, st, sweep_exec_capturing ? cudaEventRecordExternal : 0));
    // With use_pdl, rounds after the first are launched with programmatic
    // stream serialisation, so each round's launch overlaps the previous
    // round's tail.
    cudaLaunchAttribute pdl[1];
    pdl[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    pdl[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t lc = {};
    lc.gridDim = dim3(npairs);
    lc.blockDim = dim3(T);
    lc.dynamicSmemBytes = 0;
    lc.stream = st;
    for (int r = 0; r < rounds; ++r) {
        const size_t off = (size_t)r * npairs;
        lc.attrs = r > 0 && use_pdl ? pdl : nullptr;
        lc.numAttrs = r > 0 && use_pdl ? 1 : 0;
        JSVD_CUDA_TRY(cudaLaunchKernelEx(&lc, round_fn, a_w, lda, (int)m, (const int2 *)(pairs + off), tab + off, eps,
                                         counter));
    }
    JSVD_CUDA_TRY(cudaEventRecordWithFlags(ev_round_end, st, sweep_exec_capturing ? cudaEventRecordExternal : 0));
    return JSVD_OK;
}

// The V pass of a sweep (all rows of V, angles of `parity`) on `st`.
int PlainPlan::enqueue_vpass(cudaStream_t st, int parity)
{
    const int vgrid = (int)((n + vpass_rows - 1) / vpass_rows);
    pick_vpass(vpass_rows, vpass_staged)<<<vgrid, vpass_threads, vpass_smem, st>>>(v_w, ldv, (int)n,
                                                                                    parity ? cs2 : cs, rounds, npairs);
    JSVD_CUDA_TRY(cudaGetLastError());
    return JSVD_OK;
}

// Captures the rounds of a sweep for one parity of the angle table into a
// graph (done when a plan is used a second time: one-off shapes are not worth
// the instantiation).
int PlainPlan::capture_rounds(cudaStream_t st, int parity)
{
    cudaGraph_t graph = nullptr;
    JSVD_CUDA_TRY(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    sweep_exec_capturing = true;
    const int rc = enqueue_rounds(st, parity);
    sweep_exec_capturing = false;
    cudaError_t cap = cudaStreamEndCapture(st, &graph);
    if (rc != JSVD_OK) {
        if (graph) cudaGraphDestroy(graph);
        return rc;
    }
    if (cap != cudaSuccess) return cuda_failure(cap, "cudaStreamEndCapture", __FILE__, __LINE__);
    cudaGraphExec_t *dst = parity ? &sweep_exec2 : &sweep_exec;
    cudaError_t inst = cudaGraphInstantiate(dst, graph, 0);
    cudaGraphDestroy(graph);
    if (inst != cudaSuccess) return cuda_failure(inst, "cudaGraphInstantiate", __FILE__, __LINE__);
    return JSVD_OK;
}

// One persistent launch for all rounds of a sweep (angles of `parity`).
int PlainPlan::enqueue_persistent(cudaStream_t st, int parity, int g0)
{
    SweepFn sfn = pick_sweep(T, (int)m);
    double *a_arg = a_w;
    long lda_arg = lda;
    int m_arg = (int)m, n_arg = (int)n, rounds_arg = rounds, spc = slots_per_cta, np = npairs, g0_arg = g0;
    double2 *tab = parity ? cs2 : cs;
    double eps_arg = eps;
    unsigned *cnt = counter;
    int *fl = flags;
    int *status = reinterpret_cast<int *>(counter + 1);
    void *args[] = {&a_arg, &lda_arg, &m_arg, &n_arg, &rounds_arg, &spc, &tab, &np, &eps_arg, &cnt, &fl, &g0_arg,
                    &status};
    JSVD_CUDA_TRY(cudaEventRecord(ev_round_begin, st));
    JSVD_CUDA_TRY(cudaLaunchCooperativeKernel((const void *)sfn, dim3(sweep_grid), dim3(T), args, 0, st));
    JSVD_CUDA_TRY(cudaEventRecord(ev_round_end, st));
    return JSVD_OK;
}

int PlainPlan::ensure_host_staging()
{
    if (d_in) return JSVD_OK;
    JSVD_CUDA_TRY(cudaMallocAsync((void **)&d_in, sizeof(double) * m * n, stream));
    JSVD_CUDA_TRY(cudaMallocAsync((void **)&d_u, sizeof(double) * m * n, stream));
    JSVD_CUDA_TRY(cudaMallocAsync((void **)&d_sigma, sizeof(double) * n, stream));
    JSVD_CUDA_TRY(cudaMallocAsync((void **)&d_v, sizeof(double) * n * n, stream));
    JSVD_CUDA_TRY(cudaStreamSynchronize(stream));
    bytes += sizeof(double) * (2 * m * n + n + n * n);
    return JSVD_OK;
}

int PlainPlan::gram_converged(cudaStream_t st, bool &converged)
{
    if (gram == nullptr) {
        JSVD_CUDA_TRY(cudaMallocAsync((void **)&gram, sizeof(double) * n * n, stream));
        JSVD_CUDA_TRY(cudaMallocAsync((void **)&gram_count, sizeof(unsigned), stream));
        JSVD_CUDA_TRY(cudaMallocHost((void **)&h_gram_count, sizeof(unsigned)));
        JSVD_CUDA_TRY(cudaStreamSynchronize(stream));
    }
    if (const int rc = dgemm(st, 'T', 'N', (int)n, (int)n, (int)m, 1.0, a_w, lda, a_w, lda, 0.0, gram, (long)n, 1);
        rc != JSVD_OK)
        return rc;
    JSVD_CUDA_TRY(cudaMemsetAsync(gram_count, 0, sizeof(unsigned), st));
    gram_offdiag_count<<<std::min<size_t>(1184, (n * n + 255) / 256), 256, 0, st>>>(gram, (int)n, eps, gram_count);
    JSVD_CUDA_TRY(cudaGetLastError());
    JSVD_CUDA_TRY(cudaMemcpyAsync(h_gram_count, gram_count, sizeof(unsigned), cudaMemcpyDeviceToHost, st));
    JSVD_CUDA_TRY(cudaStreamSynchronize(st));
    converged = *h_gram_count == 0;
    return JSVD_OK;
}

int PlainPlan::run(const double *d_a, double *out_u, double *out_sigma, double *out_v, int max_sweeps, int *sweeps,
                   cudaStream_t stream, bool gram_stop)
{
    const int im = (int)m, in = (int)n;
    JSVD_CUDA_TRY(launch_rowmajor_to_colmajor(d_a, im, in, a_w, lda, stream));
    identity_colmajor_kernel<<<std::min<size_t>(1184, (n * n + 255) / 256), 256, 0, stream>>>(v_w, in, ldv);
    JSVD_CUDA_TRY(cudaGetLastError());

    PlainStats &st = plain_stats();
    int executed = 0;
    if (rounds == 0) {
        executed = 1;  // n == 1: one empty sweep, as the reference reports
    } else {
        if (persistent) {
            JSVD_CUDA_TRY(cudaMemsetAsync(flags, 0, sizeof(int) * (sweep_grid + 1), stream));
            JSVD_CUDA_TRY(cudaMemsetAsync(counter + 1, 0, sizeof(unsigned), stream));
        }
        if (!persistent && sweep_exec == nullptr && uses >= 1) {
            int rc = capture_rounds(stream, 0);
            if (rc == JSVD_OK) rc = capture_rounds(stream, 1);
            if (rc != JSVD_OK) return rc;
        }
        bool vpending[2] = {false, false};
        float r_ref = 0.f;  // rounds time of this solve's first sweep: no V pass runs beside it
        // V pass width: the pass runs beside the next sweep's rounds and its
        // CTAs take registers the rounds could use, so it is made as narrow
        // as it can be while it still ends well inside those rounds.  The
        // yardstick is the first sweep's rounds (uncontended; the rounds that
        // a V pass overlaps are slowed by it): halve the threads (>= 128) when
        // the pass took under 0.45 of that time, double them (<= the pair
        // count, <= 512) when it took over 0.9.  Kept in the plan.  The result
        // does not depend on the width (the slots of a round are disjoint).
        // At 1024 rows: 512 -> 128 threads, rounds 3.98 -> 3.73 us; at 8192
        // rows the pass stays at 512 (0.85 of the rounds' time).
        auto adapt_vpass = [&](float v_ms) {
            if (r_ref <= 0.f) return;
            const int cap = std::min(512, std::max(32, (npairs + 31) / 32 * 32));
            // at most kVpassSlots slots per thread (all prefetched), >= 128 threads
            const int floor_t = std::min(cap, std::max(128, (npairs + kVpassSlots - 1) / kVpassSlots + 31) / 32 * 32);
            if (v_ms < 0.45f * r_ref && vpass_threads > floor_t) vpass_threads = std::max(floor_t, vpass_threads / 2);
            else if (v_ms > 0.9f * r_ref && vpass_threads < cap) vpass_threads = std::min(cap, vpass_threads * 2);
        };
        auto collect_v = [&](int p) -> int {
            if (!vpending[p]) return JSVD_OK;
            JSVD_CUDA_TRY(cudaEventSynchronize(ev_v1[p]));
            float v_ms = 0.f;
            if (cudaEventElapsedTime(&v_ms, ev_v0[p], ev_v1[p]) == cudaSuccess) {
                st.vpass_ms += v_ms;
                if (!persistent) adapt_vpass(v_ms);
            }
            vpending[p] = false;
            return JSVD_OK;
        };
        auto launch_vpass = [&](int p, cudaStream_t vs) -> int {
            JSVD_CUDA_TRY(cudaEventRecord(ev_v0[p], vs));
            const int rc = enqueue_vpass(vs, p);
            if (rc != JSVD_OK) return rc;
            JSVD_CUDA_TRY(cudaEventRecord(ev_v1[p], vs));
            JSVD_CUDA_TRY(cudaEventRecord(ev_vpass_done[p], vs));
            vpending[p] = true;
            st.vpass_launches += 1;
            return JSVD_OK;
        };
        for (int s = 0; s < max_sweeps; ++s) {
            const int p = s & 1;
            if (vpending[p]) {
                JSVD_CUDA_TRY(cudaStreamWaitEvent(stream, ev_vpass_done[p], 0));
                const int rc = collect_v(p);
                if (rc != JSVD_OK) return rc;
            }
            JSVD_CUDA_TRY(cudaMemsetAsync(counter, 0, sizeof(unsigned), stream));
            if (persistent) {
                const int rc = enqueue_persistent(stream, p, s * rounds);
                if (rc != JSVD_OK) return rc;
                // All CTAs of a persistent sweep must be resident: its V pass
                // runs after it on the same stream.
                const int rc2 = launch_vpass(p, stream);
                if (rc2 != JSVD_OK) return rc2;
            } else {
                cudaGraphExec_t g = p ? sweep_exec2 : sweep_exec;
                if (g != nullptr) {
                    JSVD_CUDA_TRY(cudaGraphLaunch(g, stream));
                } else {
                    const int rc = enqueue_rounds(stream, p);
                    if (rc != JSVD_OK) return rc;
                }
                JSVD_CUDA_TRY(cudaEventRecord(ev_rounds_done[p], stream));
            }
            unsigned cnt[2] = {0, 0};
            JSVD_CUDA_TRY(cudaMemcpyAsync(cnt, counter, 2 * sizeof(unsigned), cudaMemcpyDeviceToHost, stream));
            JSVD_CUDA_TRY(cudaStreamSynchronize(stream));
            const unsigned rotated = cnt[0];
            if (persistent && cnt[1] != 0) {
                set_last_error(JSVD_ERR_RUNTIME, "A persistent sweep stopped at its wait limit (device status " +
                                                     std::to_string(cnt[1]) + ").");
                return JSVD_ERR_RUNTIME;
            }
            executed = s + 1;
            float r_ms = 0.f;
            if (cudaEventElapsedTime(&r_ms, ev_round_begin, ev_round_end) == cudaSuccess) st.round_ms += r_ms;
            st.round_launches += (unsigned long long)rounds;
            if (rotated == 0) break;  // V unchanged by this sweep: no V pass
            // The V pass of sweep s runs on vstream while the rounds of sweep
            // s + 1 run on `stream`; the (c, s) tables alternate between
            // sweeps, and the rounds of sweep s + 2 wait for this V pass.
            if (s == 0) r_ref = r_ms;
            if (!persistent) {
                JSVD_CUDA_TRY(cudaStreamWaitEvent(vstream, ev_rounds_done[p], 0));
                const int rc = launch_vpass(p, vstream);
                if (rc != JSVD_OK) return rc;
            }
            // Few rotations: the next sweep may rotate nothing; test every pair
            // on the Gram matrix instead of running it.
            // Only for eps >= 1e-12: the GEMM's rounding of an off-diagonal
            // entry (about sqrt(m) u relative) must stay well below eps, or
            // the test never confirms convergence (measured at eps = 1e-14).
            if (gram_stop && eps >= 1e-12 && s + 1 < max_sweeps && (size_t)rotated * 8 <= (size_t)rounds * npairs) {
                bool conv = false;
                const int rc = gram_converged(stream, conv);
                if (rc != JSVD_OK) return rc;
                st.gram_checks += 1;
                if (conv) {
                    executed = s + 2;  // the sweep that would have found no rotation
                    break;
                }
            }
        }
        for (int p = 0; p < 2; ++p) {
            if (vpending[p]) JSVD_CUDA_TRY(cudaStreamWaitEvent(stream, ev_vpass_done[p], 0));
            const int rc = collect_v(p);
            if (rc != JSVD_OK) return rc;
        }
    }
    uses += 1;
    st.solves += 1;
    st.sweeps += (unsigned long long)executed;
    st.other_launches += 2 + rowmajor_to_colmajor_launches(im) + (out_u ? 1 : 0) + (out_v ? 1 : 0);
    double *sig = out_sigma ? out_sigma : sigma_w;
    pick_sigma(T)<<<in, T, 0, stream>>>(a_w, lda, im, sig);
    JSVD_CUDA_TRY(cudaGetLastError());
    dim3 block(kTile, kTileRows);
    if (out_u) {
        dim3 grid((im + kTile - 1) / kTile, (in + kTile - 1) / kTile);
        colmajor_to_rowmajor_kernel<<<grid, block, 0, stream>>>(a_w, lda, im, in, out_u, sig, eps);
        JSVD_CUDA_TRY(cudaGetLastError());
    }
    if (out_v) {
        dim3 grid((in + kTile - 1) / kTile, (in + kTile - 1) / kTile);
        colmajor_to_rowmajor_kernel<<<grid, block, 0, stream>>>(v_w, ldv, in, in, out_v, nullptr, 0.0);
        JSVD_CUDA_TRY(cudaGetLastError());
    }
    if (sweeps) *sweeps = executed;
    return JSVD_OK;
}

}  // namespace jsvd

using namespace jsvd;

extern "C" int jsvd_test_wait_limit(int which, int limit_ms, int preset, int *device_status, double *elapsed_ms)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        if (which != 0 && which != 1) return invalid_argument("which must be 0 (round flags) or 1 (mbarrier).");
        if (limit_ms < 1 || limit_ms > 2000) return invalid_argument("limit_ms must be in [1, 2000].");
        int *d = nullptr;  // [0] the awaited flag, [1] the device status word
        JSVD_CUDA_TRY(cudaMalloc(&d, 2 * sizeof(int)));
        ScopeExit release([&] { cudaFree(d); });
        const int init[2] = {preset ? 1 : 0, 0};
        JSVD_CUDA_TRY(cudaMemcpy(d, init, sizeof(init), cudaMemcpyHostToDevice));
        cudaEvent_t ev[2] = {};
        for (auto &e : ev) JSVD_CUDA_TRY(cudaEventCreate(&e));
        ScopeExit destroy([&] {
            for (auto &e : ev) cudaEventDestroy(e);
        });
        const long long limit_ns = (long long)limit_ms * 1000000LL;
        JSVD_CUDA_TRY(cudaEventRecord(ev[0], 0));
        if (which == 0) {
            wait_limit_check_kernel<<<1, 32>>>(d, limit_ns, d + 1);
            JSVD_CUDA_TRY(cudaGetLastError());
        } else if (int rc = mixed_wait_limit_check(limit_ns, preset != 0, d + 1, 0); rc != JSVD_OK) {
            return rc;
        }
        JSVD_CUDA_TRY(cudaEventRecord(ev[1], 0));
        JSVD_CUDA_TRY(cudaEventSynchronize(ev[1]));
        int st = 0;
        JSVD_CUDA_TRY(cudaMemcpy(&st, d + 1, sizeof(int), cudaMemcpyDeviceToHost));
        float ms = 0.f;
        JSVD_CUDA_TRY(cudaEventElapsedTime(&ms, ev[0], ev[1]));
        if (device_status) *device_status = st;
        if (elapsed_ms) *elapsed_ms = ms;
        if (st == kDevWaitTimeout) {
            set_last_error(JSVD_ERR_RUNTIME, std::string(which == 0 ? "A round-flag" : "An mbarrier") +
                                                 " wait stopped at its limit (device status " + std::to_string(st) +
                                                 ").");
            return JSVD_ERR_RUNTIME;
        }
        return JSVD_OK;
    });
}

extern "C" int jsvd_round_robin_schedule(int n, int form, int *out, size_t capacity, size_t *needed)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        if (n < 1 || n > (1 << 16)) return invalid_argument("n must be in [1, 65536].");
        if (form != 0 && form != 1) return invalid_argument("form must be 0 (table) or 1 (closed form).");
        const int ne = n + (n & 1);
        const int rounds = n >= 2 ? ne - 1 : 0, npairs = n / 2;
        const size_t ints = 2 * (size_t)rounds * (size_t)npairs;
        if (needed) *needed = ints;
        if (out == nullptr) return JSVD_OK;
        if (capacity < ints) return invalid_argument("Schedule buffer too small.");
        if (form == 0) {
            std::vector<int2> pairs;
            int r_out = 0, p_out = 0;
            build_schedule(n, pairs, r_out, p_out);
            for (size_t i = 0; i < pairs.size(); ++i) {
                out[2 * i] = pairs[i].x;
                out[2 * i + 1] = pairs[i].y;
            }
        } else {
            size_t i = 0;
            for (int r = 0; r < rounds; ++r)
                for (int k = 0; k < npairs; ++k, ++i) {
                    const int2 pq = round_robin_pair(n, r, k);
                    out[2 * i] = pq.x;
                    out[2 * i + 1] = pq.y;
                }
        }
        return JSVD_OK;
    });
}
