// Shared device arithmetic for the one-sided Jacobi sweep (sm_100a).
//
// Every kernel of the plain path reproduces the reference's floating-point
// operations one for one (kleedaisuki/jacobi-svd-cuda src/kernels.cu):
//   * a dot product over m rows is split over T "virtual lanes": lane t
//     accumulates rows t, t+T, t+2T, ... with fused multiply-adds, then the T
//     partial sums meet in a halving tree  s[t] += s[t + stride],
//     stride = T/2, ..., 1                              (kernels.cu:412-472)
//   * rotation parameters use Rutishauser's formula     (kernels.cu:485-521)
//   * rotations update p and q columns                   (kernels.cu:534-575)
// Which physical thread holds which virtual lane is free; the order of the
// additions is not.  The files are compiled with --fmad=false so that the
// only fused operations are the explicit fma() calls written here.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace jsvd {

// Programmatic dependent launch (sm_90+ PTX).  launch_dependents lets the next
// kernel of the stream be scheduled before this one ends; wait blocks until
// every prerequisite grid has completed and its memory operations are
// visible.  Both are no-ops for a kernel launched without the attribute.
__device__ __forceinline__ void pdl_launch_dependents() { asm volatile("griddepcontrol.launch_dependents;" ::: "memory"); }
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }

// FMA placement for c*x - s*y and s*x + c*y.  nvcc contracts these two
// expressions in the reference; the forms below are the ones pinned against
// the reference binary's outputs (see oracle variant codes: p form | q form<<2).
#ifndef JSVD_ROT_P_FORM
#define JSVD_ROT_P_FORM 1  // 1: fma(c, x, -(s*y))   2: fma(-s, y, c*x)   0: no fusion
#endif
#ifndef JSVD_ROT_Q_FORM
#define JSVD_ROT_Q_FORM 1  // 1: fma(s, x, c*y)      2: fma(c, y, s*x)    0: no fusion
#endif
constexpr int kRotVariant = JSVD_ROT_P_FORM | (JSVD_ROT_Q_FORM << 2);

__host__ __device__ __forceinline__ double rot_p(double c, double s, double x, double y)
{
#if JSVD_ROT_P_FORM == 1
    return fma(c, x, -(s * y));
#elif JSVD_ROT_P_FORM == 2
    return fma(-s, y, c * x);
#else
    return c * x - s * y;
#endif
}

__host__ __device__ __forceinline__ double rot_q(double c, double s, double x, double y)
{
#if JSVD_ROT_Q_FORM == 1
    return fma(s, x, c * y);
#elif JSVD_ROT_Q_FORM == 2
    return fma(c, y, s * x);
#else
    return s * x + c * y;
#endif
}

// Pair k (0 <= k < n/2) of round r (0 <= r < rounds) of the reference's
// round-robin schedule (src/kernels.cu:637-678: fixed head, a dummy column for
// odd n, pair i = (circle[i], circle[ne-1-i])) in closed form: positions
// 1..ne-1 rotate by one per round, so position i >= 1 holds
// 1 + ((i - 1 - r) mod (ne - 1)); for odd n the value n is the dummy column
// and its slot is skipped.  The one definition used by every kernel that
// derives its pairs instead of reading a table, and by the host-side check
// (jsvd_round_robin_schedule).
__host__ __device__ __forceinline__ int2 round_robin_pair(int n, int r, int k)
{
    const int ne = n + (n & 1);
    const int L = ne - 1;
    int i = k;
    if (n & 1) {
        const int j = 1 + ((n - 1 + r) % L);
        const int slot = j < ne / 2 ? j : ne - 1 - j;
        if (i >= slot) i += 1;
    }
    const int i2 = ne - 1 - i;
    const int p = i == 0 ? 0 : 1 + ((i - 1 - r) % L + L) % L;
    const int q = 1 + ((i2 - 1 - r) % L + L) % L;
    return make_int2(p, q);
}

// Column at circle position pos (0 <= pos < ne) in round r of the same
// schedule, L = ne - 1; -1 for the dummy column of an odd n.  Slot k of a
// round pairs positions k and ne-1-k.
__host__ __device__ __forceinline__ int circle_col(int n, int L, int r, int pos)
{
    if (pos == 0) return 0;
    const int c = 1 + ((pos - 1 - r) % L + L) % L;
    return c == n ? -1 : c;
}

// Rutishauser rotation for the 2x2 Gram [pp pq; pq qq]; returns true when the
// pair rotates.  A pair that does not rotate reports c = 0, s = 0 (a real
// rotation always has c >= 1/sqrt(2)), which is how the deferred V update
// recognises it.
__device__ __forceinline__ bool rotation_params(double pp, double qq, double pq, double eps, double &c,
                                                double &s)
{
    const double rhs = eps * sqrt(fmax(pp, 0.0) * fmax(qq, 0.0));
    if (fabs(pq) > rhs && fabs(pq) > 1.0e-300) {
        const double tau = (qq - pp) / (2.0 * pq);
        const double h = fma(tau, tau, 1.0);
        const double t = (tau >= 0.0) ? (1.0 / (tau + sqrt(h))) : (-1.0 / (-tau + sqrt(h)));
        const double cs = 1.0 / sqrt(fma(t, t, 1.0));
        c = cs;
        s = t * cs;
        return true;
    }
    c = 0.0;
    s = 0.0;
    return false;
}

// Halving tree over W = T/32 per-lane register values followed by the
// in-warp levels 16..1.  On entry lane l holds y[w] = partial sum of virtual
// lane (32*w + l).  On exit lane 0 holds the reference's total.
template <int W>
__device__ __forceinline__ double warp_tree(double (&y)[W])
{
#pragma unroll
    for (int s = W / 2; s >= 1; s >>= 1) {
#pragma unroll
        for (int w = 0; w < s; ++w) y[w] += y[w + s];
    }
    double x = y[0];
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    return x;
}

__device__ __forceinline__ double warp_tree1(double x)
{
#pragma unroll
    for (int off = 16; off >= 1; off >>= 1) x += __shfl_down_sync(0xffffffffu, x, off);
    return x;
}

// Error codes written by kernels into a device status word (never trap).
enum DeviceStatus : int {
    kDevOk = 0,
    kDevBadShape = 1,
    kDevWaitTimeout = 2,
};

}  // namespace jsvd
