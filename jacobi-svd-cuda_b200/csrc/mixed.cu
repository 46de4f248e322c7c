// Blocked mixed-precision one-sided Jacobi SVD on sm_100a.
//
// The reference's sweep (src/kernels.cu:889-981) rotates one column pair at a
// time: every pair reads and writes two full columns, so a sweep of an m x n
// matrix moves about n^2/2 (6m + 4n) 8-byte words
// (tex/sections/03-gpu-parallel-reduction.tex:66-90).  Here the columns are
// grouped into blocks of kB = 32; a sweep pairs the blocks with the same
// fixed-head circle (round_robin_pair over blocks) and, for each block pair
// P = [X_i X_j] (m x 64):
//   1. Gram     G = P^T P (64 x 64), split over row ranges;
//   2. solve    G = W L W^T by cyclic two-sided Jacobi in FP64 (one CTA,
//               rounds of 32 disjoint index pairs; Rutishauser angles and the
//               reference's threshold |g_pq| <= tau sqrt(g_pp g_qq));
//   3. rotate   P <- P W, [V_i V_j] <- [V_i V_j] W, in place.
// A block round moves each column once instead of once per column round.
//
// Phase 1 (tensor cores).  X and V are held as pairs of FP32 arrays, a TF32
// head (low 13 mantissa bits zero) and its FP32 tail.  Grams and rotations run
// on tcgen05.mma kind::tf32 with FP32 accumulation in TMEM, operands fetched by
// TMA (no multicast):
//   Gram:   A operand = [h_i h_j l_i l_j]^T (M = 128, K-major, 128-byte
//           swizzle), B = [h_i h_j] then [l_i l_j] (N = 64): D[0:64] =
//           h^T (h+l), D[64:128] = l^T (h+l), G = D[0:64] + D[64:128].
//   Rotate: A operand = the 128-row tile of h (then l), MN-major (X is column
//           major; MN-major TF32 needs the 128-byte swizzle with 32-byte
//           atoms), B = [W_h | W_l] (N = 128, K-major): D[:, 0:64] =
//           (h+l) W_h, D[:, 64:128] = (h+l) W_l, out = their sum, split again.
// Phase 2 makes phase 1's V orthogonal in FP64 (Newton-Schulz iteration for
// the polar factor, V <- V (3I - V^T V)/2) and forms X' = X V' in FP64.
// Phase 3 sweeps X' in FP64 with the same block structure (DMMA GEMMs) until
// no pair rotates.  This is the mixed-precision preconditioned one-sided
// Jacobi scheme: a low-precision V, orthogonalised in working precision, then
// working-precision Jacobi (Zhou; Higham, Tisseur, Webb and Zhou, SIMAX 2021,
// for the symmetric eigenproblem).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "common.cuh"
#include "dgemm.hpp"
#include "internal.hpp"
#include "jsvd.h"
#include "mixed.hpp"
#include "mixed_tuning_table.h"
#include "plain.hpp"
#include "ptx.cuh"

namespace jsvd {
namespace {

constexpr int kB = 32;          // columns per block
constexpr int kW = 2 * kB;      // panel width (a block pair)
constexpr int kTileRows = 128;  // rows per rotation tile; working rows are padded to a multiple
constexpr int kColPad = 128;    // working columns padded to a multiple (block count stays even)

// ============================================================================
// Phase 1 kernels (tcgen05, 3xTF32)
// ============================================================================

constexpr int kGramStages = 4;
constexpr int kGramStageBytes = 4 * 4096;  // [h_i h_j l_i l_j], 32 rows x 32 columns each
constexpr size_t kGramTcSmem = 1024 + kGramStages * kGramStageBytes + 128;
constexpr int kGramTcThreads = 192;        // warps 0-3 epilogue, warp 4 TMA, warp 5 MMA

__device__ __forceinline__ uint8_t *align1024(uint8_t *p)
{
    const uint32_t a = smem_u32(p);
    return p + ((1024u - (a & 1023u)) & 1023u);
}

__device__ __forceinline__ void record_status(int *status, int code) { atomicCAS(status, 0, code); }

// Partial Gram of block pair blockIdx.y over row chunks [c0, c1) (32 rows
// each) of split blockIdx.x.  Output: the raw 128 x 64 FP32 accumulator,
// column-major, at part + (pair * splits + split) * 8192.
__global__ void __launch_bounds__(kGramTcThreads)
    mx_gram_tc(const __grid_constant__ CUtensorMap mh, const __grid_constant__ CUtensorMap ml, int nb, int round,
               int kchunks, int chunks_per_split, float *__restrict__ part, int *__restrict__ status)
{
    extern __shared__ uint8_t smraw[];
    uint8_t *sm = align1024(smraw);
    uint8_t *tiles = sm;
    uint64_t *full = reinterpret_cast<uint64_t *>(sm + kGramStages * kGramStageBytes);
    uint64_t *empty = full + kGramStages;
    uint64_t *accf = empty + kGramStages;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(accf + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pair = blockIdx.y, split = blockIdx.x;
    const int2 bp = round_robin_pair(nb, round, pair);
    const int c0 = split * chunks_per_split;
    const int nck = min(kchunks, c0 + chunks_per_split) - c0;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kGramStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(accf, 1);
        mbar_fence_init();
    }
    if (warp == 5) tmem_alloc(tslot, 64);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp == 4) {
        if (lane == 0) {
            tma_prefetch_desc(&mh);
            tma_prefetch_desc(&ml);
            for (int it = 0; it < nck; ++it) {
                const int s = it % kGramStages;
                const uint32_t ph = (uint32_t)(it / kGramStages) & 1u;
                if (!mbar_wait(&empty[s], ph ^ 1u)) {
                    record_status(status, kDevWaitTimeout);
                    break;
                }
                mbar_arrive_expect_tx(&full[s], kGramStageBytes);
                uint8_t *t = tiles + s * kGramStageBytes;
                const int row = (c0 + it) * 32;
                tma_load_2d(t, &mh, &full[s], row, bp.x * kB);
                tma_load_2d(t + 4096, &mh, &full[s], row, bp.y * kB);
                tma_load_2d(t + 8192, &ml, &full[s], row, bp.x * kB);
                tma_load_2d(t + 12288, &ml, &full[s], row, bp.y * kB);
            }
        }
        __syncwarp();
    } else if (warp == 5) {
        if (lane == 0) {
            constexpr uint32_t idesc = idesc_tf32(128, 64, 0, 0);
            for (int it = 0; it < nck; ++it) {
                const int s = it % kGramStages;
                const uint32_t ph = (uint32_t)(it / kGramStages) & 1u;
                if (!mbar_wait(&full[s], ph)) {
                    record_status(status, kDevWaitTimeout);
                    break;
                }
                tc_fence_after();
                const uint32_t base = smem_u32(tiles + s * kGramStageBytes);
#pragma unroll
                for (int ks = 0; ks < 4; ++ks) {  // K = 8 TF32 per MMA = 32 bytes of the 128-byte row
                    const uint64_t a = smem_desc_sw128(base + ks * 32, 16, 1024);
                    const uint64_t bh = smem_desc_sw128(base + ks * 32, 16, 1024);
                    const uint64_t bl = smem_desc_sw128(base + 8192 + ks * 32, 16, 1024);
                    tc_mma_tf32(tmem, a, bh, idesc, (it > 0 || ks > 0) ? 1u : 0u);
                    tc_mma_tf32(tmem, a, bl, idesc, 1u);
                }
                tc_commit(&empty[s]);
            }
            tc_commit(accf);
        }
        __syncwarp();
    }
    if (warp < 4) {
        const bool ok = mbar_wait(accf, 0);
        tc_fence_after();
        if (!ok) {
            record_status(status, kDevWaitTimeout);
        } else {
            float *out = part + ((size_t)pair * gridDim.x + split) * (128 * 64);
            const int r = warp * 32 + lane;
            float v[32];
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                tmem_ld32(tmem + ((uint32_t)(warp * 32) << 16) + half * 32, v);
#pragma unroll
                for (int c = 0; c < 32; ++c) out[(size_t)(half * 32 + c) * 128 + r] = v[c];
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 5) {
        tc_fence_after();
        tmem_dealloc(tmem, 64);
    }
}

constexpr int kRotTcThreads = 128;
constexpr int kRotAOff = 0;      // A: [h|l] x [block i|block j] x 4 row atoms x 4 KB = 64 KB
constexpr int kRotBOff = 65536;  // B: 2 K-atoms x 128 rows x 128 bytes = 32 KB
constexpr int kRotBarOff = 98304;
constexpr size_t kRotTcSmem = 1024 + 98304 + 64;

// Rotation of one 128-row tile of the block pair blockIdx.y, in X (tiles
// [0, x_tiles)) or in V (tiles from x_tiles on): [h + l] <- [h + l] W.  The
// tensor maps are the 32-byte-atom swizzled ones (A is MN-major): each 4 KB box
// is 32 K rows (columns of P) of 128 bytes (32 rows of P), groups of 4 K rows
// 512 bytes apart (SBO), the four 32-row atoms of the tile 4096 bytes apart
// (LBO).
// Entry W(k, n) of a pair's rotation in the rotation kernel's B operand
// image: row n (head) and row 64 + n (tail) hold column n of W along K (K
// major, 128-byte swizzle, two 32-float K atoms), 32 KB per pair, laid out
// exactly as the kernel's shared-memory B region.
__device__ __forceinline__ void rot_b_store(float *img, int k, int n, double wv)
{
    float h, l;
    split_tf32((float)wv, h, l);
    const int atom = k >> 5, kk = k & 31;
#pragma unroll
    for (int hl = 0; hl < 2; ++hl) {
        const int row = n + hl * 64;
        const int off = atom * 16384 + row * 128 + (((kk >> 2) ^ (row & 7)) << 4) + (kk & 3) * 4;
        img[off >> 2] = hl ? l : h;
    }
}

constexpr int kRotImgFloats = 8192;  // 32 KB per block pair

// B operand images of the pairs that rotate, from W (the eigen-solve writes
// them itself; this builds them from a given W).
__global__ void __launch_bounds__(256) mx_rot_image(const double *__restrict__ W, float *__restrict__ img,
                                                    const int *__restrict__ flags)
{
    const int pair = blockIdx.x;
    if (flags[pair] == 0) return;
    for (int e = threadIdx.x; e < kW * kW; e += blockDim.x)
        rot_b_store(img + (size_t)pair * kRotImgFloats, e & 63, e >> 6, W[(size_t)pair * kW * kW + e]);
}

__global__ void __launch_bounds__(kRotTcThreads)
    mx_rot_tc(const __grid_constant__ CUtensorMap mxh, const __grid_constant__ CUtensorMap mxl,
              const __grid_constant__ CUtensorMap mvh, const __grid_constant__ CUtensorMap mvl,
              float *__restrict__ xh, float *__restrict__ xl, long ldx, int x_tiles, float *__restrict__ vh,
              float *__restrict__ vl, long ldv, int nb, int round, const float *__restrict__ Wimg,
              const int *__restrict__ flags, int *__restrict__ status)
{
    const int pair = blockIdx.y;
    if (flags[pair] == 0) return;  // W = I: the tile stays as it is
    extern __shared__ uint8_t smraw[];
    uint8_t *sm = align1024(smraw);
    uint64_t *full = reinterpret_cast<uint64_t *>(sm + kRotBarOff);
    uint64_t *accf = full + 1;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(accf + 1);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const bool onV = (int)blockIdx.x >= x_tiles;
    const CUtensorMap *mh = onV ? &mvh : &mxh;
    const CUtensorMap *ml = onV ? &mvl : &mxl;
    float *oh = onV ? vh : xh;
    float *ol = onV ? vl : xl;
    const long ld = onV ? ldv : ldx;
    const int row0 = (onV ? (int)blockIdx.x - x_tiles : (int)blockIdx.x) * kTileRows;
    const int2 bp = round_robin_pair(nb, round, pair);

    if (threadIdx.x == 0) {
        mbar_init(full, 1);
        mbar_init(accf, 1);
        mbar_fence_init();
    }
    if (warp == 0) tmem_alloc(tslot, 128);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (threadIdx.x == 0) {
        // the A tiles (64 KB) and the pair's B image, [W_h | W_l] (32 KB)
        mbar_arrive_expect_tx(full, 65536 + 32768);
#pragma unroll
        for (int hl = 0; hl < 2; ++hl)
#pragma unroll
            for (int half = 0; half < 2; ++half)
#pragma unroll
                for (int g = 0; g < 4; ++g)
                    tma_load_2d(sm + kRotAOff + hl * 32768 + half * 16384 + g * 4096, hl ? ml : mh, full,
                                row0 + g * 32, (half ? bp.y : bp.x) * kB);
        bulk_load(sm + kRotBOff, Wimg + (size_t)pair * kRotImgFloats, 32768, full);
    }
    fence_proxy_async_smem();
    __syncthreads();
    if (threadIdx.x == 0) {
        constexpr uint32_t idesc = idesc_tf32(128, 128, 1, 0);
        if (!mbar_wait(full, 0)) {
            record_status(status, kDevWaitTimeout);
        } else {
            tc_fence_after();
            const uint32_t abase = smem_u32(sm + kRotAOff), bbase = smem_u32(sm + kRotBOff);
#pragma unroll
            for (int ks = 0; ks < 8; ++ks) {
                const int half = ks >> 2, g8 = ks & 3;
                const uint64_t b = smem_desc_sw128(bbase + half * 16384 + g8 * 32, 16, 1024);
                const uint64_t ah = smem_desc(abase + half * 16384 + g8 * 1024, 4096, 512, kSwizzle128B32BAtom);
                const uint64_t al =
                    smem_desc(abase + 32768 + half * 16384 + g8 * 1024, 4096, 512, kSwizzle128B32BAtom);
                tc_mma_tf32(tmem, ah, b, idesc, ks > 0 ? 1u : 0u);
                tc_mma_tf32(tmem, al, b, idesc, 1u);
            }
        }
        tc_commit(accf);
    }
    __syncwarp();
    const bool ok = mbar_wait(accf, 0);
    tc_fence_after();
    if (!ok) {
        record_status(status, kDevWaitTimeout);
    } else {
        const int r = row0 + warp * 32 + lane;
        const uint32_t lane_addr = tmem + ((uint32_t)(warp * 32) << 16);
#pragma unroll
        for (int cc = 0; cc < 2; ++cc) {
            float a[32], b[32];
            tmem_ld32(lane_addr + cc * 32, a);
            tmem_ld32(lane_addr + 64 + cc * 32, b);
            const int col0 = (cc ? bp.y : bp.x) * kB;
#pragma unroll
            for (int c = 0; c < 32; ++c) {
                float h, l;
                split_tf32(a[c] + b[c], h, l);
                const size_t idx = (size_t)r + (size_t)(col0 + c) * ld;
                oh[idx] = h;
                ol[idx] = l;
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) {
        tc_fence_after();
        tmem_dealloc(tmem, 128);
    }
}

// ============================================================================
// Phase 3 kernels (FP64, DMMA)
// ============================================================================

constexpr int kGram64Threads = 256;
constexpr int kGram64Rows = 32;             // rows of P per stage
constexpr int kGram64LD = kGram64Rows + 4;  // Ps[col][row]
constexpr int kGram64Stages = 3;
constexpr size_t kGram64Smem = sizeof(double) * kGram64Stages * kW * kGram64LD;

// Partial Gram of block pair blockIdx.y over rows [r0, r1) of split
// blockIdx.x; output 64 x 64 FP64 column-major at part + (pair*splits+split)*4096,
// upper triangle only (the 36 8 x 8 tiles (i, j), i <= j; the lower halves of
// the diagonal tiles are written too and ignored).  Warp w computes tiles
// w, w + 8, ... of the row-major list of upper tiles (4 or 5 DMMA tiles).
__device__ __forceinline__ int2 upper_tile(int t)
{
    int i = 0;
    while (t >= 8 - i) {
        t -= 8 - i;
        ++i;
    }
    return make_int2(i, i + t);
}

__global__ void __launch_bounds__(kGram64Threads)
    mx_gram_f64(const double *__restrict__ X, long ldx, int nb, int round, int rows_per_split, int rows,
                double *__restrict__ part)
{
    extern __shared__ double dsm[];
    const int pair = blockIdx.y, split = blockIdx.x;
    const int2 bp = round_robin_pair(nb, round, pair);
    const int r0 = split * rows_per_split, r1 = min(rows, r0 + rows_per_split);
    const int nst = (r1 - r0 + kGram64Rows - 1) / kGram64Rows;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int fr = lane >> 2, fk = lane & 3;
    auto issue = [&](int st) {
        double *s = dsm + (st % kGram64Stages) * kW * kGram64LD;
        const int rb = r0 + st * kGram64Rows;
        for (int e = threadIdx.x; e < kW * kGram64Rows; e += kGram64Threads) {
            const int k = e & 31, c = e >> 5;
            const int gc = (c < kB ? bp.x * kB + c : bp.y * kB + (c - kB));
            const int gr = rb + k;
            double *d = s + c * kGram64LD + k;
            if (gr < r1)
                cp_async8(d, X + (size_t)gr + (size_t)gc * ldx);
            else
                *d = 0.0;
        }
    };
    constexpr int kTiles = 36, kPerWarp = 5;
    int ti[kPerWarp], tj[kPerWarp];
#pragma unroll
    for (int u = 0; u < kPerWarp; ++u) {
        const int t = warp + 8 * u;
        const int2 ij = upper_tile(t < kTiles ? t : 0);
        ti[u] = ij.x;
        tj[u] = ij.y;
    }
    const int ntiles = warp < kTiles - 32 ? kPerWarp : kPerWarp - 1;  // warps 0-3: 5 tiles, 4-7: 4
    double acc[kPerWarp][2];
#pragma unroll
    for (int u = 0; u < kPerWarp; ++u) acc[u][0] = acc[u][1] = 0.0;
#pragma unroll
    for (int s = 0; s < kGram64Stages - 1; ++s) {
        if (s < nst) issue(s);
        cp_async_commit();
    }
    for (int st = 0; st < nst; ++st) {
        cp_async_wait<kGram64Stages - 2>();
        __syncthreads();
        if (st + kGram64Stages - 1 < nst) issue(st + kGram64Stages - 1);
        cp_async_commit();
        const double *s = dsm + (st % kGram64Stages) * kW * kGram64LD;
#pragma unroll
        for (int kk = 0; kk < kGram64Rows; kk += 4) {
            // A = P^T (row i of A = column i of P), B = P
#pragma unroll
            for (int u = 0; u < kPerWarp; ++u) {
                if (u < ntiles) {
                    const double a = s[(ti[u] * 8 + fr) * kGram64LD + kk + fk];
                    const double b = s[(tj[u] * 8 + fr) * kGram64LD + kk + fk];
                    dmma_m8n8k4(acc[u], a, b);
                }
            }
        }
    }
    cp_async_wait<0>();
    double *out = part + ((size_t)pair * gridDim.x + split) * (kW * kW);
#pragma unroll
    for (int u = 0; u < kPerWarp; ++u) {
        if (u < ntiles) {
            const int row = ti[u] * 8 + fr, col = tj[u] * 8 + 2 * fk;
            out[(size_t)col * kW + row] = acc[u][0];
            out[(size_t)(col + 1) * kW + row] = acc[u][1];
        }
    }
}

constexpr int kRot64Threads = 256;
constexpr int kRot64PLD = kTileRows + 8;  // Pt[col][row]
constexpr int kRot64WLD = kW + 4;         // Ws[col][k]
constexpr size_t kRot64Smem = sizeof(double) * (kW * kRot64PLD + kW * kRot64WLD);

// Rotation of one 128-row tile of block pair blockIdx.y (X tiles, then V
// tiles), FP64: P <- P W.  Warp w computes rows 16w..16w+15 x 64 columns.
__global__ void __launch_bounds__(kRot64Threads)
    mx_rot_f64(double *__restrict__ X, long ldx, int x_tiles, double *__restrict__ V, long ldv, int nb, int round,
               const double *__restrict__ W, const int *__restrict__ flags)
{
    const int pair = blockIdx.y;
    if (flags[pair] == 0) return;
    extern __shared__ double dsm[];
    double *Pt = dsm;                   // [64 cols][136]
    double *Ws = dsm + kW * kRot64PLD;  // [64 cols][68]
    const bool onV = (int)blockIdx.x >= x_tiles;
    double *M = onV ? V : X;
    const long ld = onV ? ldv : ldx;
    const int row0 = (onV ? (int)blockIdx.x - x_tiles : (int)blockIdx.x) * kTileRows;
    const int2 bp = round_robin_pair(nb, round, pair);
    const double *wp = W + (size_t)pair * kW * kW;
    for (int e = threadIdx.x; e < kW * kW; e += kRot64Threads) {
        const int k = e & 63, c = e >> 6;
        cp_async8(Ws + c * kRot64WLD + k, wp + e);
    }
    for (int e = threadIdx.x; e < kW * kTileRows; e += kRot64Threads) {
        const int r = e & (kTileRows - 1), c = e >> 7;
        const int gc = c < kB ? bp.x * kB + c : bp.y * kB + (c - kB);
        cp_async8(Pt + c * kRot64PLD + r, M + (size_t)(row0 + r) + (size_t)gc * ld);
    }
    cp_async_commit();
    cp_async_wait<0>();
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int fr = lane >> 2, fk = lane & 3;
    double acc[2][8][2];
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
#pragma unroll 4
    for (int kk = 0; kk < kW; kk += 4) {
        double a[2], b[8];
#pragma unroll
        for (int i = 0; i < 2; ++i) a[i] = Pt[(kk + fk) * kRot64PLD + warp * 16 + i * 8 + fr];
#pragma unroll
        for (int j = 0; j < 8; ++j) b[j] = Ws[(j * 8 + fr) * kRot64WLD + kk + fk];
#pragma unroll
        for (int i = 0; i < 2; ++i)
#pragma unroll
            for (int j = 0; j < 8; ++j) dmma_m8n8k4(acc[i][j], a[i], b[j]);
    }
    __syncthreads();  // every warp is done reading Pt
#pragma unroll
    for (int i = 0; i < 2; ++i)
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const int r = warp * 16 + i * 8 + fr, c = j * 8 + 2 * fk;
            Pt[c * kRot64PLD + r] = acc[i][j][0];
            Pt[(c + 1) * kRot64PLD + r] = acc[i][j][1];
        }
    __syncthreads();
    for (int e = threadIdx.x; e < kW * kTileRows; e += kRot64Threads) {
        const int r = e & (kTileRows - 1), c = e >> 7;
        const int gc = c < kB ? bp.x * kB + c : bp.y * kB + (c - kB);
        M[(size_t)(row0 + r) + (size_t)gc * ld] = Pt[c * kRot64PLD + r];
    }
}

// ============================================================================
// Block eigen-solve (FP64, both phases)
// ============================================================================

constexpr int kEvdThreads = 512;      // warps 0-7: W (and 48 blocks of G); warps 8-14: G; warp 15: the angles
constexpr int kEvdWThreads = 256;     // a warp per (half of the rows, quarter of the slots) of W
constexpr int kEvdBulkThreads = 224;  // warps 8-14
constexpr int kEvdQ = kW / 2 + 1;     // row stride of a quadrant of G (odd: column accesses hit distinct banks)
constexpr int kEvdQuad = (kW / 2) * kEvdQ;  // one 32 x 33 quadrant
constexpr int kEvdG = 3 * kEvdQuad;   // G: first-first, first-second, second-second quadrants
constexpr int kEvdTmpLD = kW + 1;     // the input Gram in column coordinates (set-up only)
constexpr int kOffBlocks = (kW / 2) * (kW / 2 - 1) / 2;  // 2x2 blocks (a < b) of the 32 x 32 block grid
constexpr int kEvdBulkIters = 2;      // blocks per G thread (the last 48 go to W threads 0-47)
constexpr int kEvdRounds = kW - 1;
constexpr int kEvdMaxInner = 8;
constexpr size_t kEvdSmem = sizeof(double) * (kEvdG + kW * kEvdTmpLD);  // G0, then G1 / the set-up buffer
static_assert(kOffBlocks - kEvdBulkIters * kEvdBulkThreads <= kEvdWThreads, "G blocks left for the W warps");

// Rotation of [pp pq; pq qq] that annihilates pq, with the reference's
// threshold test (|pq| > tau sqrt(pp qq), squared, and |pq| > 1e-300), in
// two parts: evd_prepare takes what depends on the diagonal only (known a
// round ahead), evd_rotation the rest once pq is known.
//   t = tan(theta), the smaller root of t^2 + 2 zeta t - 1 = 0 with
//   zeta = (qq - pp) / (2 pq) (Rutishauser's choice), c = 1 / sqrt(1 + t^2),
//   s = t c, sign(t) = sign(e) for d = qq - pp >= 0 and -sign(e) otherwise
//   (e = 2 pq).
// Small angles (x = |e| / (2 |d|) <= 2^-6): t = (sqrt(1 + 4x^2) - 1) / (2x)
// = x - x^3 + 2x^5 - 5x^7 + 14x^9 - ... (Catalan-number coefficients) and
// c = (1 + t^2)^(-1/2) = 1 - z/2 + 3z^2/8 - 5z^3/16 + 35z^4/128 - ...
// (z = t^2): the terms left out are below 2^-54 relative, so both series,
// evaluated by Horner's rule from the precomputed 1 / (2 |d|), are exact to
// rounding: ten fused operations and no square root or division.  Called by
// a full warp; the path is chosen for the whole warp.  Otherwise, with rho = 1 / sqrt(d^2 + e^2), cos 2theta =
// |d| rho and sin 2theta = |e| rho, and the half-angle identities give
//   c^2 = (1 + cos 2theta) / 2 in [1/2, 1],  c = c^2 / sqrt(c^2),
//   |s| = sin 2theta / (2c),  |t| = |s| / c:
// two reciprocal square roots, no cancellation; d and e are scaled by a
// power of two when their magnitude could over- or underflow d^2 + e^2.
struct EvdPre {
    double d;    // qq - pp
    double thr;  // tau^2 max(pp, 0) max(qq, 0)
    double r2;   // 1 / (2 |d|) (infinite for d = 0), to about one ulp
};

__device__ __forceinline__ EvdPre evd_prepare(double pp, double qq, double tau)
{
    EvdPre p;
    p.d = qq - pp;
    p.thr = (tau * tau) * (fmax(pp, 0.0) * fmax(qq, 0.0));
    // 1 / (2 |d|) by Newton's iteration r <- r (2 - |d| r) from a
    // single-precision reciprocal (two steps: 2^-23 -> 2^-46 -> rounding);
    // outside the single-precision range, by division
    const double ad = fabs(p.d);
    if (ad > 1.0e-30 && ad < 1.0e30) {
        double r = (double)__frcp_rn((float)ad);
        r = r * fma(-ad, r, 2.0);
        r = r * fma(-ad, r, 2.0);
        p.r2 = 0.5 * r;
    } else {
        p.r2 = 0.5 / ad;
    }
    return p;
}

__device__ __forceinline__ bool evd_rotation(const EvdPre &p, double pq, double &c, double &s, double &t)
{
    const bool rot = fabs(pq) > 1.0e-300 && pq * pq > p.thr;
    double d = p.d, e = 2.0 * pq;
    const double sg = ((d >= 0.0) == (e >= 0.0)) ? 1.0 : -1.0;
    const double x = fabs(e) * p.r2;
    double ta, ca, sa;
    // one path for the whole warp (the caller's 32 lanes are all active): the
    // series when every rotating lane's angle is small, else the exact form
    if (__all_sync(0xffffffffu, x <= 0x1p-6 || !rot)) {
        const double y = x * x;
        double p = fma(14.0, y, -5.0);
        p = fma(p, y, 2.0);
        p = fma(p, y, -1.0);
        p = fma(p, y, 1.0);
        ta = x * p;
        const double z = ta * ta;
        double q = fma(35.0 / 128.0, z, -5.0 / 16.0);
        q = fma(q, z, 3.0 / 8.0);
        q = fma(q, z, -0.5);
        ca = fma(q, z, 1.0);
        sa = ta * ca;
    } else {
        const double f = fmax(fabs(d), fabs(e));
        if (rot && (f > 1.0e150 || f < 1.0e-150)) {
            const int k = ilogb(f);
            d = scalbn(d, -k);
            e = scalbn(e, -k);
        }
        const double rho = rsqrt(fma(d, d, e * e));
        const double c2 = fma(0.5 * fabs(d), rho, 0.5);
        const double hs = (0.5 * fabs(e)) * rho;  // sin 2theta / 2
        const double rc = rsqrt(c2);              // 1 / c
        ca = c2 * rc;
        sa = hs * rc;
        ta = sa * rc;
    }
    c = rot ? ca : 1.0;
    s = rot ? sg * sa : 0.0;
    t = rot ? sg * ta : 0.0;
    return rot;
}

// Slots.  The 64 indices of the eigen-solve move through the circle of the
// round-robin ordering; instead of looking the pairs up per round, every
// index lives in a slot: in each inner round, pair k rotates slots 2k (its
// first index) and 2k + 1 (its second), and the round-robin advance between
// rounds is one fixed permutation of the slots, evd_next_slot:
//   first'[0] = first[0], first'[1] = second[0], first'[k] = first[k-1],
//   second'[k] = second[k+1] (k < 31), second'[31] = first[31].
// At the start (and after every full sweep of 63 rounds, the permutation's
// order) slot 2k holds index k and slot 2k+1 index 63 - k, which is pair k of
// round 0 of the circle (round_robin_pair).
__device__ __forceinline__ int evd_slot_column(int slot) { return (slot & 1) ? 63 - (slot >> 1) : (slot >> 1); }
__device__ __forceinline__ int evd_column_slot(int col) { return col < 32 ? 2 * col : 127 - 2 * col; }
__device__ __forceinline__ int evd_next_slot(int s)
{
    if (s == 0) return 0;
    if (s == 1) return 2;
    if (s == 62) return 63;
    return (s & 1) ? s - 2 : s + 2;
}
// G is symmetric; it is kept as three 32 x 33 quadrants indexed by pair:
// FF[k][l] = G(first k, first l) and SS[k][l] = G(second k, second l) for
// k <= l, FS[k][l] = G(first k, second l) for all k, l.  The update of block
// (a, b) reads FF[a][b], FS[a][b], FS[b][a], SS[a][b] and, after the circle's
// advance (first k -> first k+1, second k -> second k-1), writes
// FF[a+1][b+1], FS[a+1][b-1], FS[b+1][a-1], SS[a-1][b-1] (except at the
// circle's ends): with the odd row stride every one of those eight addresses
// falls in bank (a + b + constant) mod 16, so a warp whose 32 blocks cover
// each residue of a + b twice accesses G without bank conflicts.
__device__ __forceinline__ int evd_off(int s, int t)
{
    const int ks = s >> 1, kt = t >> 1;
    if ((s & 1) == (t & 1)) return ((s & 1) ? 2 * kEvdQuad : 0) + min(ks, kt) * kEvdQ + max(ks, kt);
    return (s & 1) ? kEvdQuad + kt * kEvdQ + ks : kEvdQuad + ks * kEvdQ + kt;
}

// The k-th off-diagonal block (a < b) with (a + b) mod 16 == r, in order of
// a + b, then a.  Residues r even have 30 blocks, odd 32.
__device__ __forceinline__ int2 evd_block_of(int r, int k)
{
    for (int d = r; d <= kW - 3; d += 16) {
        if (d < 1) continue;
        const int lo = max(0, d - (kW / 2 - 1)), hi = (d - 1) >> 1;
        const int cnt = hi - lo + 1;
        if (cnt > 0) {
            if (k < cnt) return make_int2(lo + k, d - lo - k);
            k -= cnt;
        }
    }
    return make_int2(-1, -1);
}

// W in registers, in slots.  Warp w < 8 holds rows 32 (w & 1) + lane of
// quarter q = w >> 1 of the slots (pairs 8q .. 8q+7, slots 16q .. 16q+15,
// local index j <-> pair 8q + j), w[2j] = first, w[2j+1] = second: every
// lane of a warp applies the same eight rotations (one broadcast load each).
__device__ __forceinline__ void evd_w_rotate(double (&w)[16], const double2 *cs, int q)
{
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const double2 r = cs[8 * q + j];
        const double x = w[2 * j], y = w[2 * j + 1];
        w[2 * j] = fma(r.x, x, -(r.y * y));
        w[2 * j + 1] = fma(r.y, x, r.x * y);
    }
}

// Advance of the circle for one quarter row: up = first[8q - 1] of the
// quarter below, down = second[8q + 8] of the quarter above (both from the
// warps holding them, through shared memory).
__device__ __forceinline__ void evd_w_advance(double (&w)[16], int q, double up, double down)
{
    double f[8], s[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        f[j] = w[2 * j];
        s[j] = w[2 * j + 1];
    }
    w[0] = q == 0 ? f[0] : up;
    w[2] = q == 0 ? s[0] : f[0];
#pragma unroll
    for (int j = 2; j < 8; ++j) w[2 * j] = f[j - 1];
#pragma unroll
    for (int j = 0; j < 7; ++j) w[2 * j + 1] = s[j + 1];
    w[15] = q == 3 ? f[7] : down;
}

// Input Gram of block pair blockIdx.x from `splits` partials: kind 0 = the
// tensor-core layout (128 x 64 FP32, rows r and r + 64 summed), kind 1 =
// 64 x 64 FP64 upper triangle.  Cyclic two-sided Jacobi, at most
// inner_sweeps sweeps of 63 rounds of 32 disjoint index pairs, in slot
// coordinates (above), software pipelined so that a round costs one barrier
// and the angle chain runs beside the update:
//   * G (upper triangle, slot coordinates) is double-buffered: round r reads
//     buffer r%2 and writes buffer (r+1)%2 already advanced to round r+1's
//     slots, so every thread reads and writes the same addresses in every
//     round (kept in registers, no table lookups);
//   * warps 8-14 (and threads 0-47) apply round r to the off-diagonal 2 x 2
//     blocks of slot pairs (a, b), a < b (two 16-byte loads, four stores, the
//     unrotated blocks copied: c = 1, s = 0 reproduce them);
//   * warps 0-7 apply it to W (registers; the advance of the circle across
//     quarters goes through shared memory and completes a round later);
//   * warp 15 (lane k: pair k) writes the diagonal blocks (the annihilated
//     pairs) and derives the angles of round r+1 from buffer r%2 and round
//     r's rotations: pair k of round r+1 takes its first index from pair k-1
//     of round r (pair 0 for k <= 1) and its second from pair k+1 (pair 31
//     for k = 31), so its diagonal entries are round r's annihilated
//     diagonals and its off-diagonal entry is one element of one 2 x 2 block
//     update, computed with the same operations as the update itself
//     (bit-identical to what lands in the buffer).  Everything that depends
//     on round r's angles only (the new diagonals, the neighbours' angles,
//     the diagonal part of the rotation) is done before round r's barrier.
// Writes W (64 x 64, column-major) - and, when Wimg is not null, its 3xTF32
// operand image for the tensor-core rotation - and flags[pair] = 1 when some
// pair rotated (else flags[pair] = 0 and W is left as it was).  stats[0] (as
// double bits) = running max of |g_pq| / sqrt(g_pp g_qq) over the input
// Grams, stats[1] = number of block pairs that rotated.
__global__ void __launch_bounds__(kEvdThreads, 1)
    mx_evd(const void *__restrict__ part, int kind, int splits, double tau, int inner_sweeps, int nb, int round,
           int sort, int ncols, double *__restrict__ Wout, float *__restrict__ Wimg, int *__restrict__ flags,
           unsigned long long *__restrict__ stats)
{
    extern __shared__ __align__(16) double dsm[];
    double *const G0 = dsm;                 // [64][66], buffer 0
    double *const G1 = dsm + kEvdG;         // buffer 1 (and, at set-up, the Gram in column coordinates)
    __shared__ double2 cs[2][kW / 2];       // (c, s) of the 32 pairs, by round parity (W: broadcast loads)
    __shared__ double cs_c[2][kW / 2], cs_s[2][kW / 2];  // the same, apart (G: 8-byte loads of many pairs)
    __shared__ double xf[2][4][kW];         // W advance: first[8q + 7] of quarter q, by row
    __shared__ double xs[2][4][kW];         // W advance: second[8q] of quarter q, by row
    __shared__ unsigned rot_mask[2];
    __shared__ int sweep_any[kEvdMaxInner + 1];
    __shared__ int out_col[kW];
    __shared__ unsigned long long off_bits;
    const int pair = blockIdx.x;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int nsweeps = min(inner_sweeps, kEvdMaxInner);
    if (tid == 0) off_bits = 0ull;
    if (tid <= kEvdMaxInner) sweep_any[tid] = 0;
    // the input Gram in column coordinates, in buffer 1.  Thread t sums rows
    // 4j .. 4j+3 of column c for (c, j) = ((t + 512 i) >> 4, (t + 512 i) & 15),
    // i = 0..1, over the splits: 16-byte loads, four per split in flight
    // (kind 0 adds rows r and r + 64 of the partial in the same order as the
    // element-wise sum: g += lo + hi).
    {
        constexpr int kI = kW * kW / 4 / kEvdThreads;
        double acc[kI][4];
#pragma unroll
        for (int i = 0; i < kI; ++i)
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[i][k] = 0.0;
        if (kind == 0) {
            const float *p = static_cast<const float *>(part) + (size_t)pair * splits * 8192;
#pragma unroll 4
            for (int s = 0; s < splits; ++s) {
                float4 lo[kI], hi[kI];
#pragma unroll
                for (int i = 0; i < kI; ++i) {
                    const int o = tid + kEvdThreads * i, c = o >> 4, j = o & 15;
                    const float *q = p + (size_t)s * 8192 + c * 128 + 4 * j;
                    lo[i] = __ldg(reinterpret_cast<const float4 *>(q));
                    hi[i] = __ldg(reinterpret_cast<const float4 *>(q + 64));
                }
#pragma unroll
                for (int i = 0; i < kI; ++i) {
                    acc[i][0] += (double)lo[i].x + (double)hi[i].x;
                    acc[i][1] += (double)lo[i].y + (double)hi[i].y;
                    acc[i][2] += (double)lo[i].z + (double)hi[i].z;
                    acc[i][3] += (double)lo[i].w + (double)hi[i].w;
                }
            }
        } else {
            const double *p = static_cast<const double *>(part) + (size_t)pair * splits * 4096;
#pragma unroll 4
            for (int s = 0; s < splits; ++s) {
                double2 x0[kI], x1[kI];
#pragma unroll
                for (int i = 0; i < kI; ++i) {
                    const int o = tid + kEvdThreads * i, c = o >> 4, j = o & 15;
                    const double *q = p + (size_t)s * 4096 + c * 64 + 4 * j;
                    x0[i] = __ldg(reinterpret_cast<const double2 *>(q));
                    x1[i] = __ldg(reinterpret_cast<const double2 *>(q + 2));
                }
#pragma unroll
                for (int i = 0; i < kI; ++i) {
                    acc[i][0] += x0[i].x;
                    acc[i][1] += x0[i].y;
                    acc[i][2] += x1[i].x;
                    acc[i][3] += x1[i].y;
                }
            }
        }
#pragma unroll
        for (int i = 0; i < kI; ++i) {
            const int o = tid + kEvdThreads * i, c = o >> 4, j = o & 15;
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const int r = 4 * j + k;
                if (kind == 0) {
                    G1[r * kEvdTmpLD + c] = acc[i][k];
                } else if (r <= c) {  // the FP64 Gram kernel writes the upper triangle only: mirror it
                    G1[r * kEvdTmpLD + c] = acc[i][k];
                    G1[c * kEvdTmpLD + r] = acc[i][k];
                }
            }
        }
    }
    // W: warp w < 8 holds rows 32 (w & 1) + lane, quarter w >> 1 of the slots
    const int wrow = 32 * (warp & 1) + lane, quarter = (warp >> 1) & 3;
    double w[16];
#pragma unroll
    for (int j = 0; j < 16; ++j) w[j] = (evd_slot_column(16 * quarter + j) == wrow) ? 1.0 : 0.0;
    __syncthreads();
    // symmetrise (the two triangles come from different accumulation orders)
    // into buffer 0 in slot coordinates, measure the input's largest scaled
    // off-diagonal entry, and find whether any index pair passes the rotation
    // test at all: if none does, no round can rotate (G never changes) and the
    // solve is skipped
    double off = 0.0;
    int need = 0;
    for (int e = tid; e < kW * kW; e += kEvdThreads) {
        const int r = e >> 6, c = e & 63;
        if (r <= c) {
            const double g = r < c ? 0.5 * (G1[r * kEvdTmpLD + c] + G1[c * kEvdTmpLD + r]) : G1[r * kEvdTmpLD + r];
            G0[evd_off(evd_column_slot(r), evd_column_slot(c))] = g;
            if (r < c) {
                const double a = fmax(G1[r * kEvdTmpLD + r], 0.0) * fmax(G1[c * kEvdTmpLD + c], 0.0);
                const double d = sqrt(a);
                if (d > 0.0) off = fmax(off, fabs(g) / d);
                if (fabs(g) > 1.0e-300 && g * g > (tau * tau) * a) need = 1;
            }
        }
    }
    if (off > 0.0) atomicMax(&off_bits, (unsigned long long)__double_as_longlong(off));
    // the off-diagonal 2 x 2 blocks a thread updates in every round: a group
    // of 32 blocks per warp and iteration in which each half-warp holds every
    // residue of a + b mod 16 once (shared memory serves a half-warp's 8-byte
    // accesses per wavefront; groups 0-13: G warps 8-14, two each; group 14:
    // warp 0; group 15, 16 blocks of odd residue: lanes 0-15 of warp 1).  Per block: the pair indices
    // (a | b << 8), the offsets of FF[a][b] (FS[a][b] and SS[a][b] follow at
    // fixed distances) and of FS[b][a], and the destinations of its four
    // entries after the advance, two per int
    int blk[kEvdBulkIters], rof[kEvdBulkIters], w01[kEvdBulkIters], w23[kEvdBulkIters];
#pragma unroll
    for (int j = 0; j < kEvdBulkIters; ++j) {
        int g = -1;
        if (warp >= 8 && warp < 15) g = 2 * (warp - 8) + j;
        else if (j == 0 && warp == 0) g = 14;
        else if (j == 0 && warp == 1 && lane < 16) g = 15;
        blk[j] = -1;
        rof[j] = w01[j] = w23[j] = 0;
        if (g >= 0) {
            const int2 ab = g < 15 ? evd_block_of(lane & 15, 2 * g + (lane >> 4))
                                   : evd_block_of(2 * (lane & 7) + 1, 30 + (lane >> 3));
            const int a = ab.x, b = ab.y;
            const int pa = evd_next_slot(2 * a), qa = evd_next_slot(2 * a + 1);
            const int pb = evd_next_slot(2 * b), qb = evd_next_slot(2 * b + 1);
            blk[j] = a | (b << 8);
            rof[j] = evd_off(2 * a, 2 * b) | (evd_off(2 * a + 1, 2 * b) << 16);
            w01[j] = evd_off(pa, pb) | (evd_off(pa, qb) << 16);
            w23[j] = evd_off(qa, pb) | (evd_off(qa, qb) << 16);
        }
    }
    const bool work = __syncthreads_or(need) != 0;
    // warp 15, lane k = pair k: its diagonal block's destinations, the block
    // (A, B) holding the off-diagonal entry of its next pair, and its state
    // from round to round: the pair's entries and rotation (pp, qq, pq, c, s,
    // t, rotated), the rotated diagonals nd0, nd1, the next pair's diagonal
    // part of the rotation (pre) and the angles of pairs A and B
    const int A = lane <= 1 ? 0 : lane - 1, RA = lane == 1 ? 1 : 0;
    const int B = lane <= 30 ? lane + 1 : 31, RB = lane <= 30 ? 1 : 0;
    const int dpp = evd_off(evd_next_slot(2 * lane), evd_next_slot(2 * lane));
    const int dqq = evd_off(evd_next_slot(2 * lane + 1), evd_next_slot(2 * lane + 1));
    const int dpq = evd_off(evd_next_slot(2 * lane), evd_next_slot(2 * lane + 1));
    const int rab = evd_off(2 * A, 2 * B), rba = evd_off(2 * A + 1, 2 * B);
    double a_pq = 0.0, a_c = 1.0, a_s = 0.0, a_t = 0.0, nd0 = 0.0, nd1 = 0.0, ca = 1.0, sa = 0.0, cb = 1.0, sb = 0.0;
    double n_pp = 0.0, n_qq = 0.0;
    bool me = false;
    EvdPre pre{0.0, 0.0, 0.0};
    // after the angles of a round are known: the rotated diagonals, the next
    // pair's diagonal entries and diagonal part, and the angles of A and B
    auto prepare_next = [&](double pp, double qq) {
        nd0 = fma(-a_t, a_pq, pp);
        nd1 = fma(a_t, a_pq, qq);
        // first index of pair k: pair k-1's first (k >= 2), pair 0's second
        // (k = 1), its own (k = 0); second index: pair k+1's second (k <= 30),
        // its own first (k = 31)
        const double up = __shfl_up_sync(0xffffffffu, lane == 0 ? nd1 : nd0, 1);
        const double dn = __shfl_down_sync(0xffffffffu, nd1, 1);
        ca = __shfl_sync(0xffffffffu, a_c, A);
        sa = __shfl_sync(0xffffffffu, a_s, A);
        cb = __shfl_sync(0xffffffffu, a_c, B);
        sb = __shfl_sync(0xffffffffu, a_s, B);
        n_pp = lane == 0 ? nd0 : up;
        n_qq = lane == 31 ? nd0 : dn;
        pre = evd_prepare(n_pp, n_qq, tau);
    };
    if (warp == 15 && work) {
        const double pp = G0[evd_off(2 * lane, 2 * lane)];
        const double qq = G0[evd_off(2 * lane + 1, 2 * lane + 1)];
        a_pq = G0[evd_off(2 * lane, 2 * lane + 1)];
        me = evd_rotation(evd_prepare(pp, qq, tau), a_pq, a_c, a_s, a_t);
        cs[0][lane] = make_double2(a_c, a_s);
        cs_c[0][lane] = a_c;
        cs_s[0][lane] = a_s;
        const unsigned m = __ballot_sync(0xffffffffu, me);
        if (lane == 0) {
            rot_mask[0] = m;
            if (m) sweep_any[0] = 1;
        }
        prepare_next(pp, qq);
    }
    bool rotated_any = false;
    int gr = 0;  // rounds executed so far (buffer parity)
    for (int sw = 0; sw < (work ? nsweeps : 0); ++sw) {
        for (int r = 0; r < kEvdRounds; ++r, ++gr) {
            __syncthreads();  // round gr's angles published, its input buffer complete
            const int cur = gr & 1;
            const double *Gin = cur ? G1 : G0;
            double *Gout = cur ? G0 : G1;
            if (warp < 8) {
                if (gr > 0) {  // the advance after round gr - 1 (its boundary values are published)
                    const int pb = gr & 1;
                    const double up = quarter > 0 ? xf[pb][quarter - 1][wrow] : 0.0;
                    const double down = quarter < 3 ? xs[pb][quarter + 1][wrow] : 0.0;
                    evd_w_advance(w, quarter, up, down);
                }
                if (rot_mask[cur]) evd_w_rotate(w, cs[cur], quarter);
                xf[cur ^ 1][quarter][wrow] = w[14];
                xs[cur ^ 1][quarter][wrow] = w[1];
            }
            if (warp < 15) {
#pragma unroll
                for (int j = 0; j < kEvdBulkIters; ++j) {
                    if (blk[j] < 0) continue;
                    const int ia = blk[j] & 255, ib = blk[j] >> 8;
                    const double2 P = make_double2(cs_c[cur][ia], cs_s[cur][ia]);
                    const double2 Q = make_double2(cs_c[cur][ib], cs_s[cur][ib]);
                    const double *f = Gin + (rof[j] & 0xffff);
                    const double g11 = f[0], g12 = f[kEvdQuad], g22 = f[2 * kEvdQuad], g21 = Gin[rof[j] >> 16];
                    // columns: [p' q'] = [c p - s q, s p + c q] (on the right, pair b)
                    const double h11 = fma(Q.x, g11, -(Q.y * g12)), h12 = fma(Q.y, g11, Q.x * g12);
                    const double h21 = fma(Q.x, g21, -(Q.y * g22)), h22 = fma(Q.y, g21, Q.x * g22);
                    // rows (on the left, pair a)
                    Gout[w01[j] & 0xffff] = fma(P.x, h11, -(P.y * h21));
                    Gout[w01[j] >> 16] = fma(P.x, h12, -(P.y * h22));
                    Gout[w23[j] & 0xffff] = fma(P.y, h11, P.x * h21);
                    Gout[w23[j] >> 16] = fma(P.y, h12, P.x * h22);
                }
            } else {
                // block (A, B), A < B: FF[A][B], FS[A][B], FS[B][A], SS[A][B]
                const double g11 = Gin[rab], g12 = Gin[rab + kEvdQuad], g22 = Gin[rab + 2 * kEvdQuad];
                const double g21 = Gin[rba];
                // round gr's diagonal block of pair k: g_pp - t g_pq, g_qq + t g_pq, 0
                Gout[dpp] = nd0;
                Gout[dqq] = nd1;
                Gout[dpq] = me ? 0.0 : a_pq;
                // element (RA, RB) of block (A, B) of G_out, as the update computes it
                const double h1 = RB ? fma(sb, g11, cb * g12) : fma(cb, g11, -(sb * g12));  // h1RB
                const double h2 = RB ? fma(sb, g21, cb * g22) : fma(cb, g21, -(sb * g22));  // h2RB
                a_pq = RA ? fma(sa, h1, ca * h2) : fma(ca, h1, -(sa * h2));
                me = evd_rotation(pre, a_pq, a_c, a_s, a_t);
                cs[cur ^ 1][lane] = make_double2(a_c, a_s);
                cs_c[cur ^ 1][lane] = a_c;
                cs_s[cur ^ 1][lane] = a_s;
                const unsigned m = __ballot_sync(0xffffffffu, me);
                if (lane == 0) {
                    rot_mask[cur ^ 1] = m;
                    if (m) sweep_any[r + 1 < kEvdRounds ? sw : sw + 1] = 1;
                }
                prepare_next(n_pp, n_qq);
            }
        }
        // sweep_any[sw] was last written before this sweep's final barrier
        if (!sweep_any[sw]) break;  // the same value in every thread
        rotated_any = true;
    }
    __syncthreads();  // the last round's output buffer and W boundary values are complete
    if (warp < 8 && gr > 0) {  // the advance after the last round
        const int pb = gr & 1;
        const double up = quarter > 0 ? xf[pb][quarter - 1][wrow] : 0.0;
        const double down = quarter < 3 ? xs[pb][quarter + 1][wrow] : 0.0;
        evd_w_advance(w, quarter, up, down);
    }
    const double *Gf = (gr & 1) ? G1 : G0;
    // Output order of W's columns.  With `sort`, the eigenvalues (G's
    // diagonal) are ranked and the lower-numbered block of the pair receives
    // the larger ones (decreasing norms across the blocks, de Rijk's
    // ordering for one-sided Jacobi), which speeds convergence on graded
    // spectra; it is a column permutation of W.  Only the pair's real columns
    // (global index < ncols) are reordered, among their own positions: the
    // zero padding columns never rotate and must stay at the end.  After full
    // sweeps the slots are back at their starting columns.
    if (rotated_any) {  // the same value in every thread
        // column col = tid / 8 is compared with columns 8 part .. 8 part + 7
        // (part = tid % 8) and the 8 counts meet over lanes xor 1, 2, 4
        const int col = tid >> 3, part = tid & 7;
        const int2 bp = round_robin_pair(nb, round, pair);
        const int real0 = min(max(ncols - bp.x * kB, 0), kB), real1 = min(max(ncols - bp.y * kB, 0), kB);
        auto real = [&](int c) { return c < kB ? c < real0 : c - kB < real1; };
        auto lam = [&](int c) {
            const int s = evd_column_slot(c);
            return Gf[evd_off(s, s)];
        };
        const bool desc = bp.x < bp.y;  // local order follows global order when bp.x < bp.y
        const double l1 = lam(col);
        int rank = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const int c = 8 * part + k;
            const double l2 = lam(c);
            const bool before = desc ? (l2 > l1) : (l2 < l1);
            rank += (real(c) && (before || (l2 == l1 && c < col))) ? 1 : 0;
        }
        rank += __shfl_xor_sync(0xffffffffu, rank, 1);
        rank += __shfl_xor_sync(0xffffffffu, rank, 2);
        rank += __shfl_xor_sync(0xffffffffu, rank, 4);
        if (part == 0) {
            // the rank-th real column (the real columns are a prefix of each block)
            int pos = col;
            if (sort && real(col)) pos = rank < real0 ? rank : kB + (rank - real0);
            out_col[col] = pos;
        }
    }
    __syncthreads();
    if (rotated_any && tid < kEvdWThreads) {
        // every sweep ran all 63 rounds: slot s holds column evd_slot_column(s)
        double *wo = Wout + (size_t)pair * kW * kW;
#pragma unroll
        for (int j = 0; j < 16; ++j) {
            const int col = out_col[evd_slot_column(16 * quarter + j)];
            wo[(size_t)col * kW + wrow] = w[j];
            if (Wimg != nullptr) rot_b_store(Wimg + (size_t)pair * kRotImgFloats, wrow, col, w[j]);
        }
    }
    if (tid == 0) {
        flags[pair] = rotated_any ? 1 : 0;
        if (rotated_any) atomicAdd(&stats[1], 1ull);
        if (off_bits) atomicMax(&stats[0], off_bits);
    }
}

// Wait-limit check of mbar_wait (see mixed_wait_limit_check).
__global__ void mx_wait_limit_check(long long limit_ns, int arrive, int *status)
{
    __shared__ uint64_t bar;
    if (threadIdx.x != 0) return;
    mbar_init(&bar, 1);
    mbar_fence_init();
    if (arrive) mbar_arrive(&bar);
    if (!mbar_wait(&bar, 0, limit_ns)) record_status(status, kDevWaitTimeout);
}

// ============================================================================
// Layout kernels
// ============================================================================

constexpr int kT = 32, kTR = 8;

// row-major (rows x cols) -> column-major padded (ld = rows_pad, cols_pad
// columns; the padding is zero)
__global__ void __launch_bounds__(kT *kTR)
    mx_rowmajor_to_padded(const double *__restrict__ src, int rows, int cols, double *__restrict__ dst, long ld,
                          int rows_pad, int cols_pad)
{
    __shared__ double tile[kT][kT + 1];
    const int c0 = blockIdx.x * kT, r0 = blockIdx.y * kT;
    for (int k = threadIdx.y; k < kT; k += kTR) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        tile[k][threadIdx.x] = (r < rows && c < cols) ? src[(size_t)r * cols + c] : 0.0;
    }
    __syncthreads();
    for (int k = threadIdx.y; k < kT; k += kTR) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (r < rows_pad && c < cols_pad) dst[(size_t)c * ld + r] = tile[threadIdx.x][k];
    }
}

// column-major (ld) -> row-major (rows x cols); with sigma, column c is
// divided by sigma[c] (zero when sigma[c] <= eps)
__global__ void __launch_bounds__(kT *kTR)
    mx_padded_to_rowmajor(const double *__restrict__ src, long ld, int rows, int cols, double *__restrict__ dst,
                          const double *__restrict__ sigma, double eps)
{
    __shared__ double tile[kT][kT + 1];
    const int r0 = blockIdx.x * kT, c0 = blockIdx.y * kT;
    for (int k = threadIdx.y; k < kT; k += kTR) {
        const int c = c0 + k, r = r0 + threadIdx.x;
        if (r < rows && c < cols) tile[k][threadIdx.x] = src[(size_t)c * ld + r];
    }
    __syncthreads();
    for (int k = threadIdx.y; k < kT; k += kTR) {
        const int r = r0 + k, c = c0 + threadIdx.x;
        if (r < rows && c < cols) {
            double v = tile[threadIdx.x][k];
            if (sigma) {
                const double sg = sigma[c];
                v = (sg > eps) ? v / sg : 0.0;
            }
            dst[(size_t)r * cols + c] = v;
        }
    }
}

// FP64 -> TF32 head + FP32 tail, elementwise
__global__ void mx_split(const double *__restrict__ x, size_t count, float *__restrict__ h, float *__restrict__ l)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x) {
        float hh, ll;
        split_tf32((float)x[e], hh, ll);
        h[e] = hh;
        l[e] = ll;
    }
}

__global__ void mx_join(const float *__restrict__ h, const float *__restrict__ l, size_t count, double *__restrict__ x)
{
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < count; e += (size_t)gridDim.x * blockDim.x)
        x[e] = (double)h[e] + (double)l[e];
}

// identity (n x n, ld = n): FP64 and/or the TF32 head/tail pair
__global__ void mx_identity(double *__restrict__ v, float *__restrict__ vh, float *__restrict__ vl, int n)
{
    const size_t total = (size_t)n * n;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const double d = (e / n == e % n) ? 1.0 : 0.0;
        if (v) v[e] = d;
        if (vh) vh[e] = (float)d;
        if (vl) vl[e] = 0.0f;
    }
}

// E = V^T V - I (in place) and *maxabs = max |E_ij| (double bits)
__global__ void mx_minus_identity_max(double *__restrict__ E, int n, unsigned long long *__restrict__ maxabs)
{
    const size_t total = (size_t)n * n;
    double m = 0.0;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        double v = E[e];
        if (e / n == e % n) v -= 1.0;
        E[e] = v;
        m = fmax(m, fabs(v));
        if (v != v) m = INFINITY;  // NaN
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(maxabs, (unsigned long long)__double_as_longlong(m));
}

// M = I - E / 2 (in place)
__global__ void mx_half_step(double *__restrict__ E, int n)
{
    const size_t total = (size_t)n * n;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x)
        E[e] = ((e / n == e % n) ? 1.0 : 0.0) - 0.5 * E[e];
}

// g[pair] (64 x 64 column-major FP64) = sum of the pair's Gram partials
__global__ void mx_sum_partials(const void *__restrict__ part, int kind, int splits, int npairs, double *__restrict__ g)
{
    const size_t total = (size_t)npairs * kW * kW;
    for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < total; e += (size_t)gridDim.x * blockDim.x) {
        const int pair = (int)(e / (kW * kW)), rc = (int)(e % (kW * kW));
        int r = rc & 63, c = rc >> 6;
        if (kind != 0 && r > c) {  // the FP64 Gram holds the upper triangle: read the mirror
            const int t = r;
            r = c;
            c = t;
        }
        double acc = 0.0;
        if (kind == 0) {
            const float *p = static_cast<const float *>(part) + (size_t)pair * splits * 8192;
            for (int s = 0; s < splits; ++s)
                acc += (double)p[(size_t)s * 8192 + c * 128 + r] + (double)p[(size_t)s * 8192 + c * 128 + r + 64];
        } else {
            const double *p = static_cast<const double *>(part) + (size_t)pair * splits * 4096;
            for (int s = 0; s < splits; ++s) acc += p[(size_t)s * 4096 + c * 64 + r];
        }
        g[e] = acc;
    }
}

__global__ void mx_fill_int(int *__restrict__ p, int n, int v)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = v;
}

// sigma_j = ||x_j|| (one warp per column, FP64)
__global__ void mx_sigma(const double *__restrict__ X, long ld, int rows, int cols, double *__restrict__ sigma)
{
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (w >= cols) return;
    const double *x = X + (size_t)w * ld;
    double acc = 0.0;
    for (int i = lane; i < rows; i += 32) acc = fma(x[i], x[i], acc);
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) sigma[w] = sqrt(acc);
}

// ============================================================================
// Host side
// ============================================================================

using EncodeTiledFn = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                   const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

int get_encode_fn(EncodeTiledFn *out)
{
    static EncodeTiledFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        cudaDriverEntryPointQueryResult q{};
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    if (!fn) {
        set_last_error(JSVD_ERR_CUDA, "cuTensorMapEncodeTiled is not available from the CUDA driver.");
        return JSVD_ERR_CUDA;
    }
    *out = fn;
    return JSVD_OK;
}

// 2-D map of a column-major FP32 array (rows x cols, ld = rows), box 32 x 32,
// 128-byte swizzle of 16-byte chunks (K-major operand tiles) or of 32-byte
// chunks (MN-major TF32 operand tiles).
int make_map(CUtensorMap *map, float *base, long rows, long cols, bool atom32 = false)
{
    EncodeTiledFn enc = nullptr;
    if (int rc = get_encode_fn(&enc); rc != JSVD_OK) return rc;
    const cuuint64_t dims[2] = {(cuuint64_t)rows, (cuuint64_t)cols};
    const cuuint64_t strides[1] = {(cuuint64_t)rows * sizeof(float)};
    const cuuint32_t box[2] = {32, 32};
    const cuuint32_t estr[2] = {1, 1};
    const CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, base, dims, strides, box, estr,
                           CU_TENSOR_MAP_INTERLEAVE_NONE,
                           atom32 ? CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B : CU_TENSOR_MAP_SWIZZLE_128B,
                           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_last_error(JSVD_ERR_CUDA, "cuTensorMapEncodeTiled failed (CUresult " + std::to_string((int)r) + ").");
        return JSVD_ERR_CUDA;
    }
    return JSVD_OK;
}

int init_kernel_attributes()
{
    // function attributes are per device
    static thread_local unsigned long long done_mask = 0;
    int dev = 0;
    JSVD_CUDA_TRY(cudaGetDevice(&dev));
    if (dev >= 64 || !(done_mask & (1ull << dev))) {
        JSVD_CUDA_TRY(cudaFuncSetAttribute(mx_gram_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGramTcSmem));
        JSVD_CUDA_TRY(cudaFuncSetAttribute(mx_rot_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRotTcSmem));
        JSVD_CUDA_TRY(cudaFuncSetAttribute(mx_rot_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRot64Smem));
        JSVD_CUDA_TRY(
            cudaFuncSetAttribute(mx_gram_f64, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kGram64Smem));
        JSVD_CUDA_TRY(cudaFuncSetAttribute(mx_evd, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kEvdSmem));
        if (dev < 64) done_mask |= 1ull << dev;
    }
    return JSVD_OK;
}

struct MixedStats {
    unsigned long long solves = 0, tc_sweeps = 0, f64_sweeps = 0, block_rounds = 0, fallbacks = 0;
    double qr_ms = 0, tc_ms = 0, orth_ms = 0, refine_ms = 0, out_ms = 0;
    double last_tc_off = 0, last_f64_off = 0;
    int last_tc_sweeps = 0, last_f64_sweeps = 0;
    unsigned long long tc_gram = 0, tc_rot = 0, f64_gram = 0, f64_rot = 0, evd = 0;
    unsigned long long tc_discarded = 0;
    // device time of the three kernels of sampled block rounds (rounds 0 and
    // rounds/2 of every sweep, events around each launch)
    double tc_gram_ms = 0, tc_evd_ms = 0, tc_rot_ms = 0, f64_gram_ms = 0, f64_evd_ms = 0, f64_rot_ms = 0;
    unsigned long long tc_sampled = 0, f64_sampled = 0;
    // block pairs that rotated in the sampled rounds (their rotation kernels
    // moved (rows_pad + cols_pad) x 64 elements each)
    unsigned long long tc_sampled_pairs = 0, f64_sampled_pairs = 0;
    int rows_pad = 0, cols_pad = 0, npairs = 0;  // of the last sweep's workspace
    // per sweep of the last solve: phase (1 tensor core, 3 FP64), largest
    // scaled off-diagonal Gram entry seen, block pairs that rotated
    static constexpr int kHist = 64;
    int hist_len = 0;
    int hist_phase[kHist] = {};
    double hist_off[kHist] = {};
    unsigned long long hist_rot[kHist] = {};
};

MixedStats &mixed_stats()
{
    thread_local MixedStats s;
    return s;
}

jsvd_mixed_options default_options()
{
    jsvd_mixed_options o{};
    o.precondition = 1;
    o.tc_max_sweeps = -1;
    o.tc_tol = 2e-5;
    o.inner_sweeps = 0;
    o.refine = 0;
    o.f64_max_sweeps = 0;
    o.gram_splits = 0;
    o.sort = 1;
    return o;
}

jsvd_mixed_options &thread_options()
{
    thread_local jsvd_mixed_options o = default_options();
    return o;
}

// Device workspace of one shape.
struct Work {
    int rows = 0, cols = 0, rows_pad = 0, cols_pad = 0, nb = 0, rounds = 0, npairs = 0;
    int x_tiles = 0, v_tiles = 0;
    int tc_splits = 1, tc_chunks = 0, tc_chunks_per_split = 0;
    int f64_splits = 1, f64_rows_per_split = 0;
    double *x64 = nullptr, *xr = nullptr, *v64 = nullptr, *vo = nullptr, *e64 = nullptr;
    float *xh = nullptr, *xl = nullptr, *vh = nullptr, *vl = nullptr;
    void *part = nullptr;
    double *W = nullptr, *sg = nullptr;
    float *wimg = nullptr;  // the tensor-core rotation's B operand images (phase 1)
    int *flags = nullptr, *status = nullptr;
    // [0] max off (double bits) [1] rotated pairs [2] orth max [4..7] rotated
    // pairs before/after the eigen-solve of the two sampled rounds
    unsigned long long *stats = nullptr;
    unsigned long long *h_stats = nullptr;  // pinned copy
    CUtensorMap mxh{}, mxl{}, mvh{}, mvl{};  // 16-byte-chunk swizzle (Gram operands)
    CUtensorMap rxh{}, rxl{}, rvh{}, rvl{};  // 32-byte-chunk swizzle (rotation A operands)
    void *block = nullptr;
    cudaEvent_t tev[2][4] = {};  // kernel timing of two sampled rounds per sweep
};

int split_count(int chunks, int npairs, int requested)
{
    if (requested > 0) return std::max(1, std::min(requested, chunks));
    // enough CTAs to cover the SMs about twice, at least 4 chunks per split
    int s = (2 * 148 + npairs - 1) / std::max(1, npairs);
    s = std::min(s, std::max(1, chunks / 4));
    return std::max(1, s);
}

int make_work(int rows, int cols, const jsvd_mixed_options &o, bool tc, cudaStream_t st, Work &w)
{
    w.rows = rows;
    w.cols = cols;
    w.rows_pad = (rows + kTileRows - 1) / kTileRows * kTileRows;
    w.cols_pad = (cols + kColPad - 1) / kColPad * kColPad;
    w.nb = w.cols_pad / kB;
    w.rounds = w.nb - 1;
    w.npairs = w.nb / 2;
    w.x_tiles = w.rows_pad / kTileRows;
    w.v_tiles = w.cols_pad / kTileRows;
    w.tc_chunks = w.rows_pad / 32;
    w.tc_splits = split_count(w.tc_chunks, w.npairs, o.gram_splits);
    w.tc_chunks_per_split = (w.tc_chunks + w.tc_splits - 1) / w.tc_splits;
    w.tc_splits = (w.tc_chunks + w.tc_chunks_per_split - 1) / w.tc_chunks_per_split;  // no empty split
    const int r32 = w.rows_pad / 32;
    w.f64_splits = split_count(r32, w.npairs, o.gram_splits);
    w.f64_rows_per_split = (r32 + w.f64_splits - 1) / w.f64_splits * 32;
    w.f64_splits = (w.rows_pad + w.f64_rows_per_split - 1) / w.f64_rows_per_split;
    const size_t mn = (size_t)w.rows_pad * w.cols_pad, nn = (size_t)w.cols_pad * w.cols_pad;
    const int splits = std::max(w.tc_splits, w.f64_splits);
    const size_t part_bytes = (size_t)w.npairs * splits * 4096 * sizeof(double);
    size_t bytes = 0;
    auto take = [&](size_t b) {
        const size_t off = bytes;
        bytes += (b + 255) / 256 * 256;
        return off;
    };
    const size_t o_x64 = take(mn * 8), o_xr = take(mn * 8), o_v64 = take(nn * 8), o_vo = take(nn * 8),
                 o_e = take(nn * 8);
    const size_t o_xh = tc ? take(mn * 4) : 0, o_xl = tc ? take(mn * 4) : 0, o_vh = tc ? take(nn * 4) : 0,
                 o_vl = tc ? take(nn * 4) : 0;
    const size_t o_wimg = tc ? take((size_t)w.npairs * kRotImgFloats * 4) : 0;
    const size_t o_part = take(part_bytes), o_w = take((size_t)w.npairs * kW * kW * 8), o_sg = take(w.cols_pad * 8),
                 o_flags = take(w.npairs * 4), o_status = take(4), o_stats = take(8 * 8);
    JSVD_CUDA_TRY(cudaMallocAsync(&w.block, bytes, st));
    uint8_t *b = static_cast<uint8_t *>(w.block);
    w.x64 = reinterpret_cast<double *>(b + o_x64);
    w.xr = reinterpret_cast<double *>(b + o_xr);
    w.v64 = reinterpret_cast<double *>(b + o_v64);
    w.vo = reinterpret_cast<double *>(b + o_vo);
    w.e64 = reinterpret_cast<double *>(b + o_e);
    if (tc) {
        w.xh = reinterpret_cast<float *>(b + o_xh);
        w.xl = reinterpret_cast<float *>(b + o_xl);
        w.vh = reinterpret_cast<float *>(b + o_vh);
        w.vl = reinterpret_cast<float *>(b + o_vl);
        w.wimg = reinterpret_cast<float *>(b + o_wimg);
    }
    w.part = b + o_part;
    w.W = reinterpret_cast<double *>(b + o_w);
    w.sg = reinterpret_cast<double *>(b + o_sg);
    w.flags = reinterpret_cast<int *>(b + o_flags);
    w.status = reinterpret_cast<int *>(b + o_status);
    w.stats = reinterpret_cast<unsigned long long *>(b + o_stats);
    JSVD_CUDA_TRY(cudaMallocHost((void **)&w.h_stats, 8 * sizeof(unsigned long long)));
    for (auto &row : w.tev)
        for (auto &e : row) JSVD_CUDA_TRY(cudaEventCreate(&e));
    if (tc) {
        if (int rc = make_map(&w.mxh, w.xh, w.rows_pad, w.cols_pad); rc != JSVD_OK) return rc;
        if (int rc = make_map(&w.mxl, w.xl, w.rows_pad, w.cols_pad); rc != JSVD_OK) return rc;
        if (int rc = make_map(&w.mvh, w.vh, w.cols_pad, w.cols_pad); rc != JSVD_OK) return rc;
        if (int rc = make_map(&w.mvl, w.vl, w.cols_pad, w.cols_pad); rc != JSVD_OK) return rc;
        if (int rc = make_map(&w.rxh, w.xh, w.rows_pad, w.cols_pad, true); rc != JSVD_OK) return rc;
        if (int rc = make_map(&w.rxl, w.xl, w.rows_pad, w.cols_pad, true); rc != JSVD_OK) return rc;
        if (int rc = make_map(&w.rvh, w.vh, w.cols_pad, w.cols_pad, true); rc != JSVD_OK) return rc;
        if (int rc = make_map(&w.rvl, w.vl, w.cols_pad, w.cols_pad, true); rc != JSVD_OK) return rc;
    }
    return JSVD_OK;
}

void free_work(Work &w, cudaStream_t st)
{
    if (w.block) cudaFreeAsync(w.block, st);
    if (w.h_stats) cudaFreeHost(w.h_stats);
    for (auto &row : w.tev)
        for (auto &e : row)
            if (e) cudaEventDestroy(e);
    w.block = nullptr;
    w.h_stats = nullptr;
}

unsigned grid_for(size_t count) { return (unsigned)std::min<size_t>(148 * 8, (count + 255) / 256); }

// One sweep (every block round) of phase 1 or phase 3; reads back the
// sweep's statistics.
int run_sweep(Work &w, bool tc, double tau, int inner, int sort, cudaStream_t st, double *max_off,
              unsigned long long *rotated)
{
    MixedStats &ms = mixed_stats();
    JSVD_CUDA_TRY(cudaMemsetAsync(w.stats, 0, 2 * sizeof(unsigned long long), st));
    const int sample_round[2] = {0, w.rounds / 2};
    const int nsample = w.rounds > 2 ? 2 : 1;
    for (int r = 0; r < w.rounds; ++r) {
        int si = -1;
        for (int i = 0; i < nsample; ++i)
            if (r == sample_round[i]) si = i;
        if (si >= 0) cudaEventRecord(w.tev[si][0], st);
        if (tc) {
            mx_gram_tc<<<dim3(w.tc_splits, w.npairs), kGramTcThreads, kGramTcSmem, st>>>(
                w.mxh, w.mxl, w.nb, r, w.tc_chunks, w.tc_chunks_per_split, static_cast<float *>(w.part), w.status);
            if (si >= 0) {
                cudaEventRecord(w.tev[si][1], st);
                cudaMemcpyAsync(w.stats + 4 + 2 * si, w.stats + 1, 8, cudaMemcpyDeviceToDevice, st);
            }
            mx_evd<<<w.npairs, kEvdThreads, kEvdSmem, st>>>(w.part, 0, w.tc_splits, tau, inner, w.nb, r, sort, w.cols,
                                                            w.W, w.wimg, w.flags, w.stats);
            if (si >= 0) {
                cudaMemcpyAsync(w.stats + 5 + 2 * si, w.stats + 1, 8, cudaMemcpyDeviceToDevice, st);
                cudaEventRecord(w.tev[si][2], st);
            }
            mx_rot_tc<<<dim3(w.x_tiles + w.v_tiles, w.npairs), kRotTcThreads, kRotTcSmem, st>>>(
                w.rxh, w.rxl, w.rvh, w.rvl, w.xh, w.xl, w.rows_pad, w.x_tiles, w.vh, w.vl, w.cols_pad, w.nb, r, w.wimg,
                w.flags, w.status);
            ms.tc_gram += 1;
            ms.tc_rot += 1;
        } else {
            mx_gram_f64<<<dim3(w.f64_splits, w.npairs), kGram64Threads, kGram64Smem, st>>>(
                w.xr, w.rows_pad, w.nb, r, w.f64_rows_per_split, w.rows_pad, static_cast<double *>(w.part));
            if (si >= 0) {
                cudaEventRecord(w.tev[si][1], st);
                cudaMemcpyAsync(w.stats + 4 + 2 * si, w.stats + 1, 8, cudaMemcpyDeviceToDevice, st);
            }
            mx_evd<<<w.npairs, kEvdThreads, kEvdSmem, st>>>(w.part, 1, w.f64_splits, tau, inner, w.nb, r, sort,
                                                            w.cols, w.W, nullptr, w.flags, w.stats);
            if (si >= 0) {
                cudaMemcpyAsync(w.stats + 5 + 2 * si, w.stats + 1, 8, cudaMemcpyDeviceToDevice, st);
                cudaEventRecord(w.tev[si][2], st);
            }
            mx_rot_f64<<<dim3(w.x_tiles + w.v_tiles, w.npairs), kRot64Threads, kRot64Smem, st>>>(
                w.xr, w.rows_pad, w.x_tiles, w.v64, w.cols_pad, w.nb, r, w.W, w.flags);
            ms.f64_gram += 1;
            ms.f64_rot += 1;
        }
        if (si >= 0) cudaEventRecord(w.tev[si][3], st);
        ms.evd += 1;
    }
    JSVD_CUDA_TRY(cudaGetLastError());
    ms.block_rounds += (unsigned long long)w.rounds;
    JSVD_CUDA_TRY(cudaMemcpyAsync(w.h_stats, w.stats, 2 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    JSVD_CUDA_TRY(
        cudaMemcpyAsync(w.h_stats + 4, w.stats + 4, 4 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    int dstatus = 0;
    JSVD_CUDA_TRY(cudaMemcpyAsync(&dstatus, w.status, sizeof(int), cudaMemcpyDeviceToHost, st));
    JSVD_CUDA_TRY(cudaStreamSynchronize(st));
    if (dstatus != 0) {
        set_last_error(JSVD_ERR_RUNTIME, "mixed engine: a tensor-core kernel gave up waiting for its operands "
                                         "(device status " +
                                             std::to_string(dstatus) + ").");
        return JSVD_ERR_RUNTIME;
    }
    const unsigned long long bits = w.h_stats[0];
    double off;
    std::memcpy(&off, &bits, sizeof(off));
    *max_off = off;
    *rotated = w.h_stats[1];
    for (int i = 0; i < nsample; ++i) {
        float g = 0.f, e = 0.f, t = 0.f;
        cudaEventElapsedTime(&g, w.tev[i][0], w.tev[i][1]);
        cudaEventElapsedTime(&e, w.tev[i][1], w.tev[i][2]);
        cudaEventElapsedTime(&t, w.tev[i][2], w.tev[i][3]);
        (tc ? ms.tc_gram_ms : ms.f64_gram_ms) += g;
        (tc ? ms.tc_evd_ms : ms.f64_evd_ms) += e;
        (tc ? ms.tc_rot_ms : ms.f64_rot_ms) += t;
        (tc ? ms.tc_sampled : ms.f64_sampled) += 1;
        (tc ? ms.tc_sampled_pairs : ms.f64_sampled_pairs) += w.h_stats[5 + 2 * i] - w.h_stats[4 + 2 * i];
    }
    ms.rows_pad = w.rows_pad;
    ms.cols_pad = w.cols_pad;
    ms.npairs = w.npairs;
    if (ms.hist_len < MixedStats::kHist) {
        ms.hist_phase[ms.hist_len] = tc ? 1 : 3;
        ms.hist_off[ms.hist_len] = off;
        ms.hist_rot[ms.hist_len] = *rotated;
        ++ms.hist_len;
    }
    return JSVD_OK;
}

// V <- polar factor of V (Newton-Schulz), at most `steps` steps; stops once
// max |V^T V - I| <= 4u.  Result in w.v64; *residual = max |V^T V - I| of the
// last iterate measured.
int orthogonalise(Work &w, cudaStream_t st, int steps, double *residual)
{
    *residual = INFINITY;
    const int n = w.cols_pad;
    const size_t nn = (size_t)n * n;
    for (int i = 0; i < steps; ++i) {
        if (int rc = dgemm(st, 'T', 'N', n, n, n, 1.0, w.v64, n, w.v64, n, 0.0, w.e64, n); rc != JSVD_OK) return rc;
        JSVD_CUDA_TRY(cudaMemsetAsync(w.stats + 2, 0, sizeof(unsigned long long), st));
        mx_minus_identity_max<<<grid_for(nn), 256, 0, st>>>(w.e64, n, w.stats + 2);
        JSVD_CUDA_TRY(cudaGetLastError());
        JSVD_CUDA_TRY(
            cudaMemcpyAsync(w.h_stats + 2, w.stats + 2, sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
        JSVD_CUDA_TRY(cudaStreamSynchronize(st));
        double e;
        std::memcpy(&e, &w.h_stats[2], sizeof(e));
        *residual = e;
        if (!(e <= 0.25)) break;  // not near orthogonal (or NaN): the iteration would not converge
        if (e <= 4.0 * 1.1102230246251565e-16) break;
        mx_half_step<<<grid_for(nn), 256, 0, st>>>(w.e64, n);
        if (int rc = dgemm(st, 'N', 'N', n, n, n, 1.0, w.v64, n, w.e64, n, 0.0, w.vo, n); rc != JSVD_OK) return rc;
        std::swap(w.v64, w.vo);
    }
    return JSVD_OK;
}

// Per-thread cache of workspaces (at most two shapes, 16 GiB), so that
// repeated solves of one shape allocate nothing and create no events.  A
// workspace depends on the device, the shape, whether phase 1 runs and the
// Gram row splits.
struct CachedWork {
    int device = -1, rows = 0, cols = 0, splits = 0;
    bool tc = false;
    Work w;
    ~CachedWork()
    {
        if (w.block) cudaFree(w.block);
        if (w.h_stats) cudaFreeHost(w.h_stats);
        for (auto &row : w.tev)
            for (auto &e : row)
                if (e) cudaEventDestroy(e);
    }
};

std::vector<std::unique_ptr<CachedWork>> &work_cache()
{
    thread_local std::vector<std::unique_ptr<CachedWork>> cache;
    return cache;
}

constexpr size_t kMaxCachedWorkBytes = size_t(16) << 30;

size_t work_bytes_estimate(int rows, int cols, bool tc)
{
    const size_t rp = (rows + kTileRows - 1) / kTileRows * kTileRows, cp = (cols + kColPad - 1) / kColPad * kColPad;
    return 8 * (2 * rp * cp + 3 * cp * cp) + (tc ? 8 * (rp * cp + cp * cp) : 0);
}

// The calling thread's workspace for this request: cached (repeated
// shapes) or made for this call only (*owned is then set and the caller
// frees it).
int acquire_work(int rows, int cols, const jsvd_mixed_options &o, bool tc, cudaStream_t st, Work **out, Work *owned)
{
    int dev = 0;
    JSVD_CUDA_TRY(cudaGetDevice(&dev));
    auto &cache = work_cache();
    for (size_t i = 0; i < cache.size(); ++i) {
        CachedWork &c = *cache[i];
        if (c.device == dev && c.rows == rows && c.cols == cols && c.tc == tc && c.splits == o.gram_splits) {
            std::rotate(cache.begin(), cache.begin() + i, cache.begin() + i + 1);
            *out = &cache.front()->w;
            return JSVD_OK;
        }
    }
    if (work_bytes_estimate(rows, cols, tc) > kMaxCachedWorkBytes) {
        if (int rc = make_work(rows, cols, o, tc, st, *owned); rc != JSVD_OK) return rc;
        *out = owned;
        return JSVD_OK;
    }
    auto c = std::make_unique<CachedWork>();
    c->device = dev;
    c->rows = rows;
    c->cols = cols;
    c->tc = tc;
    c->splits = o.gram_splits;
    if (int rc = make_work(rows, cols, o, tc, st, c->w); rc != JSVD_OK) return rc;
    cache.insert(cache.begin(), std::move(c));
    while (cache.size() > 2) cache.pop_back();
    *out = &cache.front()->w;
    return JSVD_OK;
}

}  // namespace

const jsvd_mixed_options &mixed_options() { return thread_options(); }

void mixed_release_thread_cache() { work_cache().clear(); }

struct MixedTuning {
    int max_cols;  // largest column count the entry covers (0 = any)
    int tc_max_sweeps, inner_sweeps, gram_splits;
};
constexpr MixedTuning kMixedTuning[] = JSVD_MIXED_TUNING_TABLE;
constexpr int kMixedTuningCount = (int)(sizeof(kMixedTuning) / sizeof(kMixedTuning[0]));

// The automatic options (tc_max_sweeps < 0, inner_sweeps <= 0, gram_splits
// <= 0) resolved from the built-in table by the input's width: on narrow
// inputs (few block pairs per round) a round costs about the same in either
// phase, the block eigen-solves dominating, so the FP64 phase, which
// converges quadratically, takes over early; on wide ones the 3xTF32 rounds
// are the cheaper and phase 1 runs until tc_tol.
jsvd_mixed_options resolve_options(const jsvd_mixed_options &o, int cols)
{
    const MixedTuning *t = &kMixedTuning[kMixedTuningCount - 1];
    for (int i = 0; i < kMixedTuningCount; ++i)
        if (kMixedTuning[i].max_cols == 0 || cols <= kMixedTuning[i].max_cols) {
            t = &kMixedTuning[i];
            break;
        }
    jsvd_mixed_options e = o;
    if (e.tc_max_sweeps < 0) e.tc_max_sweeps = t->tc_max_sweeps;
    if (e.inner_sweeps <= 0) e.inner_sweeps = t->inner_sweeps;
    if (e.gram_splits <= 0) e.gram_splits = t->gram_splits;
    return e;
}

int mixed_solve(const double *x, int rows, int cols, const jsvd_config &c, const jsvd_mixed_options &o_in,
                double *u, double *sigma, double *v, int *sweeps, cudaStream_t st)
{
    if (int rc = init_kernel_attributes(); rc != JSVD_OK) return rc;
    const jsvd_mixed_options o = resolve_options(o_in, cols);
    const int tc_max = o.tc_max_sweeps;
    const bool tc = tc_max > 0;
    Work owned;
    ScopeExit release([&] { free_work(owned, st); });
    Work *wp = nullptr;
    if (int rc = acquire_work(rows, cols, o, tc, st, &wp, &owned); rc != JSVD_OK) return rc;
    Work &w = *wp;
    MixedStats &ms = mixed_stats();
    ms.hist_len = 0;
    cudaEvent_t ev[5] = {};
    for (auto &e : ev) cudaEventCreate(&e);
    ScopeExit destroy([&] {
        for (auto &e : ev)
            if (e) cudaEventDestroy(e);
    });
    const size_t mn = (size_t)w.rows_pad * w.cols_pad, nn = (size_t)w.cols_pad * w.cols_pad;
    cudaEventRecord(ev[0], st);
    JSVD_CUDA_TRY(cudaMemsetAsync(w.status, 0, sizeof(int), st));
    mx_rowmajor_to_padded<<<dim3(w.cols_pad / kT, w.rows_pad / kT), dim3(kT, kTR), 0, st>>>(
        x, rows, cols, w.x64, w.rows_pad, w.rows_pad, w.cols_pad);
    JSVD_CUDA_TRY(cudaGetLastError());
    int tc_sweeps = 0, f64_sweeps = 0;
    double tc_off = 0.0;
    const double u53 = 1.1102230246251565e-16;
    if (tc) {
        mx_split<<<grid_for(mn), 256, 0, st>>>(w.x64, mn, w.xh, w.xl);
        mx_identity<<<grid_for(nn), 256, 0, st>>>(nullptr, w.vh, w.vl, w.cols_pad);
        JSVD_CUDA_TRY(cudaGetLastError());
        // Phase 1 rotates every pair the FP32-accurate Gram resolves: its
        // entries carry relative errors of about 2^-21 + sqrt(m) 2^-24.
        const double tau = std::max(o.tc_tol * 0.25, 4.0 * std::sqrt((double)w.rows_pad) * 5.96e-8);
        for (int s = 0; s < tc_max; ++s) {
            unsigned long long rotated = 0;
            if (int rc = run_sweep(w, true, tau, o.inner_sweeps, o.sort, st, &tc_off, &rotated); rc != JSVD_OK)
                return rc;
            ++tc_sweeps;
            if (rotated == 0 || tc_off <= o.tc_tol) break;
        }
        cudaEventRecord(ev[1], st);
        mx_join<<<grid_for(nn), 256, 0, st>>>(w.vh, w.vl, nn, w.v64);
        JSVD_CUDA_TRY(cudaGetLastError());
        double orth = INFINITY;
        if (int rc = orthogonalise(w, st, 4, &orth); rc != JSVD_OK) return rc;
        if (orth <= 1e-12) {
            if (int rc = dgemm(st, 'N', 'N', w.rows_pad, w.cols_pad, w.cols_pad, 1.0, w.x64, w.rows_pad, w.v64,
                               w.cols_pad, 0.0, w.xr, w.rows_pad);
                rc != JSVD_OK)
                return rc;
        } else {
            // phase 1 did not leave a usable V: the FP64 sweeps start from X
            ms.tc_discarded += 1;
            JSVD_CUDA_TRY(cudaMemcpyAsync(w.xr, w.x64, mn * 8, cudaMemcpyDeviceToDevice, st));
            mx_identity<<<grid_for(nn), 256, 0, st>>>(w.v64, nullptr, nullptr, w.cols_pad);
            JSVD_CUDA_TRY(cudaGetLastError());
        }
        cudaEventRecord(ev[2], st);
    } else {
        JSVD_CUDA_TRY(cudaMemcpyAsync(w.xr, w.x64, mn * 8, cudaMemcpyDeviceToDevice, st));
        mx_identity<<<grid_for(nn), 256, 0, st>>>(w.v64, nullptr, nullptr, w.cols_pad);
        JSVD_CUDA_TRY(cudaGetLastError());
        cudaEventRecord(ev[1], st);
        cudaEventRecord(ev[2], st);
    }
    // Phase 3: FP64 blocked sweeps.  The Gram's own rounding (about
    // sqrt(m) u relative) sets the smallest threshold it can decide.
    const double tau64 = std::max(c.epsilon, 4.0 * std::sqrt((double)w.rows_pad) * u53);
    const int cap = o.f64_max_sweeps > 0 ? o.f64_max_sweeps : c.max_sweeps;
    double f64_off = 0.0;
    for (int s = 0; s < cap; ++s) {
        unsigned long long rotated = 0;
        if (int rc = run_sweep(w, false, tau64, o.inner_sweeps, o.sort, st, &f64_off, &rotated); rc != JSVD_OK)
            return rc;
        ++f64_sweeps;
        if (rotated == 0) break;
    }
    cudaEventRecord(ev[3], st);
    double *sg = sigma ? sigma : w.sg;
    mx_sigma<<<(cols * 32 + 255) / 256, 256, 0, st>>>(w.xr, w.rows_pad, rows, cols, sg);
    if (u)
        mx_padded_to_rowmajor<<<dim3((rows + kT - 1) / kT, (cols + kT - 1) / kT), dim3(kT, kTR), 0, st>>>(
            w.xr, w.rows_pad, rows, cols, u, sg, c.epsilon);
    if (v)
        mx_padded_to_rowmajor<<<dim3((cols + kT - 1) / kT, (cols + kT - 1) / kT), dim3(kT, kTR), 0, st>>>(
            w.v64, w.cols_pad, cols, cols, v, nullptr, 0.0);
    JSVD_CUDA_TRY(cudaGetLastError());
    cudaEventRecord(ev[4], st);
    JSVD_CUDA_TRY(cudaStreamSynchronize(st));
    float t01 = 0, t12 = 0, t23 = 0, t34 = 0;
    cudaEventElapsedTime(&t01, ev[0], ev[1]);
    cudaEventElapsedTime(&t12, ev[1], ev[2]);
    cudaEventElapsedTime(&t23, ev[2], ev[3]);
    cudaEventElapsedTime(&t34, ev[3], ev[4]);
    ms.tc_ms += t01;
    ms.orth_ms += t12;
    ms.refine_ms += t23;
    ms.out_ms += t34;
    ms.tc_sweeps += tc_sweeps;
    ms.f64_sweeps += f64_sweeps;
    ms.last_tc_sweeps = tc_sweeps;
    ms.last_f64_sweeps = f64_sweeps;
    ms.last_tc_off = tc_off;
    ms.last_f64_off = f64_off;
    if (sweeps) *sweeps = tc_sweeps + f64_sweeps;
    return JSVD_OK;
}

int mixed_wait_limit_check(long long limit_ns, bool arrive, int *status, cudaStream_t st)
{
    mx_wait_limit_check<<<1, 32, 0, st>>>(limit_ns, arrive ? 1 : 0, status);
    JSVD_CUDA_TRY(cudaGetLastError());
    return JSVD_OK;
}

void mixed_note_solve(double qr_ms, bool fallback)
{
    MixedStats &ms = mixed_stats();
    ms.solves += 1;
    ms.qr_ms += qr_ms;
    if (fallback) ms.fallbacks += 1;
}

}  // namespace jsvd

using namespace jsvd;

// Kernel-level test hook: one block round of the engine's kernels on X
// (rows x cols, column-major FP64, device; rows and cols multiples of 128).
//   kind 0: tensor-core Gram of every block pair of `round` -> gw
//           (npairs x 64 x 64, column-major FP64, the partials summed);
//   kind 1: the FP64 Gram -> gw;
//   kind 2: tensor-core rotation X_pair <- X_pair W_pair with W from gw (X is
//           split into TF32 head and tail first and joined afterwards);
//   kind 3: the FP64 rotation.
extern "C" int jsvd_mixed_test_round(int kind, double *d_x, int rows, int cols, int round, double *d_gw)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        if (!d_x || !d_gw || rows <= 0 || cols <= 0 || rows % kTileRows || cols % kColPad || kind < 0 || kind > 3 ||
            round < 0 || round >= cols / kB - 1)
            return invalid_argument("jsvd_mixed_test_round: bad arguments.");
        cudaStream_t st = nullptr;
        if (const int e = entry_stream(nullptr, &st); e != JSVD_OK) return e;
        if (int rc = init_kernel_attributes(); rc != JSVD_OK) return rc;
        const bool tc = (kind == 0 || kind == 2);
        jsvd_mixed_options o = default_options();
        Work w;
        ScopeExit release([&] { free_work(w, st); });
        if (int rc = make_work(rows, cols, o, tc, st, w); rc != JSVD_OK) return rc;
        const size_t mn = (size_t)rows * cols;
        JSVD_CUDA_TRY(cudaMemsetAsync(w.status, 0, sizeof(int), st));
        if (tc) mx_split<<<grid_for(mn), 256, 0, st>>>(d_x, mn, w.xh, w.xl);
        if (kind == 0) {
            mx_gram_tc<<<dim3(w.tc_splits, w.npairs), kGramTcThreads, kGramTcSmem, st>>>(
                w.mxh, w.mxl, w.nb, round, w.tc_chunks, w.tc_chunks_per_split, static_cast<float *>(w.part), w.status);
            mx_sum_partials<<<grid_for((size_t)w.npairs * 4096), 256, 0, st>>>(w.part, 0, w.tc_splits, w.npairs, d_gw);
        } else if (kind == 1) {
            mx_gram_f64<<<dim3(w.f64_splits, w.npairs), kGram64Threads, kGram64Smem, st>>>(
                d_x, rows, w.nb, round, w.f64_rows_per_split, rows, static_cast<double *>(w.part));
            mx_sum_partials<<<grid_for((size_t)w.npairs * 4096), 256, 0, st>>>(w.part, 1, w.f64_splits, w.npairs,
                                                                                d_gw);
        } else {
            mx_fill_int<<<1, 256, 0, st>>>(w.flags, w.npairs, 1);
            if (kind == 2) {
                mx_rot_image<<<w.npairs, 256, 0, st>>>(d_gw, w.wimg, w.flags);
                mx_rot_tc<<<dim3(w.x_tiles, w.npairs), kRotTcThreads, kRotTcSmem, st>>>(
                    w.rxh, w.rxl, w.rvh, w.rvl, w.xh, w.xl, rows, w.x_tiles, w.vh, w.vl, cols, w.nb, round, w.wimg,
                    w.flags, w.status);
                mx_join<<<grid_for(mn), 256, 0, st>>>(w.xh, w.xl, mn, d_x);
            } else {
                mx_rot_f64<<<dim3(w.x_tiles, w.npairs), kRot64Threads, kRot64Smem, st>>>(
                    d_x, rows, w.x_tiles, w.v64, cols, w.nb, round, d_gw, w.flags);
            }
        }
        JSVD_CUDA_TRY(cudaGetLastError());
        int dstatus = 0;
        JSVD_CUDA_TRY(cudaMemcpyAsync(&dstatus, w.status, sizeof(int), cudaMemcpyDeviceToHost, st));
        JSVD_CUDA_TRY(cudaStreamSynchronize(st));
        if (dstatus != 0) {
            set_last_error(JSVD_ERR_RUNTIME, "jsvd_mixed_test_round: device status " + std::to_string(dstatus));
            return JSVD_ERR_RUNTIME;
        }
        return JSVD_OK;
    });
}

extern "C" void jsvd_mixed_options_default(jsvd_mixed_options *o)
{
    if (o) *o = default_options();
}

extern "C" int jsvd_mixed_builtin_tuning(int *out, int capacity)
{
    if (out != nullptr)
        for (int i = 0; i < kMixedTuningCount && i < capacity; ++i) {
            out[4 * i] = kMixedTuning[i].max_cols;
            out[4 * i + 1] = kMixedTuning[i].tc_max_sweeps;
            out[4 * i + 2] = kMixedTuning[i].inner_sweeps;
            out[4 * i + 3] = kMixedTuning[i].gram_splits;
        }
    return kMixedTuningCount;
}

extern "C" void jsvd_mixed_set_options(const jsvd_mixed_options *o) { thread_options() = o ? *o : default_options(); }

extern "C" void jsvd_mixed_stats_get(jsvd_mixed_stats *out)
{
    if (!out) return;
    const MixedStats &s = mixed_stats();
    out->solves = s.solves;
    out->tc_sweeps = s.tc_sweeps;
    out->f64_sweeps = s.f64_sweeps;
    out->block_rounds = s.block_rounds;
    out->fallbacks = s.fallbacks;
    out->qr_ms = s.qr_ms;
    out->tc_ms = s.tc_ms;
    out->orth_ms = s.orth_ms;
    out->refine_ms = s.refine_ms;
    out->out_ms = s.out_ms;
    out->last_tc_offdiag = s.last_tc_off;
    out->last_f64_offdiag = s.last_f64_off;
    out->last_tc_sweeps = s.last_tc_sweeps;
    out->last_f64_sweeps = s.last_f64_sweeps;
    out->tc_gram_launches = s.tc_gram;
    out->tc_rot_launches = s.tc_rot;
    out->f64_gram_launches = s.f64_gram;
    out->f64_rot_launches = s.f64_rot;
    out->evd_launches = s.evd;
    out->tc_discarded = s.tc_discarded;
    out->tc_gram_ms = s.tc_gram_ms;
    out->tc_evd_ms = s.tc_evd_ms;
    out->tc_rot_ms = s.tc_rot_ms;
    out->f64_gram_ms = s.f64_gram_ms;
    out->f64_evd_ms = s.f64_evd_ms;
    out->f64_rot_ms = s.f64_rot_ms;
    out->tc_sampled_rounds = s.tc_sampled;
    out->f64_sampled_rounds = s.f64_sampled;
    out->tc_sampled_pairs = s.tc_sampled_pairs;
    out->f64_sampled_pairs = s.f64_sampled_pairs;
    out->rows_pad = s.rows_pad;
    out->cols_pad = s.cols_pad;
    out->block_pairs = s.npairs;
}

extern "C" int jsvd_mixed_sweep_history(int *phase, double *offdiag, unsigned long long *rotated, int capacity)
{
    const MixedStats &s = mixed_stats();
    const int n = std::min(s.hist_len, std::max(0, capacity));
    for (int i = 0; i < n; ++i) {
        if (phase) phase[i] = s.hist_phase[i];
        if (offdiag) offdiag[i] = s.hist_off[i];
        if (rotated) rotated[i] = s.hist_rot[i];
    }
    return s.hist_len;
}

extern "C" void jsvd_mixed_stats_reset(void) { mixed_stats() = MixedStats{}; }
