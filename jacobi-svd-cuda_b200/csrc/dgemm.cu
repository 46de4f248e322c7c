// FP64 GEMM for sm_100a on the FP64 tensor cores.
//
// tcgen05 has no FP64 kind, so the FP64 products of this library (CholeskyQR
// Grams and triangular updates, re-orthogonalisation, U = Q U_x, V = Q1 V_x)
// run on mma.sync m8n8k4 f64 (DMMA).  Each warp owns a 32 x 32 tile of C (16
// DMMA tiles, 32 accumulators per lane); a CTA owns BM x BN; operand tiles of
// BK = 16 are staged in shared memory through a 3-stage cp.async ring.
// Every operand is stored in shared memory along the dimension that is
// contiguous in global memory, so global reads are coalesced and shared-memory
// writes conflict-free:
//   MN-contiguous [k][mn] (row length BM + 8: fragment reads of 8 x 4 doubles
//     take the minimum two wavefronts) for op(A) = N and op(B) = T;
//   K-contiguous  [mn][k] (row length BK + 4, same property) for op(A) = T and
//     op(B) = N.
#include <cuda_runtime.h>

#include <algorithm>

#include "dgemm.hpp"
#include "internal.hpp"
#include "jsvd.h"
#include "plain.hpp"
#include "ptx.cuh"

namespace jsvd {
namespace {

constexpr int kBK = 16;
constexpr int kStages = 3;

template <bool KCONTIG, int BMN>
struct OperandTile {
    // elements per stage, row length
    static constexpr int LD = KCONTIG ? (kBK + 4) : (BMN + 8);
    static constexpr int ELEMS = KCONTIG ? BMN * LD : kBK * LD;
    __device__ static int idx(int mn, int k) { return KCONTIG ? mn * LD + k : k * LD + mn; }
};

// Loads the kBK-deep slice k0 of op(X) rows [mn0, mn0 + BMN) into s.  X is
// column-major with leading dimension ldx.  For op = N of A (and op = T of B)
// the contiguous global dimension is mn; otherwise it is k.
template <bool KCONTIG, int BMN, int NT>
__device__ __forceinline__ void load_tile(double *s, const double *X, long ldx, int mn0, int k0, int MN, int K)
{
    using Tl = OperandTile<KCONTIG, BMN>;
    constexpr int TOTAL = BMN * kBK;
#pragma unroll
    for (int e0 = 0; e0 < TOTAL; e0 += NT) {
        const int e = e0 + (int)threadIdx.x;
        int mn, k;
        if (KCONTIG) {
            k = e % kBK;
            mn = e / kBK;
        } else {
            mn = e % BMN;
            k = e / BMN;
        }
        const int gm = mn0 + mn, gk = k0 + k;
        double *dst = s + Tl::idx(mn, k);
        if (gm < MN && gk < K) {
            // KCONTIG: X(k, mn) at k + mn*ldx;  MN-contiguous: X(mn, k) at mn + k*ldx
            const double *src = KCONTIG ? (X + (size_t)gk + (size_t)gm * ldx) : (X + (size_t)gm + (size_t)gk * ldx);
            cp_async8(dst, src);
        } else {
            *dst = 0.0;
        }
    }
}

template <int BM, int BN, bool TA, bool TB>
__global__ void __launch_bounds__((BM / 32) * (BN / 32) * 32)
    dgemm_kernel(int m, int n, int k, double alpha, const double *__restrict__ A, long lda,
                 const double *__restrict__ B, long ldb, double beta, double *__restrict__ C, long ldc, int lower)
{
    constexpr int WN = BN / 32;
    constexpr int NT = (BM / 32) * WN * 32;
    // op(A) = N: A(m x k) contiguous along m -> MN-contiguous; op(A) = T: K-contiguous.
    // op(B) = N: B(k x n) contiguous along k -> K-contiguous;  op(B) = T: MN-contiguous.
    constexpr bool AK = TA, BKc = !TB;
    using TA_ = OperandTile<AK, BM>;
    using TB_ = OperandTile<BKc, BN>;
    extern __shared__ double dsm[];
    double *sa = dsm;
    double *sb = dsm + kStages * TA_::ELEMS;
    const int m0 = blockIdx.x * BM, n0 = blockIdx.y * BN;
    if (lower && n0 > m0 + BM - 1) return;  // tile strictly above the diagonal
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int wm = warp / WN, wn = warp % WN;
    const int ktiles = (k + kBK - 1) / kBK;

    auto issue = [&](int kt) {
        const int s = kt % kStages;
        load_tile<AK, BM, NT>(sa + s * TA_::ELEMS, A, lda, m0, kt * kBK, m, k);
        load_tile<BKc, BN, NT>(sb + s * TB_::ELEMS, B, ldb, n0, kt * kBK, n, k);
    };

    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;

#pragma unroll
    for (int s = 0; s < kStages - 1; ++s) {
        if (s < ktiles) issue(s);
        cp_async_commit();
    }
    const int fr = lane >> 2, fk = lane & 3;
    for (int kt = 0; kt < ktiles; ++kt) {
        cp_async_wait<kStages - 2>();
        __syncthreads();
        if (kt + kStages - 1 < ktiles) issue(kt + kStages - 1);
        cp_async_commit();
        const double *ta = sa + (kt % kStages) * TA_::ELEMS;
        const double *tb = sb + (kt % kStages) * TB_::ELEMS;
#pragma unroll
        for (int kk = 0; kk < kBK; kk += 4) {
            double af[4], bf[4];
#pragma unroll
            for (int i = 0; i < 4; ++i) af[i] = ta[TA_::idx(wm * 32 + i * 8 + fr, kk + fk)];
#pragma unroll
            for (int j = 0; j < 4; ++j) bf[j] = tb[TB_::idx(wn * 32 + j * 8 + fr, kk + fk)];
#pragma unroll
            for (int i = 0; i < 4; ++i)
#pragma unroll
                for (int j = 0; j < 4; ++j) dmma_m8n8k4(acc[i][j], af[i], bf[j]);
        }
    }
    cp_async_wait<0>();
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        const int row = m0 + wm * 32 + i * 8 + fr;
        if (row >= m) continue;
#pragma unroll
        for (int j = 0; j < 4; ++j) {
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                const int col = n0 + wn * 32 + j * 8 + 2 * fk + h;
                if (col >= n || (lower && col > row)) continue;
                double *cp = C + (size_t)row + (size_t)col * ldc;
                const double v = alpha * acc[i][j][h];
                *cp = (beta == 0.0) ? v : fma(beta, *cp, v);
            }
        }
    }
}

template <int BM, int BN, bool TA, bool TB>
int launch(cudaStream_t st, int m, int n, int k, double alpha, const double *A, long lda, const double *B, long ldb,
           double beta, double *C, long ldc, int lower)
{
    constexpr int NT = (BM / 32) * (BN / 32) * 32;
    constexpr size_t smem = sizeof(double) * kStages *
                            (OperandTile<TA, BM>::ELEMS + OperandTile<!TB, BN>::ELEMS);
    static_assert(smem <= 227 * 1024, "dgemm tile does not fit shared memory");
    auto kern = dgemm_kernel<BM, BN, TA, TB>;
    if (smem > 48 * 1024)
        JSVD_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    const dim3 grid((m + BM - 1) / BM, (n + BN - 1) / BN);
    kern<<<grid, NT, smem, st>>>(m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lower);
    JSVD_CUDA_TRY(cudaGetLastError());
    return JSVD_OK;
}

template <bool TA, bool TB>
int dispatch(cudaStream_t st, int m, int n, int k, double alpha, const double *A, long lda, const double *B,
             long ldb, double beta, double *C, long ldc, int lower)
{
    // Large outputs: 128 x 128 tiles (16 warps); otherwise 64 x 64 (4 warps) so
    // that a GEMM of a 1024-column factor still fills the 148 SMs.
    const long tiles128 = (long)((m + 127) / 128) * ((n + 127) / 128);
    if (tiles128 >= 2 * 148)
        return launch<128, 128, TA, TB>(st, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lower);
    return launch<64, 64, TA, TB>(st, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lower);
}

thread_local unsigned long long t_launches = 0;

}  // namespace

unsigned long long dgemm_launches() { return t_launches; }

int dgemm(cudaStream_t st, char opA, char opB, int m, int n, int k, double alpha, const double *A, long lda,
          const double *B, long ldb, double beta, double *C, long ldc, int lower)
{
    if (m <= 0 || n <= 0) return JSVD_OK;
    if (k <= 0) return invalid_argument("dgemm: k must be positive.");
    if (m > 65535 * 64 || n > 65535 * 64) return invalid_argument("dgemm: matrix too large for the tile grid.");
    ++t_launches;
    const bool ta = (opA == 'T' || opA == 't'), tb = (opB == 'T' || opB == 't');
    if (!ta && !tb) return dispatch<false, false>(st, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lower);
    if (!ta && tb) return dispatch<false, true>(st, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lower);
    if (ta && !tb) return dispatch<true, false>(st, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lower);
    return dispatch<true, true>(st, m, n, k, alpha, A, lda, B, ldb, beta, C, ldc, lower);
}

}  // namespace jsvd

// Test and tooling entry: C = alpha op(A) op(B) + beta C on device buffers,
// on the calling thread's library stream, synchronously.
extern "C" int jsvd_dgemm_device(char op_a, char op_b, int m, int n, int k, double alpha, const double *a, long lda,
                                 const double *b, long ldb, double beta, double *c, long ldc, int lower)
{
    using namespace jsvd;
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        if (!a || !b || !c) return invalid_argument("jsvd_dgemm_device: null buffer.");
        cudaStream_t st = nullptr;
        if (const int e = entry_stream(nullptr, &st); e != JSVD_OK) return e;
        const int rc = dgemm(st, op_a, op_b, m, n, k, alpha, a, lda, b, ldb, beta, c, ldc, lower);
        if (rc != JSVD_OK) return rc;
        JSVD_CUDA_TRY(cudaStreamSynchronize(st));
        return JSVD_OK;
    });
}
