// Inline-PTX building blocks for sm_100a kernels: FP64 tensor-core MMA
// (mma.sync m8n8k4 f64), cp.async, mbarriers with bounded waits, TMA tile
// loads (cp.async.bulk.tensor, no multicast) and the tcgen05 family (TMEM
// allocation, MMA issue and commit, TMEM loads).
//
// Every wait here is bounded by a wall-clock limit read from %globaltimer:
// on expiry the caller gets `false` and must record an error and leave
// without touching the data it was waiting for.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

namespace jsvd {

constexpr long long kTcWaitLimitNs = 2000000000LL;  // 2 s per wait

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ long long tc_global_ns()
{
    long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

// ---- FP64 tensor-core MMA: D(8x8) += A(8x4, row) B(4x8, col) ---------------
// Fragments (lane = threadIdx.x % 32): a = A[lane/4][lane%4],
// b = B[lane%4][lane/4], d = {D[lane/4][2*(lane%4)], D[lane/4][2*(lane%4)+1]}.
__device__ __forceinline__ void dmma_m8n8k4(double (&d)[2], double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};"
                 : "+d"(d[0]), "+d"(d[1])
                 : "d"(a), "d"(b));
}

// ---- cp.async (8-byte elements) ---------------------------------------------
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem)
{
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_u32(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait()
{
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// ---- mbarrier -----------------------------------------------------------------
__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}
// Waits for the phase with the given parity to complete; false after
// limit_ns (kTcWaitLimitNs in the kernels; shorter in the wait-limit check).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long limit_ns = kTcWaitLimitNs)
{
    if (mbar_try_wait(bar, parity)) return true;
    const long long t0 = tc_global_ns();
    for (;;) {
        if (mbar_try_wait(bar, parity)) return true;
        if (tc_global_ns() - t0 > limit_ns) return false;
    }
}

// ---- TMA tile load (2-D tensor map, no multicast) ---------------------------
// Coordinates are in elements, innermost first; the innermost coordinate times
// the element size must be a multiple of 16 bytes (callers load 32-float boxes
// at multiples of 32).
__device__ __forceinline__ void tma_load_2d(void *smem_dst, const void *tensor_map, uint64_t *bar, int c0, int c1)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], "
        "[%2];" ::"r"(smem_u32(smem_dst)),
        "l"(tensor_map), "r"(smem_u32(bar)), "r"(c0), "r"(c1)
        : "memory");
}
// Bulk copy of `bytes` contiguous bytes from global to shared memory (no
// tensor map, no multicast), completing on an mbarrier; both addresses 16-byte
// aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void *smem_dst, const void *gmem_src, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(smem_dst)),
        "l"(gmem_src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void tma_prefetch_desc(const void *tensor_map)
{
    asm volatile("prefetch.tensormap [%0];" ::"l"(tensor_map) : "memory");
}

// Generic-proxy shared-memory writes -> visible to the async proxy (tcgen05.mma
// operand reads).
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// ---- tcgen05 ------------------------------------------------------------------
// TMEM allocation by one whole warp; the address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t *slot, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

// D[tmem] (+)= A[smem] * B[smem], kind::tf32, FP32 accumulation; one thread.
__device__ __forceinline__ void tc_mma_tf32(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                            uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate)
        : "memory");
}
// Arrives on *bar once every tcgen05.mma issued so far by this thread is done.
__device__ __forceinline__ void tc_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 consecutive FP32 columns of this thread's TMEM lane (warp w reads lanes
// 32*(w%4) .. 32*(w%4)+31; taddr carries the lane in its upper half).
__device__ __forceinline__ void tmem_ld32(uint32_t taddr, float (&v)[32])
{
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
        "%15, %16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor (tcgen05 format, version 1): start address,
// leading- and stride-dimension byte offsets, swizzle mode in bits 61-63.
//   SWIZZLE_128B (2): 16-byte chunks permuted within 128-byte rows, atoms of
//     8 rows (1024 bytes, 1024-byte aligned).  K-major operands here.
//   SWIZZLE_128B_BASE32B (1): 32-byte chunks permuted within 128-byte rows,
//     atoms of 4 rows (512 bytes).  The only layout the tensor cores accept
//     for MN-major 32-bit (TF32) operands; TMA writes it with
//     CU_TENSOR_MAP_SWIZZLE_128B_ATOM_32B.
constexpr uint32_t kSwizzle128B = 2, kSwizzle128B32BAtom = 1;
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes,
                                              uint32_t layout)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFFu);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;  // descriptor version (sm_100)
    d |= (uint64_t)layout << 61;
    return d;
}
__device__ __forceinline__ uint64_t smem_desc_sw128(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
    return smem_desc(saddr, lbo_bytes, sbo_bytes, kSwizzle128B);
}

// Instruction descriptor for kind::tf32 with FP32 accumulation: M x N tile,
// A and B K-major (0) or MN-major (1).
__host__ __device__ constexpr uint32_t idesc_tf32(int M, int N, int a_mn_major, int b_mn_major)
{
    return (1u << 4)                          // D format: F32
           | (2u << 7)                        // A format: TF32
           | (2u << 10)                       // B format: TF32
           | ((uint32_t)a_mn_major << 15)     // A major
           | ((uint32_t)b_mn_major << 16)     // B major
           | ((uint32_t)(N >> 3) << 17)       // N / 8
           | ((uint32_t)(M >> 4) << 24);      // M / 16
}

// Round-to-nearest TF32 value of x (low 13 mantissa bits zero) and the FP32
// remainder x - hi (exact).
__device__ __forceinline__ void split_tf32(float x, float &hi, float &lo)
{
    uint32_t h;
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
    hi = __uint_as_float(h);
    lo = x - hi;
}

}  // namespace jsvd
