// FP64 fused multiply-add throughput probe: the roofline denominator of the
// FP64-bound kernels (the batched solver), measured on the running device.
#include <cuda_runtime.h>

#include "internal.hpp"
#include "jsvd.h"

namespace jsvd {
namespace {

constexpr int kChains = 8;

// Eight independent FMA chains per thread; the result is written only when a
// flag the host never sets is on, so the work cannot be removed.
__global__ void __launch_bounds__(256) fp64_fma_probe(double *__restrict__ out, int iters, double a, double b,
                                                      int write)
{
    double x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-3 + c;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    if (write) out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace
}  // namespace jsvd

using namespace jsvd;

extern "C" int jsvd_probe_fp64_tflops(double *tflops)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        if (!tflops) return invalid_argument("tflops must not be null.");
        int dev = 0, sms = 0;
        JSVD_CUDA_TRY(cudaGetDevice(&dev));
        JSVD_CUDA_TRY(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
        const int grid = sms * 8, block = 256, iters = 4096;
        cudaStream_t st = nullptr;
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        ScopeExit release([&] {  // on every return path
            if (e0) cudaEventDestroy(e0);
            if (e1) cudaEventDestroy(e1);
            if (st) cudaStreamDestroy(st);
        });
        JSVD_CUDA_TRY(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        JSVD_CUDA_TRY(cudaEventCreate(&e0));
        JSVD_CUDA_TRY(cudaEventCreate(&e1));
        fp64_fma_probe<<<grid, block, 0, st>>>(nullptr, iters, 0.999999, 1e-7, 0);  // warm-up
        float best = 1e30f;
        for (int rep = 0; rep < 5; ++rep) {
            JSVD_CUDA_TRY(cudaEventRecord(e0, st));
            fp64_fma_probe<<<grid, block, 0, st>>>(nullptr, iters, 0.999999, 1e-7, 0);
            JSVD_CUDA_TRY(cudaEventRecord(e1, st));
            JSVD_CUDA_TRY(cudaEventSynchronize(e1));
            float ms = 0.f;
            JSVD_CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
            if (ms < best) best = ms;
        }
        const double flops = 2.0 * kChains * (double)iters * grid * block;
        *tflops = flops / (best * 1e-3) / 1e12;
        return JSVD_OK;
    });
}
