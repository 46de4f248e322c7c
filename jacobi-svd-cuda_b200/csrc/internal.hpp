// Host-side helpers shared by the C-ABI translation units: the per-thread
// last-error string, CUDA status checks and argument validation that mirror
// the reference's exception messages (kleedaisuki/jacobi-svd-cuda
// src/kernels.cu:29-46, 338-356, 807-833).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <exception>
#include <new>
#include <sstream>
#include <string>
#include <utility>

#include "jsvd.h"

namespace jsvd {

void set_last_error(int code, const std::string &message);
const std::string &last_error_message();

// Calls `release` when the enclosing scope ends, on every return path.
template <class F>
class ScopeExit {
public:
    explicit ScopeExit(F release) : release_(std::move(release)) {}
    ScopeExit(const ScopeExit &) = delete;
    ScopeExit &operator=(const ScopeExit &) = delete;
    ~ScopeExit() { release_(); }

private:
    F release_;
};

// *cfg, or the defaults (jsvd_config_default) written to `storage` when cfg is
// null.
inline const jsvd_config &config_or_default(const jsvd_config *cfg, jsvd_config &storage)
{
    if (cfg) return *cfg;
    jsvd_config_default(&storage);
    return storage;
}

// A device-buffer entry point (jsvd_*_svd_device).
using DeviceSolveFn = int (*)(const double *, size_t, size_t, const jsvd_config *, double *, double *, double *,
                              int *, void *);

// Host-buffer form of a device-buffer entry point: validates like the plain
// path, copies A in and the requested outputs back on the calling thread's
// library stream, synchronously.
int host_buffer_solve(DeviceSolveFn device_fn, const double *a, size_t rows, size_t columns, const jsvd_config *cfg,
                      double *u, double *sigma, double *v, int *sweeps);

// Records a C++ exception caught at a C entry point as JSVD_ERR_RUNTIME (the
// message is dropped if even that cannot be allocated).
void note_exception(const char *what) noexcept;

// Runs the body of a C entry point: a C++ exception (host allocation, thread
// creation, ...) becomes JSVD_ERR_RUNTIME and the last-error text instead of
// unwinding into a C caller.
template <class Body>
int c_entry(Body &&body) noexcept
{
    try {
        return body();
    } catch (const std::bad_alloc &) {
        note_exception("Host memory allocation failed.");
    } catch (const std::exception &e) {
        note_exception(e.what());
    } catch (...) {
        note_exception("Unknown C++ exception.");
    }
    return JSVD_ERR_RUNTIME;
}

// Formats a CUDA failure like the reference's JACOBI_CUDA_CHECK:
// "CUDA call failed: <expr> @ <file>:<line>, code=<n>, message=<text>".
inline int cuda_failure(cudaError_t status, const char *expr, const char *file, int line)
{
    std::ostringstream os;
    os << "CUDA call failed: " << expr << " @ " << file << ':' << line << ", code=" << static_cast<int>(status)
       << ", message=" << cudaGetErrorString(status);
    set_last_error(JSVD_ERR_CUDA, os.str());
    return JSVD_ERR_CUDA;
}

inline int invalid_argument(const char *message)
{
    set_last_error(JSVD_ERR_INVALID_ARGUMENT, message);
    return JSVD_ERR_INVALID_ARGUMENT;
}

// True when a rows x columns request is outside the supported range: the
// kernels index rows and columns with 32-bit integers and step them by up to
// 1024 (+ 31 in the tile kernels) past the last one, so each dimension stays
// 2048 below 2^31; byte counts of several m x n buffers must not overflow
// size_t.
inline bool dims_out_of_range(std::size_t rows, std::size_t columns)
{
    constexpr std::size_t kMaxDim = (std::size_t)0x7fffffff - 2047;
    if (rows > kMaxDim || columns > kMaxDim) return true;
    return rows * columns > SIZE_MAX / 64;  // both factors < 2^31: the product itself fits
}

// Validates a plain-path request exactly as the reference does, in the same
// order and with the same messages.  Returns JSVD_OK or an error code.
int validate_plain_request(const void *input, std::size_t rows, std::size_t columns, const jsvd_config &cfg);

// Threads-per-block normalisation of the reference (kernels.cu:685-690):
// clamp to [32, 1024] and round up to a multiple of 32.
inline int normalize_threads_per_block(int raw)
{
    int c = raw < 32 ? 32 : (raw > 1024 ? 1024 : raw);
    int a = ((c + 31) / 32) * 32;
    return a > 1024 ? 1024 : a;
}

// Reduction width actually used: the largest power of two not above the
// normalised thread count (identical to it for every power of two, which
// includes the default 256).
inline int reduction_lanes(int raw_threads)
{
    int t = normalize_threads_per_block(raw_threads);
    int p = 32;
    while (p * 2 <= t) p *= 2;
    return p;
}

// Drops the calling thread's cached QR-stage plans (precond.cu).
void pc_release_thread_plans();

}  // namespace jsvd

#define JSVD_CUDA_TRY(EXPR)                                                          \
    do {                                                                             \
        cudaError_t jsvd_status_ = (EXPR);                                           \
        if (jsvd_status_ != cudaSuccess)                                             \
            return ::jsvd::cuda_failure(jsvd_status_, #EXPR, __FILE__, __LINE__);    \
    } while (0)
