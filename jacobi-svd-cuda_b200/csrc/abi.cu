// C-ABI entry points of the plain path, per-thread plan cache and error state.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <array>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "common.cuh"
#include "blockpair.hpp"
#include "internal.hpp"
#include "mixed.hpp"
#include "jsvd.h"
#include "plain.hpp"

namespace jsvd {
namespace {

struct ErrorState {
    int code = JSVD_OK;
    std::string message;
};

ErrorState &error_state()
{
    thread_local ErrorState state;
    return state;
}

// The calling thread's library stream on one device, and the event that
// orders it after the legacy default stream (created on first use).
struct DeviceStream {
    int device = -1;
    cudaStream_t stream = nullptr;
    cudaEvent_t legacy_done = nullptr;
};

struct ThreadCache {
    std::vector<std::unique_ptr<PlainPlan>> plans;  // most recently used last
    std::vector<DeviceStream> streams;
    ~ThreadCache()
    {
        plans.clear();
        for (auto &s : streams) {
            if (s.legacy_done) cudaEventDestroy(s.legacy_done);
            cudaStreamDestroy(s.stream);
        }
    }
};

ThreadCache &thread_cache()
{
    thread_local ThreadCache cache;
    return cache;
}

constexpr size_t kMaxCachedPlans = 4;
constexpr size_t kMaxCachedBytes = size_t(8) << 30;

}  // namespace

void set_last_error(int code, const std::string &message)
{
    error_state().code = code;
    error_state().message = message;
}

const std::string &last_error_message() { return error_state().message; }

void note_exception(const char *what) noexcept
{
    ErrorState &e = error_state();
    e.code = JSVD_ERR_RUNTIME;
    try {
        e.message = what;
    } catch (...) {
        e.message.clear();
    }
}

int host_buffer_solve(DeviceSolveFn device_fn, const double *a, size_t rows, size_t columns, const jsvd_config *cfg,
                      double *u, double *sigma, double *v, int *sweeps)
{
    set_last_error(JSVD_OK, "");
    jsvd_config def;
    const jsvd_config &c = config_or_default(cfg, def);
    int rc = validate_plain_request(a, rows, columns, c);
    if (rc != JSVD_OK) return rc;
    int dev = 0;
    JSVD_CUDA_TRY(cudaGetDevice(&dev));
    cudaStream_t st = thread_stream(dev);
    if (st == nullptr) return cuda_failure(cudaGetLastError(), "cudaStreamCreateWithFlags", __FILE__, __LINE__);
    const size_t mn = rows * columns, nn = columns * columns;
    double *d = nullptr;
    JSVD_CUDA_TRY(cudaMallocAsync((void **)&d, sizeof(double) * (2 * mn + nn + columns), st));
    ScopeExit free_d([&] { cudaFreeAsync(d, st); });
    double *da = d, *du = d + mn, *dv = du + mn, *ds = dv + nn;
    JSVD_CUDA_TRY(cudaMemcpyAsync(da, a, sizeof(double) * mn, cudaMemcpyHostToDevice, st));
    rc = device_fn(da, rows, columns, &c, u ? du : nullptr, ds, v ? dv : nullptr, sweeps, st);
    if (rc != JSVD_OK) return rc;
    if (u) JSVD_CUDA_TRY(cudaMemcpyAsync(u, du, sizeof(double) * mn, cudaMemcpyDeviceToHost, st));
    if (sigma) JSVD_CUDA_TRY(cudaMemcpyAsync(sigma, ds, sizeof(double) * columns, cudaMemcpyDeviceToHost, st));
    if (v) JSVD_CUDA_TRY(cudaMemcpyAsync(v, dv, sizeof(double) * nn, cudaMemcpyDeviceToHost, st));
    JSVD_CUDA_TRY(cudaStreamSynchronize(st));
    return JSVD_OK;
}

namespace {
// The calling thread's stream record for `device`, created on first use;
// nullptr when the stream cannot be created.
DeviceStream *device_stream(int device)
{
    auto &cache = thread_cache();
    for (auto &s : cache.streams)
        if (s.device == device) return &s;
    cudaStream_t st = nullptr;
    if (cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    DeviceStream rec;
    rec.device = device;
    rec.stream = st;
    cache.streams.push_back(rec);
    // The library's workspaces come from the device's default stream-ordered
    // pool.  With the pool's default release threshold (0) every synchronise
    // hands freed memory back to the driver and the next call maps it again
    // (tens of ms for the workspace of a 4096 x 1024 solve); keep up to 4 GiB
    // cached in this process instead.
    static std::atomic<unsigned long long> pools_set{0};
    if (device >= 0 && device < 64 && !(pools_set.fetch_or(1ull << device) & (1ull << device))) {
        cudaMemPool_t pool = nullptr;
        if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
            unsigned long long keep = 4ull << 30;
            cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        }
    }
    return &cache.streams.back();
}
}  // namespace

cudaStream_t thread_stream(int device)
{
    DeviceStream *s = device_stream(device);
    return s ? s->stream : nullptr;
}

int entry_stream(void *caller_stream, cudaStream_t *out)
{
    if (caller_stream != nullptr) {
        *out = static_cast<cudaStream_t>(caller_stream);
        return JSVD_OK;
    }
    int dev = 0;
    JSVD_CUDA_TRY(cudaGetDevice(&dev));
    DeviceStream *s = device_stream(dev);
    if (s == nullptr) return cuda_failure(cudaGetLastError(), "cudaStreamCreateWithFlags", __FILE__, __LINE__);
    if (s->legacy_done == nullptr)
        JSVD_CUDA_TRY(cudaEventCreateWithFlags(&s->legacy_done, cudaEventDisableTiming));
    JSVD_CUDA_TRY(cudaEventRecord(s->legacy_done, cudaStreamLegacy));
    JSVD_CUDA_TRY(cudaStreamWaitEvent(s->stream, s->legacy_done, 0));
    *out = s->stream;
    return JSVD_OK;
}

int acquire_plain_plan(size_t m, size_t n, int T, double eps, cudaStream_t stream, PlainPlan **out)
{
    int dev = 0;
    JSVD_CUDA_TRY(cudaGetDevice(&dev));
    auto &plans = thread_cache().plans;
    for (size_t i = 0; i < plans.size(); ++i) {
        PlainPlan *p = plans[i].get();
        if (p->device == dev && p->m == m && p->n == n && p->T == T && p->eps == eps && p->mode == sweep_mode() &&
            p->vpass_global_forced == vpass_global_forced()) {
            std::rotate(plans.begin() + i, plans.begin() + i + 1, plans.end());
            *out = plans.back().get();
            return JSVD_OK;
        }
    }
    // Plans allocate and release on the library's own per-thread stream (a
    // caller's stream may be destroyed before the plan is evicted).
    cudaStream_t own = thread_stream(dev);
    if (own == nullptr) return cuda_failure(cudaGetLastError(), "cudaStreamCreateWithFlags", __FILE__, __LINE__);
    if (own != stream) JSVD_CUDA_TRY(cudaStreamSynchronize(stream));
    std::unique_ptr<PlainPlan> plan;
    int rc = PlainPlan::create(dev, m, n, T, eps, own, plan);
    if (rc != JSVD_OK) return rc;
    plan->mode = sweep_mode();
    plan->use_pdl = plan->mode == 2;
    plan->angle_once = plan->mode != 3;
    plans.push_back(std::move(plan));
    size_t total = 0;
    for (auto &p : plans) total += p->bytes;
    while (plans.size() > 1 && (plans.size() > kMaxCachedPlans || total > kMaxCachedBytes)) {
        JSVD_CUDA_TRY(cudaStreamSynchronize(stream));
        total -= plans.front()->bytes;
        plans.erase(plans.begin());
    }
    *out = plans.back().get();
    return JSVD_OK;
}

int validate_plain_request(const void *input, size_t rows, size_t columns, const jsvd_config &cfg)
{
    // Order and wording follow src/kernels.cu:807-833 and :338-356.
    if (rows == 0 || columns == 0) return invalid_argument("Input matrix shape must be non-zero.");
    if (rows < columns)
        return invalid_argument("One-sided Jacobi SVD requires rows >= columns in this implementation.");
    if (input == nullptr) return invalid_argument("Input buffer size mismatch.");
    if (!(cfg.epsilon > 0.0)) return invalid_argument("epsilon must be positive.");
    if (cfg.max_sweeps <= 0) return invalid_argument("max_sweeps must be positive.");
    if (cfg.layout_transpose_min_columns <= 0)
        return invalid_argument("layout_transpose_min_columns must be positive.");
    if (cfg.layout_transpose_min_elements == 0)
        return invalid_argument("layout_transpose_min_elements must be positive.");
    if (cfg.layout_transpose_benchmark_repetitions <= 0)
        return invalid_argument("layout_transpose_benchmark_repetitions must be positive.");
    if (cfg.layout_transpose_benchmark_sweeps <= 0)
        return invalid_argument("layout_transpose_benchmark_sweeps must be positive.");
    if (cfg.layout_transpose_mode < JSVD_LAYOUT_AUTO || cfg.layout_transpose_mode > JSVD_LAYOUT_FORCE_DISABLE)
        return invalid_argument("layout_transpose_mode is not a valid LayoutTransposeMode.");
    if (dims_out_of_range(rows, columns)) {
        set_last_error(JSVD_ERR_OVERFLOW, "Matrix dimensions exceed the supported range.");
        return JSVD_ERR_OVERFLOW;
    }
    return JSVD_OK;
}

namespace {

int plain_device_impl(const double *d_a, size_t rows, size_t cols, const jsvd_config *cfg, double *d_u,
                      double *d_sigma, double *d_v, int *sweeps, cudaStream_t stream, bool gram_stop = false)
{
    jsvd_config def;
    const jsvd_config &c = config_or_default(cfg, def);
    int rc = validate_plain_request(d_a, rows, cols, c);
    if (rc != JSVD_OK) return rc;
    rc = entry_stream(stream, &stream);
    if (rc != JSVD_OK) return rc;
    PlainPlan *plan = nullptr;
    rc = acquire_plain_plan(rows, cols, reduction_lanes(c.threads_per_block), c.epsilon, stream, &plan);
    if (rc != JSVD_OK) return rc;
    rc = plan->run(d_a, d_u, d_sigma, d_v, c.max_sweeps, sweeps, stream, gram_stop);
    if (rc != JSVD_OK) return rc;
    JSVD_CUDA_TRY(cudaStreamSynchronize(stream));
    return JSVD_OK;
}

}  // namespace

int plain_device_solve(const double *d_a, size_t rows, size_t cols, const jsvd_config *cfg, double *d_u,
                       double *d_sigma, double *d_v, int *sweeps, cudaStream_t stream, bool gram_stop)
{
    set_last_error(JSVD_OK, "");
    return plain_device_impl(d_a, rows, cols, cfg, d_u, d_sigma, d_v, sweeps, stream, gram_stop);
}

}  // namespace jsvd

using namespace jsvd;

extern "C" {

void jsvd_config_default(jsvd_config *cfg)
{
    if (!cfg) return;
    // Defaults of JacobiSvdConfig, include/kernels.hpp:78-124.
    cfg->epsilon = 1.0e-9;
    cfg->max_sweeps = 128;
    cfg->threads_per_block = 256;
    cfg->layout_transpose_mode = JSVD_LAYOUT_AUTO;
    cfg->layout_transpose_min_columns = 16;
    cfg->layout_transpose_min_elements = 4096;
    cfg->layout_transpose_auto_tune = 0;
    cfg->layout_transpose_benchmark_repetitions = 2;
    cfg->layout_transpose_benchmark_sweeps = 8;
}

int jsvd_last_error(char *buf, size_t len)
{
    const auto &st = error_state();
    if (buf && len > 0) {
        size_t k = std::min(len - 1, st.message.size());
        std::memcpy(buf, st.message.data(), k);
        buf[k] = '\0';
    }
    return st.code;
}

const char *jsvd_version(void) { return "jsvd-b200 0.1.0 (sm_100a)"; }

int jsvd_plain_arith_variant(void) { return kRotVariant; }

int jsvd_plain_svd_device(const double *d_a, size_t rows, size_t columns, const jsvd_config *cfg, double *d_u,
                          double *d_sigma, double *d_v, int *sweeps, void *stream)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        return plain_device_impl(d_a, rows, columns, cfg, d_u, d_sigma, d_v, sweeps, (cudaStream_t)stream);
    });
}

int jsvd_plain_svd(const double *a, size_t rows, size_t columns, const jsvd_config *cfg, double *u, double *sigma,
                   double *v, int *sweeps)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        jsvd_config def;
        const jsvd_config &c = config_or_default(cfg, def);
        int rc = validate_plain_request(a, rows, columns, c);
        if (rc != JSVD_OK) return rc;
        int dev = 0;
        JSVD_CUDA_TRY(cudaGetDevice(&dev));
        cudaStream_t stream = thread_stream(dev);
        if (stream == nullptr) return cuda_failure(cudaGetLastError(), "cudaStreamCreateWithFlags", __FILE__, __LINE__);
        PlainPlan *plan = nullptr;
        rc = acquire_plain_plan(rows, columns, reduction_lanes(c.threads_per_block), c.epsilon, stream, &plan);
        if (rc != JSVD_OK) return rc;
        rc = plan->ensure_host_staging();
        if (rc != JSVD_OK) return rc;
        JSVD_CUDA_TRY(cudaMemcpyAsync(plan->d_in, a, sizeof(double) * rows * columns, cudaMemcpyHostToDevice, stream));
        rc = plan->run(plan->d_in, u ? plan->d_u : nullptr, plan->d_sigma, v ? plan->d_v : nullptr, c.max_sweeps,
                       sweeps, stream);
        if (rc != JSVD_OK) return rc;
        if (u)
            JSVD_CUDA_TRY(
                cudaMemcpyAsync(u, plan->d_u, sizeof(double) * rows * columns, cudaMemcpyDeviceToHost, stream));
        if (sigma)
            JSVD_CUDA_TRY(
                cudaMemcpyAsync(sigma, plan->d_sigma, sizeof(double) * columns, cudaMemcpyDeviceToHost, stream));
        if (v)
            JSVD_CUDA_TRY(
                cudaMemcpyAsync(v, plan->d_v, sizeof(double) * columns * columns, cudaMemcpyDeviceToHost, stream));
        JSVD_CUDA_TRY(cudaStreamSynchronize(stream));
        return JSVD_OK;
    });
}

int jsvd_auto_tune_layout(const jsvd_config *cfg, jsvd_autotune_report *report)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        jsvd_config def;
        const jsvd_config &c = config_or_default(cfg, def);
        if (!report) return invalid_argument("report must not be null.");
        // Validation order of src/kernels.cu:1078-1086.
        if (c.layout_transpose_min_columns <= 0)
            return invalid_argument("layout_transpose_min_columns must be positive.");
        if (c.layout_transpose_min_elements == 0)
            return invalid_argument("layout_transpose_min_elements must be positive.");
        if (c.layout_transpose_benchmark_repetitions <= 0)
            return invalid_argument("layout_transpose_benchmark_repetitions must be positive.");
        if (c.layout_transpose_benchmark_sweeps <= 0)
            return invalid_argument("layout_transpose_benchmark_sweeps must be positive.");
        if (c.max_sweeps <= 0) return invalid_argument("max_sweeps must be positive.");

        jsvd_config bench = c;
        bench.layout_transpose_auto_tune = 0;
        bench.max_sweeps = std::min(c.max_sweeps, std::max(1, c.layout_transpose_benchmark_sweeps));
        const std::array<int, 8> widths = {8, 12, 16, 24, 32, 48, 64, 96};
        report->executed = 1;
        report->recommended_min_columns = c.layout_transpose_min_columns;
        report->recommended_min_elements = c.layout_transpose_min_elements;
        report->estimated_best_speedup = 1.0;
        report->sample_count = widths.size();
        bool selected = false;
        for (int cols : widths) {
            const size_t rows = (size_t)cols * 2;
            // Deterministic benchmark matrix of src/kernels.cu:1012-1025.
            std::vector<double> a(rows * cols);
            for (size_t r = 0; r < rows; ++r)
                for (size_t k = 0; k < (size_t)cols; ++k)
                    a[r * cols + k] = std::sin(0.013 * (double)((r + 1) * (k + 1))) +
                                      std::cos(0.017 * (double)((r + 3) * (k + 5)));
            std::vector<double> u(rows * cols), s(cols), v((size_t)cols * cols);
            double ms[2] = {0.0, 0.0};
            for (int mode = 0; mode < 2; ++mode) {
                bench.layout_transpose_mode = mode == 0 ? JSVD_LAYOUT_FORCE_DISABLE : JSVD_LAYOUT_FORCE_ENABLE;
                int sw = 0;
                int rc = jsvd_plain_svd(a.data(), rows, cols, &bench, u.data(), s.data(), v.data(), &sw);
                if (rc != JSVD_OK) return rc;
                double acc = 0.0;
                for (int rep = 0; rep < c.layout_transpose_benchmark_repetitions; ++rep) {
                    auto t0 = std::chrono::steady_clock::now();
                    rc = jsvd_plain_svd(a.data(), rows, cols, &bench, u.data(), s.data(), v.data(), &sw);
                    auto t1 = std::chrono::steady_clock::now();
                    if (rc != JSVD_OK) return rc;
                    acc += std::chrono::duration<double, std::milli>(t1 - t0).count();
                }
                ms[mode] = acc / c.layout_transpose_benchmark_repetitions;
            }
            const double speedup = ms[0] / std::max(ms[1], 1e-300);
            report->estimated_best_speedup = std::max(report->estimated_best_speedup, speedup);
            if (!selected && ms[1] < ms[0]) {
                report->recommended_min_columns = cols;
                report->recommended_min_elements = rows * (size_t)cols;
                selected = true;
            }
        }
        return JSVD_OK;
    });
}

void jsvd_plain_stats_get(jsvd_plain_stats *out)
{
    if (!out) return;
    const PlainStats &s = plain_stats();
    out->solves = s.solves;
    out->sweeps = s.sweeps;
    out->round_launches = s.round_launches;
    out->vpass_launches = s.vpass_launches;
    out->other_launches = s.other_launches;
    out->round_ms = s.round_ms;
    out->vpass_ms = s.vpass_ms;
    out->gram_checks = s.gram_checks;
}

void jsvd_plain_stats_reset(void) { plain_stats() = PlainStats{}; }

void jsvd_plain_set_sweep_mode(int mode) { set_sweep_mode(mode); }

int jsvd_plain_get_sweep_mode(void) { return sweep_mode(); }

void jsvd_plain_set_vpass_in_global(int enable) { set_vpass_global_forced(enable != 0); }

void jsvd_release_thread_cache(void)
{
    auto &cache = thread_cache();
    for (auto &s : cache.streams) cudaStreamSynchronize(s.stream);
    cache.plans.clear();
    bp_release_thread_plans();
    pc_release_thread_plans();
    mixed_release_thread_cache();
}

}  // extern "C"
