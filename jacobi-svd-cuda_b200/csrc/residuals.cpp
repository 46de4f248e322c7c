// Host-side validation metrics of one SVD result, as the reference's design
// defines them (kleedaisuki/jacobi-svd-cuda
// tex/sections/03-gpu-parallel-reduction.tex:30-40):
//   rho_A = ||A - U S V^T||_F / max(1, ||A||_F)
//   rho_U = ||U^T U - I||_F   over the columns with sigma > 0 (the solver
//                             writes zero U columns where sigma <= eps)
//   rho_V = ||V^T V - I||_F   (computed as ||V V^T - I||_F: for a square V the
//                             two matrices have the same eigenvalues)
// Row-major operands as the C ABI returns them.  Every inner product runs over
// contiguous memory (U is transposed once); rows or column pairs are
// interleaved over host threads.  No CUDA call.
#include <algorithm>
#include <cmath>
#include <exception>
#include <system_error>
#include <thread>
#include <vector>

#include "internal.hpp"
#include "jsvd.h"

namespace jsvd {
namespace {

// Four-way unrolled dot product (independent partial sums).
double dot(const double *x, const double *y, size_t len)
{
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    size_t i = 0;
    for (; i + 4 <= len; i += 4) {
        s0 += x[i] * y[i];
        s1 += x[i + 1] * y[i + 1];
        s2 += x[i + 2] * y[i + 2];
        s3 += x[i + 3] * y[i + 3];
    }
    for (; i < len; ++i) s0 += x[i] * y[i];
    return (s0 + s1) + (s2 + s3);
}

// Sum over threads of body(k, t), where part k of t handles the indices
// i = k, k + t, k + 2t, ... of the caller's loop.  A part whose thread cannot
// be started runs on the calling thread; an exception thrown by a part is
// rethrown here once every thread has been joined.
template <class Body>
double parallel_sum(int threads, Body body)
{
    if (threads <= 1) return body(0, 1);
    std::vector<double> part((size_t)threads, 0.0);
    std::vector<std::exception_ptr> errors((size_t)threads);
    auto run = [&](int k) {
        try {
            part[(size_t)k] = body(k, threads);
        } catch (...) {
            errors[(size_t)k] = std::current_exception();
        }
    };
    std::vector<std::thread> pool;
    pool.reserve((size_t)threads);
    int started = 0;
    try {
        for (; started < threads; ++started) pool.emplace_back(run, started);
    } catch (const std::system_error &) {
        // no further thread could be started: the remaining parts run below
    }
    for (int k = started; k < threads; ++k) run(k);
    for (auto &th : pool) th.join();
    for (const auto &e : errors)
        if (e) std::rethrow_exception(e);
    double s = 0.0;
    for (double p : part) s += p;
    return s;
}

// ||X X^T - I||_F^2 for X with `count` rows of length `len` at stride `ld`.
double row_gram_minus_identity_sq(const double *x, size_t count, size_t len, size_t ld, int threads)
{
    return parallel_sum(threads, [&](int k, int t) {
        double local = 0.0;
        for (size_t a = (size_t)k; a < count; a += (size_t)t) {
            const double *xa = x + a * ld;
            for (size_t b = a; b < count; ++b) {
                const double d = dot(xa, x + b * ld, len) - (a == b ? 1.0 : 0.0);
                local += (a == b ? 1.0 : 2.0) * d * d;
            }
        }
        return local;
    });
}

// Threads for a phase of `flops` multiply-adds split over `items` rows or
// column pairs: about 2M per thread (a thread start costs tens of
// microseconds), at most the host's threads and 64.
int host_threads(double flops, size_t items)
{
    const unsigned hc = std::thread::hardware_concurrency();
    const size_t cap = std::min<size_t>(hc == 0 ? 1 : hc, 64);
    const size_t by_work = (size_t)std::max(1.0, flops / (double)(1 << 21));
    return (int)std::max<size_t>(1, std::min({cap, by_work, items}));
}

}  // namespace
}  // namespace jsvd

using namespace jsvd;

extern "C" int jsvd_residuals(const double *a, const double *u, const double *sigma, const double *v, size_t rows,
                              size_t columns, jsvd_residual_report *out)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        if (out == nullptr || sigma == nullptr || v == nullptr)
            return invalid_argument("Residual buffers must not be null.");
        if (rows == 0 || columns == 0) return invalid_argument("Input matrix shape must be non-zero.");
        if (rows < columns)
            return invalid_argument("One-sided Jacobi SVD requires rows >= columns in this implementation.");
        if (dims_out_of_range(rows, columns)) {
            set_last_error(JSVD_ERR_OVERFLOW, "Matrix dimensions exceed the supported range.");
            return JSVD_ERR_OVERFLOW;
        }
        const size_t m = rows, n = columns;
        *out = jsvd_residual_report{};
        out->rho_a = -1.0;
        out->rho_u = -1.0;
        const double dm = (double)m, dn = (double)n;

        // rho_V: rows of V are contiguous
        out->rho_v = std::sqrt(row_gram_minus_identity_sq(v, n, n, n, host_threads(dn * dn * dn / 2, n)));

        if (u != nullptr) {
            // rho_U: U^T U over the columns with sigma > 0, from a transposed copy
            std::vector<size_t> keep;
            for (size_t j = 0; j < n; ++j)
                if (sigma[j] > 0.0) keep.push_back(j);
            std::vector<double> ut(keep.size() * m);
            for (size_t i = 0; i < m; ++i)
                for (size_t c = 0; c < keep.size(); ++c) ut[c * m + i] = u[i * n + keep[c]];
            const double kept = (double)keep.size();
            out->rho_u = std::sqrt(row_gram_minus_identity_sq(ut.data(), keep.size(), m, m,
                                                              host_threads(kept * kept * dm / 2, keep.size())));

            if (a != nullptr) {
                // rho_A: row i of U S V^T is (u_i .* sigma) . v_j over j
                double norm_a = 0.0;
                const double err = parallel_sum(host_threads(dm * dn * dn, m), [&](int k, int t) {
                    std::vector<double> w(n);
                    double local = 0.0;
                    for (size_t i = (size_t)k; i < m; i += (size_t)t) {
                        for (size_t c = 0; c < n; ++c) w[c] = u[i * n + c] * sigma[c];
                        for (size_t j = 0; j < n; ++j) {
                            const double d = a[i * n + j] - dot(w.data(), v + j * n, n);
                            local += d * d;
                        }
                    }
                    return local;
                });
                norm_a = std::sqrt(dot(a, a, m * n));
                out->rho_a = std::sqrt(err) / std::max(1.0, norm_a);
            }
        }
        double smax = 0.0;
        for (size_t j = 0; j < n; ++j) smax = std::max(smax, sigma[j]);
        out->sigma_max = smax;
        return JSVD_OK;
    });
}
