// Test-only shim: exposes the reference's own solver
// (jacobi::svd::one_sided_jacobi_svd, kleedaisuki/jacobi-svd-cuda
// include/kernels.hpp:295-298) through a C symbol so the golden-vector script
// can call the unmodified reference on seeded inputs.  Compiled together with
// the reference's src/kernels.cu into oracle/_ref/ by oracle/Makefile; never
// linked into the product.
#include "kernels.hpp"

#include <cstddef>
#include <cstring>
#include <exception>
#include <span>
#include <stdexcept>
#include <string>

namespace {
thread_local std::string g_error;
}

extern "C" int ref_plain_svd(const double *a, std::size_t m, std::size_t n, double eps, int max_sweeps,
                             int threads_per_block, int layout_mode, double *u, double *sigma, double *v,
                             int *sweeps)
{
    try {
        jacobi::svd::JacobiSvdConfig cfg;
        cfg.epsilon = eps;
        cfg.max_sweeps = max_sweeps;
        cfg.threads_per_block = threads_per_block;
        cfg.layout_transpose_mode = static_cast<jacobi::svd::LayoutTransposeMode>(layout_mode);
        const auto r = jacobi::svd::one_sided_jacobi_svd(std::span<const double>(a, m * n), m, n, cfg);
        if (u) std::memcpy(u, r.u.data(), sizeof(double) * r.u.size());
        if (sigma) std::memcpy(sigma, r.sigma.data(), sizeof(double) * r.sigma.size());
        if (v) std::memcpy(v, r.v.data(), sizeof(double) * r.v.size());
        if (sweeps) *sweeps = r.sweeps;
        return 0;
    } catch (const std::invalid_argument &e) {
        g_error = e.what();
        return 1;
    } catch (const jacobi::svd::CudaError &e) {
        g_error = e.what();
        return 2;
    } catch (const std::exception &e) {
        g_error = e.what();
        return 4;
    }
}

extern "C" const char *ref_last_error() { return g_error.c_str(); }
