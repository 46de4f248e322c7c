// jacobi::svd C++ API (include/kernels.hpp) over the C ABI (include/jsvd.h).
// Status codes become the reference's exception types with the same messages
// (kleedaisuki/jacobi-svd-cuda src/kernels.cu:29-46, 698-796, 807-833,
// 1066-1126).
#include "kernels.hpp"

#include <cuda_runtime.h>

#include "kernels_ext.hpp"

#include <new>
#include <sstream>
#include <string>
#include <utility>

#include "jsvd.h"

namespace jacobi::svd
{
    namespace
    {
        [[noreturn]] void rethrow_status(int code)
        {
            char buf[2048];
            jsvd_last_error(buf, sizeof(buf));
            switch (code)
            {
            case JSVD_ERR_INVALID_ARGUMENT:
                throw std::invalid_argument(buf);
            case JSVD_ERR_CUDA:
                throw CudaError(buf);
            case JSVD_ERR_OVERFLOW:
                throw std::overflow_error(buf);
            default:
                throw std::runtime_error(buf);
            }
        }

        void check_cuda(cudaError_t status, const char *expr, const char *file, int line)
        {
            if (status == cudaSuccess)
                return;
            std::ostringstream os;
            os << "CUDA call failed: " << expr << " @ " << file << ':' << line << ", code=" << static_cast<int>(status)
               << ", message=" << cudaGetErrorString(status);
            throw CudaError(os.str().c_str());
        }

        jsvd_config to_c(const JacobiSvdConfig &c)
        {
            jsvd_config out{};
            out.epsilon = c.epsilon;
            out.max_sweeps = c.max_sweeps;
            out.threads_per_block = c.threads_per_block;
            out.layout_transpose_mode = c.layout_transpose_mode == LayoutTransposeMode::force_enable
                                            ? JSVD_LAYOUT_FORCE_ENABLE
                                            : (c.layout_transpose_mode == LayoutTransposeMode::force_disable
                                                   ? JSVD_LAYOUT_FORCE_DISABLE
                                                   : JSVD_LAYOUT_AUTO);
            out.layout_transpose_min_columns = c.layout_transpose_min_columns;
            out.layout_transpose_min_elements = c.layout_transpose_min_elements;
            out.layout_transpose_auto_tune = c.layout_transpose_auto_tune ? 1 : 0;
            out.layout_transpose_benchmark_repetitions = c.layout_transpose_benchmark_repetitions;
            out.layout_transpose_benchmark_sweeps = c.layout_transpose_benchmark_sweeps;
            return out;
        }
    } // namespace

#define JSVD_CXX_CUDA(EXPR) check_cuda((EXPR), #EXPR, __FILE__, __LINE__)

    CudaError::CudaError(const char *message) : std::runtime_error(message) {}

    DeviceMatrix::DeviceMatrix(std::size_t rows, std::size_t columns) { reset(rows, columns); }

    DeviceMatrix::~DeviceMatrix()
    {
        if (data_ != nullptr)
            (void)cudaFree(data_);
    }

    DeviceMatrix::DeviceMatrix(DeviceMatrix &&other) noexcept
        : rows_(std::exchange(other.rows_, 0)), columns_(std::exchange(other.columns_, 0)),
          data_(std::exchange(other.data_, nullptr))
    {
    }

    DeviceMatrix &DeviceMatrix::operator=(DeviceMatrix &&other) noexcept
    {
        if (this != &other)
        {
            if (data_ != nullptr)
                (void)cudaFree(data_);
            rows_ = std::exchange(other.rows_, 0);
            columns_ = std::exchange(other.columns_, 0);
            data_ = std::exchange(other.data_, nullptr);
        }
        return *this;
    }

    void DeviceMatrix::reset(std::size_t rows, std::size_t columns)
    {
        if (rows == 0 || columns == 0)
            throw std::invalid_argument("DeviceMatrix dimensions must be positive.");
        if (data_ != nullptr)
        {
            JSVD_CXX_CUDA(cudaFree(data_));
            data_ = nullptr;
        }
        rows_ = rows;
        columns_ = columns;
        JSVD_CXX_CUDA(cudaMalloc(reinterpret_cast<void **>(&data_), bytes()));
    }

    std::size_t DeviceMatrix::rows() const noexcept { return rows_; }
    std::size_t DeviceMatrix::columns() const noexcept { return columns_; }
    std::size_t DeviceMatrix::size() const noexcept { return rows_ * columns_; }
    std::size_t DeviceMatrix::bytes() const noexcept { return size() * sizeof(double); }
    double *DeviceMatrix::data() noexcept { return data_; }
    const double *DeviceMatrix::data() const noexcept { return data_; }

    void DeviceMatrix::copy_from_host(std::span<const double> host_values)
    {
        if (host_values.size() != size())
            throw std::invalid_argument("Host data size does not match device matrix shape.");
        JSVD_CXX_CUDA(cudaMemcpy(data_, host_values.data(), bytes(), cudaMemcpyHostToDevice));
    }

    std::vector<double> DeviceMatrix::copy_to_host() const
    {
        std::vector<double> host(size());
        JSVD_CXX_CUDA(cudaMemcpy(host.data(), data_, bytes(), cudaMemcpyDeviceToHost));
        return host;
    }

    JacobiSvdResult one_sided_jacobi_svd(std::span<const double> host_input,
                                         std::size_t rows,
                                         std::size_t columns,
                                         const JacobiSvdConfig &config)
    {
        return jacobi_svd(host_input, rows, columns, config, SvdSolver::plain);
    }

    JacobiSvdResult jacobi_svd(std::span<const double> host_input,
                               std::size_t rows,
                               std::size_t columns,
                               const JacobiSvdConfig &config,
                               SvdSolver solver)
    {
        // Shape checks in the reference's order; the buffer-size check can only
        // be made here, where the span's length is known.
        if (rows == 0 || columns == 0)
            throw std::invalid_argument("Input matrix shape must be non-zero.");
        if (rows < columns)
            throw std::invalid_argument("One-sided Jacobi SVD requires rows >= columns in this implementation.");
        if (host_input.size() != rows * columns)
            throw std::invalid_argument("Input buffer size mismatch.");
        const jsvd_config c = to_c(config);
        JacobiSvdResult result;
        result.rows = rows;
        result.columns = columns;
        result.u.resize(rows * columns);
        result.sigma.resize(columns);
        result.v.resize(columns * columns);
        using HostEntry = int (*)(const double *, std::size_t, std::size_t, const jsvd_config *, double *, double *,
                                  double *, int *);
        HostEntry entry = jsvd_plain_svd;
        switch (solver)
        {
        case SvdSolver::plain:
            entry = jsvd_plain_svd;
            break;
        case SvdSolver::precond:
            entry = jsvd_precond_svd;
            break;
        case SvdSolver::blockpair:
            entry = jsvd_blockpair_svd;
            break;
        case SvdSolver::blocked:
            entry = jsvd_blocked_svd;
            break;
        case SvdSolver::mixed:
            entry = jsvd_mixed_svd;
            break;
        default:
            throw std::invalid_argument("Unknown SvdSolver.");
        }
        const int rc = entry(host_input.data(), rows, columns, &c, result.u.data(), result.sigma.data(),
                             result.v.data(), &result.sweeps);
        if (rc != JSVD_OK)
            rethrow_status(rc);
        return result;
    }

    SvdResiduals residuals(std::span<const double> host_input, const JacobiSvdResult &result)
    {
        const std::size_t m = result.rows, n = result.columns;
        if (m == 0 || n == 0)
            throw std::invalid_argument("Input matrix shape must be non-zero.");
        if (m < n)
            throw std::invalid_argument("One-sided Jacobi SVD requires rows >= columns in this implementation.");
        if (host_input.size() != m * n || result.u.size() != m * n || result.sigma.size() != n ||
            result.v.size() != n * n)
            throw std::invalid_argument("Result buffers do not match rows and columns.");
        jsvd_residual_report r{};
        const int rc = jsvd_residuals(host_input.data(), result.u.data(), result.sigma.data(), result.v.data(), m, n,
                                      &r);
        if (rc != JSVD_OK)
            rethrow_status(rc);
        return SvdResiduals{r.rho_a, r.rho_u, r.rho_v};
    }

    LayoutTransposeAutoTuneReport auto_tune_layout_transpose_threshold(const JacobiSvdConfig &config)
    {
        const jsvd_config c = to_c(config);
        jsvd_autotune_report r{};
        const int rc = jsvd_auto_tune_layout(&c, &r);
        if (rc != JSVD_OK)
            rethrow_status(rc);
        LayoutTransposeAutoTuneReport out;
        out.executed = r.executed != 0;
        out.recommended_min_columns = r.recommended_min_columns;
        out.recommended_min_elements = r.recommended_min_elements;
        out.estimated_best_speedup = r.estimated_best_speedup;
        out.sample_count = r.sample_count;
        return out;
    }
} // namespace jacobi::svd
