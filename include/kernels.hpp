// jacobi::svd domain API - source-compatible with kleedaisuki/jacobi-svd-cuda
// include/kernels.hpp (same namespace, types, members, defaults and function
// signatures), implemented on top of the C ABI in jsvd.h by
// jacobi-svd-cuda_b200/csrc/kernels.cpp.  Code written against the reference
// header compiles and links against libjsvd.so unchanged.
#pragma once

#include <cstddef>
#include <span>
#include <stdexcept>
#include <vector>

namespace jacobi::svd
{
    /// Layout-transpose policy (reference include/kernels.hpp:13-29).  Kept for
    /// source compatibility: this implementation always sweeps a column-major
    /// working copy, so the policy changes no arithmetic and no result.
    enum class LayoutTransposeMode
    {
        auto_select,
        force_enable,
        force_disable
    };

    /// Result of auto_tune_layout_transpose_threshold (reference :34-60).
    struct LayoutTransposeAutoTuneReport final
    {
        bool executed = false;
        int recommended_min_columns = 16;
        std::size_t recommended_min_elements = 4096;
        double estimated_best_speedup = 1.0;
        std::size_t sample_count = 0;
    };

    /// Thrown when a CUDA runtime call fails (reference :65-73).  The message
    /// has the form "CUDA call failed: <expr> @ <file>:<line>, code=<n>,
    /// message=<text>".
    class CudaError final : public std::runtime_error
    {
    public:
        explicit CudaError(const char *message);
    };

    /// Solver settings (reference :78-124).  epsilon is the relative
    /// orthogonality threshold |a_p . a_q| <= epsilon * ||a_p|| * ||a_q||;
    /// threads_per_block sets the width of the dot-product reduction tree.
    struct JacobiSvdConfig final
    {
        double epsilon = 1.0e-9;
        int max_sweeps = 128;
        int threads_per_block = 256;
        LayoutTransposeMode layout_transpose_mode = LayoutTransposeMode::auto_select;
        int layout_transpose_min_columns = 16;
        std::size_t layout_transpose_min_elements = 4096;
        bool layout_transpose_auto_tune = false;
        int layout_transpose_benchmark_repetitions = 2;
        int layout_transpose_benchmark_sweeps = 8;
    };

    /// Move-only owner of a row-major FP64 matrix in device memory
    /// (reference :130-244).
    class DeviceMatrix final
    {
    public:
        DeviceMatrix() = default;
        DeviceMatrix(std::size_t rows, std::size_t columns);
        ~DeviceMatrix();
        DeviceMatrix(const DeviceMatrix &) = delete;
        DeviceMatrix &operator=(const DeviceMatrix &) = delete;
        DeviceMatrix(DeviceMatrix &&other) noexcept;
        DeviceMatrix &operator=(DeviceMatrix &&other) noexcept;

        /// Reallocates for a rows x columns matrix (both must be positive).
        void reset(std::size_t rows, std::size_t columns);

        [[nodiscard]] std::size_t rows() const noexcept;
        [[nodiscard]] std::size_t columns() const noexcept;
        [[nodiscard]] std::size_t size() const noexcept;
        [[nodiscard]] std::size_t bytes() const noexcept;
        [[nodiscard]] double *data() noexcept;
        [[nodiscard]] const double *data() const noexcept;

        /// Copies rows*columns row-major values from the host.
        void copy_from_host(std::span<const double> host_values);
        /// Copies the matrix back to a new host vector.
        [[nodiscard]] std::vector<double> copy_to_host() const;

    private:
        std::size_t rows_ = 0;
        std::size_t columns_ = 0;
        double *data_ = nullptr;
    };

    /// Host-side result (reference :249-280): U is m x n and V is n x n, both
    /// row-major; sigma is unsorted, in the column order the sweep leaves;
    /// sweeps == max_sweeps signals that the tolerance was not reached.
    struct JacobiSvdResult final
    {
        std::size_t rows = 0;
        std::size_t columns = 0;
        std::vector<double> u;
        std::vector<double> sigma;
        std::vector<double> v;
        int sweeps = 0;
    };

    /// One-sided Jacobi SVD of a row-major m x n matrix, m >= n (reference
    /// :295-298).  Throws std::invalid_argument for bad shapes or settings and
    /// CudaError for CUDA failures.  Thread-safe; synchronous.
    [[nodiscard]] JacobiSvdResult one_sided_jacobi_svd(std::span<const double> host_input,
                                                       std::size_t rows,
                                                       std::size_t columns,
                                                       const JacobiSvdConfig &config = {});

    /// Scans matrix sizes and recommends layout thresholds (reference
    /// :306-307).
    [[nodiscard]] LayoutTransposeAutoTuneReport auto_tune_layout_transpose_threshold(
        const JacobiSvdConfig &config = {});
} // namespace jacobi::svd
