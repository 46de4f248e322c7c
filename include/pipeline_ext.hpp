// Extensions of the pipeline that have no counterpart in the reference.
#pragma once

#include <cstddef>
#include <filesystem>
#include <string>

namespace jacobi::svd::pipeline
{
    /// Solver used for testcases too large for the batched kernel.
    enum class LargeSolver
    {
        plain,   ///< the plain sweep: bit-identical to the reference (default)
        precond, ///< shifted CholeskyQR3 + Jacobi on R^T: faster on tall and
                 ///< ill-conditioned inputs, accurate to working precision
        mixed    ///< the QR stage + blocked sweeps, tensor-core (3xTF32) phase
                 ///< and FP64 refinement (jsvd_mixed_svd): fastest on large
                 ///< inputs, accurate to working precision
    };

    /// Selects the large-testcase solver for pipelines run afterwards in this
    /// process (process-wide setting).
    void set_large_solver(LargeSolver solver) noexcept;
    [[nodiscard]] LargeSolver large_solver() noexcept;

    /// Validation record of one testcase: the fields the reference's design
    /// asks a test report to carry (tex/sections/03-gpu-parallel-reduction.tex:53-58).
    struct ResidualRecord
    {
        std::size_t index = 0; ///< testcase position in the input stream
        std::size_t rows = 0, columns = 0;
        double epsilon = 0.0;
        int max_sweeps = 0, sweeps = 0;
        double rho_a = 0.0, rho_u = 0.0, rho_v = 0.0; ///< as jsvd_residuals computes them
    };

    /// The record as one JSON object on one line (no newline), numbers with
    /// enough digits to round-trip.
    [[nodiscard]] std::string residual_record_json(const ResidualRecord &record);

    /// When set to a non-empty path, pipelines run afterwards in this process
    /// compute every testcase's record on the host (jsvd_residuals, which
    /// keeps a copy of each in-flight input) and write it to that file as
    /// one JSON line, in input order; the file is truncated at the start of a
    /// run.  Empty (the default) turns this off.  Process-wide setting.
    void set_residual_report(const std::filesystem::path &path);
    [[nodiscard]] std::filesystem::path residual_report();

    /// Serving-core figures of the last pipeline run that completed in this
    /// process (zeros before the first).
    struct RunServiceStats
    {
        std::size_t batches = 0;           ///< batched launches of small testcases
        std::size_t batched_testcases = 0; ///< testcases solved in those launches
        std::size_t large_solves = 0;      ///< testcases solved one per stream
        double latency_p50_ms = 0.0;       ///< submission to completion
        double latency_p99_ms = 0.0;
        double latency_mean_ms = 0.0;
        std::size_t peak_device_bytes = 0; ///< admitted footprint high-water mark
    };
    [[nodiscard]] RunServiceStats last_run_service_stats();
} // namespace jacobi::svd::pipeline
