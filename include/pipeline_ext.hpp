// Extensions of the pipeline that have no counterpart in the reference.
#pragma once

namespace jacobi::svd::pipeline
{
    /// Solver used for testcases too large for the batched kernel.
    enum class LargeSolver
    {
        plain,   ///< the plain sweep: bit-identical to the reference (default)
        precond  ///< shifted CholeskyQR3 + Jacobi on R^T: faster on tall and
                 ///< ill-conditioned inputs, accurate to working precision
    };

    /// Selects the large-testcase solver for pipelines run afterwards in this
    /// process (process-wide setting).
    void set_large_solver(LargeSolver solver) noexcept;
    [[nodiscard]] LargeSolver large_solver() noexcept;
} // namespace jacobi::svd::pipeline
