// Extensions of the jacobi::svd C++ API (include/kernels.hpp) that have no
// counterpart in the reference: the faster solver paths and the validation
// metrics, with the reference's result type and exception types.
#pragma once

#include <cstddef>
#include <span>

#include "kernels.hpp"

namespace jacobi::svd
{
    /// Solver of jacobi_svd.
    enum class SvdSolver
    {
        plain,     ///< the reference's sweep, bit-identical (= one_sided_jacobi_svd)
        precond,   ///< two CholeskyQR factorisations, then the sweep on the
                   ///< triangular factor (accurate to working precision)
        blockpair, ///< block-pair ordering of the FP64 sweep (working precision)
        blocked,   ///< Gram-blocked FP64 sweep (working precision)
        mixed      ///< blocked sweeps with a tensor-core (3xTF32) phase and FP64
                   ///< refinement after the QR stage (working precision)
    };

    /// one_sided_jacobi_svd through the chosen solver.  Same arguments,
    /// validation, result layout and exceptions as one_sided_jacobi_svd.
    [[nodiscard]] JacobiSvdResult jacobi_svd(std::span<const double> host_input,
                                             std::size_t rows,
                                             std::size_t columns,
                                             const JacobiSvdConfig &config = {},
                                             SvdSolver solver = SvdSolver::precond);

    /// Validation metrics of a result against its input, as the reference's
    /// design defines them: rho_a = ||A - U S V^T||_F / max(1, ||A||_F),
    /// rho_u = ||U^T U - I||_F over the columns with sigma > 0,
    /// rho_v = ||V^T V - I||_F.  Host threads; no CUDA call.
    struct SvdResiduals final
    {
        double rho_a = 0.0;
        double rho_u = 0.0;
        double rho_v = 0.0;
    };
    [[nodiscard]] SvdResiduals residuals(std::span<const double> host_input, const JacobiSvdResult &result);
} // namespace jacobi::svd
