// jacobi::svd::pipeline - source-compatible with kleedaisuki/jacobi-svd-cuda
// include/pipeline.hpp (same types, members, defaults and functions).
// Implemented by jacobi-svd-cuda_b200/csrc/pipeline.cpp on top of the serving
// core (jsvd_server_* in jsvd.h): testcases are admitted against a device
// memory budget, solved concurrently on the GPU, and their U, Sigma (1 x n)
// and V written in input order.
#pragma once

#include "kernels.hpp"

#include <cstddef>
#include <filesystem>

namespace jacobi::svd::pipeline
{
    /// Stream format of a pipeline file.
    enum class MatrixFileFormat
    {
        auto_detect, ///< from the extension: .mat or .txt (case-insensitive)
        mat,
        txt
    };

    /// Pipeline settings (reference pipeline.hpp:42-73).
    struct PipelineConfig final
    {
        std::filesystem::path input_path;
        std::filesystem::path output_path;
        MatrixFileFormat input_format = MatrixFileFormat::auto_detect;
        MatrixFileFormat output_format = MatrixFileFormat::auto_detect;
        /// Accepted for source compatibility (the reference's in-flight bound).
        /// Here the serving core sets the window: at most 8192 testcases and
        /// 4 GiB of inputs in flight, because small testcases are batched
        /// into one launch and a window of a few would leave them unbatched.
        /// Output order is the input order either way.
        std::size_t max_queued_results = 4;
        JacobiSvdConfig kernel_config{};
    };

    /// What a run did (reference pipeline.hpp:78-119).
    struct PipelineReport final
    {
        std::size_t testcase_count = 0;
        std::size_t emitted_matrix_count = 0; ///< 3 per testcase: U, Sigma, V
        std::size_t total_sweeps = 0;
        LayoutTransposeMode layout_transpose_mode = LayoutTransposeMode::auto_select;
        int layout_transpose_min_columns = 16;
        std::size_t layout_transpose_min_elements = 4096;
        bool layout_transpose_auto_tuned = false;
        double layout_transpose_estimated_best_speedup = 1.0;
    };

    /// testcases -> solver -> ordered output, as one object.
    class JacobiSvdPipeline final
    {
    public:
        explicit JacobiSvdPipeline(PipelineConfig config);
        /// Runs the whole stream; for each testcase writes U, Sigma (1 x n) and V.
        [[nodiscard]] PipelineReport run() const;

    private:
        PipelineConfig config_;
    };

    [[nodiscard]] PipelineReport run_pipeline(const PipelineConfig &config);
} // namespace jacobi::svd::pipeline
