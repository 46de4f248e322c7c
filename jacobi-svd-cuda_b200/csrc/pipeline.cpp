// jacobi::svd::pipeline implementation (include/pipeline.hpp).
//
// Same contract as kleedaisuki/jacobi-svd-cuda src/pipeline.cpp:754-863:
// read testcases (*.mat through MatDispatchReader, *.txt through the text
// policy), solve each, write U, Sigma (1 x n), V per testcase in input order,
// report counts and sweeps.  The execution is different: testcases go to the
// serving core (jsvd_server_*), which batches the small ones into persistent
// launches and overlaps the large ones on worker streams; a writer thread
// collects tickets in submission order (the reorder buffer of the reference's
// FutureQueueOutputStage, src/pipeline.cpp:400-656).
#include "pipeline.hpp"

#include <algorithm>
#include <atomic>
#include <cctype>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <exception>
#include <fstream>
#include <iomanip>
#include <limits>
#include <locale>
#include <memory>
#include <mutex>
#include <sstream>
#include <stdexcept>
#include <string>
#include <thread>
#include <utility>
#include <vector>

#include "io.hpp"
#include "jsvd.h"
#include "pipeline_ext.hpp"

namespace jacobi::svd::pipeline
{
    namespace
    {
        // In-flight window of the reader: testcases submitted but not yet
        // written (bounded in count and in host bytes held by the server).
        constexpr std::size_t kMaxInFlight = 8192;
        constexpr std::size_t kMaxInFlightBytes = std::size_t(4) << 30;

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

        MatrixFileFormat resolve(MatrixFileFormat requested, const std::filesystem::path &path)
        {
            if (requested != MatrixFileFormat::auto_detect)
                return requested;
            std::string ext = path.extension().string();
            std::transform(ext.begin(), ext.end(), ext.begin(),
                           [](unsigned char c) { return static_cast<char>(std::tolower(c)); });
            if (ext == ".mat")
                return MatrixFileFormat::mat;
            if (ext == ".txt")
                return MatrixFileFormat::txt;
            throw std::invalid_argument("Cannot auto-detect file format for path: " + path.string());
        }

        void validate_testcase(const io::Matrix &m, std::size_t index)
        {
            if (m.rows == 0 || m.columns == 0)
                throw std::invalid_argument("Testcase[" + std::to_string(index) + "] has zero dimension.");
            if (m.columns != 0 && m.rows > std::numeric_limits<std::size_t>::max() / m.columns)
                throw std::overflow_error("Matrix element count overflow.");
            if (m.values.size() != m.rows * m.columns)
                throw std::invalid_argument("Testcase[" + std::to_string(index) +
                                            "] payload size does not match rows*columns.");
        }

        jsvd_config to_c(const JacobiSvdConfig &c)
        {
            jsvd_config out{};
            jsvd_config_default(&out);
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

        // Writes U, Sigma, V of each testcase in order, in either format.
        class OrderedSink
        {
        public:
            OrderedSink(const std::filesystem::path &path, MatrixFileFormat fmt) : fmt_(fmt)
            {
                if (fmt_ == MatrixFileFormat::mat)
                    mat_ = std::make_unique<io::MatOutputStream>(path);
                else
                    txt_ = std::make_unique<io::TxtOutputStream>(path);
            }
            void write(const io::Matrix &m)
            {
                if (mat_)
                    mat_->write_one(m);
                else
                    txt_->write_one(m);
            }
            void flush()
            {
                if (mat_)
                    mat_->flush();
                else
                    txt_->flush();
            }

        private:
            MatrixFileFormat fmt_;
            std::unique_ptr<io::MatOutputStream> mat_;
            std::unique_ptr<io::TxtOutputStream> txt_;
        };

        struct Pending
        {
            std::uint64_t ticket;
            std::size_t rows, columns, bytes;
            std::shared_ptr<const std::vector<double>> input; ///< kept only for the residual report
        };

        struct ServerHandle
        {
            jsvd_server *s = nullptr;
            ~ServerHandle()
            {
                if (s)
                    jsvd_server_destroy(s);
            }
        };
    } // namespace

    namespace
    {
        std::atomic<int> g_large_solver{0};
        std::mutex g_report_mu;
        std::filesystem::path g_report_path;
        RunServiceStats g_last_run; // guarded by g_report_mu

        void json_number(std::ostream &os, double x)
        {
            if (std::isfinite(x))
                os << x;
            else
                os << "null";
        }
    } // namespace

    void set_residual_report(const std::filesystem::path &path)
    {
        std::lock_guard<std::mutex> lk(g_report_mu);
        g_report_path = path;
    }

    std::filesystem::path residual_report()
    {
        std::lock_guard<std::mutex> lk(g_report_mu);
        return g_report_path;
    }

    RunServiceStats last_run_service_stats()
    {
        std::lock_guard<std::mutex> lk(g_report_mu);
        return g_last_run;
    }

    std::string residual_record_json(const ResidualRecord &r)
    {
        std::ostringstream os;
        os.imbue(std::locale::classic());
        os << std::setprecision(std::numeric_limits<double>::max_digits10);
        os << "{\"index\": " << r.index << ", \"rows\": " << r.rows << ", \"columns\": " << r.columns
           << ", \"epsilon\": ";
        json_number(os, r.epsilon);
        os << ", \"max_sweeps\": " << r.max_sweeps << ", \"sweeps\": " << r.sweeps << ", \"rho_A\": ";
        json_number(os, r.rho_a);
        os << ", \"rho_U\": ";
        json_number(os, r.rho_u);
        os << ", \"rho_V\": ";
        json_number(os, r.rho_v);
        os << '}';
        return os.str();
    }

    void set_large_solver(LargeSolver solver) noexcept
    {
        g_large_solver.store(solver == LargeSolver::precond ? 1 : solver == LargeSolver::mixed ? 2 : 0);
    }

    LargeSolver large_solver() noexcept
    {
        const int s = g_large_solver.load();
        return s == 1 ? LargeSolver::precond : s == 2 ? LargeSolver::mixed : LargeSolver::plain;
    }

    JacobiSvdPipeline::JacobiSvdPipeline(PipelineConfig config) : config_(std::move(config)) {}

    PipelineReport JacobiSvdPipeline::run() const
    {
        if (config_.input_path.empty())
            throw std::invalid_argument("Pipeline input path is empty.");
        if (config_.output_path.empty())
            throw std::invalid_argument("Pipeline output path is empty.");
        const MatrixFileFormat in_fmt = resolve(config_.input_format, config_.input_path);
        const MatrixFileFormat out_fmt = resolve(config_.output_format, config_.output_path);
        const std::filesystem::path parent = config_.output_path.parent_path();
        if (!parent.empty())
            std::filesystem::create_directories(parent);

        JacobiSvdConfig kernel = config_.kernel_config;
        LayoutTransposeAutoTuneReport tuning{};
        if (kernel.layout_transpose_auto_tune)
        {
            tuning = auto_tune_layout_transpose_threshold(kernel);
            kernel.layout_transpose_min_columns = tuning.recommended_min_columns;
            kernel.layout_transpose_min_elements = tuning.recommended_min_elements;
        }
        // Settings errors surface before any file is written, as in the reference.
        if (!(kernel.epsilon > 0.0))
            throw std::invalid_argument("epsilon must be positive.");
        if (kernel.max_sweeps <= 0)
            throw std::invalid_argument("max_sweeps must be positive.");

        jsvd_server_options opt;
        jsvd_server_options_default(&opt);
        opt.cfg = to_c(kernel);
        opt.large_path = static_cast<int>(g_large_solver.load());
        ServerHandle server;
        if (const int rc = jsvd_server_create(&opt, &server.s); rc != JSVD_OK)
            rethrow_status(rc);

        OrderedSink sink(config_.output_path, out_fmt);
        const std::filesystem::path report_path = residual_report();
        const bool reporting = !report_path.empty();
        std::ofstream report_out;
        if (reporting)
        {
            report_out.open(report_path, std::ios::out | std::ios::trunc);
            if (!report_out)
                throw std::runtime_error("Cannot open residual report file: " + report_path.string());
        }
        std::mutex mu;
        std::condition_variable cv;
        std::deque<Pending> queue;
        std::size_t queued_bytes = 0;
        bool reader_done = false;
        std::exception_ptr writer_error;
        std::atomic<std::size_t> total_sweeps{0};
        std::size_t written = 0;

        std::thread writer([&] {
            try
            {
                for (std::size_t index = 0;; ++index)
                {
                    Pending p;
                    {
                        std::unique_lock<std::mutex> lk(mu);
                        cv.wait(lk, [&] { return !queue.empty() || reader_done; });
                        if (queue.empty())
                            return;
                        p = queue.front();
                    }
                    io::Matrix u{p.rows, p.columns, std::vector<double>(p.rows * p.columns)};
                    io::Matrix s{1, p.columns, std::vector<double>(p.columns)};
                    io::Matrix v{p.columns, p.columns, std::vector<double>(p.columns * p.columns)};
                    int sweeps = 0;
                    const int rc = jsvd_server_wait(server.s, p.ticket, u.values.data(), s.values.data(),
                                                    v.values.data(), &sweeps, nullptr);
                    if (rc != JSVD_OK)
                        rethrow_status(rc);
                    sink.write(u);
                    sink.write(s);
                    sink.write(v);
                    total_sweeps.fetch_add(static_cast<std::size_t>(sweeps));
                    if (reporting)
                    {
                        jsvd_residual_report rr{};
                        if (const int rrc = jsvd_residuals(p.input->data(), u.values.data(), s.values.data(),
                                                           v.values.data(), p.rows, p.columns, &rr);
                            rrc != JSVD_OK)
                            rethrow_status(rrc);
                        ResidualRecord rec;
                        rec.index = index;
                        rec.rows = p.rows;
                        rec.columns = p.columns;
                        rec.epsilon = kernel.epsilon;
                        rec.max_sweeps = kernel.max_sweeps;
                        rec.sweeps = sweeps;
                        rec.rho_a = rr.rho_a;
                        rec.rho_u = rr.rho_u;
                        rec.rho_v = rr.rho_v;
                        report_out << residual_record_json(rec) << '\n';
                    }
                    {
                        std::lock_guard<std::mutex> lk(mu);
                        queue.pop_front();
                        queued_bytes -= p.bytes;
                        ++written;
                    }
                    cv.notify_all();
                }
            }
            catch (...)
            {
                std::lock_guard<std::mutex> lk(mu);
                writer_error = std::current_exception();
                cv.notify_all();
            }
        });

        std::size_t submitted = 0;
        std::exception_ptr reader_error;
        auto submit = [&](const io::Matrix &m) {
            validate_testcase(m, submitted);
            // the residual report keeps a copy of the input until its result is written
            const std::size_t bytes = sizeof(double) * m.values.size() * (reporting ? 2 : 1);
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] {
                    return writer_error != nullptr ||
                           (queue.size() < kMaxInFlight && (queue.empty() || queued_bytes + bytes <= kMaxInFlightBytes));
                });
                if (writer_error)
                    return false;
            }
            std::uint64_t ticket = 0;
            if (const int rc = jsvd_server_submit(server.s, m.values.data(), m.rows, m.columns, 1, &ticket);
                rc != JSVD_OK)
                rethrow_status(rc);
            std::shared_ptr<const std::vector<double>> input;
            if (reporting)
                input = std::make_shared<const std::vector<double>>(m.values);
            {
                std::lock_guard<std::mutex> lk(mu);
                queue.push_back({ticket, m.rows, m.columns, bytes, std::move(input)});
                queued_bytes += bytes;
            }
            cv.notify_all();
            ++submitted;
            return true;
        };
        try
        {
            if (in_fmt == MatrixFileFormat::mat)
            {
                io::MatDispatchReader reader(config_.input_path);
                io::MatDispatchTask task;
                while (reader.read_next(task))
                    if (!submit(io::decode_dispatch_task_matrix(task)))
                        break;
            }
            else
            {
                io::TxtInputStream reader(config_.input_path);
                io::Matrix m;
                while (reader.read_one(m))
                    if (!submit(m))
                        break;
            }
        }
        catch (...)
        {
            reader_error = std::current_exception();
        }
        {
            std::lock_guard<std::mutex> lk(mu);
            reader_done = true;
        }
        cv.notify_all();
        writer.join();
        if (reader_error)
            std::rethrow_exception(reader_error);
        if (writer_error)
            std::rethrow_exception(writer_error);
        sink.flush();
        if (reporting)
        {
            report_out.flush();
            if (!report_out)
                throw std::runtime_error("Failed to write residual report file: " + report_path.string());
        }
        jsvd_server_stats st{};
        if (jsvd_server_get_stats(server.s, &st) == JSVD_OK)
        {
            RunServiceStats run;
            run.batches = st.batches;
            run.batched_testcases = st.batched_requests;
            run.large_solves = st.large_solves;
            run.latency_p50_ms = st.p50_ms;
            run.latency_p99_ms = st.p99_ms;
            run.latency_mean_ms = st.mean_ms;
            run.peak_device_bytes = st.peak_device_bytes;
            std::lock_guard<std::mutex> lk(g_report_mu);
            g_last_run = run;
        }

        PipelineReport report;
        report.testcase_count = submitted;
        report.emitted_matrix_count = submitted * 3;
        report.total_sweeps = total_sweeps.load();
        report.layout_transpose_mode = kernel.layout_transpose_mode;
        report.layout_transpose_min_columns = kernel.layout_transpose_min_columns;
        report.layout_transpose_min_elements = kernel.layout_transpose_min_elements;
        report.layout_transpose_auto_tuned = tuning.executed;
        report.layout_transpose_estimated_best_speedup = tuning.estimated_best_speedup;
        return report;
    }

    PipelineReport run_pipeline(const PipelineConfig &config) { return JacobiSvdPipeline(config).run(); }
} // namespace jacobi::svd::pipeline
