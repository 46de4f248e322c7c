// jacobi-svd-b200: command-line driver with the option surface, defaults,
// output-path rules, reports and exit codes of the reference CLI
// (kleedaisuki/jacobi-svd-cuda src/main.cpp:877-1300): exit 0 on success,
// 2 on argument errors, 1 on execution errors.
#include <algorithm>
#include <cctype>
#include <chrono>
#include <cmath>
#include <filesystem>
#include <iomanip>
#include <iostream>
#include <limits>
#include <optional>
#include <stdexcept>
#include <string>
#include <string_view>
#include <vector>

#include "io.hpp"
#include "jsvd.h"
#include "kernels.hpp"
#include "pipeline.hpp"
#include "pipeline_ext.hpp"

namespace
{
    using jacobi::svd::LayoutTransposeMode;
    using jacobi::svd::pipeline::MatrixFileFormat;

    struct ArgError : std::runtime_error
    {
        using std::runtime_error::runtime_error;
    };

    struct Options
    {
        std::filesystem::path input, output;
        MatrixFileFormat input_format = MatrixFileFormat::auto_detect;
        MatrixFileFormat output_format = MatrixFileFormat::auto_detect;
        double epsilon = 1.0e-9;
        int max_sweeps = 128;
        int threads_per_block = 256;
        LayoutTransposeMode layout_mode = LayoutTransposeMode::auto_select;
        int layout_min_cols = 16;
        std::size_t layout_min_elems = 4096;
        bool layout_auto_tune = false;
        int layout_bench_reps = 2;
        int layout_bench_sweeps = 8;
        std::size_t queue_capacity = 4;
        bool force = false, dry_run = false, print_config = false, json = false, quiet = false;
        bool help = false, version = false;
        std::string solver = "plain";  // plain | precond | mixed
        std::filesystem::path residual_report;  // empty: off
        std::filesystem::path verify;           // empty: solve; else check this result file
    };

    struct Flag
    {
        const char *long_name;
        char short_name;
        bool takes_value;
        const char *hint;
        const char *help;
    };

    const std::vector<Flag> kFlags = {
        {"input", 'i', true, "PATH", "Input matrix stream file path."},
        {"output", 'o', true, "PATH", "Output matrix stream file path."},
        {"input-format", '\0', true, "FMT", "Input format: auto|mat|txt."},
        {"output-format", '\0', true, "FMT", "Output format: auto|mat|txt."},
        {"format", 'f', true, "FMT", "Set both input/output format: auto|mat|txt."},
        {"epsilon", 'e', true, "NUM", "Convergence epsilon (>0)."},
        {"max-sweeps", 's', true, "N", "Maximum sweep count (>0)."},
        {"threads-per-block", 't', true, "N", "Reduction width of the dot products (>0)."},
        {"layout-transpose-mode", '\0', true, "MODE", "Layout-transpose mode: auto|on|off."},
        {"layout-transpose-min-cols", '\0', true, "N", "Auto-mode threshold: minimum columns (>0)."},
        {"layout-transpose-min-elems", '\0', true, "N", "Auto-mode threshold: minimum elements (>0)."},
        {"layout-transpose-auto-tune", '\0', false, "", "Run the layout threshold scan before the pipeline."},
        {"layout-transpose-bench-reps", '\0', true, "N", "Auto-tune repetitions per scanned size (>0)."},
        {"layout-transpose-bench-sweeps", '\0', true, "N", "Auto-tune sweep cap per run (>0)."},
        {"queue-capacity", 'c', true, "N", "In-flight/reorder window size (>0)."},
        {"force", 'y', false, "", "Overwrite existing output file."},
        {"dry-run", '\0', false, "", "Validate arguments and print config only."},
        {"print-config", '\0', false, "", "Print effective config before execution."},
        {"json-report", '\0', false, "", "Print execution report in JSON."},
        {"quiet", 'q', false, "", "Suppress text report."},
        {"solver", '\0', true, "NAME", "Large-testcase solver: plain (bit-identical, default) | precond | mixed."},
        {"residual-report", '\0', true, "PATH",
         "Write each testcase's rows, columns, epsilon, sweeps, rho_A, rho_U, rho_V as a JSON line."},
        {"verify", '\0', true, "PATH",
         "Check the result file PATH (U, Sigma, V per testcase) against the input: print rho_A, rho_U, rho_V "
         "per testcase as JSON lines; nothing is solved."},
        {"help", 'h', false, "", "Show this help message."},
        {"version", 'v', false, "", "Show version information."},
    };

    std::string lower(std::string_view s)
    {
        std::string o(s);
        std::transform(o.begin(), o.end(), o.begin(), [](unsigned char c) { return (char)std::tolower(c); });
        return o;
    }

    MatrixFileFormat parse_format(std::string_view v, std::string_view name)
    {
        const std::string l = lower(v);
        if (l == "auto")
            return MatrixFileFormat::auto_detect;
        if (l == "mat")
            return MatrixFileFormat::mat;
        if (l == "txt")
            return MatrixFileFormat::txt;
        throw ArgError("Invalid value for --" + std::string(name) + ": expected auto|mat|txt.");
    }

    LayoutTransposeMode parse_layout(std::string_view v, std::string_view name)
    {
        const std::string l = lower(v);
        if (l == "auto")
            return LayoutTransposeMode::auto_select;
        if (l == "on")
            return LayoutTransposeMode::force_enable;
        if (l == "off")
            return LayoutTransposeMode::force_disable;
        throw ArgError("Invalid value for --" + std::string(name) + ": expected auto|on|off.");
    }

    long long parse_int(std::string_view v, std::string_view name, bool size_range)
    {
        const std::string t(v);
        std::size_t used = 0;
        long long x = 0;
        try
        {
            x = size_range ? (long long)std::stoull(t, &used, 10) : std::stoi(t, &used, 10);
        }
        catch (const std::exception &)
        {
            throw ArgError("Invalid integer value for --" + std::string(name) + ".");
        }
        if (used != t.size())
            throw ArgError("Invalid integer value for --" + std::string(name) + ".");
        if (x <= 0)
            throw ArgError("Option --" + std::string(name) + " must be positive.");
        return x;
    }

    double parse_double(std::string_view v, std::string_view name)
    {
        const std::string t(v);
        std::size_t used = 0;
        double x = 0.0;
        try
        {
            x = std::stod(t, &used);
        }
        catch (const std::exception &)
        {
            throw ArgError("Invalid floating-point value for --" + std::string(name) + ".");
        }
        if (used != t.size())
            throw ArgError("Invalid floating-point value for --" + std::string(name) + ".");
        if (!std::isfinite(x) || x <= 0.0)
            throw ArgError("Option --" + std::string(name) + " must be a positive finite number.");
        return x;
    }

    void apply(Options &o, const Flag &f, std::string_view v)
    {
        const std::string n = f.long_name;
        if (n == "input") o.input = std::string(v);
        else if (n == "output") o.output = std::string(v);
        else if (n == "input-format") o.input_format = parse_format(v, n);
        else if (n == "output-format") o.output_format = parse_format(v, n);
        else if (n == "format") o.input_format = o.output_format = parse_format(v, n);
        else if (n == "epsilon") o.epsilon = parse_double(v, n);
        else if (n == "max-sweeps") o.max_sweeps = (int)parse_int(v, n, false);
        else if (n == "threads-per-block") o.threads_per_block = (int)parse_int(v, n, false);
        else if (n == "layout-transpose-mode") o.layout_mode = parse_layout(v, n);
        else if (n == "layout-transpose-min-cols") o.layout_min_cols = (int)parse_int(v, n, false);
        else if (n == "layout-transpose-min-elems") o.layout_min_elems = (std::size_t)parse_int(v, n, true);
        else if (n == "layout-transpose-auto-tune") o.layout_auto_tune = true;
        else if (n == "layout-transpose-bench-reps") o.layout_bench_reps = (int)parse_int(v, n, false);
        else if (n == "layout-transpose-bench-sweeps") o.layout_bench_sweeps = (int)parse_int(v, n, false);
        else if (n == "queue-capacity") o.queue_capacity = (std::size_t)parse_int(v, n, true);
        else if (n == "force") o.force = true;
        else if (n == "dry-run") o.dry_run = true;
        else if (n == "print-config") o.print_config = true;
        else if (n == "json-report") o.json = true;
        else if (n == "quiet") o.quiet = true;
        else if (n == "solver")
        {
            const std::string l = lower(v);
            if (l != "plain" && l != "precond" && l != "mixed")
                throw ArgError("Invalid value for --solver: expected plain|precond|mixed.");
            o.solver = l;
        }
        else if (n == "residual-report") o.residual_report = std::string(v);
        else if (n == "verify") o.verify = std::string(v);
        else if (n == "help") o.help = true;
        else if (n == "version") o.version = true;
    }

    std::optional<MatrixFileFormat> ext_format(const std::filesystem::path &p)
    {
        const std::string e = lower(p.extension().string());
        if (e == ".mat")
            return MatrixFileFormat::mat;
        if (e == ".txt")
            return MatrixFileFormat::txt;
        return std::nullopt;
    }

    const char *ext_for(MatrixFileFormat f) { return f == MatrixFileFormat::txt ? ".txt" : ".mat"; }

    const char *format_name(MatrixFileFormat f)
    {
        return f == MatrixFileFormat::mat ? "mat" : (f == MatrixFileFormat::txt ? "txt" : "auto");
    }

    const char *layout_name(LayoutTransposeMode m)
    {
        return m == LayoutTransposeMode::force_enable ? "on"
                                                      : (m == LayoutTransposeMode::force_disable ? "off" : "auto");
    }

    // Output-path and format defaults of the reference (src/main.cpp:682-779).
    void normalize(Options &o)
    {
        if (o.input.empty())
            throw ArgError("Missing input file. Use --input <path>.");
        const auto in_ext = ext_format(o.input);
        if (o.input_format == MatrixFileFormat::auto_detect && !in_ext)
            throw ArgError("Cannot infer input format from extension. Use --input-format {mat|txt}.");
        if (o.output.empty())
        {
            MatrixFileFormat f = o.output_format;
            if (f == MatrixFileFormat::auto_detect)
            {
                f = o.input_format != MatrixFileFormat::auto_detect ? o.input_format
                                                                      : (in_ext ? *in_ext : MatrixFileFormat::mat);
                o.output_format = f;
            }
            std::string stem = o.input.stem().string();
            if (stem.empty())
                stem = "result";
            o.output = o.input.parent_path() / (stem + ".svd" + ext_for(f));
        }
        if (o.output_format == MatrixFileFormat::auto_detect && !ext_format(o.output))
        {
            MatrixFileFormat fb = o.input_format != MatrixFileFormat::auto_detect
                                      ? o.input_format
                                      : (in_ext ? *in_ext : MatrixFileFormat::mat);
            if (o.output.extension().empty())
                o.output += ext_for(fb);
            o.output_format = fb;
        }
    }

    std::filesystem::path comparable(const std::filesystem::path &p)
    {
        std::error_code ec;
        auto a = std::filesystem::absolute(p, ec);
        return ec ? p.lexically_normal() : a.lexically_normal();
    }

    void validate(const Options &o)
    {
        if (!std::filesystem::exists(o.input))
            throw ArgError("Input file does not exist: " + o.input.string());
        if (std::filesystem::is_directory(o.input))
            throw ArgError("Input path is a directory, expected a file: " + o.input.string());
        if (std::filesystem::is_directory(o.output))
            throw ArgError("Output path points to a directory: " + o.output.string());
        if (comparable(o.input) == comparable(o.output))
            throw ArgError("Input and output paths must be different files.");
        if (!o.residual_report.empty() && (comparable(o.residual_report) == comparable(o.input) ||
                                           comparable(o.residual_report) == comparable(o.output)))
            throw ArgError("--residual-report must name a file other than the input and output.");
        if (std::filesystem::exists(o.output) && !o.force)
            throw ArgError("Output file already exists. Use --force to overwrite: " + o.output.string());
    }

    Options parse(int argc, char **argv)
    {
        Options o;
        std::vector<std::string> positional;
        auto need_value = [&](const Flag &f, int &i) -> std::string {
            if (i + 1 >= argc)
                throw ArgError("Missing value for --" + std::string(f.long_name) + ".");
            return argv[++i];
        };
        for (int i = 1; i < argc; ++i)
        {
            const std::string tok = argv[i] ? argv[i] : "";
            if (tok.empty())
                continue;
            if (tok == "--")
            {
                for (++i; i < argc; ++i)
                    positional.emplace_back(argv[i]);
                break;
            }
            if (tok.rfind("--", 0) == 0)
            {
                const std::string body = tok.substr(2);
                const auto eq = body.find('=');
                const std::string name = body.substr(0, eq);
                auto it = std::find_if(kFlags.begin(), kFlags.end(), [&](const Flag &f) { return name == f.long_name; });
                if (it == kFlags.end())
                    throw ArgError("Unknown option: --" + name);
                if (it->takes_value)
                    apply(o, *it, eq != std::string::npos ? body.substr(eq + 1) : need_value(*it, i));
                else if (eq != std::string::npos)
                    throw ArgError("Option --" + std::string(it->long_name) + " does not take a value.");
                else
                    apply(o, *it, "");
                continue;
            }
            if (tok.size() > 1 && tok[0] == '-')
            {
                for (std::size_t k = 1; k < tok.size(); ++k)
                {
                    auto it = std::find_if(kFlags.begin(), kFlags.end(),
                                           [&](const Flag &f) { return f.short_name == tok[k]; });
                    if (it == kFlags.end())
                        throw ArgError(std::string("Unknown short option: -") + tok[k]);
                    if (!it->takes_value)
                    {
                        apply(o, *it, "");
                        continue;
                    }
                    apply(o, *it, k + 1 < tok.size() ? tok.substr(k + 1) : need_value(*it, i));
                    break;
                }
                continue;
            }
            positional.push_back(tok);
        }
        std::size_t p = 0;
        if (o.input.empty() && p < positional.size())
            o.input = positional[p++];
        if (o.output.empty() && p < positional.size())
            o.output = positional[p++];
        if (p < positional.size())
            throw ArgError("Unexpected positional argument: " + positional[p]);
        if (!o.verify.empty() && !o.help && !o.version)
        {
            if (o.input.empty())
                throw ArgError("Missing input file. Use --input <path>.");
            for (const auto &f : {o.input, o.verify})
                if (!std::filesystem::is_regular_file(f))
                    throw ArgError("Input file does not exist: " + f.string());
        }
        else if (!o.help && !o.version)
        {
            normalize(o);
            validate(o);
        }
        return o;
    }

    void json_number(std::ostream &os, double x)
    {
        if (std::isfinite(x))
            os << x;
        else
            os << "null";
    }

    // --verify: the validation metrics of every testcase of the input against
    // the result file's U, Sigma (1 x n), V records, without solving.
    int run_verify(const Options &o)
    {
        using namespace jacobi::svd;
        auto read_file = [](const std::filesystem::path &p, MatrixFileFormat f) {
            if (f == MatrixFileFormat::auto_detect)
            {
                const auto e = ext_format(p);
                if (!e)
                    throw ArgError("Cannot infer format from extension: " + p.string() + ".");
                f = *e;
            }
            return f == MatrixFileFormat::txt ? io::read_txt_file(p) : io::read_mat_file(p);
        };
        const std::vector<io::Matrix> in = read_file(o.input, o.input_format);
        const std::vector<io::Matrix> res = read_file(o.verify, o.output_format);
        if (res.size() != 3 * in.size())
            throw std::runtime_error("Result file holds " + std::to_string(res.size()) +
                                     " matrices; expected 3 (U, Sigma, V) for each of the " +
                                     std::to_string(in.size()) + " testcases.");
        std::cout << std::setprecision(std::numeric_limits<double>::max_digits10);
        for (std::size_t k = 0; k < in.size(); ++k)
        {
            const io::Matrix &a = in[k], &u = res[3 * k], &sg = res[3 * k + 1], &v = res[3 * k + 2];
            const std::size_t m = a.rows, n = a.columns;
            if (u.rows != m || u.columns != n || sg.rows != 1 || sg.columns != n || v.rows != n || v.columns != n)
                throw std::runtime_error("Testcase[" + std::to_string(k) + "] result shapes do not match the input.");
            jsvd_residual_report r{};
            if (jsvd_residuals(a.values.data(), u.values.data(), sg.values.data(), v.values.data(), m, n, &r) !=
                JSVD_OK)
            {
                char buf[512];
                jsvd_last_error(buf, sizeof(buf));
                throw std::runtime_error("Testcase[" + std::to_string(k) + "]: " + buf);
            }
            std::cout << "{\"index\": " << k << ", \"rows\": " << m << ", \"columns\": " << n << ", \"rho_A\": ";
            json_number(std::cout, r.rho_a);
            std::cout << ", \"rho_U\": ";
            json_number(std::cout, r.rho_u);
            std::cout << ", \"rho_V\": ";
            json_number(std::cout, r.rho_v);
            std::cout << ", \"sigma_max\": ";
            json_number(std::cout, r.sigma_max);
            std::cout << "}\n";
        }
        return 0;
    }

    void print_help(const std::string &exe)
    {
        std::cout << "Jacobi SVD (B200) CLI\n\nUsage:\n  " << exe << " [OPTIONS] <input> [output]\n\nOptions:\n";
        for (const Flag &f : kFlags)
        {
            std::string names = f.short_name ? std::string("-") + f.short_name + ", " : "    ";
            names += std::string("--") + f.long_name;
            if (f.takes_value)
                names += std::string(" ") + f.hint;
            std::cout << "  " << names << std::string(names.size() < 32 ? 32 - names.size() : 1, ' ') << f.help
                      << '\n';
        }
        std::cout << "\nNotes:\n  - When [output] is omitted, default output is <input-stem>.svd.{mat|txt}.\n"
                     "  - Existing output file requires --force to overwrite.\n";
    }

    void print_config(const Options &o)
    {
        std::cout << "input           : " << o.input.string() << '\n'
                  << "output          : " << o.output.string() << '\n'
                  << "input-format    : " << format_name(o.input_format) << '\n'
                  << "output-format   : " << format_name(o.output_format) << '\n'
                  << "epsilon         : " << o.epsilon << '\n'
                  << "max-sweeps      : " << o.max_sweeps << '\n'
                  << "threads-per-blk : " << o.threads_per_block << '\n'
                  << "layout-mode     : " << layout_name(o.layout_mode) << '\n'
                  << "layout-min-cols : " << o.layout_min_cols << '\n'
                  << "layout-min-elem : " << o.layout_min_elems << '\n'
                  << "layout-auto-tune: " << (o.layout_auto_tune ? "true" : "false") << '\n'
                  << "layout-bench-rep: " << o.layout_bench_reps << '\n'
                  << "layout-bench-swp: " << o.layout_bench_sweeps << '\n'
                  << "queue-capacity  : " << o.queue_capacity << '\n'
                  << "force-overwrite : " << (o.force ? "true" : "false") << '\n'
                  << "solver          : " << o.solver << '\n'
                  << "residual-report : " << (o.residual_report.empty() ? "off" : o.residual_report.string())
                  << '\n';
    }
} // namespace

int main(int argc, char **argv)
{
    try
    {
        const std::string exe =
            argc > 0 && argv[0] ? std::filesystem::path(argv[0]).filename().string() : "jacobi-svd-b200";
        Options o = parse(argc, argv);
        if (o.help)
        {
            print_help(exe);
            return 0;
        }
        if (o.version)
        {
            std::cout << "jacobi-svd-b200 CLI v0.1.0 (sm_100a)\n";
            return 0;
        }
        if (!o.verify.empty())
            return run_verify(o);
        if (o.dry_run)
        {
            std::cout << "Dry run: pipeline was not executed.\n";
            print_config(o);
            return 0;
        }
        if (o.print_config)
        {
            std::cout << "Effective configuration:\n";
            print_config(o);
            std::cout << '\n';
        }
        jacobi::svd::pipeline::set_residual_report(o.residual_report);
        using jacobi::svd::pipeline::LargeSolver;
        jacobi::svd::pipeline::set_large_solver(o.solver == "precond" ? LargeSolver::precond
                                                : o.solver == "mixed" ? LargeSolver::mixed
                                                                      : LargeSolver::plain);
        jacobi::svd::pipeline::PipelineConfig cfg;
        cfg.input_path = o.input;
        cfg.output_path = o.output;
        cfg.input_format = o.input_format;
        cfg.output_format = o.output_format;
        cfg.max_queued_results = o.queue_capacity;
        cfg.kernel_config = jacobi::svd::JacobiSvdConfig{
            .epsilon = o.epsilon,
            .max_sweeps = o.max_sweeps,
            .threads_per_block = o.threads_per_block,
            .layout_transpose_mode = o.layout_mode,
            .layout_transpose_min_columns = o.layout_min_cols,
            .layout_transpose_min_elements = o.layout_min_elems,
            .layout_transpose_auto_tune = o.layout_auto_tune,
            .layout_transpose_benchmark_repetitions = o.layout_bench_reps,
            .layout_transpose_benchmark_sweeps = o.layout_bench_sweeps,
        };
        const auto t0 = std::chrono::steady_clock::now();
        const auto report = jacobi::svd::pipeline::run_pipeline(cfg);
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (!o.quiet)
        {
            std::cout << "Pipeline completed.\n"
                      << "testcases       : " << report.testcase_count << '\n'
                      << "emitted-matrices: " << report.emitted_matrix_count << '\n'
                      << "total-sweeps    : " << report.total_sweeps << '\n'
                      << "layout-mode     : " << layout_name(report.layout_transpose_mode) << '\n'
                      << "layout-min-cols : " << report.layout_transpose_min_columns << '\n'
                      << "layout-min-elem : " << report.layout_transpose_min_elements << '\n'
                      << "layout-auto-tune: " << (report.layout_transpose_auto_tuned ? "true" : "false") << '\n'
                      << "layout-best-spd : " << std::fixed << std::setprecision(3)
                      << report.layout_transpose_estimated_best_speedup << '\n'
                      << "elapsed-ms      : " << std::fixed << std::setprecision(3) << ms << '\n';
        }
        if (o.json)
        {
            std::cout << "{\n  \"testcase_count\": " << report.testcase_count << ",\n  \"emitted_matrix_count\": "
                      << report.emitted_matrix_count << ",\n  \"total_sweeps\": " << report.total_sweeps
                      << ",\n  \"layout_transpose_mode\": \"" << layout_name(report.layout_transpose_mode)
                      << "\",\n  \"layout_transpose_min_columns\": " << report.layout_transpose_min_columns
                      << ",\n  \"layout_transpose_min_elements\": " << report.layout_transpose_min_elements
                      << ",\n  \"layout_transpose_auto_tuned\": "
                      << (report.layout_transpose_auto_tuned ? "true" : "false")
                      << ",\n  \"layout_transpose_estimated_best_speedup\": " << std::fixed << std::setprecision(3)
                      << report.layout_transpose_estimated_best_speedup << ",\n  \"elapsed_ms\": " << std::fixed
                      << std::setprecision(3) << ms;
            // serving-core figures of this run (no counterpart in the reference's report)
            const auto svc = jacobi::svd::pipeline::last_run_service_stats();
            const double rate = ms > 0.0 ? 1e3 * (double)report.testcase_count / ms : 0.0;
            std::cout << ",\n  \"testcases_per_s\": " << std::setprecision(3) << rate
                      << ",\n  \"latency_p50_ms\": " << svc.latency_p50_ms
                      << ",\n  \"latency_p99_ms\": " << svc.latency_p99_ms
                      << ",\n  \"latency_mean_ms\": " << svc.latency_mean_ms
                      << ",\n  \"batches\": " << svc.batches << ",\n  \"batched_testcases\": "
                      << svc.batched_testcases << ",\n  \"large_solves\": " << svc.large_solves
                      << ",\n  \"peak_device_bytes\": " << svc.peak_device_bytes << "\n}\n";
        }
        return 0;
    }
    catch (const ArgError &e)
    {
        std::cerr << "Argument error: " << e.what() << '\n' << "Use --help for usage.\n";
        return 2;
    }
    catch (const std::exception &e)
    {
        std::cerr << "Execution failed: " << e.what() << '\n';
        return 1;
    }
}
