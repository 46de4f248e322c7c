// GPU driver for the reference-compatible C++ API (include/kernels.hpp and
// the jacobi_svd extension of include/kernels_ext.hpp), built and run by
// tests/test_cxx_api_gpu.py on a machine with a GPU.  Commands:
//   solve IN OUT EPS T SOLVER
//          IN: int64 rows, int64 columns, then rows*columns row-major
//          doubles; runs one_sided_jacobi_svd (SOLVER "reference") or
//          jacobi_svd with the named solver, and writes OUT: int32 sweeps,
//          then sigma (columns), U (rows*columns), V (columns*columns)
//   device-matrix
//          DeviceMatrix round trip, move construction and assignment, reset;
//          prints one "name value" line per check
//   auto-tune
//          auto_tune_layout_transpose_threshold with a short scan; prints the
//          report's fields
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <utility>
#include <vector>

#include "kernels_ext.hpp"

using namespace jacobi::svd;

namespace
{
    int solve(const char *in_path, const char *out_path, double eps, int threads, const std::string &solver)
    {
        std::ifstream in(in_path, std::ios::binary);
        std::int64_t dims[2] = {0, 0};
        in.read(reinterpret_cast<char *>(dims), sizeof(dims));
        std::vector<double> a(static_cast<std::size_t>(dims[0] * dims[1]));
        in.read(reinterpret_cast<char *>(a.data()), static_cast<std::streamsize>(a.size() * sizeof(double)));
        if (!in)
            return 65;
        JacobiSvdConfig cfg;
        cfg.epsilon = eps;
        cfg.threads_per_block = threads;
        JacobiSvdResult r;
        if (solver == "reference")
            r = one_sided_jacobi_svd(a, dims[0], dims[1], cfg);
        else
        {
            SvdSolver s = SvdSolver::plain;
            if (solver == "precond")
                s = SvdSolver::precond;
            else if (solver == "blockpair")
                s = SvdSolver::blockpair;
            else if (solver == "blocked")
                s = SvdSolver::blocked;
            else if (solver == "mixed")
                s = SvdSolver::mixed;
            else if (solver != "plain")
                return 64;
            r = jacobi_svd(a, dims[0], dims[1], cfg, s);
        }
        std::ofstream out(out_path, std::ios::binary);
        const std::int32_t sw = r.sweeps;
        out.write(reinterpret_cast<const char *>(&sw), sizeof(sw));
        for (const auto *vec : {&r.sigma, &r.u, &r.v})
            out.write(reinterpret_cast<const char *>(vec->data()),
                      static_cast<std::streamsize>(vec->size() * sizeof(double)));
        return out ? 0 : 66;
    }

    int device_matrix()
    {
        std::vector<double> host(12);
        for (std::size_t i = 0; i < host.size(); ++i)
            host[i] = 0.5 * static_cast<double>(i) - 2.0;
        DeviceMatrix d(3, 4);
        std::cout << "shape " << d.rows() << 'x' << d.columns() << ' ' << d.size() << ' ' << d.bytes() << '\n';
        d.copy_from_host(host);
        std::cout << "round_trip " << (d.copy_to_host() == host ? 1 : 0) << '\n';
        const double *p = d.data();
        DeviceMatrix moved(std::move(d));
        std::cout << "move_construct " << (moved.data() == p && d.data() == nullptr && d.size() == 0 ? 1 : 0)
                  << ' ' << (moved.copy_to_host() == host ? 1 : 0) << '\n';
        DeviceMatrix other(2, 2);
        other = std::move(moved);
        std::cout << "move_assign " << (other.data() == p && other.rows() == 3 ? 1 : 0) << ' '
                  << (other.copy_to_host() == host ? 1 : 0) << '\n';
        other.reset(5, 2);
        std::cout << "reset " << other.rows() << 'x' << other.columns() << ' ' << other.size() << '\n';
        std::vector<double> h2(10, 7.25);
        other.copy_from_host(h2);
        std::cout << "reset_round_trip " << (other.copy_to_host() == h2 ? 1 : 0) << '\n';
        try
        {
            other.copy_from_host(host);  // 12 values for a 5 x 2 matrix
            std::cout << "size_check none\n";
        }
        catch (const std::invalid_argument &e)
        {
            std::cout << "size_check " << e.what() << '\n';
        }
        return 0;
    }

    int auto_tune()
    {
        JacobiSvdConfig cfg;
        cfg.layout_transpose_benchmark_repetitions = 1;
        cfg.layout_transpose_benchmark_sweeps = 2;
        const LayoutTransposeAutoTuneReport r = auto_tune_layout_transpose_threshold(cfg);
        std::cout << "executed " << (r.executed ? 1 : 0) << '\n'
                  << "recommended_min_columns " << r.recommended_min_columns << '\n'
                  << "recommended_min_elements " << r.recommended_min_elements << '\n'
                  << "estimated_best_speedup " << r.estimated_best_speedup << '\n'
                  << "sample_count " << r.sample_count << '\n';
        return 0;
    }
} // namespace

int main(int argc, char **argv)
{
    if (argc < 2)
        return 64;
    const std::string cmd = argv[1];
    try
    {
        if (cmd == "solve" && argc == 7)
            return solve(argv[2], argv[3], std::stod(argv[4]), std::stoi(argv[5]), argv[6]);
        if (cmd == "device-matrix")
            return device_matrix();
        if (cmd == "auto-tune")
            return auto_tune();
    }
    catch (const std::exception &e)
    {
        std::cout << "exception " << e.what() << '\n';
        return 70;
    }
    return 64;
}
