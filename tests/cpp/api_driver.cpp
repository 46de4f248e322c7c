// Test driver for the jacobi::svd C++ extensions (include/kernels_ext.hpp),
// built and run by tests/test_cxx_api_host.py; no GPU needed.  Commands:
//   validate         calls jacobi_svd with each solver on invalid requests and
//                    prints the exception type and message of each
//   residuals FILE   reads rows, columns, then A, U, sigma, V (whitespace-
//                    separated doubles) from FILE and prints rho_a rho_u rho_v
//   bad-result       prints the message of residuals() on mismatched buffers
//   device-matrix    prints the messages of DeviceMatrix's argument checks
//                    (zero dimensions; a default-constructed matrix given data)
//   cuda-error       solves a valid 4 x 3 matrix with every solver and prints
//                    the exception type and message of each (for a machine
//                    without a GPU, where the first CUDA call fails)
#include <fstream>
#include <iomanip>
#include <iostream>
#include <limits>
#include <stdexcept>
#include <string>
#include <vector>

#include "kernels_ext.hpp"

using namespace jacobi::svd;

namespace
{
    const char *name(SvdSolver s)
    {
        switch (s)
        {
        case SvdSolver::plain:
            return "plain";
        case SvdSolver::precond:
            return "precond";
        case SvdSolver::blockpair:
            return "blockpair";
        default:
            return "blocked";
        }
    }

    void attempt(SvdSolver s, std::span<const double> a, std::size_t m, std::size_t n, const JacobiSvdConfig &cfg)
    {
        try
        {
            (void)jacobi_svd(a, m, n, cfg, s);
            std::cout << name(s) << " ok\n";
        }
        catch (const std::invalid_argument &e)
        {
            std::cout << name(s) << " invalid_argument " << e.what() << '\n';
        }
        catch (const std::exception &e)
        {
            std::cout << name(s) << " other " << e.what() << '\n';
        }
    }
} // namespace

int main(int argc, char **argv)
{
    if (argc < 2)
        return 64;
    const std::string cmd = argv[1];
    if (cmd == "validate")
    {
        std::vector<double> a(12, 1.0);
        for (SvdSolver s : {SvdSolver::plain, SvdSolver::precond, SvdSolver::blockpair, SvdSolver::blocked})
        {
            attempt(s, a, 3, 4, {});  // rows < columns
            attempt(s, a, 4, 4, {});  // buffer holds 12 values, not 16
            JacobiSvdConfig bad;
            bad.epsilon = 0.0;
            attempt(s, a, 4, 3, bad);
        }
        return 0;
    }
    if (cmd == "residuals" && argc == 3)
    {
        std::ifstream in(argv[2]);
        std::size_t m = 0, n = 0;
        in >> m >> n;
        std::vector<double> a(m * n);
        JacobiSvdResult r;
        r.rows = m;
        r.columns = n;
        r.u.resize(m * n);
        r.sigma.resize(n);
        r.v.resize(n * n);
        for (auto *vec : {&a, &r.u, &r.sigma, &r.v})
            for (double &x : *vec)
                in >> x;
        if (!in)
            return 65;
        const SvdResiduals res = residuals(a, r);
        std::cout << std::setprecision(std::numeric_limits<double>::max_digits10) << res.rho_a << ' ' << res.rho_u
                  << ' ' << res.rho_v << '\n';
        return 0;
    }
    if (cmd == "device-matrix")
    {
        for (auto [r, c] : {std::pair<std::size_t, std::size_t>{0, 3}, {3, 0}})
        {
            try
            {
                DeviceMatrix d(r, c);
                std::cout << "constructed\n";
            }
            catch (const std::invalid_argument &e)
            {
                std::cout << e.what() << '\n';
            }
        }
        try
        {
            DeviceMatrix d;  // 0 x 0, no allocation
            const std::vector<double> host(6, 1.0);
            d.copy_from_host(host);
            std::cout << "copied\n";
        }
        catch (const std::invalid_argument &e)
        {
            std::cout << e.what() << '\n';
        }
        return 0;
    }
    if (cmd == "cuda-error")
    {
        const std::vector<double> a = {4, 1, 0, 1, 3, 1, 0, 1, 2, 1, 1, 1};
        for (SvdSolver s : {SvdSolver::plain, SvdSolver::precond, SvdSolver::blockpair, SvdSolver::blocked})
        {
            try
            {
                (void)jacobi_svd(a, 4, 3, {}, s);
                std::cout << name(s) << " ok\n";
            }
            catch (const CudaError &e)
            {
                std::cout << name(s) << " CudaError " << e.what() << '\n';
            }
            catch (const std::exception &e)
            {
                std::cout << name(s) << " other " << e.what() << '\n';
            }
        }
        return 0;
    }
    if (cmd == "bad-result")
    {
        JacobiSvdResult r;
        r.rows = 4;
        r.columns = 3;
        r.u.resize(12);
        r.sigma.resize(3);
        r.v.resize(8);
        std::vector<double> a(12);
        try
        {
            (void)residuals(a, r);
        }
        catch (const std::invalid_argument &e)
        {
            std::cout << e.what() << '\n';
        }
        return 0;
    }
    return 64;
}
