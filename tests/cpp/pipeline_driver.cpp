// Test driver for the host-side pipeline extensions (include/pipeline_ext.hpp),
// built and run by tests/test_pipeline_host.py; no GPU needed.  Commands:
//   record-json   prints residual_record_json of a fixed record and of one
//                 with a NaN residual, one per line
//   report-path P sets the residual report path to P, prints what it reads
//                 back, clears it and prints the cleared value in brackets
//   last-run      prints the fields of last_run_service_stats (no run yet)
#include <cmath>
#include <iostream>
#include <limits>
#include <string>

#include "pipeline_ext.hpp"

using namespace jacobi::svd::pipeline;

int main(int argc, char **argv)
{
    if (argc < 2)
        return 64;
    const std::string cmd = argv[1];
    if (cmd == "record-json")
    {
        ResidualRecord r;
        r.index = 7;
        r.rows = 300;
        r.columns = 260;
        r.epsilon = 1e-14;
        r.max_sweeps = 128;
        r.sweeps = 13;
        r.rho_a = 3.0000000000000001e-15;
        r.rho_u = 1.25e-13;
        r.rho_v = 0.1;
        std::cout << residual_record_json(r) << '\n';
        r.rho_a = std::numeric_limits<double>::quiet_NaN();
        r.rho_u = -1.0;
        std::cout << residual_record_json(r) << '\n';
        return 0;
    }
    if (cmd == "report-path" && argc == 3)
    {
        set_residual_report(argv[2]);
        std::cout << residual_report().string() << '\n';
        set_residual_report({});
        std::cout << '[' << residual_report().string() << "]\n";
        return 0;
    }
    if (cmd == "last-run")
    {
        const RunServiceStats r = last_run_service_stats();
        std::cout << r.batches << ' ' << r.batched_testcases << ' ' << r.large_solves << ' ' << r.latency_p50_ms << ' '
                  << r.latency_p99_ms << ' ' << r.latency_mean_ms << ' ' << r.peak_device_bytes << '\n';
        return 0;
    }
    return 64;
}
