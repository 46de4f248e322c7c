// Concurrency stress of the serving core (jsvd_server_*), built with the
// library's host code under ThreadSanitizer by tests/test_server_host.py.
// Runs where no GPU is present: every request fails fast with a CUDA error,
// which still exercises queues, admission, completion, polls, waits and
// destroy from many threads.  Prints one summary line per scenario.
// Usage: server_stress DIR (DIR receives the pipeline scenario's files).
#include <atomic>
#include <cstdio>
#include <thread>
#include <vector>

#include "io.hpp"
#include "jsvd.h"
#include "pipeline.hpp"

namespace
{
    // 4 submitters, 4 waiters that poll then wait, one stats reader.
    int mixed()
    {
        jsvd_server_options opt;
        jsvd_server_options_default(&opt);
        opt.small_workers = 2;
        opt.large_workers = 2;
        jsvd_server *s = nullptr;
        if (jsvd_server_create(&opt, &s) != JSVD_OK)
            return 1;
        std::vector<double> small(40 * 30, 1.0), large(300 * 260, 1.0);
        const int per = 200;
        std::vector<uint64_t> tickets(4 * per, 0);
        std::vector<std::atomic<int>> ready(4 * per);
        std::atomic<int> collected{0};
        std::vector<std::thread> th;
        for (int k = 0; k < 4; ++k)
            th.emplace_back([&, k] {
                for (int i = 0; i < per; ++i)
                {
                    const bool big = i % 7 == 0;
                    uint64_t t = 0;
                    jsvd_server_submit(s, big ? large.data() : small.data(), big ? 300 : 40, big ? 260 : 30, i % 2,
                                       &t);
                    tickets[k * per + i] = t;
                    ready[k * per + i].store(1, std::memory_order_release);
                }
            });
        for (int k = 0; k < 4; ++k)
            th.emplace_back([&, k] {
                std::vector<double> u(300 * 260), sg(260), v(260 * 260);
                for (int i = k; i < 4 * per; i += 4)
                {
                    while (!ready[i].load(std::memory_order_acquire))
                        std::this_thread::yield();
                    int done = 0, sw = 0;
                    double lat = 0;
                    jsvd_server_poll(s, tickets[i], &done);
                    jsvd_server_wait(s, tickets[i], u.data(), sg.data(), v.data(), &sw, &lat);
                    collected.fetch_add(1);
                }
            });
        th.emplace_back([&] {
            jsvd_server_stats st;
            for (int i = 0; i < 200; ++i)
                jsvd_server_get_stats(s, &st);
        });
        for (auto &t : th)
            t.join();
        jsvd_server_stats st;
        jsvd_server_get_stats(s, &st);
        jsvd_server_destroy(s);
        std::printf("mixed %d %llu %llu\n", collected.load(), st.submitted, st.completed + st.failed);
        return 0;
    }

    // destroy while a thread waits on the last of 300 queued requests
    int destroy_with_waiter()
    {
        for (int trial = 0; trial < 10; ++trial)
        {
            jsvd_server_options opt;
            jsvd_server_options_default(&opt);
            opt.small_workers = 1;
            opt.large_workers = 1;
            jsvd_server *s = nullptr;
            if (jsvd_server_create(&opt, &s) != JSVD_OK)
                return 1;
            std::vector<double> a(40 * 30, 1.0);
            std::vector<uint64_t> t(300);
            for (auto &x : t)
                jsvd_server_submit(s, a.data(), 40, 30, 0, &x);
            std::thread w([&] {
                std::vector<double> sg(30), v(900);
                (void)jsvd_server_wait(s, t.back(), nullptr, sg.data(), v.data(), nullptr, nullptr);
            });
            int done = 0;
            while (jsvd_server_poll(s, t.back(), &done) == JSVD_OK)  // until the waiter holds the ticket
                std::this_thread::yield();
            jsvd_server_destroy(s);
            w.join();
        }
        std::printf("destroy 10\n");
        return 0;
    }
    // the pipeline's reader and writer threads on its failure path: the
    // first collected result fails, the writer records it, the reader stops
    // and run_pipeline rethrows
    int pipeline_failure(const std::filesystem::path &dir)
    {
        using namespace jacobi::svd;
        const std::filesystem::path in = dir / "stress_in.mat";
        const std::filesystem::path out = dir / "stress_out.mat";
        std::vector<io::Matrix> mats;
        for (int i = 0; i < 60; ++i)
            mats.push_back(io::Matrix{20, 10, std::vector<double>(200, 1.0 + i)});
        io::write_mat_file(in, mats);
        int failures = 0;
        for (int trial = 0; trial < 20; ++trial)
        {
            pipeline::PipelineConfig cfg;
            cfg.input_path = in;
            cfg.output_path = out;
            try
            {
                (void)pipeline::run_pipeline(cfg);
            }
            catch (const std::exception &)
            {
                ++failures;
            }
        }
        std::filesystem::remove(in);
        std::filesystem::remove(out);
        std::printf("pipeline %d\n", failures);
        return 0;
    }
} // namespace

// argv[1]: a directory for the pipeline scenario's files
int main(int argc, char **argv)
{
    if (argc != 2)
        return 64;
    return mixed() | destroy_with_waiter() | pipeline_failure(argv[1]);
}
