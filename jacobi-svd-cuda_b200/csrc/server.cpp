// Serving core: continuous batching of SVD requests on one GPU.
//
// This is what the reference's pipeline does with a host thread pool calling
// one_sided_jacobi_svd per testcase (kleedaisuki/jacobi-svd-cuda
// src/pipeline.cpp:234-394, 754-863), reorganised for the device:
//   * submit() copies the request and queues it; nothing touches the GPU yet;
//   * admission reserves the request's device footprint against a memory
//     budget and waits while the budget is exhausted;
//   * "small" requests (the working copy of A fits a CTA's shared memory) are
//     batched at sweep granularity: a worker keeps every request it admitted
//     on the device (A and V stay resident), runs one sweep of all of them per
//     step (one CTA each), retires the ones whose sweep rotated nothing and,
//     before the next step, admits queued requests into the room they freed -
//     a request that arrives while others are on the GPU joins at the next
//     sweep, not after the whole batch; two such workers overlap on the device;
//   * "large" requests go to worker threads that each drive their own stream
//     (plain path, per-thread plan cache), so several large solves overlap;
//   * every path uses the plain path's arithmetic, so a request's result does
//     not depend on what else was in flight.
// Latency = completion - submission (host steady clock).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "batched.hpp"
#include "internal.hpp"
#include "jsvd.h"
#include "plain.hpp"

namespace jsvd {
namespace {

using Clock = std::chrono::steady_clock;

// A request may use the batched solver when A's FP64 working copy plus the
// round scratch fits one CTA's shared memory.
bool is_small(size_t m, size_t n) { return sizeof(double) * (m * n + 5 * (n / 2 + 2)) <= 200 * 1024; }

size_t small_footprint(size_t m, size_t n, bool want_u)
{
    // state (A, V) + the FP64 input + outputs (sigma, V, optional U)
    return sizeof(double) * (2 * m * n + n + 2 * n * n + (want_u ? m * n : 0));
}

size_t large_footprint(size_t m, size_t n, int path)
{
    // I/O buffers (A, U, sigma, V) + plan (A_w, V_w, sigma, schedule and
    // angles) + the preconditioned path's Q and seven n x n scratch matrices;
    // the mixed path adds its working set on the padded n x n factor (five
    // FP64 and four FP32 matrices)
    const size_t np = (n + 127) / 128 * 128;
    return sizeof(double) * (2 * m * n + n + n * n) + sizeof(double) * (m * n + n * n + n) + 24 * n * n +
           sizeof(double) * (m * n + 7 * n * n) + (path == 2 ? (5 * 8 + 4 * 4) * np * np : 0);
}

struct Request {
    uint64_t id = 0;
    size_t m = 0, n = 0;
    bool want_u = false, small = false;
    std::vector<double> a, u, sigma, v;
    int sweeps = 0;
    int status = JSVD_OK;
    std::string error;
    size_t footprint = 0;
    Clock::time_point t_submit, t_done;
    bool done = false;
    bool claimed = false;  // a wait() has taken this ticket
};

// Pinned host staging that grows and is reused by one worker.
struct Pinned {
    void *p = nullptr;
    size_t cap = 0;
    ~Pinned()
    {
        if (p) cudaFreeHost(p);
    }
    int ensure(size_t bytes)
    {
        if (bytes <= cap) return JSVD_OK;
        if (p) cudaFreeHost(p);
        p = nullptr;
        size_t c = std::max<size_t>(bytes, cap * 2);
        JSVD_CUDA_TRY(cudaMallocHost(&p, c));
        cap = c;
        return JSVD_OK;
    }
};

}  // namespace

class Server {
public:
    explicit Server(const jsvd_server_options &o) : opt_(o)
    {
        cudaGetDevice(&device_);
        try {
            for (int i = 0; i < opt_.small_workers; ++i) threads_.emplace_back([this] { small_loop(); });
            for (int i = 0; i < opt_.large_workers; ++i) threads_.emplace_back([this] { large_loop(); });
        } catch (...) {
            stop();  // the workers already started must be joined before the vector goes away
            throw;
        }
    }

    // Fails the requests still queued (their waiters wake with an error) and
    // returns once no thread is inside wait().
    ~Server()
    {
        stop();
        std::unique_lock<std::mutex> lk(mu_);
        cv_done_.wait(lk, [&] { return waiters_ == 0; });
    }

    int submit(const double *a, size_t m, size_t n, int want_u, uint64_t *ticket)
    {
        if (a == nullptr || ticket == nullptr) return invalid_argument("Request buffers must not be null.");
        if (m == 0 || n == 0) return invalid_argument("Input matrix shape must be non-zero.");
        if (m < n) return invalid_argument("One-sided Jacobi SVD requires rows >= columns in this implementation.");
        if (dims_out_of_range(m, n)) {
            set_last_error(JSVD_ERR_OVERFLOW, "Matrix dimensions exceed the supported range.");
            return JSVD_ERR_OVERFLOW;
        }
        auto r = std::make_unique<Request>();
        r->m = m;
        r->n = n;
        r->want_u = want_u != 0;
        // The batched solver reduces with T = 256; other widths take the plain path.
        r->small = is_small(m, n) && reduction_lanes(opt_.cfg.threads_per_block) == 256;
        r->footprint = r->small ? small_footprint(m, n, r->want_u) : large_footprint(m, n, opt_.large_path);
        if (r->footprint > opt_.device_budget_bytes) {
            set_last_error(JSVD_ERR_BUDGET, "Request needs " + std::to_string(r->footprint) +
                                                " bytes of device memory, more than the serving budget of " +
                                                std::to_string(opt_.device_budget_bytes) + ".");
            return JSVD_ERR_BUDGET;
        }
        r->a.assign(a, a + m * n);
        r->t_submit = Clock::now();
        std::lock_guard<std::mutex> lk(mu_);
        if (stopping_) {
            set_last_error(JSVD_ERR_RUNTIME, "The server is being destroyed.");
            return JSVD_ERR_RUNTIME;
        }
        r->id = next_id_++;
        *ticket = r->id;
        Request *raw = r.get();
        requests_.emplace(r->id, std::move(r));
        (raw->small ? small_q_ : large_q_).push_back(raw);
        ++submitted_;
        cv_work_.notify_all();
        return JSVD_OK;
    }

    int wait(uint64_t ticket, double *u, double *sigma, double *v, int *sweeps, double *latency_ms)
    {
        std::unique_ptr<Request> r;
        {
            std::unique_lock<std::mutex> lk(mu_);
            auto it = requests_.find(ticket);
            if (it == requests_.end() || it->second->claimed)
                return invalid_argument("Unknown or already collected ticket.");
            Request *raw = it->second.get();
            raw->claimed = true;
            ++waiters_;
            // The wait releases the lock: a submit() may rehash the map, so the
            // iterator is looked up again afterwards (the element itself stays put).
            cv_done_.wait(lk, [&] { return raw->done; });
            it = requests_.find(ticket);
            r = std::move(it->second);
            requests_.erase(it);
            --waiters_;
            // Under the lock: a destructor waiting for the last waiter cannot
            // proceed before this scope ends, and after it this thread only
            // touches its own request.
            cv_done_.notify_all();
        }
        if (r->status != JSVD_OK) {
            set_last_error(r->status, r->error);
            return r->status;
        }
        if (u && r->want_u) std::memcpy(u, r->u.data(), sizeof(double) * r->m * r->n);
        if (sigma) std::memcpy(sigma, r->sigma.data(), sizeof(double) * r->n);
        if (v) std::memcpy(v, r->v.data(), sizeof(double) * r->n * r->n);
        if (sweeps) *sweeps = r->sweeps;
        if (latency_ms) *latency_ms = std::chrono::duration<double, std::milli>(r->t_done - r->t_submit).count();
        return JSVD_OK;
    }

    int poll(uint64_t ticket, int *done)
    {
        if (done == nullptr) return invalid_argument("done must not be null.");
        std::lock_guard<std::mutex> lk(mu_);
        auto it = requests_.find(ticket);
        if (it == requests_.end() || it->second->claimed)
            return invalid_argument("Unknown or already collected ticket.");
        *done = it->second->done ? 1 : 0;
        return JSVD_OK;
    }

    void stats(jsvd_server_stats *s)
    {
        std::lock_guard<std::mutex> lk(mu_);
        std::memset(s, 0, sizeof(*s));
        s->submitted = submitted_;
        s->completed = completed_;
        s->failed = failed_;
        s->batches = batches_;
        s->batched_requests = batched_requests_;
        s->large_solves = large_solves_;
        s->peak_device_bytes = peak_bytes_;
        s->device_bytes_in_use = in_use_;
        if (!lat_.empty()) {
            std::vector<double> l = lat_;
            std::sort(l.begin(), l.end());
            auto pct = [&](double q) { return l[std::min(l.size() - 1, (size_t)(q * (l.size() - 1) + 0.5))]; };
            s->p50_ms = pct(0.50);
            s->p99_ms = pct(0.99);
            double sum = 0;
            for (double x : l) sum += x;
            s->mean_ms = sum / l.size();
        }
    }

private:
    void stop()
    {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stopping_ = true;
        }
        cv_work_.notify_all();
        cv_budget_.notify_all();
        for (auto &t : threads_)
            if (t.joinable()) t.join();
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (auto *q : {&small_q_, &large_q_}) {
                for (Request *r : *q) {
                    r->status = JSVD_ERR_RUNTIME;
                    r->error = "The server was destroyed before the request ran.";
                    r->done = true;
                    ++failed_;
                }
                q->clear();
            }
        }
        cv_done_.notify_all();
    }

    // Takes requests from q while their footprints fit the budget; blocks while
    // the first one does not fit.  Returns an empty list when stopping.
    std::vector<Request *> admit(std::deque<Request *> &q, size_t max_count)
    {
        std::unique_lock<std::mutex> lk(mu_);
        cv_work_.wait(lk, [&] { return stopping_ || !q.empty(); });
        std::vector<Request *> got;
        while (!stopping_ && got.empty()) {
            while (!q.empty() && got.size() < max_count && in_use_ + q.front()->footprint <= opt_.device_budget_bytes) {
                in_use_ += q.front()->footprint;
                got.push_back(q.front());
                q.pop_front();
            }
            if (got.empty()) {
                if (q.empty()) {
                    cv_work_.wait(lk, [&] { return stopping_ || !q.empty(); });
                } else {
                    cv_budget_.wait(lk);
                }
            }
        }
        peak_bytes_ = std::max(peak_bytes_, in_use_);
        return got;
    }

    // Takes queued requests while their footprints fit the budget, up to
    // max_count, without waiting.
    std::vector<Request *> try_admit(std::deque<Request *> &q, size_t max_count)
    {
        std::lock_guard<std::mutex> lk(mu_);
        std::vector<Request *> got;
        while (!stopping_ && !q.empty() && got.size() < max_count &&
               in_use_ + q.front()->footprint <= opt_.device_budget_bytes) {
            in_use_ += q.front()->footprint;
            got.push_back(q.front());
            q.pop_front();
        }
        peak_bytes_ = std::max(peak_bytes_, in_use_);
        return got;
    }

    void finish(const std::vector<Request *> &rs, int status, const std::string &err)
    {
        const auto now = Clock::now();
        {
            std::lock_guard<std::mutex> lk(mu_);
            for (Request *r : rs) {
                in_use_ -= r->footprint;
                r->status = status;
                r->error = err;
                r->t_done = now;
                r->done = true;
                if (status == JSVD_OK) {
                    ++completed_;
                    lat_.push_back(std::chrono::duration<double, std::milli>(now - r->t_submit).count());
                } else {
                    ++failed_;
                }
            }
        }
        cv_budget_.notify_all();
        cv_done_.notify_all();
    }

    // A small request on the device: one allocation holding its state (A,
    // V), its input and its outputs (sigma, V, U).
    struct Slot {
        Request *r = nullptr;
        double *d = nullptr;
        int sweeps = 0;
        bool first = true;
    };

    StepDesc slot_desc(const Slot &s) const
    {
        const size_t m = s.r->m, n = s.r->n;
        StepDesc d{};
        d.m = (int)m;
        d.n = (int)n;
        d.a = s.d;
        d.v = s.d + m * n;
        d.in = s.first ? s.d + m * n + n * n : nullptr;
        d.s_out = s.d + 2 * m * n + n * n;
        d.v_out = d.s_out + n;
        d.u_out = s.r->want_u ? d.v_out + n * n : nullptr;
        return d;
    }

    // Uploads the fresh requests (they join `active`), runs one sweep of every
    // active request, then collects the ones that converged or reached
    // max_sweeps into `done` (their outputs are on the host, their device
    // memory released).
    int step_once(std::vector<Slot> &active, std::vector<Request *> &fresh, std::vector<Slot> &done,
                  cudaStream_t st, Pinned &stage, StepScratch &sc)
    {
        size_t up = 0;
        for (Request *r : fresh) up += r->m * r->n;
        if (up > 0) {
            if (int rc = stage.ensure(sizeof(double) * up); rc != JSVD_OK) return rc;
            JSVD_CUDA_TRY(cudaStreamSynchronize(st));  // the staging buffer is free again
        }
        size_t off = 0;
        double *h = static_cast<double *>(stage.p);
        while (!fresh.empty()) {
            Request *r = fresh.back();
            const size_t m = r->m, n = r->n;
            Slot s;
            s.r = r;
            JSVD_CUDA_TRY(cudaMallocAsync((void **)&s.d, sizeof(double) * (3 * m * n + n + 2 * n * n), st));
            fresh.pop_back();
            active.push_back(s);
            std::memcpy(h + off, r->a.data(), sizeof(double) * m * n);
            JSVD_CUDA_TRY(cudaMemcpyAsync(s.d + m * n + n * n, h + off, sizeof(double) * m * n,
                                          cudaMemcpyHostToDevice, st));
            off += m * n;
        }
        std::vector<StepDesc> descs(active.size());
        for (size_t i = 0; i < active.size(); ++i) descs[i] = slot_desc(active[i]);
        std::vector<int> rotated(active.size());
        if (int rc = batch_step(descs, opt_.cfg.epsilon, rotated.data(), sc, st); rc != JSVD_OK) return rc;
        {
            std::lock_guard<std::mutex> lk(mu_);
            ++batches_;
        }
        std::vector<Slot> keep;
        std::vector<StepDesc> fin;
        for (size_t i = 0; i < active.size(); ++i) {
            Slot &s = active[i];
            s.first = false;
            ++s.sweeps;
            if (rotated[i] == 0 || s.sweeps >= opt_.cfg.max_sweeps) {
                done.push_back(s);
                fin.push_back(slot_desc(s));
            } else {
                keep.push_back(s);
            }
        }
        active.swap(keep);
        if (done.empty()) return JSVD_OK;
        if (int rc = batch_finish(fin, opt_.cfg.epsilon, sc, st); rc != JSVD_OK) return rc;
        size_t out = 0;
        for (const Slot &s : done) out += s.r->n + s.r->n * s.r->n + (s.r->want_u ? s.r->m * s.r->n : 0);
        if (int rc = stage.ensure(sizeof(double) * out); rc != JSVD_OK) return rc;
        h = static_cast<double *>(stage.p);
        off = 0;
        for (const Slot &s : done) {
            const size_t m = s.r->m, n = s.r->n, k = n + n * n + (s.r->want_u ? m * n : 0);
            JSVD_CUDA_TRY(cudaMemcpyAsync(h + off, s.d + 2 * m * n + n * n, sizeof(double) * k,
                                          cudaMemcpyDeviceToHost, st));
            off += k;
        }
        JSVD_CUDA_TRY(cudaStreamSynchronize(st));
        off = 0;
        for (Slot &s : done) {
            Request *r = s.r;
            const size_t m = r->m, n = r->n;
            r->sigma.assign(h + off, h + off + n);
            r->v.assign(h + off + n, h + off + n + n * n);
            if (r->want_u) r->u.assign(h + off + n + n * n, h + off + n + n * n + m * n);
            r->sweeps = s.sweeps;
            off += n + n * n + (r->want_u ? m * n : 0);
            cudaFreeAsync(s.d, st);
            s.d = nullptr;
        }
        return JSVD_OK;
    }

    void small_loop()
    {
        cudaSetDevice(device_);
        cudaStream_t st = nullptr;
        cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        Pinned stage;
        StepScratch sc;
        std::vector<Slot> active;
        for (;;) {
            const size_t cap = (size_t)std::max(1, opt_.max_batch);
            const size_t room = cap > active.size() ? cap - active.size() : 0;
            // with nothing on the device, block for work; else take what is queued
            std::vector<Request *> fresh = active.empty() ? admit(small_q_, room) : try_admit(small_q_, room);
            if (active.empty() && fresh.empty()) break;
            std::vector<Slot> done;
            // a C++ exception (a host allocation) fails these requests, not the process
            const int rc = c_entry([&] { return step_once(active, fresh, done, st, stage, sc); });
            if (rc != JSVD_OK) {
                // every request on the device (and any not yet uploaded) fails
                const std::string err = last_error_message();
                std::vector<Request *> failed(fresh.begin(), fresh.end());
                for (Slot &s : active) {
                    failed.push_back(s.r);
                    if (s.d) cudaFreeAsync(s.d, st);
                }
                for (Slot &s : done) {
                    failed.push_back(s.r);
                    if (s.d) cudaFreeAsync(s.d, st);
                }
                active.clear();
                cudaStreamSynchronize(st);
                finish(failed, rc, err);
                continue;
            }
            if (!done.empty()) {
                std::vector<Request *> rs;
                for (const Slot &s : done) rs.push_back(s.r);
                {
                    std::lock_guard<std::mutex> lk(mu_);
                    batched_requests_ += rs.size();
                }
                finish(rs, JSVD_OK, std::string());
            }
        }
        if (st) cudaStreamDestroy(st);
    }

    int run_large(Request *r, Pinned &stage)
    {
        const size_t m = r->m, n = r->n;
        const size_t doubles = m * n + n + n * n + (r->want_u ? m * n : 0);
        int rc = stage.ensure(sizeof(double) * doubles);
        if (rc != JSVD_OK) return rc;
        cudaStream_t st = thread_stream(device_);
        if (st == nullptr) return cuda_failure(cudaGetLastError(), "cudaStreamCreateWithFlags", __FILE__, __LINE__);
        double *h = static_cast<double *>(stage.p);
        std::memcpy(h, r->a.data(), sizeof(double) * m * n);
        double *d = nullptr;
        JSVD_CUDA_TRY(cudaMallocAsync((void **)&d, sizeof(double) * doubles, st));
        ScopeExit free_d([&] { cudaFreeAsync(d, st); });  // stream-ordered, on every path
        JSVD_CUDA_TRY(cudaMemcpyAsync(d, h, sizeof(double) * m * n, cudaMemcpyHostToDevice, st));
        double *ds = d + m * n, *dv = ds + n, *du = r->want_u ? dv + n * n : nullptr;
        rc = opt_.large_path == 1   ? jsvd_precond_svd_device(d, m, n, &opt_.cfg, du, ds, dv, &r->sweeps, st)
             : opt_.large_path == 2 ? jsvd_mixed_svd_device(d, m, n, &opt_.cfg, du, ds, dv, &r->sweeps, st)
                                    : jsvd_plain_svd_device(d, m, n, &opt_.cfg, du, ds, dv, &r->sweeps, st);
        if (rc != JSVD_OK) return rc;
        JSVD_CUDA_TRY(cudaMemcpyAsync(h + m * n, ds, sizeof(double) * (doubles - m * n), cudaMemcpyDeviceToHost, st));
        JSVD_CUDA_TRY(cudaStreamSynchronize(st));
        r->sigma.assign(h + m * n, h + m * n + n);
        r->v.assign(h + m * n + n, h + m * n + n + n * n);
        if (r->want_u) r->u.assign(h + m * n + n + n * n, h + m * n + n + n * n + m * n);
        return JSVD_OK;
    }

    void large_loop()
    {
        cudaSetDevice(device_);
        Pinned stage;
        for (;;) {
            std::vector<Request *> rs = admit(large_q_, 1);
            if (rs.empty()) break;
            const int rc = c_entry([&] { return run_large(rs[0], stage); });
            {
                std::lock_guard<std::mutex> lk(mu_);
                ++large_solves_;
            }
            finish(rs, rc, rc == JSVD_OK ? std::string() : last_error_message());
        }
        jsvd_release_thread_cache();
    }

    jsvd_server_options opt_;
    int device_ = 0;
    std::mutex mu_;
    std::condition_variable cv_work_, cv_done_, cv_budget_;
    std::deque<Request *> small_q_, large_q_;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> requests_;
    std::vector<std::thread> threads_;
    bool stopping_ = false;
    int waiters_ = 0;  // threads inside wait()
    uint64_t next_id_ = 1;
    size_t in_use_ = 0, peak_bytes_ = 0;
    unsigned long long submitted_ = 0, completed_ = 0, failed_ = 0, batches_ = 0, batched_requests_ = 0,
                       large_solves_ = 0;
    std::vector<double> lat_;
};

}  // namespace jsvd

using namespace jsvd;

struct jsvd_server {
    std::unique_ptr<Server> impl;
};

extern "C" {

void jsvd_server_options_default(jsvd_server_options *o)
{
    if (!o) return;
    std::memset(o, 0, sizeof(*o));
    o->device_budget_bytes = size_t(40) << 30;
    o->small_workers = 2;
    o->large_workers = 4;
    o->max_batch = 4096;
    jsvd_config_default(&o->cfg);
}

int jsvd_server_create(const jsvd_server_options *opt, jsvd_server **out)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        if (!out) return invalid_argument("out must not be null.");
        jsvd_server_options o;
        jsvd_server_options_default(&o);
        if (opt) o = *opt;
        if (o.device_budget_bytes == 0) o.device_budget_bytes = size_t(40) << 30;
        if (o.small_workers <= 0) o.small_workers = 2;
        if (o.large_workers <= 0) o.large_workers = 4;
        if (o.max_batch <= 0) o.max_batch = 4096;
        if (!(o.cfg.epsilon > 0.0)) return invalid_argument("epsilon must be positive.");
        if (o.cfg.max_sweeps <= 0) return invalid_argument("max_sweeps must be positive.");
        auto s = std::make_unique<jsvd_server>();
        s->impl = std::make_unique<Server>(o);
        *out = s.release();
        return JSVD_OK;
    });
}

int jsvd_server_submit(jsvd_server *s, const double *a, size_t rows, size_t columns, int want_u, uint64_t *ticket)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        if (!s) return invalid_argument("server must not be null.");
        return s->impl->submit(a, rows, columns, want_u, ticket);
    });
}

int jsvd_server_wait(jsvd_server *s, uint64_t ticket, double *u, double *sigma, double *v, int *sweeps,
                     double *latency_ms)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        if (!s) return invalid_argument("server must not be null.");
        return s->impl->wait(ticket, u, sigma, v, sweeps, latency_ms);
    });
}

int jsvd_server_poll(jsvd_server *s, uint64_t ticket, int *done)
{
    return c_entry([&]() -> int {
        set_last_error(JSVD_OK, "");
        if (!s) return invalid_argument("server must not be null.");
        return s->impl->poll(ticket, done);
    });
}

int jsvd_server_get_stats(jsvd_server *s, jsvd_server_stats *out)
{
    return c_entry([&]() -> int {
        if (!s || !out) return invalid_argument("server and out must not be null.");
        s->impl->stats(out);
        return JSVD_OK;
    });
}

void jsvd_server_destroy(jsvd_server *s) { delete s; }

}  // extern "C"
