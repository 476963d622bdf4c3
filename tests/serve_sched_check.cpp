// Host-only checks of the scoring server's scheduler (cracklingplusplus_gpu_b200/csrc/serve_sched.hpp)
// with a fake executor: results reach the right requests, batching and overlap happen, batches
// respect the guide limit and the slot's memory budget, admission is in arrival order, the
// footprint estimate grows with what batches used, requests too large for one batch are scored in
// parts, waits time out, and shutdown drains the queue.
// Prints "ok" and exits 0 when every check holds.
#include <atomic>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <thread>

#include "serve_sched.hpp"

using namespace issl::serve;

#define CHECK(c)                                                          \
    do {                                                                  \
        if (!(c)) {                                                       \
            std::fprintf(stderr, "check failed line %d: %s\n", __LINE__, #c); \
            std::exit(1);                                                 \
        }                                                                 \
    } while (0)

struct FakeExec {
    std::atomic<int> running{0}, peak{0};
    std::atomic<uint64_t> max_batch{0};
    uint64_t limit_guides = ~0ull;
    double us_per_guide = 2.0;
    double cand_per_guide = 10.0;
    std::mutex mu;
    std::vector<uint64_t> admitted;  // tickets in admission order
    int run(uint32_t, std::vector<Request*>& batch, uint64_t* cands, std::string*) {
        const int r = ++running;
        int p = peak.load();
        while (r > p && !peak.compare_exchange_weak(p, r)) {}
        uint64_t n = 0;
        {
            std::lock_guard<std::mutex> lk(mu);
            for (Request* q : batch) {
                admitted.push_back(q->ticket);
                n += q->sigs.size();
            }
        }
        CHECK(n <= limit_guides);
        uint64_t m = max_batch.load();
        while (n > m && !max_batch.compare_exchange_weak(m, n)) {}
        std::this_thread::sleep_for(std::chrono::microseconds(static_cast<int64_t>(500 + us_per_guide * n)));
        for (Request* q : batch) {
            const size_t k = q->sigs.size();
            q->mit.resize(k);
            q->cfd.resize(k);
            q->code.resize(k);
            q->count.resize(k);
            for (size_t i = 0; i < k; i++) {
                q->mit[i] = static_cast<double>(q->sigs[i]) * 0.5 + q->method;
                q->cfd[i] = q->threshold;
                q->code[i] = (q->sigs[i] & 1) ? '1' : '0';
                q->count[i] = q->sigs[i] + static_cast<uint64_t>(q->max_dist);
            }
        }
        *cands = static_cast<uint64_t>(cand_per_guide * static_cast<double>(n));
        --running;
        return ISSL_OK;
    }
};

std::unique_ptr<Request> make(uint64_t seed, size_t n, int method, double thr, int md) {
    auto r = std::make_unique<Request>();
    r->sigs.resize(n);
    for (size_t i = 0; i < n; i++) r->sigs[i] = seed * 1000003ull + i * 7919ull;
    r->method = method;
    r->threshold = thr;
    r->max_dist = md;
    return r;
}

void check_results(const Request& r, uint64_t seed) {
    for (size_t i = 0; i < r.sigs.size(); i++) {
        const uint64_t s = seed * 1000003ull + i * 7919ull;
        CHECK(r.sigs[i] == s);
        CHECK(r.mit[i] == static_cast<double>(s) * 0.5 + r.method);
        CHECK(r.cfd[i] == r.threshold);
        CHECK(r.code[i] == ((s & 1) ? '1' : '0'));
        CHECK(r.count[i] == s + static_cast<uint64_t>(r.max_dist));
    }
}

int main() {
    {  // many submitters: right results, batching, overlap, latency summary
        FakeExec ex;
        Config cfg;
        cfg.n_slots = 3;
        cfg.max_batch_guides = 20000;
        Footprint fp;
        fp.fixed = 1000;
        fp.per_guide = 10;
        fp.per_candidate = 1;
        fp.candidates_per_guide = 10;
        cfg.slot_budget_bytes = fp.bytes(cfg.max_batch_guides) * 2;
        ex.limit_guides = cfg.max_batch_guides;
        Scheduler<FakeExec> s(cfg, fp, ex);
        std::vector<std::thread> th;
        std::atomic<int> done{0};
        for (int t = 0; t < 8; t++)
            th.emplace_back([&, t] {
                std::mt19937 rng(t);
                for (int k = 0; k < 50; k++) {
                    const uint64_t seed = t * 1000 + k;
                    const size_t n = 1 + rng() % 2000;
                    uint64_t ticket = 0;
                    std::string err;
                    CHECK(s.submit(make(seed, n, k % 5, 50.0 + k, k % 5), &ticket, &err) == ISSL_OK);
                    std::unique_ptr<Request> r;
                    CHECK(s.wait(ticket, -1, &r, &err) == ISSL_OK);
                    CHECK(r->sigs.size() == n && r->done);
                    CHECK(r->batch_guides >= n && r->batch_requests >= 1);
                    check_results(*r, seed);
                    std::string e2;
                    std::unique_ptr<Request> again;
                    CHECK(s.wait(ticket, 0, &again, &e2) == ISSL_ERR_ARG);  // a ticket is collected once
                    done++;
                }
            });
        for (auto& t : th) t.join();
        CHECK(done == 400);
        Stats st = s.stats(false);
        CHECK(st.requests == 400);
        CHECK(st.batches < 400);  // requests that arrive together share a batch
        CHECK(st.peak_in_flight >= 2 && st.peak_in_flight <= 3);
        CHECK(ex.peak >= 2);
        CHECK(st.p50_ms > 0 && st.p50_ms <= st.p99_ms && st.p99_ms <= st.max_ms);
        Stats st2 = s.stats(true);
        CHECK(st2.requests == 400);
        CHECK(s.stats(false).requests == 0);
        std::printf("{\"batches\": %llu, \"peak_in_flight\": %u, \"p50_ms\": %.3f, \"p99_ms\": %.3f}\n",
                    static_cast<unsigned long long>(st.batches), st.peak_in_flight, st.p50_ms, st.p99_ms);
    }
    {  // admission by footprint, limits, arrival order, estimate growth
        FakeExec ex;
        ex.cand_per_guide = 0;
        Config cfg;
        cfg.n_slots = 1;
        cfg.max_batch_guides = 1000;
        Footprint fp;
        fp.fixed = 1000;
        fp.per_guide = 100;
        fp.per_candidate = 10;
        fp.candidates_per_guide = 0;
        cfg.slot_budget_bytes = fp.bytes(500);  // 500 guides fit a slot
        ex.limit_guides = 500;
        Scheduler<FakeExec> s(cfg, fp, ex);
        uint64_t ticket;
        std::string err;
        {  // needs more than a slot's memory (600 > 500 guides) and exceeds the batch limit (1001 > 1000):
           // both are scored in parts of at most 500 guides, with every guide's result in place
            uint64_t t1, t2;
            CHECK(s.submit(make(1, 600, 2, 75, 4), &t1, &err) == ISSL_OK);
            CHECK(s.submit(make(2, 1001, 1, 60, 3), &t2, &err) == ISSL_OK);
            std::unique_ptr<Request> r1, r2;
            CHECK(s.wait(t1, -1, &r1, &err) == ISSL_OK && r1->sigs.size() == 600 && r1->parts.size() == 2);
            CHECK(s.wait(t2, -1, &r2, &err) == ISSL_OK && r2->sigs.size() == 1001 && r2->parts.size() == 3);
            check_results(*r1, 1);
            check_results(*r2, 2);
            CHECK(r1->t_submit <= r1->t_admit && r1->t_admit <= r1->t_done);
            CHECK(ex.max_batch <= 500);
            ex.admitted.clear();
        }
        std::vector<uint64_t> tickets;
        for (int k = 0; k < 12; k++) {
            CHECK(s.submit(make(100 + k, 200, 2, 75, 4), &ticket, &err) == ISSL_OK);
            tickets.push_back(ticket);
        }
        for (size_t k = 0; k < tickets.size(); k++) {
            std::unique_ptr<Request> r;
            CHECK(s.wait(tickets[k], -1, &r, &err) == ISSL_OK);
            CHECK(r->batch_guides <= 500 && r->batch_requests <= 2);
            check_results(*r, 100 + k);
        }
        CHECK(ex.max_batch <= 500);
        for (size_t k = 1; k < ex.admitted.size(); k++) CHECK(ex.admitted[k] > ex.admitted[k - 1]);  // FIFO
        // a batch that used many candidates raises the estimate: 400 guides no longer fit one batch
        // and run in parts
        ex.cand_per_guide = 8;
        CHECK(s.submit(make(7, 100, 2, 75, 4), &ticket, &err) == ISSL_OK);
        std::unique_ptr<Request> r;
        CHECK(s.wait(ticket, -1, &r, &err) == ISSL_OK);
        ex.max_batch = 0;
        CHECK(s.submit(make(8, 400, 2, 75, 4), &ticket, &err) == ISSL_OK);
        CHECK(s.wait(ticket, -1, &r, &err) == ISSL_OK && r->parts.size() >= 2);
        check_results(*r, 8);
        CHECK(ex.max_batch < 400);
        CHECK(s.submit(make(9, 0, 2, 75, 4), &ticket, &err) == ISSL_OK);  // empty request completes at once
        CHECK(s.wait(ticket, 0, &r, &err) == ISSL_OK && r->sigs.empty());
        CHECK(s.stats(false).requests == 16);  // a request scored in parts counts once
    }
    {  // refused only when not even one guide fits a slot
        FakeExec ex;
        Config cfg;
        cfg.n_slots = 1;
        Footprint fp;
        fp.fixed = 1000;
        fp.per_guide = 100;
        cfg.slot_budget_bytes = 1050;
        Scheduler<FakeExec> s(cfg, fp, ex);
        uint64_t ticket;
        std::string err;
        CHECK(s.submit(make(1, 3, 2, 75, 4), &ticket, &err) == ISSL_ERR_BUSY);
    }
    {  // timeouts and draining on shutdown
        FakeExec ex;
        ex.us_per_guide = 50;
        Config cfg;
        cfg.n_slots = 1;
        cfg.max_batch_guides = 5000;
        Footprint fp;
        cfg.slot_budget_bytes = 1ull << 40;
        std::vector<uint64_t> tickets;
        {
            Scheduler<FakeExec> s(cfg, fp, ex);
            uint64_t ticket;
            std::string err;
            CHECK(s.submit(make(3, 4000, 0, 75, 4), &ticket, &err) == ISSL_OK);
            std::unique_ptr<Request> r;
            CHECK(s.wait(ticket, 1, &r, &err) == ISSL_ERR_TIMEOUT);  // 200 ms of work
            CHECK(s.wait(ticket, -1, &r, &err) == ISSL_OK);
            for (int k = 0; k < 5; k++) {
                CHECK(s.submit(make(50 + k, 1000, 1, 60, 3), &ticket, &err) == ISSL_OK);
                tickets.push_back(ticket);
            }
        }  // destructor: the five pending requests are scored before the slots stop
        CHECK(ex.admitted.size() >= 2);
        CHECK(ex.admitted.back() == tickets.back());
    }
    std::printf("ok\n");
    return 0;
}
