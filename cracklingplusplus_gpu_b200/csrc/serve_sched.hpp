// Request scheduling of the scoring server: admission by device-memory footprint and
// continuous batching over several slots that run at the same time.
//
// A slot is one worker thread with its own scoring workspace on the GPU (its own buffers and
// captured graph). A free slot takes the waiting requests in arrival order and packs them into
// one batch while the batch stays within the per-batch guide limit and its modelled device
// footprint stays within the slot's share of the free device memory; the batch is scored as one
// pass (each request is one guide set with its own method / threshold / mismatch bound). Other
// slots keep taking requests meanwhile, so requests that arrive while batches are on the GPU
// are admitted as soon as a slot frees up, and the batches overlap on the device. A request too
// large for one batch (guide limit or footprint) is queued as consecutive parts of equal size.
//
// This file has no GPU code: the executor that scores a batch is a template parameter, so the
// same scheduler runs in the library (a GPU executor) and in host-only tests (a fake one).
#pragma once

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "issl_b200.h"

namespace issl {
namespace serve {

using Clock = std::chrono::steady_clock;

inline double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Config {
    uint32_t n_slots = 3;
    uint32_t max_wait_us = 0;
    uint64_t max_batch_guides = 131072;
    uint64_t slot_budget_bytes = 0;  // device bytes one slot's batch may occupy
};

// Device bytes of a scoring workspace holding a batch of n guides: a fixed part (bucket tables,
// scan scratch), a per-guide part (probe lists, scan units, outputs) and the candidate-hit
// buffers, sized by a running estimate of candidates per guide that grows with what batches
// actually produced.
struct Footprint {
    uint64_t fixed = 0;
    uint64_t per_guide = 0;
    uint64_t per_candidate = 0;
    double candidates_per_guide = 64.0;
    uint64_t bytes(uint64_t n) const {
        return fixed + n * per_guide + static_cast<uint64_t>(static_cast<double>(n) * candidates_per_guide) *
                                           per_candidate;
    }
    // the most guides whose footprint stays within `budget` (0 if not even one fits)
    uint64_t guides_within(uint64_t budget) const {
        if (budget < bytes(1)) return 0;
        const double per = static_cast<double>(per_guide) + candidates_per_guide * static_cast<double>(per_candidate);
        uint64_t m = static_cast<uint64_t>(static_cast<double>(budget - fixed) / per);
        while (m > 1 && bytes(m) > budget) m--;
        return m ? m : 1;
    }
};

struct Request {
    uint64_t ticket = 0;
    std::vector<uint64_t> sigs;
    int method = ISSL_METHOD_MIT_AND_CFD;
    int max_dist = 4;
    double threshold = 75.0;
    std::vector<double> mit, cfd;
    std::vector<char> code;
    std::vector<uint64_t> count;
    Clock::time_point t_submit, t_admit, t_done;
    uint64_t batch_guides = 0;
    uint32_t batch_requests = 0, slot = 0;
    int status = ISSL_OK;
    std::string error;
    bool done = false;
    // a request larger than one batch may hold is scored as consecutive parts: each part is a
    // request of its own in the queue, `parent` the caller's request, which completes with its last
    Request* parent = nullptr;
    uint64_t part_off = 0;  // first guide of the part within the parent
    uint32_t parts_left = 0;
    std::vector<std::unique_ptr<Request>> parts;
};

struct Stats {
    uint64_t requests = 0, guides = 0, batches = 0;
    double p50_ms = 0, p99_ms = 0, max_ms = 0, mean_batch_guides = 0;
    uint32_t slots = 0, peak_in_flight = 0;
    uint64_t slot_budget_bytes = 0, peak_batch_bytes = 0;
};

// Exec must provide:
//   int run(uint32_t slot, std::vector<Request*>& batch, uint64_t* candidates, std::string* err);
// which scores every request of the batch into its result vectors and reports the candidate
// hit slots the pass used (for the footprint estimate). It is called from the slot's thread.
template <class Exec>
class Scheduler {
public:
    Scheduler(const Config& cfg, const Footprint& fp, Exec& exec) : cfg_(cfg), fp_(fp), exec_(exec) {
        for (uint32_t s = 0; s < cfg_.n_slots; s++) workers_.emplace_back([this, s] { worker(s); });
    }

    // Finishes every request already submitted, then stops the slots.
    ~Scheduler() {
        {
            std::lock_guard<std::mutex> lk(mu_);
            stop_ = true;
        }
        work_cv_.notify_all();
        for (auto& t : workers_) t.join();
    }

    Scheduler(const Scheduler&) = delete;
    Scheduler& operator=(const Scheduler&) = delete;

    // A request above the batch limit, or whose modelled footprint exceeds a slot's share of the
    // device memory, is scored as consecutive parts of equal size (guides are independent); only
    // a request of which not even one guide fits a slot is refused (ISSL_ERR_BUSY).
    int submit(std::unique_ptr<Request> r, uint64_t* ticket, std::string* err) {
        const uint64_t n = r->sigs.size();
        std::lock_guard<std::mutex> lk(mu_);
        const uint64_t fit = std::min<uint64_t>(cfg_.max_batch_guides, fp_.guides_within(cfg_.slot_budget_bytes));
        if (n && fit == 0) {
            *err = "request needs more device memory than a slot may use (" + std::to_string(fp_.bytes(1)) +
                   " > " + std::to_string(cfg_.slot_budget_bytes) + " bytes for one guide)";
            return ISSL_ERR_BUSY;
        }
        r->ticket = ++next_ticket_;
        r->t_submit = Clock::now();
        *ticket = r->ticket;
        Request* p = r.get();
        requests_[r->ticket] = std::move(r);
        if (n == 0) {  // nothing to score
            p->t_admit = p->t_done = p->t_submit;
            p->done = true;
            done_cv_.notify_all();
            return ISSL_OK;
        }
        if (n <= fit) {
            pending_.push_back(p);
        } else {
            const uint64_t k = (n + fit - 1) / fit, m = (n + k - 1) / k;
            p->mit.resize(n);
            p->cfd.resize(n);
            p->code.resize(n);
            p->count.resize(n);
            p->parts_left = static_cast<uint32_t>(k);
            for (uint64_t off = 0; off < n; off += m) {
                auto part = std::make_unique<Request>();
                part->sigs.assign(p->sigs.begin() + off, p->sigs.begin() + std::min(n, off + m));
                part->method = p->method;
                part->max_dist = p->max_dist;
                part->threshold = p->threshold;
                part->ticket = p->ticket;
                part->t_submit = p->t_submit;
                part->parent = p;
                part->part_off = off;
                pending_.push_back(part.get());
                p->parts.push_back(std::move(part));
            }
        }
        pending_guides_ += n;
        work_cv_.notify_one();
        return ISSL_OK;
    }

    // Waits up to timeout_ms (< 0: without limit) for the request; on completion hands it over
    // and forgets the ticket. ISSL_ERR_TIMEOUT: not finished yet (the ticket stays valid).
    int wait(uint64_t ticket, int timeout_ms, std::unique_ptr<Request>* out, std::string* err) {
        std::unique_lock<std::mutex> lk(mu_);
        auto it = requests_.find(ticket);
        if (it == requests_.end()) {
            *err = "unknown or already collected ticket";
            return ISSL_ERR_ARG;
        }
        Request* r = it->second.get();
        auto ready = [&] { return r->done; };
        if (timeout_ms < 0)
            done_cv_.wait(lk, ready);
        else if (!done_cv_.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
            *err = "request not finished yet";
            return ISSL_ERR_TIMEOUT;
        }
        *out = std::move(it->second);
        requests_.erase(it);
        if ((*out)->status != ISSL_OK) *err = (*out)->error;
        return (*out)->status;
    }

    Stats stats(bool reset) {
        std::lock_guard<std::mutex> lk(mu_);
        Stats s;
        s.requests = latencies_.size();
        s.guides = guides_done_;
        s.batches = batches_;
        s.slots = cfg_.n_slots;
        s.peak_in_flight = peak_in_flight_;
        s.slot_budget_bytes = cfg_.slot_budget_bytes;
        s.peak_batch_bytes = peak_batch_bytes_;
        s.mean_batch_guides = batches_ ? static_cast<double>(guides_done_) / batches_ : 0.0;
        if (!latencies_.empty()) {
            std::vector<double> v = latencies_;
            auto pct = [&](double q) {
                const size_t k = std::min(v.size() - 1, static_cast<size_t>(q * (v.size() - 1) + 0.5));
                std::nth_element(v.begin(), v.begin() + k, v.end());
                return v[k];
            };
            s.p50_ms = pct(0.50);
            s.p99_ms = pct(0.99);
            s.max_ms = *std::max_element(v.begin(), v.end());
        }
        if (reset) {
            latencies_.clear();
            guides_done_ = batches_ = 0;
            peak_in_flight_ = in_flight_;
            peak_batch_bytes_ = 0;
        }
        return s;
    }

private:
    void worker(uint32_t slot) {
        for (;;) {
            std::unique_lock<std::mutex> lk(mu_);
            work_cv_.wait(lk, [&] { return stop_ || !pending_.empty(); });
            if (pending_.empty()) {
                if (stop_) return;
                continue;
            }
            if (cfg_.max_wait_us && !stop_ && pending_guides_ < cfg_.max_batch_guides) {
                // gather arrivals a little longer before dispatching a small batch
                const auto until = Clock::now() + std::chrono::microseconds(cfg_.max_wait_us);
                work_cv_.wait_until(lk, until, [&] { return stop_ || pending_guides_ >= cfg_.max_batch_guides; });
                if (pending_.empty()) continue;  // another slot took them
            }
            // admission: arrival order, while the batch fits the guide limit and the slot's memory
            std::vector<Request*> batch;
            uint64_t n = 0;
            while (!pending_.empty()) {
                Request* r = pending_.front();
                const uint64_t n2 = n + r->sigs.size();
                if (!batch.empty() && (n2 > cfg_.max_batch_guides || fp_.bytes(n2) > cfg_.slot_budget_bytes)) break;
                batch.push_back(r);
                pending_.pop_front();
                n = n2;
            }
            pending_guides_ -= n;
            const uint64_t bytes = fp_.bytes(n);
            peak_batch_bytes_ = std::max(peak_batch_bytes_, bytes);
            in_flight_++;
            peak_in_flight_ = std::max(peak_in_flight_, in_flight_);
            const auto t_admit = Clock::now();
            for (Request* r : batch) {
                r->t_admit = t_admit;
                r->batch_guides = n;
                r->batch_requests = static_cast<uint32_t>(batch.size());
                r->slot = slot;
            }
            if (!pending_.empty()) work_cv_.notify_one();  // let another free slot take the rest
            lk.unlock();

            uint64_t candidates = 0;
            std::string err;
            int st = ISSL_OK;
            try {
                st = exec_.run(slot, batch, &candidates, &err);
            } catch (const std::exception& e) {
                st = ISSL_ERR_CUDA;
                err = e.what();
            }

            lk.lock();
            if (st == ISSL_OK && n)
                fp_.candidates_per_guide =
                    std::max(fp_.candidates_per_guide, 1.25 * static_cast<double>(candidates) / static_cast<double>(n));
            in_flight_--;
            batches_++;
            const auto t_done = Clock::now();
            for (Request* r : batch) {
                r->t_done = t_done;
                r->status = st;
                r->error = err;
                r->done = true;
                guides_done_ += r->sigs.size();
                Request* q = r->parent;
                if (!q) {
                    latencies_.push_back(ms_between(r->t_submit, t_done));
                    continue;
                }
                // a part: its results go to the caller's request, which is done with its last part
                if (st == ISSL_OK) {
                    std::copy(r->mit.begin(), r->mit.end(), q->mit.begin() + r->part_off);
                    std::copy(r->cfd.begin(), r->cfd.end(), q->cfd.begin() + r->part_off);
                    std::copy(r->code.begin(), r->code.end(), q->code.begin() + r->part_off);
                    std::copy(r->count.begin(), r->count.end(), q->count.begin() + r->part_off);
                } else if (q->status == ISSL_OK) {
                    q->status = st;
                    q->error = err;
                }
                std::vector<double>().swap(r->mit);
                std::vector<double>().swap(r->cfd);
                if (q->parts_left == static_cast<uint32_t>(q->parts.size()) || r->t_admit < q->t_admit)
                    q->t_admit = r->t_admit;  // the first part's admission
                q->batch_guides = std::max(q->batch_guides, r->batch_guides);
                q->batch_requests = std::max(q->batch_requests, r->batch_requests);
                q->slot = r->slot;
                if (--q->parts_left == 0) {
                    q->t_done = t_done;
                    q->done = true;
                    latencies_.push_back(ms_between(q->t_submit, t_done));
                }
            }
            lk.unlock();
            done_cv_.notify_all();
        }
    }

    Config cfg_;
    Footprint fp_;
    Exec& exec_;
    std::mutex mu_;
    std::condition_variable work_cv_, done_cv_;
    std::deque<Request*> pending_;
    uint64_t pending_guides_ = 0;
    std::map<uint64_t, std::unique_ptr<Request>> requests_;
    uint64_t next_ticket_ = 0;
    bool stop_ = false;
    uint32_t in_flight_ = 0, peak_in_flight_ = 0;
    uint64_t batches_ = 0, guides_done_ = 0, peak_batch_bytes_ = 0;
    std::vector<double> latencies_;
    std::vector<std::thread> workers_;
};

}  // namespace serve
}  // namespace issl
