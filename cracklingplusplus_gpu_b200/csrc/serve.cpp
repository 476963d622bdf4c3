// The scoring server: the scheduler of serve_sched.hpp driving one batch context per slot.
#include <cuda_runtime.h>

#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "issl_internal.cuh"
#include "serve_sched.hpp"

namespace issl {
namespace {

constexpr uint64_t kDefaultHeadroom = 16ull << 30;
constexpr uint64_t kDefaultBatchGuides = 131072;
constexpr uint32_t kDefaultSlots = 3;

// Scores a batch of requests on one slot: signatures gathered into the slot's pinned staging,
// one guide set per request, one graph replay, results scattered back to the requests.
struct GpuExec {
    struct Slot {
        issl_batch* batch = nullptr;
        uint64_t* sigs = nullptr;
        double* mit = nullptr;
        double* cfd = nullptr;
        char* code = nullptr;
        uint64_t* count = nullptr;
    };
    issl_index* ix = nullptr;
    std::vector<Slot> slots;

    int run(uint32_t slot, std::vector<serve::Request*>& batch, uint64_t* candidates, std::string* err) {
        Slot& S = slots[slot];
        if (cudaSetDevice(ix->device) != cudaSuccess) {
            *err = "cudaSetDevice failed";
            return ISSL_ERR_CUDA;
        }
        std::vector<issl_guide_set> sets;
        sets.reserve(batch.size());
        uint64_t n = 0;
        for (serve::Request* r : batch) {
            std::memcpy(S.sigs + n, r->sigs.data(), r->sigs.size() * sizeof(uint64_t));
            sets.push_back(issl_guide_set{r->sigs.size(), r->method, r->max_dist, r->threshold});
            n += r->sigs.size();
        }
        const int rc = issl_batch_score_host(S.batch, S.sigs, n, sets.data(), sets.size(), S.mit, S.cfd, S.code,
                                             S.count);
        if (rc != ISSL_OK) {
            *err = issl_last_error();
            return rc;
        }
        issl_score_stats st{};
        issl_batch_stats(S.batch, &st);
        *candidates = st.candidates;
        uint64_t off = 0;
        for (serve::Request* r : batch) {
            const uint64_t k = r->sigs.size();
            r->mit.assign(S.mit + off, S.mit + off + k);
            r->cfd.assign(S.cfd + off, S.cfd + off + k);
            r->code.assign(S.code + off, S.code + off + k);
            r->count.assign(S.count + off, S.count + off + k);
            off += k;
        }
        return ISSL_OK;
    }
};

}  // namespace
}  // namespace issl

struct issl_server {
    issl::GpuExec exec;
    std::unique_ptr<issl::serve::Scheduler<issl::GpuExec>> sched;
    ~issl_server() {
        sched.reset();  // drains the queue, joins the slots
        cudaSetDevice(exec.ix->device);
        for (auto& s : exec.slots) {
            if (s.batch) issl_batch_destroy(s.batch);
            for (void* p : {static_cast<void*>(s.sigs), static_cast<void*>(s.mit), static_cast<void*>(s.cfd),
                            static_cast<void*>(s.code), static_cast<void*>(s.count)})
                if (p) cudaFreeHost(p);
        }
    }
};

using issl::guarded;

extern "C" {

int issl_server_create(issl_index* ix, const issl_server_config* config, issl_server** out) {
    return guarded([&] {
        ISSL_REQUIRE(ix && out, ISSL_ERR_ARG, "issl_server_create: null argument");
        *out = nullptr;
        issl_server_config c{};
        if (config) c = *config;
        issl::serve::Config cfg;
        cfg.n_slots = c.n_slots ? c.n_slots : issl::kDefaultSlots;
        cfg.max_wait_us = c.max_wait_us;
        cfg.max_batch_guides = c.max_batch_guides ? c.max_batch_guides : issl::kDefaultBatchGuides;
        const uint64_t headroom = c.headroom_bytes ? c.headroom_bytes : issl::kDefaultHeadroom;
        ISSL_REQUIRE(cfg.n_slots <= 64, ISSL_ERR_ARG, "issl_server_create: at most 64 slots");
        ISSL_REQUIRE(cfg.max_batch_guides < (1ull << 26), ISSL_ERR_ARG, "issl_server_create: batch limit above 2^26");
        ISSL_CUDA(cudaSetDevice(ix->device));
        size_t free_b = 0, total_b = 0;
        ISSL_CUDA(cudaMemGetInfo(&free_b, &total_b));
        issl::serve::Footprint fp;
        issl::workspace_model(ix, &fp.fixed, &fp.per_guide, &fp.per_candidate);
        const uint64_t budget = free_b > headroom ? free_b - headroom : 0;
        cfg.slot_budget_bytes = budget / cfg.n_slots;
        ISSL_REQUIRE(cfg.slot_budget_bytes >= fp.bytes(1), ISSL_ERR_NOMEM,
                     "not enough free device memory for the server's slots beside the index and the headroom");
        auto srv = std::make_unique<issl_server>();
        srv->exec.ix = ix;
        srv->exec.slots.resize(cfg.n_slots);
        const uint64_t cap = cfg.max_batch_guides;
        for (auto& s : srv->exec.slots) {
            if (issl_batch_create(ix, &s.batch) != ISSL_OK) throw issl::Error(ISSL_ERR_CUDA, issl_last_error());
            // the slot's workspace takes its whole share at its first batch and keeps it
            issl::batch_set_capacity_floor(s.batch, cap, cfg.slot_budget_bytes);
            ISSL_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&s.sigs), cap * 8, cudaHostAllocDefault));
            ISSL_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&s.mit), cap * 8, cudaHostAllocDefault));
            ISSL_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&s.cfd), cap * 8, cudaHostAllocDefault));
            ISSL_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&s.code), cap, cudaHostAllocDefault));
            ISSL_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&s.count), cap * 8, cudaHostAllocDefault));
        }
        srv->sched = std::make_unique<issl::serve::Scheduler<issl::GpuExec>>(cfg, fp, srv->exec);
        *out = srv.release();
    });
}

int issl_server_submit(issl_server* srv, const uint64_t* sigs, size_t n, int method, double threshold, int max_dist,
                       uint64_t* ticket) {
    return guarded([&] {
        ISSL_REQUIRE(srv && ticket && (sigs || n == 0), ISSL_ERR_ARG, "issl_server_submit: null argument");
        ISSL_REQUIRE(method >= ISSL_METHOD_MIT && method <= ISSL_METHOD_AVG_MIT_CFD, ISSL_ERR_ARG,
                     "Scoring method is not valid.");
        ISSL_REQUIRE(max_dist >= 0 && max_dist <= issl::kMaxDist, ISSL_ERR_ARG, "max_dist must be 0..4");
        auto r = std::make_unique<issl::serve::Request>();
        r->sigs.assign(sigs, sigs + n);
        r->method = method;
        r->threshold = threshold;
        r->max_dist = max_dist;
        std::string err;
        const int rc = srv->sched->submit(std::move(r), ticket, &err);
        if (rc != ISSL_OK) throw issl::Error(rc, err);
    });
}

int issl_server_wait(issl_server* srv, uint64_t ticket, int timeout_ms, double* mit, double* cfd, char* code,
                     uint64_t* count, issl_request_info* info) {
    return guarded([&] {
        ISSL_REQUIRE(srv, ISSL_ERR_ARG, "issl_server_wait: null server");
        std::unique_ptr<issl::serve::Request> r;
        std::string err;
        const int rc = srv->sched->wait(ticket, timeout_ms, &r, &err);
        if (rc != ISSL_OK) throw issl::Error(rc, err);
        const size_t n = r->sigs.size();
        if (mit && n) std::memcpy(mit, r->mit.data(), n * 8);
        if (cfd && n) std::memcpy(cfd, r->cfd.data(), n * 8);
        if (code && n) std::memcpy(code, r->code.data(), n);
        if (count && n) std::memcpy(count, r->count.data(), n * 8);
        if (info) {
            info->queue_ms = issl::serve::ms_between(r->t_submit, r->t_admit);
            info->service_ms = issl::serve::ms_between(r->t_admit, r->t_done);
            info->latency_ms = issl::serve::ms_between(r->t_submit, r->t_done);
            info->batch_guides = r->batch_guides;
            info->batch_requests = r->batch_requests;
            info->slot = r->slot;
        }
    });
}

int issl_server_stats(issl_server* srv, issl_server_summary* out, int reset) {
    return guarded([&] {
        ISSL_REQUIRE(srv && out, ISSL_ERR_ARG, "issl_server_stats: null argument");
        const issl::serve::Stats s = srv->sched->stats(reset != 0);
        out->requests = s.requests;
        out->guides = s.guides;
        out->batches = s.batches;
        out->p50_ms = s.p50_ms;
        out->p99_ms = s.p99_ms;
        out->max_ms = s.max_ms;
        out->mean_batch_guides = s.mean_batch_guides;
        out->slots = s.slots;
        out->peak_in_flight = s.peak_in_flight;
        out->slot_budget_bytes = s.slot_budget_bytes;
        out->peak_batch_bytes = s.peak_batch_bytes;
    });
}

void issl_server_destroy(issl_server* srv) { delete srv; }

}  // extern "C"
