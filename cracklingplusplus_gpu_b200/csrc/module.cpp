// ISSLScoringModule on the B200 library: lib/ISSLScoringModule.cpp:13-513 with the scoring loop
// replaced by issl_score() and the per-call file read replaced by a resident index.
#include "issl_b200_module.hpp"

#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <iostream>
#include <map>
#include <mutex>
#include <stdexcept>

namespace issl {
void set_last_error(const std::string& msg);
}

namespace {

// keeps the library status next to the reference's exception type
struct ModuleError : std::runtime_error {
    int code;
    ModuleError(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

std::mutex g_cache_mu;
std::map<std::string, issl_index*> g_cache;  // indexes kept open, keyed by (path, device, mapped)

// The index of a path, opened on first use and kept for the process. memoryMapped selects the
// host-list index (ISSLScoringModuleMMF's role); ISSL_WINDOW_SLICES sets its window (default 4).
issl_index* resident_index(const std::string& path, int device, bool mapped) {
    std::lock_guard<std::mutex> lock(g_cache_mu);
    const std::string key = path + "#" + std::to_string(device) + (mapped ? "#mapped" : "");
    auto it = g_cache.find(key);
    if (it != g_cache.end()) return it->second;
    issl_index* ix = nullptr;
    const char* w = std::getenv("ISSL_WINDOW_SLICES");
    const int rc = mapped ? issl_open_mapped(path.c_str(), device, w ? static_cast<uint32_t>(std::atoi(w)) : 4u, &ix)
                          : issl_open(path.c_str(), device, &ix);
    if (rc != ISSL_OK) throw ModuleError(rc, issl_last_error());
    g_cache[key] = ix;
    return ix;
}

}  // namespace

ISSLScoringModule::ISSLScoringModule(const cracklingConfig& cfg) {
    // specificityModule::specificityModule, lib/specificityModule.cpp:3-8
    toolIsSelected = cfg.offTarget.enabled;
    optimsationLevel = cfg.general.optimisation;
    consensusN = cfg.consensus.n;
    config = cfg.offTarget;
    ISSLIndex = cfg.input.offtargetSites;
    const char* dev = std::getenv("ISSL_DEVICE");
    device = dev ? std::atoi(dev) : 0;
    switch (config.method) {  // lib/ISSLScoringModule.cpp:24-49
        case otScoreMethod::mitAndCfd:
        case otScoreMethod::mitOrCfd:
        case otScoreMethod::avgMitCfd:
        case otScoreMethod::mit:
        case otScoreMethod::cfd:
            break;
        default:
            throw std::runtime_error("Scoring method is not valid.");
    }
}

bool ISSLScoringModule::processGuide(const guideResults& guide) const {
    // lib/ISSLScoringModule.cpp:488-513
    if (optimsationLevel == optimisationLevel::ultralow) return true;
    if (!guide.isUnique) return false;
    if (optimsationLevel == optimisationLevel::medium || optimsationLevel == optimisationLevel::high) {
        if (guide.consensusCount < consensusN) return false;
        if (guide.passedBowtie2 == ISSL_CODE_REJECTED) return false;
    }
    return true;
}

void ISSLScoringModule::run(std::vector<guideResults>& candidateGuides) {
    if (!toolIsSelected) {
        std::cout << "Off-target scoring has been configured not to run. Skipping Off-target scoring" << std::endl;
        return;
    }
    issl_index* ix = resident_index(ISSLIndex.string(), device, config.memoryMapped);
    std::vector<size_t> picked;
    picked.reserve(candidateGuides.size());
    for (size_t i = 0; i < candidateGuides.size(); i++)
        if (processGuide(candidateGuides[i])) picked.push_back(i);
    const size_t n = picked.size();
    std::vector<char> seqs(n * 20, 0);
    for (size_t k = 0; k < n; k++) {
        const std::string& s = candidateGuides[picked[k]].seq;
        std::memcpy(seqs.data() + 20 * k, s.data(), s.size() < 20 ? s.size() : 20);
    }
    std::vector<double> mit(n), cfd(n);
    std::vector<char> code(n);
    if (n) {
        const int rc = issl_score(ix, seqs.data(), 20, n, static_cast<int>(config.method), config.scoreThreshold, 4,
                                  mit.data(), cfd.data(), code.data(), nullptr, nullptr);
        if (rc != ISSL_OK) throw ModuleError(rc, issl_last_error());
    }
    size_t failed = 0;
    for (size_t k = 0; k < n; k++) {
        guideResults& g = candidateGuides[picked[k]];
        g.mitOfftargetscore = mit[k];
        g.cfdOfftargetscore = cfd[k];
        g.passedOffTargetScore = code[k];
        failed += code[k] == ISSL_CODE_REJECTED;
    }
    std::cout << "\t" << failed << " of " << n << " failed here." << std::endl;
}

extern "C" int issl_module_run(const char* index_path, int method, double threshold, int optimisation,
                               int consensus_n, int flags, size_t n, const char* seqs, size_t stride,
                               const uint8_t* is_unique, const int8_t* consensus_count, const char* passed_bowtie2,
                               double* mit_out, double* cfd_out, char* code_out) {
    try {
        if (!index_path || (n && (!seqs || !mit_out || !cfd_out || !code_out))) return ISSL_ERR_ARG;
        cracklingConfig cfg;
        cfg.input.offtargetSites = index_path;
        cfg.offTarget.method = static_cast<otScoreMethod>(method);
        cfg.offTarget.scoreThreshold = threshold;
        cfg.offTarget.enabled = (flags & ISSL_MODULE_ENABLED) != 0;
        cfg.offTarget.memoryMapped = (flags & ISSL_MODULE_MEMORY_MAPPED) != 0;
        cfg.general.optimisation = static_cast<optimisationLevel>(optimisation);
        cfg.consensus.n = static_cast<uint8_t>(consensus_n);
        std::vector<guideResults> guides(n);
        for (size_t i = 0; i < n; i++) {
            const char* s = seqs + i * stride;
            guides[i].seq.assign(s, strnlen(s, stride));
            guides[i].isUnique = is_unique ? is_unique[i] != 0 : true;
            guides[i].consensusCount = consensus_count ? consensus_count[i] : 0;
            guides[i].passedBowtie2 = passed_bowtie2 ? passed_bowtie2[i] : '?';
            // outputs are in/out: guides the filter skips keep what the caller passed in
            guides[i].mitOfftargetscore = mit_out[i];
            guides[i].cfdOfftargetscore = cfd_out[i];
            guides[i].passedOffTargetScore = code_out[i];
        }
        ISSLScoringModule module(cfg);
        module.run(guides);
        for (size_t i = 0; i < n; i++) {
            mit_out[i] = guides[i].mitOfftargetscore;
            cfd_out[i] = guides[i].cfdOfftargetscore;
            code_out[i] = guides[i].passedOffTargetScore;
        }
        return ISSL_OK;
    } catch (const ModuleError& e) {
        return e.code;
    } catch (const std::exception& e) {
        issl::set_last_error(e.what());
        return ISSL_ERR_ARG;
    }
}

extern "C" int issl_module_release_all(void) {
    std::lock_guard<std::mutex> lock(g_cache_mu);
    for (auto& kv : g_cache) issl_close(kv.second);
    g_cache.clear();
    return ISSL_OK;
}
