// The C entry points behind the header-only ISSLScoringModule (include/issl_b200_module.hpp):
// lib/ISSLScoringModule.cpp:13-513 with the scoring loop replaced by issl_score() and the per-call
// file read replaced by a resident index. Only C types cross this boundary, so the library
// exports no C++ symbol tied to the layout of cracklingConfig or guideResults.
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <string>
#include <vector>

#include "issl_internal.cuh"

extern "C" {
int issl_module_open(const char* index_path, int device, int memory_mapped, issl_index** out);
int issl_module_run(const char* index_path, int method, double threshold, int optimisation, int consensus_n,
                    int flags, size_t n, const char* seqs, size_t stride, const uint8_t* is_unique,
                    const int8_t* consensus_count, const char* passed_bowtie2, double* mit_out, double* cfd_out,
                    char* code_out);
int issl_module_release_all(void);
}

namespace {

constexpr int kModuleEnabled = 1;       // ISSL_MODULE_ENABLED
constexpr int kModuleMemoryMapped = 2;  // ISSL_MODULE_MEMORY_MAPPED
// optimisationLevel, include/util.hpp:21
constexpr int kUltralow = 0, kMedium = 2, kHigh = 3;

std::mutex g_cache_mu;
std::map<std::string, issl_index*> g_cache;  // indexes kept open, keyed by (path, device, mapped)

// processGuide, lib/ISSLScoringModule.cpp:488-513
bool process_guide(int optimisation, int consensus_n, bool is_unique, int consensus_count, char passed_bowtie2) {
    if (optimisation == kUltralow) return true;
    if (!is_unique) return false;
    if (optimisation == kMedium || optimisation == kHigh) {
        if (consensus_count < consensus_n) return false;
        if (passed_bowtie2 == ISSL_CODE_REJECTED) return false;
    }
    return true;
}

}  // namespace

extern "C" int issl_module_open(const char* index_path, int device, int memory_mapped, issl_index** out) {
    return issl::guarded([&] {
        ISSL_REQUIRE(index_path && out, ISSL_ERR_ARG, "issl_module_open: null argument");
        std::lock_guard<std::mutex> lock(g_cache_mu);
        const std::string key = std::string(index_path) + "#" + std::to_string(device) + (memory_mapped ? "#mapped" : "");
        auto it = g_cache.find(key);
        if (it != g_cache.end()) {
            *out = it->second;
            return;
        }
        issl_index* ix = nullptr;
        const char* w = std::getenv("ISSL_WINDOW_SLICES");
        const int rc = memory_mapped
                           ? issl_open_mapped(index_path, device, w ? static_cast<uint32_t>(std::atoi(w)) : 4u, &ix)
                           : issl_open(index_path, device, &ix);
        if (rc != ISSL_OK) throw issl::Error(rc, issl_last_error());
        g_cache[key] = ix;
        *out = ix;
    });
}

extern "C" int issl_module_run(const char* index_path, int method, double threshold, int optimisation,
                               int consensus_n, int flags, size_t n, const char* seqs, size_t stride,
                               const uint8_t* is_unique, const int8_t* consensus_count, const char* passed_bowtie2,
                               double* mit_out, double* cfd_out, char* code_out) {
    return issl::guarded([&] {
        ISSL_REQUIRE(index_path && (n == 0 || (seqs && mit_out && cfd_out && code_out)), ISSL_ERR_ARG,
                     "issl_module_run: null argument");
        // lib/ISSLScoringModule.cpp:24-49
        ISSL_REQUIRE(method >= ISSL_METHOD_MIT && method <= ISSL_METHOD_AVG_MIT_CFD, ISSL_ERR_ARG,
                     "Scoring method is not valid.");
        if (!(flags & kModuleEnabled)) return;  // the tool is not selected: nothing is touched
        std::vector<size_t> picked;
        picked.reserve(n);
        for (size_t i = 0; i < n; i++)
            if (process_guide(optimisation, consensus_n, is_unique ? is_unique[i] != 0 : true,
                              consensus_count ? consensus_count[i] : 0, passed_bowtie2 ? passed_bowtie2[i] : '?'))
                picked.push_back(i);
        const size_t k = picked.size();
        if (!k) return;
        const char* dev = std::getenv("ISSL_DEVICE");
        issl_index* ix = nullptr;
        const int rc = issl_module_open(index_path, dev ? std::atoi(dev) : 0, (flags & kModuleMemoryMapped) != 0, &ix);
        if (rc != ISSL_OK) throw issl::Error(rc, issl_last_error());
        // sequenceToSignature(seq, 20) reads the first 20 characters (:219, :469-476); a shorter
        // sequence reads as if padded with A
        std::vector<char> packed(k * issl::kSeqLen, 'A');
        for (size_t j = 0; j < k; j++) {
            const char* s = seqs + picked[j] * stride;
            std::memcpy(packed.data() + j * issl::kSeqLen, s, strnlen(s, std::min<size_t>(stride, issl::kSeqLen)));
        }
        std::vector<double> mit(k), cfd(k);
        std::vector<char> code(k);
        const int rs = issl_score(ix, packed.data(), issl::kSeqLen, k, method, threshold, issl::kMaxDist, mit.data(),
                                  cfd.data(), code.data(), nullptr, nullptr);
        if (rs != ISSL_OK) throw issl::Error(rs, issl_last_error());
        for (size_t j = 0; j < k; j++) {
            mit_out[picked[j]] = mit[j];
            cfd_out[picked[j]] = cfd[j];
            code_out[picked[j]] = code[j];
        }
    });
}

extern "C" int issl_module_release_all(void) {
    std::lock_guard<std::mutex> lock(g_cache_mu);
    for (auto& kv : g_cache) issl_close(kv.second);
    g_cache.clear();
    return ISSL_OK;
}
