// Drop-in ISSLScoringModule backed by the B200 library.
//
// Same public surface as the reference's class (include/ISSLScoringModule.hpp:15-29):
//     ISSLScoringModule(const cracklingConfig& config);
//     void run(std::vector<guideResults>& candidateGuides);
// with the same configuration fields (offTarget.{enabled, method, scoreThreshold},
// input.offtargetSites, general.optimisation, consensus.n), the same per-guide filter
// (processGuide, lib/ISSLScoringModule.cpp:488-513), the same written fields
// (mitOfftargetscore, cfdOfftargetscore, passedOffTargetScore) and the same error convention
// (std::runtime_error). The difference: the index is loaded into HBM once per path and stays
// resident for every later run(), instead of being read from disk on every call.
//
// Embedding in the reference: define ISSL_B200_USE_REFERENCE_TYPES and include the reference's
// util.hpp first, so the reference's own cracklingConfig / guideResults are used (include/dropin/
// ISSLScoringModule.hpp does exactly that, in place of the reference's header). Without it, this
// header declares minimal mirrors of those types (field names and meanings as in util.hpp). The
// class is header-only and the library behind it exports only C entry points, so programs built
// against either type world link the same libissl_b200.so.
#pragma once

#include <algorithm>
#include <cstddef>
#include <cstdint>
#include <filesystem>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "issl_b200.h"

#ifndef ISSL_B200_USE_REFERENCE_TYPES
#include <cfloat>
#include <climits>

// include/util.hpp:20-21
enum otScoreMethod { mit = 0, cfd = 1, mitAndCfd = 2, mitOrCfd = 3, avgMitCfd = 4 };
enum optimisationLevel { ultralow = 0, low = 1, medium = 2, high = 3 };

struct generalConfig {
    std::string name;
    optimisationLevel optimisation = ultralow;
};
struct consensusConfig {
    uint8_t n = 0;
};
struct inputConfig {
    std::filesystem::path offtargetSites;
};
struct offTargetConfig {  // include/util.hpp:64-72
    bool enabled = true;
    bool memoryMapped = false;  // true: the lists stay in host memory (issl_open_mapped) and are
                                // streamed per call, for indexes larger than HBM
    otScoreMethod method = mitAndCfd;
    uint8_t threads = 0;        // accepted, unused: the GPU replaces the OpenMP team
    uint64_t pageLen = 0;
    double scoreThreshold = 75.0;
};
struct cracklingConfig {
    generalConfig general;
    consensusConfig consensus;
    inputConfig input;
    offTargetConfig offTarget;
};
// the fields of include/util.hpp:112-140 that the off-target module reads or writes
struct guideResults {
    std::string seq = "-";
    bool isUnique = false;
    int8_t consensusCount = 0;
    char passedBowtie2 = '?';
    char passedOffTargetScore = '?';
    double mitOfftargetscore = -DBL_MAX;
    double cfdOfftargetscore = -DBL_MAX;
};
#endif

extern "C" {
// C entries behind the class below (and the language bindings). They take plain C types only, so
// the shared library exports no C++ symbol that depends on the layout of cracklingConfig or
// guideResults: the class is compiled in the caller's type world, the reference's or the mirrors.
//
// issl_module_open: the resident index of a path, opened on first use and kept for the process
// (keyed by path, device and memory_mapped; memory_mapped selects the host-list index of
// issl_open_mapped, ISSL_WINDOW_SLICES sets its window, default 4).
int issl_module_open(const char* index_path, int device, int memory_mapped, issl_index** out);
// issl_module_run: ISSLScoringModule::run on a guide batch. Per guide the 20+ character sequence
// (at seqs + i*stride), isUnique, consensusCount and passedBowtie2 in; mitOfftargetscore,
// cfdOfftargetscore and passedOffTargetScore in/out (guides the processGuide filter skips keep the
// values passed in, as run() leaves them untouched). flags: ISSL_MODULE_ENABLED
// (offTarget.enabled), ISSL_MODULE_MEMORY_MAPPED (offTarget.memoryMapped). The index is on the
// device named by ISSL_DEVICE (default 0). Returns ISSL_OK or an ISSL_ERR_* code.
#define ISSL_MODULE_ENABLED 1
#define ISSL_MODULE_MEMORY_MAPPED 2
int issl_module_run(const char* index_path, int method, double threshold, int optimisation, int consensus_n,
                    int flags, size_t n, const char* seqs, size_t stride, const uint8_t* is_unique,
                    const int8_t* consensus_count, const char* passed_bowtie2, double* mit_out, double* cfd_out,
                    char* code_out);
// Drops every index the module keeps resident (process-lifetime cache keyed by path).
int issl_module_release_all(void);
}

// Header-only: every member is defined inline here, so each program compiles the class against
// its own cracklingConfig / guideResults (include/ISSLScoringModule.hpp:15-29 of the reference for
// the surface, lib/ISSLScoringModule.cpp for the behaviour).
class ISSLScoringModule {
   public:
    explicit ISSLScoringModule(const cracklingConfig& cfg)
        : config(cfg.offTarget),
          ISSLIndex(cfg.input.offtargetSites),
          toolIsSelected(cfg.offTarget.enabled),
          optimsationLevel(cfg.general.optimisation),
          consensusN(cfg.consensus.n) {
        // specificityModule::specificityModule (lib/specificityModule.cpp:3-8) and the method
        // check of lib/ISSLScoringModule.cpp:24-49
        switch (config.method) {
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

    // lib/ISSLScoringModule.cpp:154-466: scores every guide that passes the processGuide filter
    // (:488-513) and writes its MIT and CFD scores and its accept code
    void run(std::vector<guideResults>& candidateGuides) {
        if (!toolIsSelected) {
            std::cout << "Off-target scoring has been configured not to run. Skipping Off-target scoring"
                      << std::endl;
            return;
        }
        const size_t n = candidateGuides.size();
        size_t stride = 20;
        for (const guideResults& g : candidateGuides) stride = std::max(stride, g.seq.size());
        std::vector<char> seqs(n * stride, 0);
        std::vector<uint8_t> uniq(n);
        std::vector<int8_t> cons(n);
        std::vector<char> bt2(n), code(n, 0);  // code 0: marks guides the filter skips
        std::vector<double> mit(n), cfd(n);
        for (size_t i = 0; i < n; i++) {
            const guideResults& g = candidateGuides[i];
            std::copy(g.seq.begin(), g.seq.end(), seqs.begin() + static_cast<std::ptrdiff_t>(i * stride));
            uniq[i] = g.isUnique ? 1 : 0;
            cons[i] = g.consensusCount;
            bt2[i] = g.passedBowtie2;
            mit[i] = g.mitOfftargetscore;
            cfd[i] = g.cfdOfftargetscore;
        }
        const int flags = ISSL_MODULE_ENABLED | (config.memoryMapped ? ISSL_MODULE_MEMORY_MAPPED : 0);
        const int rc = issl_module_run(ISSLIndex.string().c_str(), static_cast<int>(config.method),
                                       config.scoreThreshold, static_cast<int>(optimsationLevel), consensusN, flags,
                                       n, seqs.data(), stride, uniq.data(), cons.data(), bt2.data(), mit.data(),
                                       cfd.data(), code.data());
        if (rc != ISSL_OK) throw std::runtime_error(issl_last_error());
        size_t tested = 0, failed = 0;
        for (size_t i = 0; i < n; i++) {
            if (code[i] == 0) continue;  // skipped by the filter: left as it was
            guideResults& g = candidateGuides[i];
            g.mitOfftargetscore = mit[i];
            g.cfdOfftargetscore = cfd[i];
            g.passedOffTargetScore = code[i];
            tested++;
            failed += code[i] == ISSL_CODE_REJECTED;
        }
        std::cout << "\t" << failed << " of " << tested << " failed here." << std::endl;
    }

   private:
    offTargetConfig config;
    std::filesystem::path ISSLIndex;
    bool toolIsSelected;
    optimisationLevel optimsationLevel;
    uint8_t consensusN;
};
