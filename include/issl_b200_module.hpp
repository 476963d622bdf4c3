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
// util.hpp first, so the reference's own cracklingConfig / guideResults are used. Without it, this
// header declares minimal mirrors of those types (field names and meanings as in util.hpp).
#pragma once

#include <cstdint>
#include <filesystem>
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

class ISSLScoringModule {
   public:
    explicit ISSLScoringModule(const cracklingConfig& config);
    void run(std::vector<guideResults>& candidateGuides);

   private:
    bool processGuide(const guideResults& guide) const;
    offTargetConfig config;
    std::filesystem::path ISSLIndex;
    bool toolIsSelected;
    optimisationLevel optimsationLevel;
    uint8_t consensusN;
    int device;
};

extern "C" {
// C entry used by language bindings to drive ISSLScoringModule::run on a guide batch:
// per guide the 20+ character sequence (at seqs + i*stride), isUnique, consensusCount and
// passedBowtie2 in; mitOfftargetscore, cfdOfftargetscore and passedOffTargetScore in/out (guides
// the filter skips keep the values passed in, as run() leaves them untouched). flags:
// ISSL_MODULE_ENABLED (offTarget.enabled), ISSL_MODULE_MEMORY_MAPPED (offTarget.memoryMapped).
// Returns ISSL_OK or an ISSL_ERR_* code.
#define ISSL_MODULE_ENABLED 1
#define ISSL_MODULE_MEMORY_MAPPED 2
int issl_module_run(const char* index_path, int method, double threshold, int optimisation, int consensus_n,
                    int flags, size_t n, const char* seqs, size_t stride, const uint8_t* is_unique,
                    const int8_t* consensus_count, const char* passed_bowtie2, double* mit_out, double* cfd_out,
                    char* code_out);
// Drops every index the module keeps resident (process-lifetime cache keyed by path).
int issl_module_release_all(void);
}
