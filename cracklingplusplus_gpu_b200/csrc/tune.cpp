// Autotuner of the scan's unit sizes (per bucket-size class), staging depth and persistent grid.
//
// Everything goes through the library's own C ABI: the sample is scored with
// issl_score_device under each candidate tuning and the pipeline's device time
// (issl_last_stats().total_ms, CUDA events) is compared. A candidate is kept only when it beats
// the best so far by more than 2%, so noise does not move the tuning. Results never depend on
// the tuning, only the time does.
#include <cuda_runtime.h>

#include <algorithm>
#include <fstream>
#include <sstream>
#include <string>

#include "issl_internal.cuh"

namespace issl {
namespace {

struct Sample {
    issl_index* ix;
    const uint64_t* d_sigs;
    size_t n;
    int method, max_dist;
    double threshold;
    DevBuf<double> mit, cfd;
    DevBuf<char> code;
    DevBuf<uint64_t> count;
};

// best of `reps` runs of the pipeline under tuning t (after one untimed run)
double time_tuning(Sample& s, const issl_tuning& t, issl_score_stats* last, int reps = 3) {
    if (issl_set_tuning(s.ix, &t) != ISSL_OK) throw Error(ISSL_ERR_ARG, issl_last_error());
    double best = 1e30;
    for (int r = 0; r <= reps; r++) {
        const int rc = issl_score_device(s.ix, s.d_sigs, s.n, s.method, s.threshold, s.max_dist, s.mit.p, s.cfd.p,
                                         s.code.p, s.count.p, nullptr, nullptr);
        if (rc == ISSL_ERR_NOMEM) return 1e30;  // this tuning needs more memory than there is: skip it
        if (rc != ISSL_OK) throw Error(rc, issl_last_error());
        issl_score_stats st{};
        issl_last_stats(s.ix, &st);
        if (r > 0) best = std::min(best, st.total_ms);
        if (last) *last = st;
    }
    return best;
}

std::string cache_key(const issl_index* ix, size_t n) {
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, ix->device);
    std::ostringstream k;
    k << prop.name << "|sm" << prop.multiProcessorCount << "|sites" << ix->n_sites << "|n" << n << "|masks";
    for (uint64_t m : ix->masks) k << ':' << std::hex << m << std::dec;
    std::string s = k.str();
    std::replace(s.begin(), s.end(), ' ', '_');
    return s;
}

bool cache_lookup(const char* path, const std::string& key, issl_tuning& t) {
    std::ifstream f(path);
    std::string line;
    bool found = false;
    while (std::getline(f, line)) {  // the last entry of a key wins
        std::istringstream in(line);
        std::string k;
        issl_tuning c{};
        if (in >> k >> c.chunk[0] >> c.chunk[1] >> c.chunk[2] >> c.stages >> c.blocks_per_sm >> c.first_wave &&
            k == key) {
            t = c;
            found = true;
        }
    }
    return found;
}

void cache_store(const char* path, const std::string& key, const issl_tuning& t) {
    std::ofstream f(path, std::ios::app);
    ISSL_REQUIRE(f.good(), ISSL_ERR_IO, std::string("autotune: cannot write the cache file ") + path);
    f << key << ' ' << t.chunk[0] << ' ' << t.chunk[1] << ' ' << t.chunk[2] << ' ' << t.stages << ' '
      << t.blocks_per_sm << ' ' << t.first_wave << '\n';
}

}  // namespace
}  // namespace issl

extern "C" int issl_autotune(issl_index* ix, const uint64_t* d_sigs, size_t n, int method, double threshold,
                             int max_dist, const char* cache_path, issl_tuning* out, issl_tune_report* report) {
    using namespace issl;
    issl_tuning start{};
    if (ix) start = ix->tuning;
    const int rc = guarded([&] {
        ISSL_REQUIRE(ix && d_sigs && n > 0, ISSL_ERR_ARG, "issl_autotune: needs an index and a sample of guides");
        issl_tune_report rep{};
        const std::string key = cache_key(ix, n);
        issl_tuning best = ix->tuning;
        if (cache_path && cache_lookup(cache_path, key, best)) {
            if (issl_set_tuning(ix, &best) != ISSL_OK) throw Error(ISSL_ERR_FORMAT, issl_last_error());
            rep.from_cache = 1;
        } else {
            ISSL_CUDA(cudaSetDevice(ix->device));
            Sample s{ix, d_sigs, n, method, max_dist, threshold, {}, {}, {}, {}};
            s.mit.reserve(n);
            s.cfd.reserve(n);
            s.code.reserve(n);
            s.count.reserve(n);
            issl_score_stats st{};
            double best_ms = time_tuning(s, best, &st);
            rep.default_ms = best_ms;
            rep.configs_timed = 1;
            for (int c = 0; c < 3; c++) rep.class_probes[c] = st.class_probes[c];
            auto consider = [&](const issl_tuning& t) {
                const double ms = time_tuning(s, t, nullptr);
                rep.configs_timed++;
                if (ms < best_ms * 0.98) {
                    best_ms = ms;
                    best = t;
                }
            };
            // 1. staging depth
            const issl_tuning base = best;
            for (uint32_t stages = 2; stages <= 4; stages++)
                if (stages != base.stages) {
                    issl_tuning t = base;
                    t.stages = stages;
                    consider(t);
                }
            // 2. unit size of each bucket-size class the sample reaches, heaviest class first
            for (int c = 2; c >= 0; c--) {
                if (!rep.class_probes[c]) continue;
                const issl_tuning cur = best;
                for (uint32_t chunk : {1024u, 512u, 256u})
                    if (chunk != cur.chunk[c]) {
                        issl_tuning t = cur;
                        t.chunk[c] = chunk;
                        consider(t);
                    }
            }
            // 3. persistent grid: fewer blocks per SM than fit
            const issl_tuning cur = best;
            for (uint32_t b : {2u, 3u, 4u})
                if (b != cur.blocks_per_sm) {
                    issl_tuning t = cur;
                    t.blocks_per_sm = b;
                    consider(t);
                }
            // 4. slice waves
            const issl_tuning cur2 = best;
            for (uint32_t fw : {0u, 1u, 2u, 4u})
                if (fw != cur2.first_wave) {
                    issl_tuning t = cur2;
                    t.first_wave = fw;
                    consider(t);
                }
            rep.best_ms = best_ms;
            if (issl_set_tuning(ix, &best) != ISSL_OK) throw Error(ISSL_ERR_ARG, issl_last_error());
            if (cache_path) cache_store(cache_path, key, best);
        }
        if (out) *out = best;
        if (report) *report = rep;
    });
    // a failed sweep leaves the tuning the index had before the call
    if (rc != ISSL_OK && ix) {
        ix->tuning = start;
        ix->tuning_version++;
    }
    return rc;
}
