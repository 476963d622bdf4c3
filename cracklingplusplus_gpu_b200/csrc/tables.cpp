// Penalty tables of the MIT and CFD off-target scores (host side).
//
// MIT: the reference looks each 1..4-mismatch mask up in a 6,195-entry hash map
// (precalculatedMITScores, lib/otScorePenalties.cpp:3-6199) whose values are the MIT local
// score of Hsu et al. 2013 (nbt.2647), as written out in calcMITLocalScore
// (ISSLCreateIndex/ISSLCreateIndex.cpp:235-261). Here the table is computed from that formula
// with the same operation order (this file is compiled with -ffp-contract=off) and stored
// densely by the combinatorial rank of the mismatch-position subset, so a device lookup is one
// load instead of a hash probe. A test checks every entry bit for bit against the reference map.
//
// CFD: position and PAM penalty tables of Doench et al. 2016 in the reference's index layout.
#include <cstdint>
#include <vector>

#include "issl_internal.cuh"

namespace issl {
namespace {
#include "cfd_tables.inc"

// Mismatch penalty per position (Hsu et al. 2013), ISSLCreateIndex.cpp:239.
const double kMitPenalty[20] = {0.0,   0.0,   0.014, 0.0,   0.0,   0.395, 0.317,
                                0.0,   0.389, 0.079, 0.445, 0.508, 0.613, 0.851,
                                0.732, 0.828, 0.615, 0.804, 0.685, 0.583};

double mit_local_score(const uint64_t* pos, uint64_t length) {
    double t1 = 1.0, t2, t3, d = 0.0;
    for (uint64_t i = 0; i < length; ++i) t1 = t1 * (1.0 - kMitPenalty[pos[i]]);
    if (length == 1) {
        d = 19.0;
    } else {
        for (uint64_t i = 0; i < length - 1; ++i) d += static_cast<double>(pos[i + 1] - pos[i]);
        d = d / static_cast<double>(length - 1);
    }
    t2 = 1.0 / ((19.0 - d) / 19.0 * 4.0 + 1);
    t3 = 1.0 / static_cast<double>(length * length);
    return t1 * t2 * t3 * 100;
}

uint64_t binom(uint64_t n, uint64_t k) {
    if (k > n) return 0;
    uint64_t r = 1;
    for (uint64_t i = 1; i <= k; i++) r = r * (n - k + i) / i;
    return r;
}
}  // namespace

// rank of a 1..4-subset {p_1 < ... < p_k} of 20 positions:
//   base[k] + sum_i C(p_i, i)   (combinatorial number system; base = 0, 20, 210, 1350)
uint32_t mit_rank(uint32_t mask20) {
    static const uint32_t base[5] = {0, 0, 20, 210, 1350};
    uint32_t r = 0, i = 0;
    for (uint32_t p = 0; p < 20; p++)
        if (mask20 >> p & 1u) r += static_cast<uint32_t>(binom(p, ++i));
    return base[i] + r;
}

const std::vector<double>& mit_rank_table() {
    static const std::vector<double> table = [] {
        std::vector<double> t(6195, 0.0);
        for (uint32_t m = 1; m < (1u << 20); m++) {
            int k = __builtin_popcount(m);
            if (k > 4) continue;
            uint64_t p[4];
            int n = 0;
            for (uint64_t j = 0; j < 20; j++)
                if (m >> j & 1u) p[n++] = j;
            t[mit_rank(m)] = mit_local_score(p, static_cast<uint64_t>(n));
        }
        return t;
    }();
    return table;
}

const double* cfd_pos_table() { return kCfdPos; }
const double* cfd_pam_table() { return kCfdPam; }

}  // namespace issl

extern "C" int issl_tables(uint64_t* mit_masks, double* mit_scores, double* cfd_pos320,
                           double* cfd_pam16) {
    return issl::guarded([&] {
        const auto& t = issl::mit_rank_table();
        int n = 0;
        for (uint32_t m = 1; m < (1u << 20); m++) {
            if (__builtin_popcount(m) > 4) continue;
            uint64_t wide = 0;
            for (int p = 0; p < 20; p++) wide |= static_cast<uint64_t>((m >> p) & 1u) << (2 * p);
            if (mit_masks) mit_masks[n] = wide;
            if (mit_scores) mit_scores[n] = t[issl::mit_rank(m)];
            n++;
        }
        if (cfd_pos320)
            for (int i = 0; i < 320; i++) cfd_pos320[i] = issl::cfd_pos_table()[i];
        if (cfd_pam16)
            for (int i = 0; i < 16; i++) cfd_pam16[i] = issl::cfd_pam_table()[i];
    });
}
