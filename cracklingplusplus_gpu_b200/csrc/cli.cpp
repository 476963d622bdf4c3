// issl_score_offtargets: the ISSLScoreOfftargets command line (ISSLScoreOfftargets.cpp:36-647) on
// the B200 library.
//
//   issl_score_offtargets <issltable> <query file> <max distance> <score-threshold>
//                         <and|or|avg|mit|cfd> [output file]
//
// Same argument meaning, query-file check (20 nt + LF per line, :252-265), stdout lines
// "seq<TAB>MIT<TAB>CFD" with %f (or -1 for a score the method does not compute, :597-608), timing
// lines, and the stderr execution summary with per-query off-target counts and the distinct
// off-target count (:528-556). Differences: the detailed results file is written to the path
// given as the sixth argument (the reference writes under a fixed Windows directory and needs the
// argument to exist), and max distance values other than 4 are clamped to 4, since the reference
// scores every site within 4 mismatches whatever the argument says (:292, :369).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "issl_b200.h"

namespace {
double secs(std::chrono::high_resolution_clock::time_point a, std::chrono::high_resolution_clock::time_point b) {
    return std::chrono::duration<double>(b - a).count();
}
}  // namespace

int main(int argc, char** argv) {
    using clk = std::chrono::high_resolution_clock;
    const auto t_total = clk::now();
    if (argc < 6) {
        std::fprintf(stderr,
                     "Usage: %s [issltable] [query file] [max distance] [score-threshold] [score-method] "
                     "[output-file-optional]\n",
                     argv[0]);
        return 1;
    }
    int max_dist = std::atoi(argv[3]);
    if (max_dist != 4) {
        std::fprintf(stderr, "Note: clamping maxDist from %d to 4 to match the reference's fixed bound.\n", max_dist);
        max_dist = 4;
    }
    const double threshold = std::atof(argv[4]);
    const std::string m = argv[5];
    int method;
    if (m == "and")
        method = ISSL_METHOD_MIT_AND_CFD;
    else if (m == "or")
        method = ISSL_METHOD_MIT_OR_CFD;
    else if (m == "avg")
        method = ISSL_METHOD_AVG_MIT_CFD;
    else if (m == "mit")
        method = ISSL_METHOD_MIT;
    else if (m == "cfd")
        method = ISSL_METHOD_CFD;
    else {
        std::fprintf(stderr, "Invalid scoring method. Acceptable options are: 'and', 'or', 'avg', 'mit', 'cfd'");
        return 1;
    }
    const bool calc_mit = method != ISSL_METHOD_CFD, calc_cfd = method != ISSL_METHOD_MIT;
    const char* dev = std::getenv("ISSL_DEVICE");

    const auto t_load = clk::now();
    issl_index* ix = nullptr;
    if (issl_open(argv[1], dev ? std::atoi(dev) : 0, &ix) != ISSL_OK) {
        std::fprintf(stderr, "%s\n", issl_last_error());
        return 1;
    }
    const auto t_load_end = clk::now();
    std::printf("Index loading time: %g seconds\n", secs(t_load, t_load_end));

    const auto t_query = clk::now();
    const size_t line = 21;
    FILE* fp = std::fopen(argv[2], "rb");
    if (!fp) {
        std::fprintf(stderr, "Failed to read in query file.\n");
        return 1;
    }
    std::fseek(fp, 0, SEEK_END);
    const long size = std::ftell(fp);
    std::fseek(fp, 0, SEEK_SET);
    if (size < 0 || static_cast<size_t>(size) % line != 0) {
        std::fprintf(stderr, "Error: query file is not a multiple of the expected line length (%zu)\n", line);
        std::fprintf(stderr, "The sequence length may be incorrect; alternatively, the line endings\n");
        std::fprintf(stderr, "may be something other than LF, or there may be junk at the end of the file.\n");
        return 1;
    }
    const size_t nq = static_cast<size_t>(size) / line;
    std::vector<char> data(static_cast<size_t>(size) + 1);
    if (size && std::fread(data.data(), static_cast<size_t>(size), 1, fp) < 1) {
        std::fprintf(stderr, "Failed to read in query file.\n");
        return 1;
    }
    std::fclose(fp);
    std::printf("Query loading time: %g seconds\n", secs(t_query, clk::now()));

    std::vector<double> mit(nq), cfd(nq);
    std::vector<char> code(nq);
    std::vector<uint64_t> count(nq);
    uint64_t distinct = 0;
    const auto t_issl = clk::now();
    if (issl_score(ix, data.data(), line, nq, method, threshold, max_dist, mit.data(), cfd.data(), code.data(),
                   count.data(), &distinct) != ISSL_OK) {
        std::fprintf(stderr, "%s\n", issl_last_error());
        return 1;
    }
    const auto t_issl_end = clk::now();
    std::printf("ISSL scoring time: %g seconds\n", secs(t_issl, t_issl_end));

    uint64_t total = 0;
    for (auto c : count) total += c;
    const double ms = secs(t_issl, t_issl_end) * 1000.0;
    std::fprintf(stderr, "\n=== EXECUTION SUMMARY ===\n");
    std::fprintf(stderr, "Total queries processed: %zu\n", nq);
    std::fprintf(stderr, "Total off-targets scored: %llu\n", static_cast<unsigned long long>(total));
    std::fprintf(stderr, "Average off-targets per query: %.2f\n", nq ? static_cast<double>(total) / nq : 0.0);
    std::fprintf(stderr, "Processing rate: %.2f queries/sec\n", ms > 0 ? nq * 1000.0 / ms : 0.0);
    std::fprintf(stderr, "Off-target scoring rate: %.2f off-targets/sec\n", ms > 0 ? total * 1000.0 / ms : 0.0);
    std::fprintf(stderr, "Distinct off-targets: %llu\n", static_cast<unsigned long long>(distinct));
    std::fprintf(stderr, "========================\n\n");

    FILE* out = nullptr;
    if (argc > 6) {
        out = std::fopen(argv[6], "w");
        if (out)
            std::fprintf(out, "# Query\tMIT_Score\tCFD_Score\tOfftarget_Count\n");
        else
            std::fprintf(stderr, "Error: Could not open output file: %s\n", argv[6]);
    }
    static const char kBase[4] = {'A', 'C', 'G', 'T'};
    char seq[21];
    seq[20] = 0;
    for (size_t i = 0; i < nq; i++) {
        // the printed sequence is decoded from the signature (signatureToSequence, :28-34)
        for (int j = 0; j < 20; j++) {
            const char c = data[i * line + j];
            seq[j] = kBase[c == 'C' ? 1 : c == 'G' ? 2 : c == 'T' ? 3 : 0];
        }
        std::printf("%s\t", seq);
        if (calc_mit) std::printf("%f\t", mit[i]); else std::printf("-1\t");
        if (calc_cfd) std::printf("%f\n", cfd[i]); else std::printf("-1\n");
        if (out) {
            std::fprintf(out, "%s\t", seq);
            if (calc_mit) std::fprintf(out, "%f\t", mit[i]); else std::fprintf(out, "-1\t");
            if (calc_cfd) std::fprintf(out, "%f\t", cfd[i]); else std::fprintf(out, "-1\t");
            std::fprintf(out, "%llu\n", static_cast<unsigned long long>(count[i]));
        }
    }
    if (out) {
        std::fclose(out);
        std::fprintf(stderr, "Detailed results saved to: %s\n", argv[6]);
    }
    issl_close(ix);
    std::printf("Total execution time: %g seconds\n", secs(t_total, clk::now()));
    return 0;
}
