// Test-infrastructure driver around the reference's own ISSLScoringModule.
//
// This file is part of the CPU checker, never of the shipped library. It is compiled
// together with the reference's lib/ISSLScoringModule.cpp, lib/specificityModule.cpp,
// lib/util.cpp and lib/otScorePenalties.cpp (read in place, see oracle/Makefile) and
// drives the drop-in entry point `ISSLScoringModule::run(std::vector<guideResults>&)`
// (include/ISSLScoringModule.hpp:15-29) exactly as the pipeline driver does
// (src/CracklingPlusPlus.cpp:74-81), then prints every guide's scores with full
// double precision so that restatements can be compared bit for bit.
//
// usage: ref_module_driver <index.issl> <guides.tsv> <method> <threshold>
//                          <optimisation> <consensusN> <enabled> <out.tsv>
//   guides.tsv: one guide per line: seq \t isUnique(0/1) \t consensusCount \t passedBowtie2 char
//   method: mit|cfd|mitAndCfd|mitOrCfd|avgMitCfd      optimisation: ultralow|low|medium|high
//   out.tsv: seq \t mit(%.17g) \t cfd(%.17g) \t passedOffTargetScore char
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "ISSLScoringModule.hpp"

int main(int argc, char** argv) {
    if (argc != 9) {
        std::fprintf(stderr,
                     "usage: %s index guides.tsv method threshold optimisation consensusN enabled out.tsv\n",
                     argv[0]);
        return 2;
    }
    cracklingConfig cfg{};
    cfg.input.offtargetSites = argv[1];
    cfg.offTarget.method = otScoreMethodMap.at(argv[3]);
    cfg.offTarget.scoreThreshold = std::atof(argv[4]);
    cfg.offTarget.threads = 8;
    cfg.offTarget.enabled = std::atoi(argv[7]) != 0;
    cfg.offTarget.memoryMapped = false;
    cfg.offTarget.pageLen = 0;
    cfg.general.optimisation = optimisationMap.at(argv[5]);
    cfg.consensus.n = static_cast<uint8_t>(std::atoi(argv[6]));

    std::vector<guideResults> guides;
    std::ifstream in(argv[2]);
    for (std::string line; std::getline(in, line);) {
        if (line.empty()) continue;
        std::istringstream ls(line);
        std::string seq, uniq, cons, bt2;
        std::getline(ls, seq, '\t');
        std::getline(ls, uniq, '\t');
        std::getline(ls, cons, '\t');
        std::getline(ls, bt2, '\t');
        guideResults g;
        g.seq = seq;
        g.isUnique = uniq.empty() ? true : (std::atoi(uniq.c_str()) != 0);
        g.consensusCount = static_cast<int8_t>(cons.empty() ? 0 : std::atoi(cons.c_str()));
        g.passedBowtie2 = bt2.empty() ? CODE_UNTESTED : bt2[0];
        guides.push_back(g);
    }

    ISSLScoringModule module(cfg);
    module.run(guides);

    FILE* out = std::fopen(argv[8], "w");
    if (!out) return 3;
    for (const auto& g : guides) {
        std::fprintf(out, "%s\t%.17g\t%.17g\t%c\n", g.seq.c_str(), g.mitOfftargetscore,
                     g.cfdOfftargetscore, g.passedOffTargetScore);
    }
    std::fclose(out);
    return 0;
}
