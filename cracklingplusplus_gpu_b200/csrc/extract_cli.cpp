// Command-line mirror of ExtractOfftargets (ExtractOfftargets/ExtractOfftargets.cpp:19-370):
//   issl_extract_offtargets <output-file> {<input-file-1> <input-file-2> ... | <input-dir>}
// Same arguments and output file (every site, sorted, one 20-mer per line); the work runs on the
// GPU (ISSL_DEVICE selects it, default 0).
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <vector>

#include "issl_b200.h"

int main(int argc, char** argv) {
    if (argc < 3) {
        std::fprintf(stderr, "Usage: %s <output-file>  {<input-file-1> <input-file-2> ... <input-file-n> | <input-dir>}\n",
                     argv[0]);
        return 1;
    }
    const char* dev = std::getenv("ISSL_DEVICE");
    const auto t0 = std::chrono::steady_clock::now();
    std::vector<const char*> inputs(argv + 2, argv + argc);
    uint64_t n = 0;
    if (issl_extract_offtargets(inputs.data(), inputs.size(), argv[1], dev ? std::atoi(dev) : 0, &n) != ISSL_OK) {
        std::fprintf(stderr, "%s\n", issl_last_error());
        return 1;
    }
    const double s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    std::printf("Extracted %llu off-target sites in %.3f seconds\n", static_cast<unsigned long long>(n), s);
    return 0;
}
