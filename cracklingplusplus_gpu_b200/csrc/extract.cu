// Off-target extraction on the GPU: ExtractOfftargets/ExtractOfftargets.cpp:16-370.
//
// The reference splits its inputs into sequences (FASTA records, or one sequence per line of a
// plain text file; lines trimmed and upper-cased, :66-104), finds every site matching
//   forward  (?=([ACG][ACGT]{19}[ACGT][AG]G))   -> the match's first 20 bases          (:16, :124-138)
//   reverse  (?=(C[CT][ACGT][ACGT]{19}[TGC]))   -> the first 20 bases of its reverse complement
//                                                  (:17, :140-154; rc of lib/util.cpp:50-64)
// at every position (the lookahead makes matches overlap), and writes all of them sorted as text,
// one 20-mer per line, duplicates kept (:160-365, external merge sort of 30M-line batches).
// ISSLCreateIndex then counts the duplicates as occurrences (ISSLCreateIndex.cpp:393-417).
//
// Here the host only parses the inputs into one byte buffer of sequences separated by a
// non-base byte (no match can span two sequences); the device scans every position for both
// patterns, encodes each site as a 40-bit key with the first base most significant (so numeric
// order is the reference's lexicographic order), sorts the keys with the LSD radix sort, and
// either prints the sorted lines or run-length counts them into (signature, occurrences) pairs
// that build the resident index directly.
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <string>
#include <vector>

#include "issl_internal.cuh"
#include "scan.cuh"

namespace issl {
namespace {

constexpr int kSiteLen = 20;
constexpr int kMatchLen = 23;
constexpr uint8_t kSep = '\n';  // between sequences: not a base, so no match spans it

// ---- host: inputs -> sequences ------------------------------------------------------------
// boost::algorithm::trim / to_upper on ASCII (std::isspace / std::toupper in the C locale)
std::string trim_upper(const std::string& s) {
    size_t a = 0, b = s.size();
    while (a < b && std::isspace(static_cast<unsigned char>(s[a]))) a++;
    while (b > a && std::isspace(static_cast<unsigned char>(s[b - 1]))) b--;
    std::string r = s.substr(a, b - a);
    for (char& c : r) c = static_cast<char>(std::toupper(static_cast<unsigned char>(c)));
    return r;
}

// Appends the sequences of one input file to `out`, each followed by kSep (:66-104): a file whose
// first line starts with '>' is FASTA (records start at header lines, their lines concatenated);
// anything else holds one sequence per line.
void append_sequences(const std::string& path, std::string& out) {
    std::ifstream in(path, std::ios::binary);
    ISSL_REQUIRE(in.good(), ISSL_ERR_IO, "cannot open input " + path);
    std::string line;
    if (!std::getline(in, line)) return;
    if (!line.empty() && line[0] == '>') {
        while (std::getline(in, line)) {
            const std::string t = trim_upper(line);
            if (!t.empty() && t[0] == '>')
                out.push_back(static_cast<char>(kSep));
            else
                out += t;
        }
        out.push_back(static_cast<char>(kSep));
    } else {
        do {
            out += trim_upper(line);
            out.push_back(static_cast<char>(kSep));
        } while (std::getline(in, line));
    }
}

std::vector<std::string> expand_inputs(const char* const* inputs, size_t n) {
    namespace fs = std::filesystem;
    std::vector<std::string> files;
    for (size_t i = 0; i < n; i++) {
        ISSL_REQUIRE(inputs[i], ISSL_ERR_ARG, "null input path");
        const fs::path p(inputs[i]);
        std::error_code ec;
        if (fs::is_regular_file(p, ec)) {
            files.push_back(p.string());
        } else if (fs::is_directory(p, ec)) {  // every file of the directory (:41-48)
            std::vector<std::string> in_dir;
            for (const auto& e : fs::directory_iterator(p)) in_dir.push_back(e.path().string());
            std::sort(in_dir.begin(), in_dir.end());
            files.insert(files.end(), in_dir.begin(), in_dir.end());
        } else {
            throw Error(ISSL_ERR_IO, std::string("no such input file or directory: ") + inputs[i]);
        }
    }
    return files;
}

// ---- device: matches -> keys ----------------------------------------------------------------
__device__ __forceinline__ int base_code(uint8_t c) {  // A C G T -> 0 1 2 3, anything else -1
    return c == 'A' ? 0 : c == 'C' ? 1 : c == 'G' ? 2 : c == 'T' ? 3 : -1;
}

// Forward site at i: s[i] in ACG, s[i+1..i+20] bases, s[i+21] in AG, s[i+22] == G.
// Reverse site at i: s[i] == C, s[i+1] in CT, s[i+2..i+21] bases, s[i+22] in CGT; the site is the
// reverse complement of s[i+3..i+22]. Key: base j of the 20-mer at bits 2 (19 - j).
__device__ __forceinline__ void match_at(const uint8_t* s, uint64_t i, uint64_t n, bool& fwd, bool& rev,
                                         uint64_t& kf, uint64_t& kr) {
    fwd = rev = false;
    if (i + kMatchLen > n) return;
    const uint8_t c0 = s[i], c1 = s[i + 1], c21 = s[i + 21], c22 = s[i + 22];
    const bool f_ends = (c0 == 'A' || c0 == 'C' || c0 == 'G') && (c21 == 'A' || c21 == 'G') && c22 == 'G';
    const bool r_ends = c0 == 'C' && (c1 == 'C' || c1 == 'T') && (c22 == 'C' || c22 == 'G' || c22 == 'T');
    if (!f_ends && !r_ends) return;
    bool ok = true;
    uint64_t key = 0;
    for (int j = 1; j <= 21; j++) {  // positions 1..21 must all be bases for either pattern
        const int b = base_code(s[i + j]);
        if (b < 0) {
            ok = false;
            break;
        }
    }
    if (!ok) return;
    if (f_ends) {
        for (int j = 0; j < kSiteLen; j++) key = (key << 2) | static_cast<uint64_t>(base_code(s[i + j]));
        kf = key;
        fwd = true;
    }
    if (r_ends) {
        key = 0;
        for (int j = 0; j < kSiteLen; j++)  // complement of s[i+22-j]
            key = (key << 2) | static_cast<uint64_t>(3 - base_code(s[i + 22 - j]));
        kr = key;
        rev = true;
    }
}

__global__ void k_count_matches(const uint8_t* __restrict__ s, uint64_t n, uint64_t per, uint32_t* __restrict__ cnt,
                                uint64_t nchunks) {
    for (uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; c < nchunks;
         c += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint32_t k = 0;
        const uint64_t e = std::min<uint64_t>(n, (c + 1) * per);
        for (uint64_t i = c * per; i < e; i++) {
            bool f, r;
            uint64_t kf, kr;
            match_at(s, i, n, f, r, kf, kr);
            k += f + r;
        }
        cnt[c] = k;
    }
}

// Keys in the reference's emission order inside a chunk (forward, then reverse, per position;
// the order does not matter after the sort).
__global__ void k_emit_keys(const uint8_t* __restrict__ s, uint64_t n, uint64_t per, const uint64_t* __restrict__ off,
                            uint64_t nchunks, uint64_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    for (uint64_t c = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; c < nchunks;
         c += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t o = off[c];
        const uint64_t e = std::min<uint64_t>(n, (c + 1) * per);
        for (uint64_t i = c * per; i < e; i++) {
            bool f, r;
            uint64_t kf, kr;
            match_at(s, i, n, f, r, kf, kr);
            if (f) {
                keys[o] = kf;
                vals[o] = static_cast<uint32_t>(o);
                o++;
            }
            if (r) {
                keys[o] = kr;
                vals[o] = static_cast<uint32_t>(o);
                o++;
            }
        }
    }
}

__global__ void k_keys_to_text(const uint64_t* __restrict__ keys, uint64_t n, char* __restrict__ out) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t k = keys[i];
        char* o = out + i * (kSiteLen + 1);
        for (int j = 0; j < kSiteLen; j++) o[j] = "ACGT"[(k >> (2 * (kSiteLen - 1 - j))) & 3u];
        o[kSiteLen] = '\n';
    }
}

// run heads of the sorted keys: 1 where a new site starts
__global__ void k_run_heads(const uint64_t* __restrict__ keys, uint64_t n, uint32_t* __restrict__ head) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        head[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

struct LoadU32 {
    const uint32_t* p;
    __device__ uint32_t operator()(uint64_t i) const { return p[i]; }
};
struct StoreExcl {
    uint32_t* p;
    __device__ void operator()(uint64_t i, uint32_t ex, uint32_t) const { p[i] = ex; }
};
struct LoadU32As64 {
    const uint32_t* p;
    __device__ uint64_t operator()(uint64_t i) const { return p[i]; }
};
struct StoreExcl64 {
    uint64_t* p;
    __device__ void operator()(uint64_t i, uint64_t ex, uint64_t) const { p[i] = ex; }
};

// Site u = run u of the sorted keys: its ISSL signature (base j at bits 2j, the reference's
// sequenceToSignature) and its length (occurrences).
__global__ void k_runs_to_sites(const uint64_t* __restrict__ keys, uint64_t n, const uint32_t* __restrict__ head,
                                const uint32_t* __restrict__ rank, uint64_t* __restrict__ sigs,
                                uint32_t* __restrict__ start) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (!head[i]) continue;
        const uint64_t k = keys[i];
        uint64_t sig = 0;
        for (int j = 0; j < kSiteLen; j++) sig |= ((k >> (2 * (kSiteLen - 1 - j))) & 3ull) << (2 * j);
        sigs[rank[i]] = sig;
        start[rank[i]] = static_cast<uint32_t>(i);
    }
}

__global__ void k_run_lengths(const uint32_t* __restrict__ start, uint64_t u, uint64_t n, uint32_t* __restrict__ occ) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < u;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        occ[i] = (i + 1 < u ? start[i + 1] : static_cast<uint32_t>(n)) - start[i];
}

inline unsigned grid_for(uint64_t n, unsigned threads = 256) {
    uint64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148ull * 32) b = 148ull * 32;
    return static_cast<unsigned>(b);
}

// The sorted site keys of the inputs, on the device.
struct Extracted {
    DevBuf<uint64_t> keys_a, keys_b;
    DevBuf<uint32_t> vals_a, vals_b;
    uint64_t* keys = nullptr;  // sorted, n entries
    uint64_t n = 0;
};

void extract_sorted(const std::vector<std::string>& files, Extracted& x, cudaStream_t st) {
    std::string seq;
    for (const auto& f : files) append_sequences(f, seq);
    const uint64_t n = seq.size();
    ISSL_REQUIRE(n < (1ull << 40), ISSL_ERR_UNSUPPORTED, "inputs above 2^40 bytes");
    if (n == 0) return;
    DevBuf<uint8_t> d_seq;
    d_seq.reserve(n + kMatchLen);
    ISSL_CUDA(cudaMemcpyAsync(d_seq.p, seq.data(), n, cudaMemcpyHostToDevice, st));
    ISSL_CUDA(cudaMemsetAsync(d_seq.p + n, 0, kMatchLen, st));
    const uint64_t per = 64;  // positions per chunk
    const uint64_t nchunks = (n + per - 1) / per;
    ISSL_REQUIRE(nchunks < 0xFFFFFFFFull, ISSL_ERR_UNSUPPORTED, "inputs too large");
    DevBuf<uint32_t> cnt;
    DevBuf<uint64_t> off, total, scan_tmp;
    cnt.reserve(nchunks);
    off.reserve(nchunks + 1);
    total.reserve(1);
    scan_tmp.reserve(kScanBlocks + 4);
    k_count_matches<<<grid_for(nchunks), 256, 0, st>>>(d_seq.p, n, per, cnt.p, nchunks);
    device_scan<uint64_t, OpSum>(LoadU32As64{cnt.p}, StoreExcl64{off.p}, nullptr, nchunks, scan_tmp.p, total.p, st);
    uint64_t m = 0;
    ISSL_CUDA(cudaMemcpyAsync(&m, total.p, 8, cudaMemcpyDeviceToHost, st));
    ISSL_CUDA(cudaStreamSynchronize(st));
    ISSL_REQUIRE(m < 0xFFFFFFFFull, ISSL_ERR_UNSUPPORTED, "2^32 or more off-target sites");
    x.n = m;
    if (m == 0) return;
    x.keys_a.reserve(m);
    x.keys_b.reserve(m);
    x.vals_a.reserve(m);
    x.vals_b.reserve(m);
    k_emit_keys<<<grid_for(nchunks), 256, 0, st>>>(d_seq.p, n, per, off.p, nchunks, x.keys_a.p, x.vals_a.p);
    ISSL_CUDA(cudaGetLastError());
    const size_t tb = radix_sort_temp_bytes(m, true);
    DevBuf<uint8_t> temp;
    temp.reserve(tb);
    uint64_t* ko = nullptr;
    uint32_t* vo = nullptr;
    radix_sort_pairs_u64(x.keys_a.p, x.vals_a.p, x.keys_b.p, x.vals_b.p, m, 2 * kSiteLen, temp.p, tb, st, &ko, &vo);
    x.keys = ko;
    ISSL_CUDA(cudaStreamSynchronize(st));
}

}  // namespace
}  // namespace issl

using issl::guarded;

extern "C" {

int issl_extract_offtargets(const char* const* inputs, size_t n_inputs, const char* out_path, int device,
                            uint64_t* n_offtargets) {
    return guarded([&] {
        ISSL_REQUIRE(inputs && n_inputs > 0 && out_path, ISSL_ERR_ARG, "issl_extract_offtargets: null argument");
        ISSL_CUDA(cudaSetDevice(device));
        const auto files = issl::expand_inputs(inputs, n_inputs);
        cudaStream_t st;
        ISSL_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        struct G {
            cudaStream_t s;
            ~G() { cudaStreamDestroy(s); }
        } g{st};
        issl::Extracted x;
        issl::extract_sorted(files, x, st);
        FILE* fp = std::fopen(out_path, "wb");
        ISSL_REQUIRE(fp, ISSL_ERR_IO, std::string("cannot write ") + out_path);
        struct F {
            FILE* f;
            ~F() { std::fclose(f); }
        } ff{fp};
        // the text, produced on the device in slices of at most 64M lines
        const uint64_t line = issl::kSiteLen + 1, slab = 64ull << 20;
        if (x.n) {
            issl::DevBuf<char> d_txt;
            std::vector<char> h_txt;
            const uint64_t lines = std::min<uint64_t>(x.n, slab);
            d_txt.reserve(lines * line);
            h_txt.resize(lines * line);
            for (uint64_t i = 0; i < x.n; i += slab) {
                const uint64_t k = std::min<uint64_t>(slab, x.n - i);
                issl::k_keys_to_text<<<issl::grid_for(k), 256, 0, st>>>(x.keys + i, k, d_txt.p);
                ISSL_CUDA(cudaMemcpyAsync(h_txt.data(), d_txt.p, k * line, cudaMemcpyDeviceToHost, st));
                ISSL_CUDA(cudaStreamSynchronize(st));
                ISSL_REQUIRE(std::fwrite(h_txt.data(), 1, k * line, fp) == k * line, ISSL_ERR_IO,
                             std::string("short write to ") + out_path);
            }
        }
        if (n_offtargets) *n_offtargets = x.n;
    });
}

int issl_build_from_sequences(const char* const* inputs, size_t n_inputs, const uint64_t* slice_masks,
                              uint64_t n_slices, int device, issl_index** out, uint64_t* n_offtargets) {
    return guarded([&] {
        ISSL_REQUIRE(inputs && n_inputs > 0 && slice_masks && out, ISSL_ERR_ARG,
                     "issl_build_from_sequences: null argument");
        *out = nullptr;
        ISSL_CUDA(cudaSetDevice(device));
        const auto files = issl::expand_inputs(inputs, n_inputs);
        cudaStream_t st;
        ISSL_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        struct G {
            cudaStream_t s;
            ~G() { cudaStreamDestroy(s); }
        } g{st};
        uint64_t u = 0;
        auto ix = std::make_unique<issl_index>();
        ix->device = device;
        ix->seq_len = issl::kSiteLen;
        ix->n_slices = n_slices;
        ix->masks.assign(slice_masks, slice_masks + n_slices);
        {
            issl::Extracted x;
            issl::extract_sorted(files, x, st);
            ISSL_REQUIRE(x.n > 0, ISSL_ERR_FORMAT, "the inputs hold no off-target sites");
            // unique sites (ids in sorted order, as ISSLCreateIndex assigns them) and their counts
            issl::DevBuf<uint32_t> head, rank, start, total32, scan_tmp;
            head.reserve(x.n);
            rank.reserve(x.n);
            total32.reserve(1);
            scan_tmp.reserve(issl::kScanBlocks + 4);
            issl::k_run_heads<<<issl::grid_for(x.n), 256, 0, st>>>(x.keys, x.n, head.p);
            issl::device_scan<uint32_t, issl::OpSum>(issl::LoadU32{head.p}, issl::StoreExcl{rank.p}, nullptr, x.n,
                                                     scan_tmp.p, total32.p, st);
            uint32_t uu = 0;
            ISSL_CUDA(cudaMemcpyAsync(&uu, total32.p, 4, cudaMemcpyDeviceToHost, st));
            ISSL_CUDA(cudaStreamSynchronize(st));
            u = uu;
            ix->n_sites = u;
            ix->sigs.reserve(u);
            ix->occ.reserve(u);
            start.reserve(u);
            issl::k_runs_to_sites<<<issl::grid_for(x.n), 256, 0, st>>>(x.keys, x.n, head.p, rank.p, ix->sigs.p,
                                                                        start.p);
            issl::k_run_lengths<<<issl::grid_for(u), 256, 0, st>>>(start.p, u, x.n, ix->occ.p);
            ISSL_CUDA(cudaGetLastError());
            ISSL_CUDA(cudaStreamSynchronize(st));
            if (n_offtargets) *n_offtargets = x.n;
        }  // the keys are freed before the index is built
        issl::build_from_device_sites(ix.get(), ix->sigs.p, ix->occ.p, st);
        *out = ix.release();
    });
}

}  // extern "C"
