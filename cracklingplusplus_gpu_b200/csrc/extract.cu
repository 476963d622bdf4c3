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
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <cctype>
#include <cstdio>
#include <cstring>
#include <filesystem>
#include <fstream>
#include <string>
#include <thread>
#include <vector>

#include "issl_internal.cuh"
#include "scan.cuh"

namespace issl {
namespace {

constexpr int kSiteLen = 20;
constexpr uint8_t kSep = '\n';  // between sequences: not a base, so no match spans it

// ---- host: inputs -> sequences ------------------------------------------------------------
// boost::algorithm::trim / to_upper on ASCII (std::isspace / std::toupper in the C locale), as a
// table over bytes
struct CharTables {
    bool space[256];
    char upper[256];
    CharTables() {
        for (int c = 0; c < 256; c++) {
            space[c] = std::isspace(c) != 0;
            upper[c] = static_cast<char>(std::toupper(c));
        }
    }
};
const CharTables& char_tables() {
    static const CharTables t;
    return t;
}

// Appends line [b, e) trimmed and upper-cased, except a FASTA header line (fasta and its first
// character is '>'); returns its first character after trimming (0 if none).
char append_trimmed(const char* b, const char* e, bool fasta, std::string& out) {
    const CharTables& T = char_tables();
    while (b < e && T.space[static_cast<unsigned char>(*b)]) b++;
    while (e > b && T.space[static_cast<unsigned char>(e[-1])]) e--;
    if (b == e) return 0;
    const char first = T.upper[static_cast<unsigned char>(*b)];
    if (fasta && first == '>') return first;  // a header: not sequence
    const size_t at = out.size();
    out.resize(at + static_cast<size_t>(e - b));
    char* o = &out[at];
    for (; b < e; b++) *o++ = T.upper[static_cast<unsigned char>(*b)];
    return first;
}

// Whole lines [p, end) of one input: FASTA header lines become kSep (a new record), sequence
// lines are appended trimmed and upper-cased (their record's lines concatenate); in a plain file
// every line is followed by kSep. Lines end at '\n' as std::getline ends them.
void parse_lines(const char* p, const char* end, bool fasta, std::string& out) {
    while (p < end) {
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', static_cast<size_t>(end - p)));
        const char* e = nl ? nl : end;
        const char first = append_trimmed(p, e, fasta, out);
        if (!fasta || first == '>') out.push_back(static_cast<char>(kSep));
        p = nl ? nl + 1 : end;
    }
}

// Appends the sequences of one input file to `out`, each followed by kSep (:66-104): a file whose
// first line starts with '>' is FASTA (records start at header lines, their lines concatenated;
// the first header is skipped); anything else holds one sequence per line. Large files are cut
// at line starts into one piece per host thread; the pieces are parsed in parallel and joined in
// order, which gives exactly the sequential result (a piece's output depends only on its lines).
void append_sequences(const std::string& path, std::string& out) {
    FILE* fp = std::fopen(path.c_str(), "rb");
    ISSL_REQUIRE(fp, ISSL_ERR_IO, "cannot open input " + path);
    std::vector<char> buf;
    {
        std::fseek(fp, 0, SEEK_END);
        const long size = std::ftell(fp);
        std::fseek(fp, 0, SEEK_SET);
        buf.resize(size > 0 ? static_cast<size_t>(size) : 0);
        const size_t got = buf.empty() ? 0 : std::fread(buf.data(), 1, buf.size(), fp);
        std::fclose(fp);
        ISSL_REQUIRE(got == buf.size(), ISSL_ERR_IO, "short read of " + path);
    }
    if (buf.empty()) return;
    const char* p = buf.data();
    const char* end = p + buf.size();
    const bool fasta = *p == '>';  // the raw first line starts with '>'
    if (fasta) {
        const char* nl = static_cast<const char*>(std::memchr(p, '\n', buf.size()));
        p = nl ? nl + 1 : end;
    }
    const size_t bytes = static_cast<size_t>(end - p);
    const unsigned hw = std::max(1u, std::min(32u, std::thread::hardware_concurrency()));
    const unsigned T = bytes >= (8u << 20) ? hw : 1u;
    std::vector<const char*> cut(T + 1);
    cut[0] = p;
    cut[T] = end;
    for (unsigned t = 1; t < T; t++) {  // piece t starts at the first line start at or after its share
        const char* c = std::max(cut[t - 1], p + bytes / T * t);
        if (c > p && c < end && c[-1] != '\n') {
            const char* nl = static_cast<const char*>(std::memchr(c, '\n', static_cast<size_t>(end - c)));
            c = nl ? nl + 1 : end;
        }
        cut[t] = c;
    }
    std::vector<std::string> part(T);
    if (T == 1) {
        parse_lines(cut[0], cut[1], fasta, part[0]);
    } else {
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < T; t++)
            pool.emplace_back([&, t] {
                part[t].reserve(static_cast<size_t>(cut[t + 1] - cut[t]) + 16);
                parse_lines(cut[t], cut[t + 1], fasta, part[t]);
            });
        for (auto& th : pool) th.join();
    }
    size_t at = out.size(), total = 0;
    for (auto& s : part) total += s.size();
    out.resize(at + total + (fasta ? 1 : 0));
    std::vector<size_t> off(T);
    for (unsigned t = 0; t < T; t++) {
        off[t] = at;
        at += part[t].size();
    }
    if (T == 1) {
        std::memcpy(&out[off[0]], part[0].data(), part[0].size());
    } else {
        std::vector<std::thread> pool;
        for (unsigned t = 0; t < T; t++)
            pool.emplace_back([&, t] { std::memcpy(&out[off[t]], part[t].data(), part[t].size()); });
        for (auto& th : pool) th.join();
    }
    if (fasta) out[at] = static_cast<char>(kSep);  // the last record's end
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
// Tiles of kTile positions, one 32-position word per thread. The block first packs the tile's
// bases into shared memory, one word per thread, the last thread packing the word after the tile
// (which the last windows reach into) and testing none: per word,
// the 2-bit codes (A C G T -> 0 1 2 3, base j at bits 2j) and three bit planes with one bit per
// position: valid (the byte is A, C, G or T), lo and hi (the code's two bits). Each thread then
// tests its 32 positions at once with shifts of the planes of its word and the next:
//   forward at k   positions k..k+22 all bases, code(k) != T, code(k+21) in {A, G}, code(k+22) == G
//   reverse at k   positions k..k+22 all bases, code(k) == C, code(k+1) in {C, T}, code(k+22) != A
// (the reference's patterns; position k+1..k+20 / k+2..k+21 of each are [ACGT]). Keys, for the
// matches only: base j of the 20-mer at bits 2 (19 - j), so numeric order is lexicographic order:
//   forward  codes k..k+19, the first most significant (a 2-bit-group reversal of the window)
//   reverse  the reverse complement of codes k+3..k+22: code k+22-j complemented (x ^ 3) as base
//            j, which is the window's codes k+3..k+22 in place, complemented
constexpr uint32_t kTileThreads = 256, kTileWords = kTileThreads, kTile = (kTileWords - 1) * 32;
constexpr uint64_t kSeqPad = kTile + 64;  // zero bytes after the sequences: every tile read is in bounds
constexpr uint64_t kMask40 = (1ull << 40) - 1;

__device__ __forceinline__ uint32_t gather_byte_lsbs(uint32_t x) {  // bit 0 of byte i -> bit i
    return ((x & 0x01010101u) * 0x10204080u) >> 28;
}

__device__ __forceinline__ uint64_t msb_first(uint64_t x) {  // codes 0..19 at bits 2j -> at bits 2 (19 - j)
    uint64_t z = __brevll(x);                                 // code j at bits 63-2j (low), 62-2j (high)
    z = ((z >> 1) & 0x5555555555555555ull) | ((z & 0x5555555555555555ull) << 1);
    return z >> 24;
}

struct TilePlanes {
    uint64_t codes[kTileWords];
    uint32_t valid[kTileWords], lo[kTileWords], hi[kTileWords];
};

// ASCII A C G T = 0x41 0x43 0x47 0x54: ((c >> 1) ^ (c >> 2)) & 3 maps them to 0 1 2 3, four bytes
// at a time (the bits kept come from the byte itself).
__device__ __forceinline__ void pack_tile(const uint8_t* __restrict__ s, uint64_t t0, TilePlanes& t) {
    for (uint32_t u = threadIdx.x; u < kTileWords; u += kTileThreads) {
        const uint4* src = reinterpret_cast<const uint4*>(s + t0 + 32ull * u);
        const uint4 w0 = src[0], w1 = src[1];
        const uint32_t w[8] = {w0.x, w0.y, w0.z, w0.w, w1.x, w1.y, w1.z, w1.w};
        uint64_t c = 0;
        uint32_t v = 0, lo = 0, hi = 0;
#pragma unroll
        for (int q = 0; q < 8; q++) {
            const uint32_t c4 = ((w[q] >> 1) ^ (w[q] >> 2)) & 0x03030303u;
            const uint32_t ok4 = __vcmpeq4(w[q], 0x41414141u) | __vcmpeq4(w[q], 0x43434343u) |
                                 __vcmpeq4(w[q], 0x47474747u) | __vcmpeq4(w[q], 0x54545454u);
            v |= gather_byte_lsbs(ok4) << (4 * q);
            lo |= gather_byte_lsbs(c4) << (4 * q);
            hi |= gather_byte_lsbs(c4 >> 1) << (4 * q);
            const uint32_t m = c4 | (c4 >> 6);  // codes 0, 1 at bits 0-3; codes 2, 3 at bits 16-19
            c |= static_cast<uint64_t>((m & 0xFu) | ((m >> 12) & 0xF0u)) << (8 * q);
        }
        t.codes[u] = c;
        t.valid[u] = v;
        t.lo[u] = lo;
        t.hi[u] = hi;
    }
}

// the forward and reverse match bits of the 32 positions of word u
__device__ __forceinline__ void match_word(const TilePlanes& t, uint32_t u, uint32_t& fwd, uint32_t& rev) {
    const uint64_t V = t.valid[u] | static_cast<uint64_t>(t.valid[u + 1]) << 32;
    const uint64_t L = t.lo[u] | static_cast<uint64_t>(t.lo[u + 1]) << 32;
    const uint64_t H = t.hi[u] | static_cast<uint64_t>(t.hi[u + 1]) << 32;
    const uint64_t a2 = V & (V >> 1), a4 = a2 & (a2 >> 2), a8 = a4 & (a4 >> 4);
    const uint64_t all23 = a8 & (a8 >> 8) & (a8 >> 15);  // positions k..k+22 all bases
    fwd = static_cast<uint32_t>(all23 & ~(L & H) & ~(L >> 21) & ((H & ~L) >> 22));
    rev = static_cast<uint32_t>(all23 & (L & ~H) & (L >> 1) & ((L | H) >> 22));
}

// the codes of the 32 positions from position k of word u
__device__ __forceinline__ uint64_t window(const TilePlanes& t, uint32_t u, uint32_t k) {
    return k ? (t.codes[u] >> (2 * k)) | (t.codes[u + 1] << (64 - 2 * k)) : t.codes[u];
}

// Count mode (keys == nullptr): matches per tile into cnt. Emit mode: the tile's keys from
// off[tile] (the exclusive scan of the counts) in position order, forward before reverse at a
// position.
__global__ void __launch_bounds__(kTileThreads) k_pam_tiles(const uint8_t* __restrict__ s, uint64_t ntiles,
                                                           uint32_t* __restrict__ cnt, const uint64_t* __restrict__ off,
                                                           uint64_t* __restrict__ keys) {
    __shared__ TilePlanes t;
    __shared__ uint32_t wsum[kTileThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint64_t tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
        pack_tile(s, tile * kTile, t);
        __syncthreads();
        // positions at or past the end read the zero padding: never bases, never a match
        uint32_t fwd = 0, rev = 0;
        if (threadIdx.x + 1 < kTileWords) match_word(t, threadIdx.x, fwd, rev);
        const uint32_t mine = __popc(fwd) + __popc(rev);
        uint32_t incl = mine;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t x = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= d) incl += x;
        }
        if (lane == 31) wsum[warp] = incl;
        __syncthreads();
        uint32_t before = incl - mine, total = 0;
#pragma unroll
        for (int w = 0; w < kTileThreads / 32; w++) {
            if (w < warp) before += wsum[w];
            total += wsum[w];
        }
        if (!keys) {
            if (threadIdx.x == 0) cnt[tile] = total;
        } else {
            uint64_t o = off[tile] + before;
            for (uint32_t m = fwd | rev; m; m &= m - 1) {
                const uint32_t k = __ffs(m) - 1;
                const uint64_t x = window(t, threadIdx.x, k);
                if ((fwd >> k) & 1u) keys[o++] = msb_first(x & kMask40);
                if ((rev >> k) & 1u) keys[o++] = ((x >> 6) & kMask40) ^ kMask40;
            }
        }
        __syncthreads();  // the planes and wsum are refilled next
    }
}

// 256 keys per block: their 21-byte lines are built in shared memory and stored with 16-byte
// writes (a block's lines start at a multiple of 256 x 21 bytes, a multiple of 16).
__global__ void __launch_bounds__(256) k_keys_to_text(const uint64_t* __restrict__ keys, uint64_t n,
                                                      char* __restrict__ out) {
    __shared__ __align__(16) char txt[256 * (kSiteLen + 1)];
    for (uint64_t b0 = blockIdx.x * 256ull; b0 < n; b0 += gridDim.x * 256ull) {
        const uint64_t i = b0 + threadIdx.x;
        const uint32_t cnt = static_cast<uint32_t>(n - b0 < 256 ? n - b0 : 256);
        if (i < n) {
            const uint64_t k = keys[i];
            char* o = txt + threadIdx.x * (kSiteLen + 1);
            for (int j = 0; j < kSiteLen; j++) o[j] = "ACGT"[(k >> (2 * (kSiteLen - 1 - j))) & 3u];
            o[kSiteLen] = '\n';
        }
        __syncthreads();
        const uint32_t bytes = cnt * (kSiteLen + 1);
        char* dst = out + b0 * (kSiteLen + 1);
        for (uint32_t w = threadIdx.x; w < bytes / 16; w += 256)
            reinterpret_cast<uint4*>(dst)[w] = reinterpret_cast<const uint4*>(txt)[w];
        for (uint32_t c = bytes / 16 * 16 + threadIdx.x; c < bytes; c += 256) dst[c] = txt[c];
        __syncthreads();
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
    d_seq.reserve(n + kSeqPad);
    ISSL_CUDA(cudaMemcpyAsync(d_seq.p, seq.data(), n, cudaMemcpyHostToDevice, st));
    ISSL_CUDA(cudaMemsetAsync(d_seq.p + n, 0, kSeqPad, st));
    const uint64_t nchunks = (n + kTile - 1) / kTile;  // tiles
    DevBuf<uint32_t> cnt;
    DevBuf<uint64_t> off, total, scan_tmp;
    cnt.reserve(nchunks);
    off.reserve(nchunks + 1);
    total.reserve(1);
    scan_tmp.reserve(kScanBlocks + 4);
    const unsigned tgrid = static_cast<unsigned>(std::min<uint64_t>(nchunks, 148ull * 8));
    k_pam_tiles<<<tgrid, kTileThreads, 0, st>>>(d_seq.p, nchunks, cnt.p, nullptr, nullptr);
    device_scan<uint64_t, OpSum>(LoadU32As64{cnt.p}, StoreExcl64{off.p}, nullptr, nchunks, scan_tmp.p, total.p, st);
    uint64_t m = 0;
    ISSL_CUDA(cudaMemcpyAsync(&m, total.p, 8, cudaMemcpyDeviceToHost, st));
    ISSL_CUDA(cudaStreamSynchronize(st));
    ISSL_REQUIRE(m < 0xFFFFFFFFull, ISSL_ERR_UNSUPPORTED, "2^32 or more off-target sites");
    x.n = m;
    if (m == 0) return;
    x.keys_a.reserve(m);
    x.keys_b.reserve(m);
    k_pam_tiles<<<tgrid, kTileThreads, 0, st>>>(d_seq.p, nchunks, nullptr, off.p, x.keys_a.p);
    ISSL_CUDA(cudaGetLastError());
    const size_t tb = radix_sort_temp_bytes(m, true);
    DevBuf<uint8_t> temp;
    temp.reserve(tb);
    uint64_t* ko = nullptr;
    uint32_t* vo = nullptr;
    radix_sort_pairs_u64(x.keys_a.p, nullptr, x.keys_b.p, nullptr, m, 2 * kSiteLen, temp.p, tb, st, &ko, &vo);
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
        const int fd = ::open(out_path, O_WRONLY | O_CREAT | O_TRUNC, 0644);
        ISSL_REQUIRE(fd >= 0, ISSL_ERR_IO, std::string("cannot write ") + out_path);
        struct F {
            int fd;
            ~F() { ::close(fd); }
        } ff{fd};
        // The text, made on the device in slabs of up to 16M lines and copied into two page-locked
        // host buffers: slab i+1 is converted and copied while the host threads write slab i at
        // its file offset.
        const uint64_t line = issl::kSiteLen + 1, slab = 16ull << 20;
        if (x.n) {
            const uint64_t lines = std::min<uint64_t>(x.n, slab);
            issl::DevBuf<char> d_txt[2];
            issl::PinnedBuf<char> h_txt[2];
            cudaEvent_t ready[2];
            for (int b = 0; b < 2; b++) {
                d_txt[b].reserve(lines * line);
                h_txt[b].reserve(lines * line);
                ISSL_CUDA(cudaEventCreateWithFlags(&ready[b], cudaEventDisableTiming));
            }
            struct E {
                cudaEvent_t* e;
                ~E() {
                    cudaEventDestroy(e[0]);
                    cudaEventDestroy(e[1]);
                }
            } ee{ready};
            const uint64_t n_slabs = (x.n + slab - 1) / slab;
            auto issue = [&](uint64_t i) {
                const int b = static_cast<int>(i & 1);
                const uint64_t k = std::min<uint64_t>(slab, x.n - i * slab);
                issl::k_keys_to_text<<<issl::grid_for(k), 256, 0, st>>>(x.keys + i * slab, k, d_txt[b].p);
                ISSL_CUDA(cudaMemcpyAsync(h_txt[b].p, d_txt[b].p, k * line, cudaMemcpyDeviceToHost, st));
                ISSL_CUDA(cudaEventRecord(ready[b], st));
            };
            const unsigned T = std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
            issue(0);
            for (uint64_t i = 0; i < n_slabs; i++) {
                if (i + 1 < n_slabs) issue(i + 1);  // its buffer held slab i-1, already written
                const int b = static_cast<int>(i & 1);
                ISSL_CUDA(cudaEventSynchronize(ready[b]));
                const uint64_t bytes = std::min<uint64_t>(slab, x.n - i * slab) * line, base = i * slab * line;
                std::vector<std::thread> pool;
                std::vector<int> ok(T, 1);
                for (unsigned t = 0; t < T; t++)
                    pool.emplace_back([&, t] {
                        uint64_t o = bytes / T * t;
                        const uint64_t e = t + 1 == T ? bytes : bytes / T * (t + 1);
                        while (o < e) {
                            const ssize_t w = ::pwrite(fd, h_txt[b].p + o, e - o, static_cast<off_t>(base + o));
                            if (w <= 0) {
                                ok[t] = 0;
                                return;
                            }
                            o += static_cast<uint64_t>(w);
                        }
                    });
                for (auto& th : pool) th.join();
                for (int v : ok) ISSL_REQUIRE(v, ISSL_ERR_IO, std::string("short write to ") + out_path);
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
