// The resident index: .issl loading, validation, GPU construction and export.
//
// Device layout (slice-major, list order of the reference file kept):
//   sigs    [N]      u64  2-bit packed site signatures (the file's offtargets array)
//   occ     [N]      u32  occurrence count per site (the high word of every list entry)
//   ids     [S*N]    u32  packed list entry: site id + occurrence code (see IndexView); the one
//                         random read per scored hit
//   rbits   [...]    u32  residual codes (the site's bases outside the slice), bit-sliced in
//                         blocks of 32 list positions, one word per residual bit
//   offsets [G+1]    u64  bucket starts in global entry numbering (slice s, position j -> s*N + j);
//                         buckets are numbered slice by slice, so off[g+1] - off[g] is always the
//                         size of bucket g, across slice boundaries too
// The reference stores (occ << 32) | id per entry and gathers offtargets[id] for every entry it
// scans (ISSLScoringModule.cpp:248-286). Here the scan streams rbits only (2 * rwidth bits per
// entry: 3 bytes for 8-nt slices) because the slice positions of every entry in a bucket equal
// the query's by construction; bit-slicing lets one lane compare a guide with 32 entries at a time.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "device_util.cuh"
#include "issl_internal.cuh"
#include "scan.cuh"

namespace issl {

namespace {
thread_local std::string g_last_error;
}
void set_last_error(const std::string& m) { g_last_error = m; }

std::vector<SliceGeom> make_geometry(const std::vector<uint64_t>& masks, uint64_t seq_len, uint64_t n_sites) {
    ISSL_REQUIRE(seq_len >= 1 && seq_len <= kSeqLen, ISSL_ERR_UNSUPPORTED,
                 "only indexes of 20-nt (or shorter) sites are supported, got seqLength " +
                     std::to_string(seq_len));
    ISSL_REQUIRE(!masks.empty() && masks.size() <= static_cast<size_t>(kMaxSlices), ISSL_ERR_UNSUPPORTED,
                 "slice count must be 1.." + std::to_string(kMaxSlices) + ", got " +
                     std::to_string(masks.size()));
    std::vector<SliceGeom> geom(masks.size());
    uint64_t bbase = 0, wbase = 0;
    const uint64_t valid = (1ull << seq_len) - 1;
    for (size_t s = 0; s < masks.size(); s++) {
        SliceGeom& g = geom[s];
        std::memset(&g, 0, sizeof g);
        const uint64_t pm = masks[s] & valid;  // positions >= seqLength are ignored (:107-113)
        g.pmask = static_cast<uint32_t>(pm);
        int w = 0, r = 0;
        for (int p = 0; p < kSeqLen; p++) {
            if (pm >> p & 1u)
                g.pos[w++] = static_cast<uint8_t>(p);
            else
                g.rpos[r++] = static_cast<uint8_t>(p);
        }
        ISSL_REQUIRE(w >= 4 && w <= 13, ISSL_ERR_UNSUPPORTED,
                     "slice " + std::to_string(s) + " has width " + std::to_string(w) +
                         "; supported widths are 4..13 positions");
        g.width = static_cast<uint8_t>(w);
        g.rwidth = static_cast<uint8_t>(r);
        g.wpb = static_cast<uint8_t>(2 * r + 1);
        g.wbase = wbase;
        wbase += blocks_per_slice(n_sites) * g.wpb;
        g.bbase = static_cast<uint32_t>(bbase);
        bbase += 1ull << (2 * w);
        ISSL_REQUIRE(bbase + masks.size() + 1 < (1ull << 32), ISSL_ERR_UNSUPPORTED,
                     "too many buckets over all slices");
    }
    return geom;
}

uint32_t choose_entry_words(uint64_t n_sites, uint64_t n_slices, uint64_t rbits_bytes) {
    if (const char* e = std::getenv("ISSL_ENTRY_BYTES")) {
        const std::string v(e);
        ISSL_REQUIRE(v == "4" || v == "8", ISSL_ERR_ARG, "ISSL_ENTRY_BYTES must be 4 or 8");
        return v == "8" ? 2u : 1u;
    }
    size_t free_b = 0, total_b = 0;
    ISSL_CUDA(cudaMemGetInfo(&free_b, &total_b));
    // what the 8-byte lists and the residual codes take, and what must stay free for scoring
    const uint64_t need = n_sites * n_slices * 8 + rbits_bytes;
    const uint64_t keep = std::max<uint64_t>(32ull << 30, total_b / 5);
    return free_b > need + keep ? 2u : 1u;
}

uint64_t bitsliced_words(const std::vector<SliceGeom>& geom, uint64_t n_sites) {
    uint64_t w = 0;
    for (auto& g : geom) w += blocks_per_slice(n_sites) * g.wpb;
    return w;
}

namespace {

__global__ void k_slice_keys(const uint64_t* __restrict__ sigs, uint64_t n, SliceGeom g,
                             uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        keys[i] = slice_key(sigs[i], g);
        vals[i] = static_cast<uint32_t>(i);
    }
}

// off[k] = base + first position whose key >= k, for k in [0, nb]; keys sorted ascending.
__global__ void k_offsets_from_sorted(const uint32_t* __restrict__ keys, uint64_t n, uint32_t nb, uint64_t base,
                                      uint64_t* __restrict__ off) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i <= n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const int64_t prev = i == 0 ? -1 : static_cast<int64_t>(keys[i - 1]);
        const int64_t cur = i == n ? static_cast<int64_t>(nb) : static_cast<int64_t>(keys[i]);
        for (int64_t k = prev + 1; k <= cur; k++) off[k] = base + i;
    }
}

// Bit-sliced residual codes of one slice: a warp per block of 32 list positions; lane e holds the
// residual code of entry e and a ballot per bit collects word j = bit j of the 32 codes.
// With 8-byte entries (ew == 2) it also stores each entry's residual code beside its packed id.
__global__ void k_rbits(uint32_t* __restrict__ ids, uint32_t ew, uint32_t id_bits, const uint64_t* __restrict__ sigs,
                        uint64_t n, SliceGeom g, uint32_t* __restrict__ out) {
    const int lane = threadIdx.x & 31;
    const uint64_t nblk = blocks_per_slice(n);
    for (uint64_t b = (blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x) >> 5; b < nblk;
         b += (static_cast<uint64_t>(gridDim.x) * blockDim.x) >> 5) {
        const uint64_t pos = b * 32 + lane;
        const uint32_t r = pos < n ? slice_residual(sigs[entry_id(ids[pos * ew], id_bits)], g) : 0u;
        if (ew == 2 && pos < n) ids[pos * 2 + 1] = r;
        uint32_t mine = 0;
        const int nbits = 2 * g.rwidth;  // data words; word nbits is the zero padding word
        for (int j = 0; j < nbits; j++) {
            const uint32_t w = __ballot_sync(0xffffffffu, (r >> j) & 1u);
            if (lane == j) mine = w;
        }
        if (lane < nbits) out[g.wbase + b * g.wpb + lane] = mine;
        if (lane == 0) out[g.wbase + b * g.wpb + nbits] = 0u;
    }
}

// bucket_of[j] for every list position j of one slice (off: the slice's nb+1 global starts)
__global__ void k_fill_bucket_of(const uint64_t* __restrict__ off, uint32_t nb, uint64_t base,
                                 uint32_t* __restrict__ bucket_of) {
    for (uint64_t k = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; k < nb;
         k += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        for (uint64_t j = off[k] - base; j < off[k + 1] - base; j++) bucket_of[j] = static_cast<uint32_t>(k);
}

enum : uint32_t { kBadId = 1u, kDupId = 2u, kOccMismatch = 4u, kWrongBucket = 8u };

// Splits file entries (occ << 32 | id) of slice s, list positions [j0, j0+cnt), into ids/occ and
// validates them: id < N, each id once per slice, one occurrence count per site across slices,
// and the entry sits in the bucket of its own slice key.
__global__ void k_split_entries(const uint64_t* __restrict__ entries, uint64_t j0, uint64_t cnt, uint64_t n_sites,
                                int first_slice, SliceGeom g, const uint64_t* __restrict__ sigs,
                                const uint32_t* __restrict__ bucket_of, uint32_t* __restrict__ ids_slice, uint32_t ew,
                                uint32_t id_bits, uint32_t occ_esc, uint32_t* __restrict__ occ,
                                uint32_t* __restrict__ seen, uint32_t* flags) {
    for (uint64_t t = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; t < cnt;
         t += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t e = entries[t];
        const uint64_t id = e & 0xFFFFFFFFull;
        const uint32_t o = static_cast<uint32_t>(e >> 32);
        const uint64_t j = j0 + t;
        if (id >= n_sites) {
            atomicOr(flags, kBadId);
            ids_slice[j * ew] = 0;
            continue;
        }
        ids_slice[j * ew] = pack_entry(static_cast<uint32_t>(id), o, id_bits, occ_esc);
        const uint32_t bit = 1u << (id & 31);
        if (atomicOr(&seen[id >> 5], bit) & bit) atomicOr(flags, kDupId);
        if (first_slice)
            occ[id] = o;
        else if (occ[id] != o)
            atomicOr(flags, kOccMismatch);
        if (slice_key(sigs[id], g) != bucket_of[j]) atomicOr(flags, kWrongBucket);
    }
}

// packed entries of one slice from the sorted site ids
__global__ void k_pack_entries(const uint32_t* __restrict__ sorted_ids, const uint32_t* __restrict__ occ, uint64_t cnt,
                               uint32_t id_bits, uint32_t occ_esc, uint32_t ew, uint32_t* __restrict__ out) {
    for (uint64_t j = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; j < cnt;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t id = sorted_ids[j];
        out[j * ew] = pack_entry(id, occ[id], id_bits, occ_esc);
    }
}

__global__ void k_join_entries(const uint32_t* __restrict__ ids, uint32_t ew, uint32_t id_bits,
                               const uint32_t* __restrict__ occ, uint64_t cnt, uint64_t* __restrict__ out) {
    for (uint64_t j = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; j < cnt;
         j += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t id = entry_id(ids[j * ew], id_bits);
        out[j] = (static_cast<uint64_t>(occ[id]) << 32) | id;
    }
}

inline unsigned grid_for(uint64_t n, unsigned threads = 256) {
    uint64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > 148ull * 32) b = 148ull * 32;
    return static_cast<unsigned>(b);
}

uint64_t count_buckets(const std::vector<SliceGeom>& g) {
    uint64_t t = 0;
    for (auto& s : g) t += 1ull << (2 * s.width);
    return t;
}

// Where a builder puts slice s: straight into the resident arrays, or, for a host-list index,
// into one slice's worth of device memory that is copied out to the page-locked host arrays once
// the slice is complete (the whole lists never need to fit on the device).
struct SliceSink {
    issl_index* ix;
    DevBuf<uint32_t> ids1, rbits1;
    explicit SliceSink(issl_index* x) : ix(x) {
        const uint64_t N = ix->n_sites, ew = ix->entry_words, words = rbits_words(ix);
        if (ix->host_lists) {
            ix->h_ids.reserve(ix->n_slices * N * ew);
            ix->h_rbits.reserve(words);
            std::memset(ix->h_rbits.p + (words - 4), 0, 16);  // the padding words
            uint64_t most = 0;
            for (auto& g : ix->geom) most = std::max<uint64_t>(most, blocks_per_slice(N) * g.wpb);
            ids1.reserve(N * ew);
            rbits1.reserve(most);
        } else {
            ix->ids.reserve(ix->n_slices * N * ew);
            ix->rbits.reserve(words);
        }
    }
    uint32_t* ids(uint64_t s) { return ix->host_lists ? ids1.p : ix->ids.p + s * ix->n_sites * ix->entry_words; }
    // slice s's geometry and array for k_rbits (the one-slice buffer starts at the slice's first word)
    SliceGeom geom(uint64_t s) const {
        SliceGeom g = ix->geom[s];
        if (ix->host_lists) g.wbase = 0;
        return g;
    }
    uint32_t* rbits() { return ix->host_lists ? rbits1.p : ix->rbits.p; }
    void done(uint64_t s, cudaStream_t st) {
        if (!ix->host_lists) return;
        const uint64_t N = ix->n_sites, ew = ix->entry_words;
        const SliceGeom& g = ix->geom[s];
        ISSL_CUDA(cudaMemcpyAsync(ix->h_ids.p + s * N * ew, ids1.p, N * ew * 4, cudaMemcpyDeviceToHost, st));
        ISSL_CUDA(cudaMemcpyAsync(ix->h_rbits.p + g.wbase, rbits1.p, blocks_per_slice(N) * g.wpb * 4,
                                  cudaMemcpyDeviceToHost, st));
        ISSL_CUDA(cudaStreamSynchronize(st));  // the one-slice buffers are refilled next
    }
};

// list entry width: 8 bytes when HBM leaves room (host-list indexes always, their lists are not
// on the device), unless ISSL_ENTRY_BYTES forces one
uint32_t entry_words_for(const issl_index* ix) {
    if (ix->host_lists && !std::getenv("ISSL_ENTRY_BYTES")) return 2u;
    return choose_entry_words(ix->n_sites, ix->n_slices, rbits_words(ix) * 4);
}

// ---- sequential sources for the loader: the .issl byte stream, from a file or from arrays ----
struct Source {
    virtual ~Source() = default;
    virtual void read(void* dst, size_t bytes, const char* what) = 0;
};

struct FileSource : Source {
    FILE* fp;
    explicit FileSource(const char* path) : fp(std::fopen(path, "rb")) {
        ISSL_REQUIRE(fp != nullptr, ISSL_ERR_IO, std::string("Error reading index: could not open file ") + path);
    }
    ~FileSource() override {
        if (fp) std::fclose(fp);
    }
    void read(void* dst, size_t bytes, const char* what) override {
        if (bytes == 0) return;
        ISSL_REQUIRE(std::fread(dst, 1, bytes, fp) == bytes, ISSL_ERR_IO,
                     std::string("Error reading index: ") + what + " (file truncated)");
    }
};

struct ArraySource : Source {
    // segments of the virtual stream in order
    std::vector<std::pair<const uint8_t*, size_t>> segs;
    size_t seg = 0, off = 0;
    void read(void* dst, size_t bytes, const char* what) override {
        uint8_t* d = static_cast<uint8_t*>(dst);
        while (bytes) {
            ISSL_REQUIRE(seg < segs.size(), ISSL_ERR_ARG, std::string("index arrays too short: ") + what);
            const size_t take = std::min(bytes, segs[seg].second - off);
            std::memcpy(d, segs[seg].first + off, take);
            d += take;
            bytes -= take;
            off += take;
            if (off == segs[seg].second) {
                seg++;
                off = 0;
            }
        }
    }
};

struct PinnedStaging {
    static constexpr size_t kBytes = 64ull << 20;
    void* h[2] = {nullptr, nullptr};
    uint64_t* d[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr};
    PinnedStaging() {
        for (int i = 0; i < 2; i++) {
            ISSL_CUDA(cudaMallocHost(&h[i], kBytes));
            ISSL_CUDA(cudaMalloc(reinterpret_cast<void**>(&d[i]), kBytes));
            ISSL_CUDA(cudaEventCreateWithFlags(&done[i], cudaEventDisableTiming));
        }
    }
    ~PinnedStaging() {
        for (int i = 0; i < 2; i++) {
            if (h[i]) cudaFreeHost(h[i]);
            if (d[i]) cudaFree(d[i]);
            if (done[i]) cudaEventDestroy(done[i]);
        }
    }
};

void load_stream(issl_index* ix, Source& src, int device) {
    ISSL_CUDA(cudaSetDevice(device));
    ix->device = device;
    uint64_t hdr[3];
    src.read(hdr, sizeof hdr, "header invalid");
    ix->n_sites = hdr[0];
    ix->seq_len = hdr[1];
    ix->n_slices = hdr[2];
    ISSL_REQUIRE(ix->n_sites < (1ull << 32), ISSL_ERR_FORMAT, "index has 2^32 or more sites");
    ISSL_REQUIRE(ix->n_slices >= 1 && ix->n_slices <= static_cast<uint64_t>(kMaxSlices), ISSL_ERR_FORMAT,
                 "Error reading index: header invalid (slice count " + std::to_string(ix->n_slices) + ")");
    ISSL_REQUIRE(ix->seq_len >= 1 && ix->seq_len <= 64, ISSL_ERR_FORMAT, "Error reading index: header invalid");
    const uint64_t N = ix->n_sites, S = ix->n_slices;
    entry_packing(N, &ix->id_bits, &ix->occ_esc);
    cudaStream_t st;
    ISSL_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    struct StreamGuard {
        cudaStream_t s;
        ~StreamGuard() { cudaStreamDestroy(s); }
    } sg{st};
    PinnedStaging stg;
    const size_t per = PinnedStaging::kBytes / 8;

    // signatures
    ix->sigs.reserve(N);
    for (uint64_t i = 0, b = 0; i < N; b ^= 1) {
        const uint64_t cnt = std::min<uint64_t>(per, N - i);
        ISSL_CUDA(cudaEventSynchronize(stg.done[b]));
        src.read(stg.h[b], cnt * 8, "loading off-target sequences failed");
        ISSL_CUDA(cudaMemcpyAsync(ix->sigs.p + i, stg.h[b], cnt * 8, cudaMemcpyHostToDevice, st));
        ISSL_CUDA(cudaEventRecord(stg.done[b], st));
        i += cnt;
    }
    ix->masks.resize(S);
    src.read(ix->masks.data(), S * 8, "reading slice masks failed");
    ix->geom = make_geometry(ix->masks, ix->seq_len, N);
    ix->n_buckets = count_buckets(ix->geom);
    ix->d_geom.reserve(S);
    ISSL_CUDA(cudaMemcpyAsync(ix->d_geom.p, ix->geom.data(), S * sizeof(SliceGeom), cudaMemcpyHostToDevice, st));

    ix->occ.reserve(N);
    ix->entry_words = entry_words_for(ix);
    SliceSink sink(ix);
    ix->offsets.reserve(ix->n_buckets + 1);
    DevBuf<uint32_t> seen, bucket_of, flags;
    seen.reserve(N / 32 + 1);
    bucket_of.reserve(N);
    flags.reserve(1);
    ISSL_CUDA(cudaMemsetAsync(flags.p, 0, 4, st));
    std::vector<uint64_t> sizes, off64;
    uint64_t bbase = 0;
    for (uint64_t s = 0; s < S; s++) {
        const SliceGeom& g = ix->geom[s];
        const uint64_t nb = 1ull << (2 * g.width);
        sizes.resize(nb);
        src.read(sizes.data(), nb * 8, "reading slice list sizes failed");
        off64.resize(nb + 1);
        uint64_t acc = 0;
        for (uint64_t k = 0; k < nb; k++) {
            off64[k] = s * N + acc;
            acc += sizes[k];
            ISSL_REQUIRE(acc <= N, ISSL_ERR_FORMAT,
                         "Error reading index: slice " + std::to_string(s) + " list sizes exceed the site count");
        }
        ISSL_REQUIRE(acc == N, ISSL_ERR_FORMAT,
                     "Error reading index: slice " + std::to_string(s) + " list sizes sum to " +
                         std::to_string(acc) + ", expected " + std::to_string(N));
        off64[nb] = s * N + N;  // = first start of the next slice
        // the previous slice's kernels read bucket_of / seen: order through the stream
        ISSL_CUDA(cudaMemcpyAsync(ix->offsets.p + bbase, off64.data(), (nb + 1) * 8, cudaMemcpyHostToDevice, st));
        ISSL_CUDA(cudaStreamSynchronize(st));  // off64 is reused next slice
        k_fill_bucket_of<<<grid_for(nb), 256, 0, st>>>(ix->offsets.p + bbase, static_cast<uint32_t>(nb), s * N,
                                                      bucket_of.p);
        ISSL_CUDA(cudaMemsetAsync(seen.p, 0, (N / 32 + 1) * 4, st));
        for (uint64_t j = 0, b = 0; j < N; b ^= 1) {
            const uint64_t cnt = std::min<uint64_t>(per, N - j);
            ISSL_CUDA(cudaEventSynchronize(stg.done[b]));
            src.read(stg.h[b], cnt * 8, "reading slice contents failed");
            ISSL_CUDA(cudaMemcpyAsync(stg.d[b], stg.h[b], cnt * 8, cudaMemcpyHostToDevice, st));
            k_split_entries<<<grid_for(cnt), 256, 0, st>>>(stg.d[b], j, cnt, N, s == 0, g, ix->sigs.p, bucket_of.p,
                                                           sink.ids(s), ix->entry_words, ix->id_bits,
                                                           ix->occ_esc, ix->occ.p, seen.p, flags.p);
            ISSL_CUDA(cudaEventRecord(stg.done[b], st));
            j += cnt;
        }
        k_rbits<<<grid_for(blocks_per_slice(N) * 32), 256, 0, st>>>(sink.ids(s), ix->entry_words, ix->id_bits,
                                                                    ix->sigs.p, N, sink.geom(s), sink.rbits());
        ISSL_CUDA(cudaGetLastError());
        sink.done(s, st);
        uint32_t f = 0;
        ISSL_CUDA(cudaMemcpyAsync(&f, flags.p, 4, cudaMemcpyDeviceToHost, st));
        ISSL_CUDA(cudaStreamSynchronize(st));
        const std::string where = "Error reading index: slice " + std::to_string(s) + ": ";
        ISSL_REQUIRE(!(f & kBadId), ISSL_ERR_FORMAT, where + "site id out of range");
        ISSL_REQUIRE(!(f & kDupId), ISSL_ERR_FORMAT, where + "a site id is listed twice");
        ISSL_REQUIRE(!(f & kOccMismatch), ISSL_ERR_FORMAT,
                     where + "occurrence count of a site differs from slice 0 (unsupported)");
        ISSL_REQUIRE(!(f & kWrongBucket), ISSL_ERR_FORMAT, where + "a site is listed under a bucket other than its key");
        bbase += nb;
    }
    ISSL_CUDA(cudaStreamSynchronize(st));
}

}  // namespace

void build_from_device_sites(issl_index* ix, const uint64_t* d_sigs, const uint32_t* d_occ, cudaStream_t st) {
    const uint64_t N = ix->n_sites, S = ix->n_slices;
    ISSL_REQUIRE(N < (1ull << 32), ISSL_ERR_UNSUPPORTED, "2^32 or more sites");
    entry_packing(N, &ix->id_bits, &ix->occ_esc);
    ix->geom = make_geometry(ix->masks, ix->seq_len, N);
    ix->n_buckets = count_buckets(ix->geom);
    if (ix->sigs.p != d_sigs) {
        ix->sigs.reserve(N);
        ISSL_CUDA(cudaMemcpyAsync(ix->sigs.p, d_sigs, N * 8, cudaMemcpyDeviceToDevice, st));
    }
    if (ix->occ.p != d_occ) {
        ix->occ.reserve(N);
        ISSL_CUDA(cudaMemcpyAsync(ix->occ.p, d_occ, N * 4, cudaMemcpyDeviceToDevice, st));
    }
    ix->d_geom.reserve(S);
    ISSL_CUDA(cudaMemcpyAsync(ix->d_geom.p, ix->geom.data(), S * sizeof(SliceGeom), cudaMemcpyHostToDevice, st));
    ix->entry_words = entry_words_for(ix);
    SliceSink sink(ix);
    ix->offsets.reserve(ix->n_buckets + 1);
    DevBuf<uint32_t> keys, vals, keys2, vals2;
    DevBuf<uint8_t> temp;
    keys.reserve(N);
    vals.reserve(N);
    keys2.reserve(N);
    vals2.reserve(N);
    const size_t tb = radix_sort_temp_bytes(N, false);
    temp.reserve(tb);
    uint64_t bbase = 0;
    for (uint64_t s = 0; s < S; s++) {
        const SliceGeom& g = ix->geom[s];
        const uint32_t nb = 1u << (2 * g.width);
        k_slice_keys<<<grid_for(N), 256, 0, st>>>(ix->sigs.p, N, g, keys.p, vals.p);
        uint32_t *ko = keys.p, *vo = vals.p;
        // stable by key: ids stay ascending inside each bucket (ISSLCreateIndex.cpp:455-468)
        radix_sort_pairs_u32(keys.p, vals.p, keys2.p, vals2.p, N, 2 * g.width, temp.p, tb, st, &ko, &vo);
        k_pack_entries<<<grid_for(N), 256, 0, st>>>(vo, ix->occ.p, N, ix->id_bits, ix->occ_esc, ix->entry_words,
                                                    sink.ids(s));
        k_offsets_from_sorted<<<grid_for(N + 1), 256, 0, st>>>(ko, N, nb, s * N, ix->offsets.p + bbase);
        k_rbits<<<grid_for(blocks_per_slice(N) * 32), 256, 0, st>>>(sink.ids(s), ix->entry_words, ix->id_bits,
                                                                    ix->sigs.p, N, sink.geom(s), sink.rbits());
        ISSL_CUDA(cudaGetLastError());
        sink.done(s, st);
        bbase += nb;
    }
    ISSL_CUDA(cudaStreamSynchronize(st));
}

void export_slice_lists(const issl_index* ix, uint64_t s, uint64_t* host_lists, cudaStream_t st) {
    const uint64_t N = ix->n_sites;
    if (!N) return;
    DevBuf<uint64_t> tmp;
    tmp.reserve(N);
    const uint32_t* ids = ix->ids.p + s * N * ix->entry_words;
    DevBuf<uint32_t> staged;  // host-list index: the slice's entries brought to the device
    if (ix->host_lists) {
        staged.reserve(N * ix->entry_words);
        ISSL_CUDA(cudaMemcpyAsync(staged.p, ix->h_ids.p + s * N * ix->entry_words, N * ix->entry_words * 4,
                                  cudaMemcpyHostToDevice, st));
        ids = staged.p;
    }
    k_join_entries<<<grid_for(N), 256, 0, st>>>(ids, ix->entry_words, ix->id_bits, ix->occ.p, N, tmp.p);
    ISSL_CUDA(cudaGetLastError());
    ISSL_CUDA(cudaMemcpyAsync(host_lists, tmp.p, N * 8, cudaMemcpyDeviceToHost, st));
    ISSL_CUDA(cudaStreamSynchronize(st));
}

std::vector<uint64_t> export_sizes(const issl_index* ix) {
    std::vector<uint64_t> sizes;
    sizes.reserve(ix->n_buckets);
    std::vector<uint64_t> off(ix->n_buckets + 1);
    ISSL_CUDA(cudaMemcpy(off.data(), ix->offsets.p, (ix->n_buckets + 1) * 8, cudaMemcpyDeviceToHost));
    for (uint64_t g = 0; g < ix->n_buckets; g++) sizes.push_back(off[g + 1] - off[g]);
    return sizes;
}

}  // namespace issl

issl::IndexView issl_index::view() const {
    issl::IndexView v;
    v.sigs = sigs.p;
    v.occ = occ.p;
    v.ids = ids.p;
    v.rbits = rbits.p;
    v.ids_base = 0;
    v.rbits_base = 0;
    v.offsets = offsets.p;
    v.geom = d_geom.p;
    v.n_sites = n_sites;
    v.n_slices = static_cast<uint32_t>(n_slices);
    v.n_buckets = static_cast<uint32_t>(n_buckets);
    v.id_bits = id_bits;
    v.occ_esc = occ_esc;
    v.entry_words = entry_words;
    return v;
}

using issl::guarded;

extern "C" {

const char* issl_last_error(void) { return issl::g_last_error.c_str(); }

int issl_open(const char* path, int device, issl_index** out) {
    return guarded([&] {
        ISSL_REQUIRE(path && out, ISSL_ERR_ARG, "issl_open: null argument");
        *out = nullptr;
        auto ix = std::make_unique<issl_index>();
        issl::FileSource src(path);
        issl::load_stream(ix.get(), src, device);
        *out = ix.release();
    });
}

int issl_open_mapped(const char* path, int device, uint32_t window_slices, issl_index** out) {
    return guarded([&] {
        ISSL_REQUIRE(path && out, ISSL_ERR_ARG, "issl_open_mapped: null argument");
        ISSL_REQUIRE(window_slices >= 1 && window_slices <= static_cast<uint32_t>(issl::kMaxSlices), ISSL_ERR_ARG,
                     "issl_open_mapped: window_slices must be 1..64");
        *out = nullptr;
        auto ix = std::make_unique<issl_index>();
        ix->host_lists = true;
        ix->window_slices = window_slices;
        issl::FileSource src(path);
        issl::load_stream(ix.get(), src, device);
        *out = ix.release();
    });
}

int issl_open_arrays(const uint64_t* sigs, uint64_t n_sites, uint64_t seq_len, const uint64_t* slice_masks,
                     uint64_t n_slices, const uint64_t* list_sizes, const uint64_t* lists, int device,
                     issl_index** out) {
    return guarded([&] {
        ISSL_REQUIRE(out && slice_masks && list_sizes && (lists || n_sites == 0) && (sigs || n_sites == 0),
                     ISSL_ERR_ARG, "issl_open_arrays: null argument");
        *out = nullptr;
        ISSL_REQUIRE(n_slices >= 1 && n_slices <= static_cast<uint64_t>(issl::kMaxSlices), ISSL_ERR_ARG,
                     "issl_open_arrays: slice count out of range");
        static thread_local uint64_t hdr[3];
        hdr[0] = n_sites;
        hdr[1] = seq_len;
        hdr[2] = n_slices;
        issl::ArraySource src;
        src.segs.push_back({reinterpret_cast<const uint8_t*>(hdr), sizeof hdr});
        src.segs.push_back({reinterpret_cast<const uint8_t*>(sigs), n_sites * 8});
        src.segs.push_back({reinterpret_cast<const uint8_t*>(slice_masks), n_slices * 8});
        uint64_t base = 0;
        const uint64_t valid = seq_len >= 64 ? ~0ull : ((1ull << seq_len) - 1);
        for (uint64_t s = 0; s < n_slices; s++) {
            const uint64_t w = static_cast<uint64_t>(__builtin_popcountll(slice_masks[s] & valid));
            ISSL_REQUIRE(w <= 13, ISSL_ERR_UNSUPPORTED, "slice wider than 13 positions");
            const uint64_t nb = 1ull << (2 * w);
            src.segs.push_back({reinterpret_cast<const uint8_t*>(list_sizes + base), nb * 8});
            src.segs.push_back({reinterpret_cast<const uint8_t*>(lists + s * n_sites), n_sites * 8});
            base += nb;
        }
        auto ix = std::make_unique<issl_index>();
        issl::load_stream(ix.get(), src, device);
        *out = ix.release();
    });
}

int issl_build(const uint64_t* sigs, const uint32_t* occ, uint64_t n_sites, const uint64_t* slice_masks,
               uint64_t n_slices, int device, issl_index** out) {
    return guarded([&] {
        ISSL_REQUIRE(out && slice_masks && (n_sites == 0 || (sigs && occ)), ISSL_ERR_ARG, "issl_build: null argument");
        *out = nullptr;
        ISSL_CUDA(cudaSetDevice(device));
        auto ix = std::make_unique<issl_index>();
        ix->device = device;
        ix->n_sites = n_sites;
        ix->seq_len = issl::kSeqLen;
        ix->n_slices = n_slices;
        ix->masks.assign(slice_masks, slice_masks + n_slices);
        ix->sigs.reserve(n_sites);
        ix->occ.reserve(n_sites);
        if (n_sites) {
            ISSL_CUDA(cudaMemcpy(ix->sigs.p, sigs, n_sites * 8, cudaMemcpyHostToDevice));
            ISSL_CUDA(cudaMemcpy(ix->occ.p, occ, n_sites * 4, cudaMemcpyHostToDevice));
        }
        cudaStream_t st;
        ISSL_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        try {
            issl::build_from_device_sites(ix.get(), ix->sigs.p, ix->occ.p, st);
        } catch (...) {
            cudaStreamDestroy(st);
            throw;
        }
        cudaStreamDestroy(st);
        *out = ix.release();
    });
}

int issl_close(issl_index* index) {
    return guarded([&] {
        if (!index) return;
        cudaSetDevice(index->device);
        delete index;
    });
}

int issl_index_get_info(const issl_index* ix, issl_index_info* out) {
    return guarded([&] {
        ISSL_REQUIRE(ix && out, ISSL_ERR_ARG, "issl_index_get_info: null argument");
        out->n_sites = ix->n_sites;
        out->seq_len = ix->seq_len;
        out->n_slices = ix->n_slices;
        out->n_buckets = ix->n_buckets;
        out->device_bytes = ix->sigs.bytes() + ix->occ.bytes() + ix->ids.bytes() + ix->rbits.bytes() +
                            ix->offsets.bytes() + ix->d_geom.bytes();
        out->entry_bytes = static_cast<int>(4 * ix->entry_words);
        out->host_bytes = ix->h_ids.bytes() + ix->h_rbits.bytes();
        out->window_slices = ix->host_lists ? static_cast<int>(ix->window_slices) : 0;
        out->device = ix->device;
        int mn = 64, mx = 0;
        for (auto& g : ix->geom) {
            mn = std::min<int>(mn, g.width);
            mx = std::max<int>(mx, g.width);
        }
        out->min_width = mn;
        out->max_width = mx;
    });
}

int issl_export(const issl_index* ix, uint64_t* sigs, uint64_t* slice_masks, uint64_t* list_sizes, uint64_t* lists) {
    return guarded([&] {
        ISSL_REQUIRE(ix, ISSL_ERR_ARG, "issl_export: null index");
        ISSL_CUDA(cudaSetDevice(ix->device));
        if (sigs && ix->n_sites) ISSL_CUDA(cudaMemcpy(sigs, ix->sigs.p, ix->n_sites * 8, cudaMemcpyDeviceToHost));
        if (slice_masks) std::memcpy(slice_masks, ix->masks.data(), ix->n_slices * 8);
        if (list_sizes) {
            auto sz = issl::export_sizes(ix);
            std::memcpy(list_sizes, sz.data(), sz.size() * 8);
        }
        if (lists) {
            cudaStream_t st;
            ISSL_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            for (uint64_t s = 0; s < ix->n_slices; s++) issl::export_slice_lists(ix, s, lists + s * ix->n_sites, st);
            cudaStreamDestroy(st);
        }
    });
}

int issl_save(const issl_index* ix, const char* path) {
    return guarded([&] {
        ISSL_REQUIRE(ix && path, ISSL_ERR_ARG, "issl_save: null argument");
        ISSL_CUDA(cudaSetDevice(ix->device));
        FILE* fp = std::fopen(path, "wb");
        ISSL_REQUIRE(fp, ISSL_ERR_IO, std::string("cannot create ") + path);
        struct Closer {
            FILE* f;
            ~Closer() {
                if (f) std::fclose(f);
            }
        } closer{fp};
        auto put = [&](const void* p, size_t bytes) {
            ISSL_REQUIRE(std::fwrite(p, 1, bytes, fp) == bytes, ISSL_ERR_IO, std::string("short write to ") + path);
        };
        const uint64_t hdr[3] = {ix->n_sites, ix->seq_len, ix->n_slices};
        put(hdr, sizeof hdr);
        std::vector<uint64_t> buf(ix->n_sites);
        if (ix->n_sites) ISSL_CUDA(cudaMemcpy(buf.data(), ix->sigs.p, ix->n_sites * 8, cudaMemcpyDeviceToHost));
        put(buf.data(), ix->n_sites * 8);
        put(ix->masks.data(), ix->n_slices * 8);
        auto sizes = issl::export_sizes(ix);
        cudaStream_t st;
        ISSL_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        uint64_t base = 0;
        for (uint64_t s = 0; s < ix->n_slices; s++) {
            const uint64_t nb = 1ull << (2 * ix->geom[s].width);
            put(sizes.data() + base, nb * 8);
            issl::export_slice_lists(ix, s, buf.data(), st);
            put(buf.data(), ix->n_sites * 8);
            base += nb;
        }
        cudaStreamDestroy(st);
        ISSL_REQUIRE(std::fclose(fp) == 0, ISSL_ERR_IO, std::string("cannot close ") + path);
        closer.f = nullptr;
    });
}

}  // extern "C"
