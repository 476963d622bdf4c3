// Internal declarations of the issl_b200 library (not part of the public C ABI).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <vector>

#include "issl_b200.h"

namespace issl {

constexpr int kSeqLen = 20;     // protospacer length scored by the reference (20 nt)
constexpr int kMaxSlices = 64;  // slices per index supported by the device tables
constexpr int kMaxDist = 4;     // the reference's fixed mismatch bound (ISSLScoringModule.cpp:292)

// ---- errors ---------------------------------------------------------------------------
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};
void set_last_error(const std::string& msg);

#define ISSL_CUDA(expr)                                                                         \
    do {                                                                                        \
        cudaError_t e_ = (expr);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            throw ::issl::Error(e_ == cudaErrorMemoryAllocation ? ISSL_ERR_NOMEM : ISSL_ERR_CUDA, \
                                std::string(#expr) + ": " + cudaGetErrorString(e_));            \
    } while (0)

#define ISSL_REQUIRE(cond, code, msg)                   \
    do {                                                \
        if (!(cond)) throw ::issl::Error((code), (msg)); \
    } while (0)

// Runs f, converting exceptions into a status code + thread-local message.
template <class F>
int guarded(F&& f) {
    try {
        f();
        return ISSL_OK;
    } catch (const Error& e) {
        set_last_error(e.what());
        return e.code;
    } catch (const std::bad_alloc&) {
        set_last_error("host allocation failed");
        return ISSL_ERR_NOMEM;
    } catch (const std::exception& e) {
        set_last_error(e.what());
        return ISSL_ERR_CUDA;
    }
}

// ---- device memory ---------------------------------------------------------------------
template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() { release(); }
    void release() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    // (re)allocates when the capacity is short; contents are not preserved
    void reserve(size_t count) {
        if (count <= n && p) return;
        release();
        size_t bytes = (count ? count : 1) * sizeof(T);
        ISSL_CUDA(cudaMalloc(reinterpret_cast<void**>(&p), bytes));
        n = count;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// page-locked host memory (device copies from it run at full link speed)
template <class T>
struct PinnedBuf {
    T* p = nullptr;
    size_t n = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf&) = delete;
    PinnedBuf& operator=(const PinnedBuf&) = delete;
    ~PinnedBuf() { release(); }
    void release() {
        if (p) cudaFreeHost(p);
        p = nullptr;
        n = 0;
    }
    void reserve(size_t count) {
        if (count <= n && p) return;
        release();
        ISSL_CUDA(cudaMallocHost(reinterpret_cast<void**>(&p), (count ? count : 1) * sizeof(T)));
        n = count;
    }
    size_t bytes() const { return n * sizeof(T); }
};

// ---- slice geometry ----------------------------------------------------------------------
// Per-slice constants. A slice is a set of `width` protospacer positions; the key of a
// signature is the 2-bit bases at those positions packed in ascending position order
// (ISSLScoringModule.cpp:235-239). The residual is the bases at the other positions packed
// the same way; it is what the scan compares, since the key positions match by construction.
//
// The residual codes of a slice are stored bit-transposed ("bit-sliced") in blocks of 32
// consecutive list positions: word j of a block holds bit j of the residual code of each of the
// block's 32 entries (entry e at bit e). A block has wpb = 2 * rwidth + 1 words (the last one is
// zero padding): an odd block stride puts the 32 blocks of a staged chunk in 32 different shared
// memory banks, so lane l reading word j of block l never conflicts with another lane.
struct SliceGeom {
    uint64_t wbase;       // first word of this slice's blocks in the bit-sliced array
    uint32_t pmask;       // 20-bit position mask
    uint32_t bbase;       // first global bucket id of this slice (sum of 4^w of earlier slices)
    uint8_t width;        // positions in the slice
    uint8_t rwidth;       // positions outside the slice (20 - width)
    uint8_t wpb;          // words per block of 32 entries
    uint8_t pad;
    uint8_t pos[kSeqLen]; // slice positions, ascending
    uint8_t rpos[kSeqLen];// residual positions, ascending
};

constexpr int kBlockEntries = 32;
__host__ __device__ inline uint64_t blocks_per_slice(uint64_t n_sites) { return (n_sites + 31) / 32; }

std::vector<SliceGeom> make_geometry(const std::vector<uint64_t>& masks, uint64_t seq_len, uint64_t n_sites);
uint64_t bitsliced_words(const std::vector<SliceGeom>& geom, uint64_t n_sites);

// ---- the resident index ------------------------------------------------------------------
struct Workspace;

// List entries are packed in 32 bits: the site id in the low id_bits bits, the occurrence count
// in the bits above it when it is below occ_esc, else occ_esc ("look it up in occ[id]"). Up to
// 2^29 sites the code has 3 bits, so a site with 1..6 occurrences (almost all of them) is scored
// with one random read: this entry.
struct IndexView {  // POD view handed to kernels
    const uint64_t* sigs;     // N packed signatures
    const uint32_t* occ;      // N occurrence counts (one per site)
    const uint32_t* ids;      // S*N list entries in list order (slice-major), entry_words words each:
                              // the packed id, then (entry_words 2) the residual code
    const uint32_t* rbits;    // bit-sliced residual codes (see SliceGeom)
    uint64_t ids_base;        // global entry number of ids[0]: 0, or the first entry of the slice
                              // window a host-list index has staged on the device
    uint64_t rbits_base;      // global word number of rbits[0] (a multiple of 4), likewise
    const uint64_t* offsets;  // G+1 bucket starts in global entry numbering: s*N + position
    const SliceGeom* geom;    // S slice descriptors
    uint64_t n_sites;
    uint32_t n_slices;
    uint32_t n_buckets;       // sum of 4^w
    uint32_t id_bits;         // bits of the site id in a packed entry (1..32)
    uint32_t occ_esc;         // occurrence codes >= occ_esc mean "read occ[id]" (0: always)
    uint32_t entry_words;     // 2: entries carry the residual code; 1: packed id only
};

}  // namespace issl

struct issl_index {
    int device = 0;
    uint64_t n_sites = 0, seq_len = 20, n_slices = 0, n_buckets = 0;
    std::vector<uint64_t> masks;
    std::vector<issl::SliceGeom> geom;
    issl::DevBuf<uint64_t> sigs;
    issl::DevBuf<uint32_t> occ, ids, rbits;
    issl::DevBuf<uint64_t> offsets;  // n_buckets + 1 global bucket starts
    uint32_t id_bits = 32, occ_esc = 0;  // packing of the list entries (IndexView)
    uint32_t entry_words = 2;            // 32-bit words per list entry (IndexView)
    issl::DevBuf<issl::SliceGeom> d_geom;
    // Host-list index (issl_open_mapped): ids and rbits live in page-locked host memory and are
    // staged on the device window_slices slices at a time while scoring; the device arrays
    // above are then empty.
    bool host_lists = false;
    uint32_t window_slices = 0;
    issl::PinnedBuf<uint32_t> h_ids, h_rbits;
    std::unique_ptr<issl::Workspace> ws;
    issl_score_stats stats{};
    // scan unit size per bucket-size class, staging depth, blocks per SM, first slice wave
    issl_tuning tuning{{1024, 1024, 1024}, 2, 0, 1};
    uint32_t tuning_version = 0;
    issl::IndexView view() const;
    issl_index();  // defined where Workspace is complete
    ~issl_index();
};

namespace issl {

// entry packing for an index of n sites: 29 id bits and a 3-bit occurrence code (counts 0..6
// stored, 7 = escape) up to 2^29 sites; beyond that the id takes the bits it needs and the code
// what is left (no code at 2^31 sites and more: every count is read from occ[id])
inline void entry_packing(uint64_t n, uint32_t* id_bits, uint32_t* occ_esc) {
    uint32_t b = 29;
    while (b < 32 && (1ull << b) < n) b++;
    *id_bits = b;
    *occ_esc = b < 32 ? (1u << (32 - b)) - 1u : 0u;
}
__host__ __device__ __forceinline__ uint32_t pack_entry(uint32_t id, uint32_t occ, uint32_t id_bits, uint32_t occ_esc) {
    return id_bits < 32 ? id | ((occ < occ_esc ? occ : occ_esc) << id_bits) : id;
}
__host__ __device__ __forceinline__ uint32_t entry_id(uint32_t e, uint32_t id_bits) {
    return id_bits < 32 ? e & ((1u << id_bits) - 1u) : e;
}
// occurrence count of a packed entry (one more read only for escaped counts)
__device__ __forceinline__ uint32_t entry_occ(uint32_t e, const IndexView& v) {
    const uint32_t c = v.id_bits < 32 ? e >> v.id_bits : 0u;
    return c < v.occ_esc ? c : v.occ[entry_id(e, v.id_bits)];
}

// 8-byte list entries (id + residual code) when the index leaves room for them beside the scoring
// workspaces, else 4-byte entries; ISSL_ENTRY_BYTES=4 or 8 forces a width (index.cu)
uint32_t choose_entry_words(uint64_t n_sites, uint64_t n_slices, uint64_t rbits_bytes);

// builders (index.cu)
void build_from_device_sites(issl_index* ix, const uint64_t* d_sigs, const uint32_t* d_occ,
                             cudaStream_t st);

// words of the bit-sliced array: every slice's blocks, plus 4 words of padding that the scan's
// 16-byte-rounded copies may touch
inline uint64_t rbits_words(const issl_index* ix) { return bitsliced_words(ix->geom, ix->n_sites) + 4; }

// radix sort (radix_sort.cu): stable LSD sort of (key, value) pairs on the low `bits` bits.
size_t radix_sort_temp_bytes(size_t n, bool wide_keys);
void radix_sort_pairs_u32(uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp,
                          size_t n, int bits, void* temp, size_t temp_bytes, cudaStream_t st,
                          uint32_t** keys_out, uint32_t** vals_out);
void radix_sort_pairs_u64(uint64_t* keys, uint32_t* vals, uint64_t* keys_tmp, uint32_t* vals_tmp,
                          size_t n, int bits, void* temp, size_t temp_bytes, cudaStream_t st,
                          uint64_t** keys_out, uint32_t** vals_out);

// device bytes of a scoring workspace: fixed + n * per_guide + candidates * per_candidate (score.cu)
void workspace_model(const issl_index* ix, uint64_t* fixed, uint64_t* per_guide, uint64_t* per_candidate);

// Sizes a batch context's workspace, from its next call on, for batches of up to `guides` guides
// and as many candidate slots as `budget_bytes` leaves room for, so that serving never grows (and
// reallocates, which synchronises the device) while other batches run (score.cu). Dropped again
// if the device cannot hold it.
void batch_set_capacity_floor(issl_batch* batch, uint64_t guides, uint64_t budget_bytes);

// tables (tables.cpp)
const std::vector<double>& mit_rank_table();   // 6195 entries indexed by subset rank
const double* cfd_pos_table();
const double* cfd_pam_table();

}  // namespace issl
