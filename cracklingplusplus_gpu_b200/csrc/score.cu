// ISSL scoring on the GPU: the hot path of lib/ISSLScoringModule.cpp:206-462 and
// ISSLScoreOfftargets/ISSLScoreOfftargets.cpp:308-505.
//
// Pipeline (one stream, no host round trip; sizes produced on the device are read on the device),
// run once per slice wave (the first slices, then the rest) for the guides still scoring:
//   1 probe_count   every (guide, wave slice) pair -> its global bucket; count probes per bucket
//   2 bucket scan   exclusive scan over the wave's buckets of (scan units, probes): per-bucket
//                   probe slot ranges, and unit descriptors -- a unit is (up to 32 consecutive
//                   32-entry blocks of a bucket) x (up to kGroup guides probing that bucket), so
//                   guides sharing a bucket read its entries once and heavy buckets split into
//                   many units
//   3 probe_scatter guides grouped by bucket, with each guide's residual code for that slice
//   4 scan          persistent, work-stealing: stream the bit-sliced residual codes of every unit
//                   through per-warp bulk-copy rings; a candidate is an entry whose residual
//                   differs from the guide's in <= max_dist bases; candidates are counted per guide
//   5 segments      the exclusive prefix of the per-guide candidate counts: each guide's segment
//                   of the hit buffer
//   6 resolve       per candidate: its list entry (site id, occurrences, signature); kept only in
//                   the first slice that reaches it (replacing the per-guide toggle bitset of
//                   :252-258): a site reached in slice s counts iff no earlier slice has all its
//                   positions matching; the kept ones get their MIT and CFD contributions and go
//                   to the next free slot of their guide's segment
//   7 score         per guide: exact fixed-point totals over the wave's hits plus the earlier
//                   waves'; guides whose early-exit test (:366-395) fires are ordered as the
//                   reference visits them (slice, then list position) to find the exact stop;
//                   the others are finalised (:404-459) after the last wave or carried on
#include <cuda_runtime.h>

#include <algorithm>
#include <cstddef>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "async_copy.cuh"
#include "bitslice.cuh"
#include "device_util.cuh"
#include "issl_internal.cuh"
#include "scan.cuh"

namespace issl {

constexpr int kChunk = 1024;       // largest scan unit: 32 bit-sliced blocks of 32 list positions
constexpr int kGroup = 32;         // guides per scan unit
constexpr int kScanWarps = 4;      // warps per scan block
constexpr uint32_t kEmpty = 0xFFFFFFFFu;

struct UnitDesc {   // 16 bytes
    uint32_t p0;    // first list position of the unit within its slice
    uint32_t qbeg;  // first probe slot of the unit's guides
    uint16_t len;   // list positions in the unit (<= kChunk, inside one aligned kChunk block)
    uint8_t qn;     // guides in the unit (<= kGroup)
    uint8_t s;      // slice
    uint32_t pad;
};

struct Counters {
    // per wave (cleared at the start of every wave: the fields before `overflow`)
    uint64_t bucket_total;  // hi: units, lo: probes into non-empty buckets
    unsigned long long cand_reserved;  // candidate slots reserved by the scan (may exceed capacity)
    uint32_t n_units;       // min(units, capacity)
    uint32_t n_cand;        // min(cand_reserved, capacity): the slots the later kernels read
    uint32_t hit_total;     // owned hits of the wave (the resolve pass counts them)
    uint32_t n_big;         // exiting guides with more than kWarpSort hits (block scorer)
    uint32_t n_exit;        // exiting guides with at most kWarpSort hits (warp scorer)
    uint32_t next_batch;    // work queue of the scan: next batch of 32 units to take
    // per call
    uint32_t overflow;      // 1: units, 2: hits, 4: a bounded wait in the scan gave up
    uint32_t act_n[2];      // guides still scoring after a wave (active lists A and B)
    uint32_t n_replay;      // guides rescored by k_replay (decision within the reference's rounding)
    uint64_t max_units, max_cand;        // largest wave (to size the buffers)
    uint64_t probes, units, hits, cands; // summed over the waves
    uint64_t distinct;
    uint64_t buckets;       // distinct buckets probed
    uint64_t entries;       // entries compared by the scan (per guide group)
    uint64_t rbytes;        // bit-sliced bytes the scan copies
    uint64_t class_probes[3];  // probes into buckets of < 64, 64..4095, >= 4096 entries
    uint64_t dropped;       // grouped hits whose site is farther than kMaxDist (counted for nothing)
};
constexpr size_t kWaveCounterBytes = offsetof(Counters, overflow);

struct Tables {  // device copies of the penalty tables
    double mit[6195];
    double cfd_pos[320];
    double cfd_pam[16];
    uint32_t binom[20][5];  // C(p, i) for the MIT subset rank
};

struct ScoreParams {
    int method;
    int calc_mit, calc_cfd;
    int max_dist;
    double threshold;
    double maximum_sum;  // (10000 - 100 t) / t, ISSLScoringModule.cpp:225
    int want_distinct;
    int pad;
};

// A batch of guide sets scored in one pass: the header and the set table live in device memory
// so that a captured graph can be replayed for any batch that fits the capacities.
struct SetDesc {
    ScoreParams P;
    uint32_t begin, count;  // the set's guides: [begin, begin + count) of the batch
};
struct BatchHeader {
    uint32_t n;         // guides in the batch
    uint32_t n_sets;
    int max_dist;       // largest max_dist of the sets (the scan's bound)
    uint32_t pad;
};

// Unit size per bucket-size class (autotuned per index).
struct ChunkClasses {
    uint32_t c[3];  // list positions per unit for buckets of < 64, 64..4095 and >= 4096 entries
};
__device__ __forceinline__ uint64_t chunk_of(uint64_t bucket_size, const ChunkClasses& cc) {
    return bucket_size < 64 ? cc.c[0] : bucket_size < 4096 ? cc.c[1] : cc.c[2];
}

constexpr int kMaxStages = 4;
constexpr int kStageQr = kGroup + 2;     // (guide, residual) pairs per stage + alignment slack
constexpr uint32_t kCandSlab = 256;
constexpr uint32_t kScanRecs = 64;  // per-warp buffer of candidate records (guide, lane, word)
// candidate slots of one wave are addressed with 32 bits: the capacity stays below this
constexpr size_t kMaxCandSlots = 0xFFFFFFFFull - (1ull << 20);
constexpr uint32_t kDeadCand = 0xFFFFFFFFu;  // guide field of an unused or rejected candidate slot
constexpr int kGuideBits = 26;               // candidate records pack guide | slice << 26
constexpr long long kWaitCycles = 4000000000ll;  // ~2 s at 1.965 GHz

struct StageMeta {
    uint32_t p0;   // first list position of the unit
    uint32_t len;  // list positions in the unit
    uint32_t b0;   // first block of the unit
    uint32_t nb;   // blocks in the unit
    uint32_t qoff; // offset of the unit's first guide in the staged pairs
    uint32_t qn;   // guides in the unit
    uint32_t s;    // slice
    uint32_t delta;// words between the 16-byte aligned copy start and the unit's first block
};

// per-warp shared memory, sized at launch for the widest block of the index and the stage count
struct WarpLayout {
    uint32_t stages;
    uint32_t stage_words;  // 32 blocks x words per block (largest slice)
    uint32_t qr_off, qm_off, rec_off, meta_off, bar_off, bytes;
};

__host__ __device__ inline WarpLayout warp_layout(uint32_t max_wpb, uint32_t stages) {
    WarpLayout L;
    L.stages = stages;
    L.stage_words = (32u * max_wpb + 3u + 3u) & ~3u;  // 32 blocks + alignment slack, 16-byte multiple
    L.qr_off = stages * L.stage_words * 4u;                 // 16-byte aligned (stage_words % 4 == 0)
    L.qm_off = L.qr_off + stages * kStageQr * 8u;
    L.rec_off = L.qm_off + 64u * 4u;  // two 32-word guide-mask buffers
    L.meta_off = L.rec_off + kScanRecs * 8u;
    L.bar_off = L.meta_off + stages * static_cast<uint32_t>(sizeof(StageMeta));
    L.bytes = (L.bar_off + stages * 8u + 15u) & ~15u;
    return L;
}

}  // namespace issl

// One owned hit grouped under its guide: (list position, slice, site id, occurrences) and its MIT
// and CFD contributions (each already multiplied by the occurrences; the scorers drop the one the
// guide's method does not use). 32 bytes, written whole by one thread: hits land in their guide's
// segment in arrival order, and a scattered write of less than a 32-byte sector costs a DRAM read
// of the sector when it is evicted partly written.
struct __align__(32) HitRec {
    uint4 r;
    double mit, cfd;
};
// device bytes per candidate slot: the candidate record and the grouped-hit record it may become
constexpr size_t kCandSlotBytes = sizeof(uint2) + sizeof(HitRec);

struct issl::Workspace {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaEvent_t ev[2 + 2 * kMaxSlices] = {};  // call start / end, then scan start / end of each slice wave
    size_t q_cap = 0, unit_cap = 0, cand_cap = 0;
    uint64_t g_cap = 0;
    int scan_blocks = 0;
    int scan_rw = 0;  // residual width the scan is specialised for (0: mixed)
    WarpLayout scan_layout{};
    int scan_smem = 0;
    bool zero_state_ok = false;  // bucket_cnt is all zero between calls
    DevBuf<uint64_t> qsig;
    DevBuf<char> ascii;
    size_t ascii_cap = 0;
    DevBuf<uint32_t> probe_gb;
    DevBuf<uint64_t> probe_qr;  // per probe slot: guide | residual << 32 (+2 padding)
    DevBuf<uint32_t> bucket_cnt, bucket_qstart, bucket_ustart;
    DevBuf<UnitDesc> units;
    DevBuf<uint2> cands;  // candidate slots: (guide | slice << 26, list position)
    DevBuf<HitRec> seg;   // owned hits grouped per guide
    // per guide: candidates of the wave (counted by the scan), segment start, owned hits written
    DevBuf<uint32_t> qcand, qoff, qfill, big, exitq;
    DevBuf<uint32_t> replayq;  // guides whose decision k_replay settles
    DevBuf<uint32_t> bitmap;
    DevBuf<Counters> counters;
    DevBuf<uint64_t> scan64;
    DevBuf<uint32_t> scan32;
    DevBuf<Tables> tables;
    DevBuf<double> out_mit, out_cfd;
    DevBuf<char> out_code;
    DevBuf<uint64_t> out_count, out_distinct;
    Counters last{};
    uint64_t launches = 0;  // kernels enqueued by the current call
    uint64_t staged = 0;    // host-list index: bytes the last pipeline copies from host memory
    uint32_t tuning_version = ~0u;  // version of the index's tuning the scan is configured for
    double cand_density = 64.0;     // candidate slots per guide recent runs needed (largest wave)
    uint64_t q_floor = 0, cand_floor = 0;  // capacities held whatever a call needs (server slots)
    double cand_seen = 0.0, guides_seen = 0.0;  // their decayed, size-weighted sums
    uint64_t epoch = 0;             // bumped whenever a buffer is reallocated
    // batch form: set table (header + sets) on the device and its pinned host staging, the
    // guide -> set map, and the captured pipeline
    DevBuf<uint16_t> qset;
    DevBuf<uint32_t> active[2];  // guides still scoring after a slice wave (double-buffered)
    DevBuf<uint64_t> acc;        // their running totals (5 words per guide)
    DevBuf<uint8_t> batch;
    uint8_t* h_batch = nullptr;
    size_t sets_cap = 0;
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    uint64_t graph_epoch = ~0ull;
    uint32_t graph_tuning = ~0u;
    uint64_t graph_kernels = 0;
    // host-list index: two device windows of staged slices, the stream that fills them, and the
    // events that order the fills with the scans (window b is free again once the resolve pass of
    // the wave that used it has run)
    DevBuf<uint32_t> win_ids[2], win_rbits[2];
    cudaStream_t copy_stream = nullptr;
    cudaEvent_t win_start = nullptr, win_ready[2] = {}, win_free[2] = {};
    ~Workspace() {
        if (graph) cudaGraphExecDestroy(graph);
        for (cudaEvent_t e : {win_start, win_ready[0], win_ready[1], win_free[0], win_free[1]})
            if (e) cudaEventDestroy(e);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        if (h_batch) cudaFreeHost(h_batch);
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (own_stream) cudaStreamDestroy(own_stream);
        if (cap_stream) cudaStreamDestroy(cap_stream);
    }
};

issl_index::issl_index() = default;
issl_index::~issl_index() = default;

namespace issl {
namespace {

// ---------------------------------------------------------------------------------------------
// 1. probes
__global__ void k_encode_ascii(const char* __restrict__ ascii, size_t stride, uint64_t n, uint64_t* __restrict__ qsig) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const char* p = ascii + i * stride;
        uint64_t s = 0;
#pragma unroll
        for (int j = 0; j < kSeqLen; j++) {
            const char c = p[j];
            const uint64_t b = c == 'C' ? 1u : c == 'G' ? 2u : c == 'T' ? 3u : 0u;  // nucleotideIndex, :10
            s |= b << (2 * j);
        }
        qsig[i] = s;
    }
}

// n: guides, or *d_n when the count lives on the device (batch form)
__device__ __forceinline__ uint64_t guide_count(const uint32_t* d_n, uint64_t n) { return d_n ? *d_n : n; }

// The probes of one wave: every guide still scoring x the wave's slices [s0, s0 + sw). Guides
// are the list `active` of *d_nact entries, or all guides (active == nullptr) in the first wave.
struct WaveProbes {
    const uint32_t* active;
    const uint32_t* d_nact;
    const uint32_t* d_n;
    uint64_t n;
    uint32_t s0, sw;
    __device__ uint64_t guides() const { return d_nact ? *d_nact : guide_count(d_n, n); }
    __device__ void at(uint64_t p, uint64_t& q, uint32_t& s) const {
        const uint64_t i = p / sw;
        s = s0 + static_cast<uint32_t>(p - i * sw);
        q = active ? active[i] : i;
    }
};

__global__ void k_probe_count(IndexView ix, const uint64_t* __restrict__ qsig, WaveProbes wp,
                              uint32_t* __restrict__ probe_gb, uint32_t* __restrict__ bucket_cnt,
                              const uint64_t* __restrict__ off) {
    __shared__ SliceGeom g[kMaxSlices];
    for (int i = threadIdx.x; i < static_cast<int>(ix.n_slices); i += blockDim.x) g[i] = ix.geom[i];
    __syncthreads();
    const uint64_t total = wp.guides() * wp.sw;
    for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < total;
         p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        uint64_t q;
        uint32_t s;
        wp.at(p, q, s);
        const uint32_t gb = g[s].bbase + slice_key(qsig[q], g[s]);
        const bool nonempty = off[gb + 1] > off[gb];
        probe_gb[p] = nonempty ? gb : kEmpty;
        if (nonempty) atomicAdd(&bucket_cnt[gb], 1u);
    }
}

// 2. bucket scan: value = (units << 32) | probes
// g counts from g0, the first bucket of the wave's slices
struct BucketLoad {
    const uint32_t* cnt;
    const uint64_t* off;
    uint64_t n_sites;
    ChunkClasses cc;
    uint64_t g0;
    __device__ uint64_t operator()(uint64_t gi) const {
        const uint64_t g = g0 + gi;
        const uint32_t c = cnt[g];
        if (!c) return 0;
        // a unit is up to C / 32 consecutive 32-entry blocks, counted from the bucket's first
        // block, so it never spans more than 32 blocks (one per lane)
        const uint64_t C = chunk_of(off[g + 1] - off[g], cc);
        const uint64_t sb = (off[g] / n_sites) * n_sites;
        const uint64_t chunks = (((off[g + 1] - 1 - sb) >> 5) - ((off[g] - sb) >> 5)) / (C >> 5) + 1;
        const uint64_t units = chunks * ((c + kGroup - 1) / kGroup);
        return (units << 32) | c;
    }
};

// the bucket's first probe slot and first unit (exclusive prefixes over the wave's buckets)
struct BucketStore {
    uint32_t* qstart;
    uint32_t* ustart;
    uint64_t g0;
    __device__ void operator()(uint64_t gi, uint64_t ex, uint64_t) const {
        qstart[g0 + gi] = static_cast<uint32_t>(ex);
        ustart[g0 + gi] = static_cast<uint32_t>(ex >> 32);
    }
};

// Slice of a list position in global entry numbering (s * n + position), without a 64-bit divide:
// a double estimate, corrected by one either way.
__device__ __forceinline__ uint64_t slice_of_entry(uint64_t e, uint64_t n, double inv_n) {
    uint64_t s = static_cast<uint64_t>(static_cast<double>(e) * inv_n);
    if (s * n > e) s--;
    else if ((s + 1) * n <= e) s++;
    return s;
}

// Unit descriptors. A bucket's units run over the chunk-aligned blocks of its list range (counted
// from its first block), and within a chunk over its groups of up to kGroup guides: unit r of the
// bucket is chunk r / groups, group r % groups, and lands at ustart[bucket] + r. Each lane reads
// one bucket; the units of the warp's 32 buckets are consecutive and the warp writes them 32 at a
// time, so hot buckets probed by many guides spread over the lanes too. The same pass adds up the
// wave's work counters for the roofline:
// distinct buckets scanned, entries compared and bit-sliced bytes copied (once per guide group),
// and the probes per bucket-size class.
struct UnitSpan {
    uint64_t e0, e1;   // list range of the bucket
    uint32_t c;        // guides probing it
    uint32_t ng, lc;   // guide groups, log2 of the unit size
    uint32_t u0, q0;   // first unit, first probe slot
    uint32_t s;        // slice
};
__device__ __forceinline__ void write_unit(const UnitSpan& b, uint32_t r, uint32_t n, UnitDesc* __restrict__ units) {
    const uint32_t u = b.u0 + r;
    if (u >= n) return;  // past the buffer's capacity: the host grows it and reruns
    const uint32_t k = r / b.ng, j = r - k * b.ng;
    const uint64_t B0 = b.e0 >> 5;
    const uint64_t first = (B0 + (static_cast<uint64_t>(k) << (b.lc - 5))) << 5;
    const uint64_t last = (B0 + (static_cast<uint64_t>(k + 1) << (b.lc - 5))) << 5;
    const uint64_t cb = first > b.e0 ? first : b.e0;
    const uint64_t ce = last < b.e1 ? last : b.e1;
    UnitDesc d;
    d.p0 = static_cast<uint32_t>(cb);
    d.qbeg = b.q0 + j * kGroup;
    d.len = static_cast<uint16_t>(ce - cb);
    d.qn = static_cast<uint8_t>(b.c - j * kGroup < kGroup ? b.c - j * kGroup : kGroup);
    d.s = static_cast<uint8_t>(b.s);
    d.pad = 0;
    units[u] = d;
}

__global__ void k_expand_units(const uint32_t* __restrict__ cnt, const uint64_t* __restrict__ off,
                               const uint32_t* __restrict__ qstart, const uint32_t* __restrict__ ustart, uint64_t g0,
                               uint64_t g1, uint64_t n_sites, double inv_n, ChunkClasses cc,
                               const SliceGeom* __restrict__ geom, Counters* __restrict__ ctr,
                               UnitDesc* __restrict__ units) {
    const uint32_t n = ctr->n_units;  // at most the buffer's capacity
    const int lane = threadIdx.x & 31;
    uint64_t buckets = 0, entries = 0, bytes = 0, cp[3] = {0, 0, 0};
    // warp-aligned grid stride, so that the hot-bucket path below is uniform across the warp
    const uint64_t stride = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    for (uint64_t g = g0 + blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; g - lane < g1; g += stride) {
        UnitSpan b{0, 0, 0, 1, 5, 0, 0, 0};
        uint32_t nu = 0, u0 = 0xFFFFFFFFu;  // past the wave: after every unit
        if (g < g1) {
            b.c = cnt[g];
            u0 = ustart[g];
        }
        if (b.c) {
            b.s = static_cast<uint32_t>(slice_of_entry(off[g], n_sites, inv_n));
            b.e0 = off[g] - b.s * n_sites;  // list positions
            b.e1 = off[g + 1] - b.s * n_sites;
            const uint64_t C = chunk_of(b.e1 - b.e0, cc);
            b.lc = __ffs(static_cast<uint32_t>(C)) - 1;  // unit sizes are powers of 2
            b.ng = (b.c + kGroup - 1) / kGroup;
            b.u0 = u0;
            b.q0 = qstart[g];
            const uint64_t nb = ((b.e1 - 1) >> 5) - (b.e0 >> 5) + 1;  // blocks the bucket touches
            nu = static_cast<uint32_t>((nb - 1) / (C >> 5) + 1) * b.ng;
            buckets++;
            entries += (b.e1 - b.e0) * b.ng;
            bytes += nb * geom[b.s].wpb * 4ull * b.ng;
            const uint64_t len = b.e1 - b.e0;
            cp[0] += len < 64 ? b.c : 0u;
            cp[1] += len >= 64 && len < 4096 ? b.c : 0u;
            cp[2] += len >= 4096 ? b.c : 0u;
        }
        // the warp's buckets own the consecutive units [U0, U0 + T); each round lane l writes unit
        // U0 + t0 + l (coalesced), whose bucket is that of the last lane starting at or before it
        // (an empty bucket starts where the next non-empty one does, so that lane is non-empty)
        const uint32_t T = __reduce_add_sync(0xffffffffu, nu);
        const uint32_t U0 = __shfl_sync(0xffffffffu, u0, 0);
        for (uint32_t t0 = 0; t0 < T; t0 += 32) {
            const uint32_t w = U0 + t0 + static_cast<uint32_t>(lane);
            int o = 0;
#pragma unroll
            for (int step = 16; step > 0; step >>= 1)
                if (__shfl_sync(0xffffffffu, u0, o + step) <= w) o += step;
            UnitSpan h;
            h.e0 = __shfl_sync(0xffffffffu, b.e0, o);
            h.e1 = __shfl_sync(0xffffffffu, b.e1, o);
            h.c = __shfl_sync(0xffffffffu, b.c, o);
            h.ng = __shfl_sync(0xffffffffu, b.ng, o);
            h.lc = __shfl_sync(0xffffffffu, b.lc, o);
            h.u0 = __shfl_sync(0xffffffffu, u0, o);
            h.q0 = __shfl_sync(0xffffffffu, b.q0, o);
            h.s = __shfl_sync(0xffffffffu, b.s, o);
            if (t0 + lane < T) write_unit(h, w - h.u0, n, units);
        }
    }
    for (int d = 16; d > 0; d >>= 1) {
        buckets += __shfl_down_sync(0xffffffffu, buckets, d);
        entries += __shfl_down_sync(0xffffffffu, entries, d);
        bytes += __shfl_down_sync(0xffffffffu, bytes, d);
        for (int i = 0; i < 3; i++) cp[i] += __shfl_down_sync(0xffffffffu, cp[i], d);
    }
    if (lane == 0 && buckets) {
        atomicAdd(reinterpret_cast<unsigned long long*>(&ctr->buckets), buckets);
        atomicAdd(reinterpret_cast<unsigned long long*>(&ctr->entries), entries);
        atomicAdd(reinterpret_cast<unsigned long long*>(&ctr->rbytes), bytes);
        for (int i = 0; i < 3; i++)
            if (cp[i]) atomicAdd(reinterpret_cast<unsigned long long*>(&ctr->class_probes[i]), cp[i]);
    }
}

__global__ void k_units_finalize(Counters* c, uint64_t unit_cap) {
    const uint64_t u = c->bucket_total >> 32;
    c->n_units = static_cast<uint32_t>(u < unit_cap ? u : unit_cap);
    if (u > unit_cap) atomicOr(&c->overflow, 1u);
    if (u > c->max_units) c->max_units = u;
    c->units += u;
    c->probes += c->bucket_total & 0xFFFFFFFFull;
}

// 3. guides grouped by bucket; each slot holds (guide index, guide residual code for the slice)
__global__ void k_probe_scatter(IndexView ix, const uint64_t* __restrict__ qsig, WaveProbes wp,
                                const uint32_t* __restrict__ probe_gb, uint32_t* __restrict__ bucket_cnt,
                                const uint32_t* __restrict__ qstart, uint64_t* __restrict__ probe_qr) {
    __shared__ SliceGeom g[kMaxSlices];
    for (int i = threadIdx.x; i < static_cast<int>(ix.n_slices); i += blockDim.x) g[i] = ix.geom[i];
    __syncthreads();
    const uint64_t total = wp.guides() * wp.sw;
    for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < total;
         p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t gb = probe_gb[p];
        if (gb == kEmpty) continue;
        uint64_t q;
        uint32_t s;
        wp.at(p, q, s);
        // the decrement leaves bucket_cnt all zero for the next call
        const uint32_t slot = qstart[gb] + atomicSub(&bucket_cnt[gb], 1u) - 1u;
        probe_qr[slot] = q | (static_cast<uint64_t>(slice_residual(qsig[q], g[s])) << 32);
    }
}

// ---------------------------------------------------------------------------------------------
// 4. the scan
//
// A unit is up to 32 bit-sliced blocks of 32 list positions (at most kChunk = 1024 entries; the
// unit size per bucket-size class is tunable) and up to kGroup guides. Each warp runs its own
// ring of 2..4 stages in shared memory: for unit t + stages it issues two bulk copies (cp.async.bulk, the TMA engine) -- the unit's blocks and its guides'
// (index, residual) pairs -- completing on the stage's mbarrier, while it computes unit t from
// the stage that has landed. Lane l takes block l: per guide it forms the mismatch word of every
// residual position (32 entries at once), adds them with a carry-save tree and keeps the entries
// within max_dist. Candidates (rare) are written as (guide | slice, list position) to slabs of the
// candidate buffer that the warp reserves kCandSlab at a time; k_cand_resolve then reads each one's
// list entry and applies the ownership rule with every lane busy.
struct ScanArgs {
    const uint32_t* rbits;
    uint64_t rbits_base;  // global word number of rbits[0]
    const SliceGeom* geom;
    const UnitDesc* units;
    const uint64_t* probe_qr;
    Counters* counters;
    uint2* cands;
    uint32_t* qcand;      // candidates per guide (sizes the guides' hit segments)
    uint32_t n_slices;
    uint32_t cand_cap;
    int max_dist;
    const BatchHeader* hdr;  // batch form: the bound is the largest max_dist of the sets
    WarpLayout L;
};

struct ScanShared {  // per-block slice tables
    uint64_t wbase[kMaxSlices];
    uint8_t wpb[kMaxSlices], rw[kMaxSlices];
};

struct ScanCtx {  // per-warp state of the candidate slab
    uint32_t cpos, cend;
    bool full;
};

// Writes the warp's candidate records out: record r is (guide | lane << 26, word), the entries of
// block b0 + lane within the bound for that guide. Every lane takes one record per round; the
// round's candidates are counted per guide and written as (guide | slice << 26, list position) to
// consecutive slots of the warp's slab (k_cand_resolve then reads each one's list entry and applies
// the ownership rule to the site's mismatch positions).
__device__ __forceinline__ void flush_records(const ScanArgs& a, const uint2* rec, uint32_t nrec, const StageMeta& m,
                                              int lane, ScanCtx& cx) {
    __syncwarp();  // the records are written
    for (uint32_t r0 = 0; r0 < nrec; r0 += 32) {
        const uint32_t j = r0 + static_cast<uint32_t>(lane);
        const uint2 rc = j < nrec ? rec[j] : make_uint2(0u, 0u);
        const uint32_t c = __popc(rc.y);
        // slot of the lane's first candidate within the round: usually every record holds one
        // candidate and the lane's own index is its offset; otherwise an inclusive prefix
        uint32_t inc = j < nrec ? static_cast<uint32_t>(lane) + 1u : 0u;
        uint32_t tot = nrec - r0 < 32u ? nrec - r0 : 32u;
        if (__ballot_sync(0xffffffffu, c > 1u)) {
            inc = c;
#pragma unroll
            for (int dd = 1; dd < 32; dd <<= 1) {
                const uint32_t o = __shfl_up_sync(0xffffffffu, inc, dd);
                if (lane >= dd) inc += o;
            }
            tot = __shfl_sync(0xffffffffu, inc, 31);
        }
        if (cx.cpos + tot > cx.cend) {
            // retire the rest of the slab, reserve a new one (at least the round's candidates)
            for (uint32_t i = cx.cpos + lane; i < cx.cend; i += 32)
                if (i < a.cand_cap) a.cands[i] = make_uint2(kDeadCand, 0);
            // 64-bit reservations: a wave may ask for more than 2^32 slots (the host then splits
            // the guides); a slab past the capacity is never written
            const uint32_t want = tot > kCandSlab ? tot : kCandSlab;
            uint32_t base = 0, full = 0;
            if (lane == 0) {
                const unsigned long long b = atomicAdd(&a.counters->cand_reserved, static_cast<unsigned long long>(want));
                full = b + want > a.cand_cap;
                base = full ? a.cand_cap : static_cast<uint32_t>(b);
            }
            cx.cpos = __shfl_sync(0xffffffffu, base, 0);
            cx.cend = cx.cpos + want;
            cx.full = __shfl_sync(0xffffffffu, full, 0) != 0;
        }
        if (c) {
            const uint32_t g = rc.x & ((1u << kGuideBits) - 1u);
            atomicAdd(&a.qcand[g], c);
            if (!cx.full) {
                const uint32_t gx = g | (m.s << kGuideBits), p = 32u * (m.b0 + (rc.x >> kGuideBits));
                uint32_t o = cx.cpos + inc - c;
                for (uint32_t bits = rc.y; bits; bits &= bits - 1u) a.cands[o++] = make_uint2(gx, p + __ffs(bits) - 1u);
            }
        }
        cx.cpos += tot;
    }
    __syncwarp();  // the record buffer is read
}

// Compares every guide of the unit with the lane's block (RW residual positions per entry).
template <int RW>
__device__ __forceinline__ void scan_unit(const ScanArgs& a, const uint32_t* rb, const uint64_t* qr, uint32_t* qm,
                                          uint2* rec, const StageMeta& m, uint32_t wpb, int lane, int max_dist,
                                          ScanCtx& cx) {
    constexpr int NW = 2 * RW;
    constexpr int NV = (NW + 3) / 4;
    const unsigned lt = (1u << lane) - 1u;
    uint32_t nrec = 0;  // candidate records of the unit not yet written out (uniform)
    // this lane's block and the entries of it that belong to the unit (unsigned arithmetic: list
    // positions reach 2^32 - 1; the unit starts in block b0 and ends after this lane's block start)
    uint32_t d[NW];
    uint32_t valid = 0;
    const uint32_t bl = m.b0 + lane;
    if (static_cast<uint32_t>(lane) < m.nb) {
        const uint32_t base = 32u * bl, end = m.p0 + m.len;
        const uint32_t lo = m.p0 > base ? m.p0 - base : 0u;
        const uint32_t hi = end - base >= 32u ? 32u : end - base;
        valid = (hi >= 32u ? 0xFFFFFFFFu : ((1u << hi) - 1u)) & ~((1u << lo) - 1u);
    }
    // odd block stride: the 32 lanes read 32 different banks. Words of lanes past the unit are
    // stale but masked by `valid`.
    const uint32_t* blk = rb + m.delta + lane * wpb;
#pragma unroll
    for (int j = 0; j < NW; j++) d[j] = blk[j];
    // guide bit j spread to a word (qm[j] = 0 or ~0), double-buffered: the next guide's masks are
    // written while this guide's are read, one warp barrier per guide
    if (m.qn) {
        const uint32_t rq0 = static_cast<uint32_t>(qr[m.qoff] >> 32);
        __syncwarp();  // the previous unit's reads of the mask buffers are done
        if (lane < NW) qm[lane] = 0u - ((rq0 >> lane) & 1u);
    }
    for (uint32_t k = 0; k < m.qn; k++) {
        // this guide's masks are complete; the other buffer's last reads (the previous guide's)
        // are done, so it takes the next guide's masks while this one's are read
        __syncwarp();
        const uint64_t g = qr[m.qoff + k];
        if (k + 1 < m.qn) {
            const uint32_t rqn = static_cast<uint32_t>(qr[m.qoff + k + 1] >> 32);
            if (lane < NW) qm[32u * ((k + 1) & 1u) + lane] = 0u - ((rqn >> lane) & 1u);
        }
        // mismatch word of each residual position; guide masks come as 128-bit broadcast reads,
        // two positions per read
        const uint4* qm4 = reinterpret_cast<const uint4*>(qm + 32u * (k & 1u));
        uint32_t mm[RW];
#pragma unroll
        for (int v = 0; v < NV; v++) {
            const uint4 w = qm4[v];
            if (2 * v < RW) mm[2 * v] = (d[4 * v] ^ w.x) | (d[4 * v + 1] ^ w.y);
            if (2 * v + 1 < RW) mm[2 * v + 1] = (d[4 * v + 2] ^ w.z) | (d[4 * v + 3] ^ w.w);
        }
        const uint32_t cbits = bs::within(bs::count_mismatches<RW>(mm), max_dist) & valid;
        // candidate words are rare (about two lanes per guide and unit): each lane with one
        // appends (guide | lane << 26, word) to the warp's record buffer, which is written out
        // when it may not take another guide's 32 and when the unit ends. The comparison loop
        // itself has no branch on the data.
        const unsigned hm = __ballot_sync(0xffffffffu, cbits != 0);
        if (nrec > kScanRecs - 32u) {
            flush_records(a, rec, nrec, m, lane, cx);
            nrec = 0;
        }
        if (cbits)
            rec[nrec + __popc(hm & lt)] = make_uint2(static_cast<uint32_t>(g) | (static_cast<uint32_t>(lane) << kGuideBits), cbits);
        nrec += __popc(hm);
    }
    if (nrec) flush_records(a, rec, nrec, m, lane, cx);
}

// RWFIX > 0: every slice of the index has RWFIX residual positions; 0: mixed widths.
// Persistent and work-stealing: each warp takes batches of 32 consecutive units from a global
// queue (one atomic per batch), so warps that draw heavy units (hot repeat buckets with a full
// group of guides) simply take fewer batches. The 10- and 12-position scans keep to 72 registers,
// so that seven blocks fit an SM (the shared-memory limit at two stages); the others to 96 (five).
template <int RWFIX>
__global__ void __launch_bounds__(kScanWarps * 32, RWFIX == 12 || RWFIX == 10 ? 7 : 5) k_scan(ScanArgs a) {
    extern __shared__ __align__(16) uint8_t smem_raw[];
    __shared__ ScanShared sh;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const WarpLayout L = a.L;
    const uint32_t NS = L.stages;
    uint8_t* wbase_ptr = smem_raw + static_cast<size_t>(warp) * L.bytes;
    uint32_t* rb = reinterpret_cast<uint32_t*>(wbase_ptr);
    uint64_t* qr = reinterpret_cast<uint64_t*>(wbase_ptr + L.qr_off);
    uint32_t* qm = reinterpret_cast<uint32_t*>(wbase_ptr + L.qm_off);
    uint2* rec = reinterpret_cast<uint2*>(wbase_ptr + L.rec_off);
    StageMeta* meta = reinterpret_cast<StageMeta*>(wbase_ptr + L.meta_off);
    uint64_t* bar = reinterpret_cast<uint64_t*>(wbase_ptr + L.bar_off);
    for (int i = threadIdx.x; i < static_cast<int>(a.n_slices); i += blockDim.x) {
        sh.wbase[i] = a.geom[i].wbase;
        sh.wpb[i] = a.geom[i].wpb;
        sh.rw[i] = a.geom[i].rwidth;
    }
    if (lane == 0) {
        for (uint32_t st = 0; st < NS; st++) mbar_init(&bar[st], 1);
        fence_barrier_init();
    }
    __syncthreads();
    const int max_dist = a.hdr ? a.hdr->max_dist : a.max_dist;

    const uint32_t n_units = a.counters->n_units;
    const uint32_t n_batches = (n_units + 31) / 32;
    // descriptor of unit (batch b, slot lane); len 0 marks "no unit"
    auto take_batch = [&]() -> uint4 {
        uint32_t b = 0;
        if (lane == 0) b = atomicAdd(&a.counters->next_batch, 1u);
        b = __shfl_sync(0xffffffffu, b, 0);
        const uint32_t u = b * 32u + lane;
        return (b < n_batches && u < n_units) ? __ldg(reinterpret_cast<const uint4*>(a.units) + u)
                                              : make_uint4(0, 0, 0, 0);
    };
    uint4 dA = take_batch(), dB = make_uint4(0, 0, 0, 0);
    bool have_b = false;
    uint32_t issued = 0;  // units of this warp issued so far (unit t lives in ring stage t % NS)
    uint32_t ist = 0;     // ring stage of the next unit to issue (issued % NS, kept without a divide)
    uint32_t slot = 0;    // slot of the next unit in batch A
    bool ended = false;

    // issues the copies of the warp's next unit, if there is one (all lanes call; lane 0 issues)
    auto try_issue = [&]() {
        if (ended) return;
        if (slot == 32) {
            if (!have_b) dB = take_batch();
            dA = dB;
            have_b = false;
            slot = 0;
        }
        const uint32_t dz = __shfl_sync(0xffffffffu, dA.z, slot);
        if ((dz & 0xFFFFu) == 0) {
            ended = true;
            return;
        }
        // take the following batch one unit early so its descriptor load overlaps this copy
        if (slot == 31 && !have_b) {
            dB = take_batch();
            have_b = true;
        }
        const uint32_t p0 = __shfl_sync(0xffffffffu, dA.x, slot), qbeg = __shfl_sync(0xffffffffu, dA.y, slot);
        if (lane == 0) {
            const uint32_t st = ist;
            const uint32_t len = dz & 0xFFFFu, qn = (dz >> 16) & 0xFFu, s = dz >> 24;
            const uint32_t b0 = p0 / 32u, nb = (p0 + len - 1) / 32u - b0 + 1;  // <= 32: inside one chunk
            const uint32_t wpb = sh.wpb[s];
            // blocks are wpb (odd) words long: copy from the 16-byte boundary at or below the
            // first block and skip the `delta` leading words in shared memory
            const uint64_t w0 = sh.wbase[s] + static_cast<uint64_t>(b0) * wpb, wa = w0 & ~3ull;
            const uint32_t delta = static_cast<uint32_t>(w0 - wa);
            const uint32_t nwords = (delta + nb * wpb + 3u) & ~3u;
            const uint32_t qa0 = qbeg & ~1u, qa1 = (qbeg + qn + 1) & ~1u;
            StageMeta& m = meta[st];
            m.p0 = p0;
            m.len = len;
            m.b0 = b0;
            m.nb = nb;
            m.qoff = qbeg - qa0;
            m.qn = qn;
            m.s = s;
            m.delta = delta;
            const uint32_t rbytes = nwords * 4u, qbytes = (qa1 - qa0) * 8u;
            fence_proxy_async_smem();
            mbar_arrive_expect_tx(&bar[st], rbytes + qbytes);
            bulk_copy_g2s(rb + st * L.stage_words, a.rbits + (wa - a.rbits_base), rbytes, &bar[st]);
            bulk_copy_g2s(qr + st * kStageQr, a.probe_qr + qa0, qbytes, &bar[st]);
        }
        slot++;
        issued++;
        if (++ist == NS) ist = 0;
    };

    ScanCtx cx{0u, 0u, false};
    for (uint32_t i = 0; i < NS; i++) try_issue();
    __syncwarp();

    uint32_t t = 0, st = 0, phase = 0;
    bool failed = false;
    for (; t < issued; t++) {
        const bool ok = mbar_wait_bounded(&bar[st], phase, kWaitCycles);
        if (__any_sync(0xffffffffu, !ok)) {
            failed = true;
            break;
        }
        const StageMeta m = meta[st];
        const uint32_t wpb = sh.wpb[m.s];
        const uint32_t* srb = rb + st * L.stage_words;
        const uint64_t* sqr = qr + st * kStageQr;
        if constexpr (RWFIX > 0) {
            scan_unit<RWFIX>(a, srb, sqr, qm, rec, m, wpb, lane, max_dist, cx);
        } else switch (sh.rw[m.s]) {  // uniform across the warp
            case 12: scan_unit<12>(a, srb, sqr, qm, rec, m, wpb, lane, max_dist, cx); break;
            case 10: scan_unit<10>(a, srb, sqr, qm, rec, m, wpb, lane, max_dist, cx); break;
            case 16: scan_unit<16>(a, srb, sqr, qm, rec, m, wpb, lane, max_dist, cx); break;
            case 15: scan_unit<15>(a, srb, sqr, qm, rec, m, wpb, lane, max_dist, cx); break;
            case 14: scan_unit<14>(a, srb, sqr, qm, rec, m, wpb, lane, max_dist, cx); break;
            case 13: scan_unit<13>(a, srb, sqr, qm, rec, m, wpb, lane, max_dist, cx); break;
            case 11: scan_unit<11>(a, srb, sqr, qm, rec, m, wpb, lane, max_dist, cx); break;
            case 9: scan_unit<9>(a, srb, sqr, qm, rec, m, wpb, lane, max_dist, cx); break;
            case 8: scan_unit<8>(a, srb, sqr, qm, rec, m, wpb, lane, max_dist, cx); break;
            default: scan_unit<7>(a, srb, sqr, qm, rec, m, wpb, lane, max_dist, cx); break;
        }
        __syncwarp();  // every lane is done with stage st before it is refilled
        try_issue();
        if (++st == NS) {
            st = 0;
            phase ^= 1u;
        }
    }
    if (failed) {
        // a copy did not land in time: report, then wait (bounded) for this warp's copies in flight
        if (lane == 0) atomicOr(&a.counters->overflow, 4u);
        for (uint32_t u = t; u < issued; u++) mbar_wait_bounded(&bar[u % NS], (u / NS) & 1u, kWaitCycles);
    }
    for (uint32_t i = cx.cpos + lane; i < cx.cend; i += 32)
        if (i < a.cand_cap) a.cands[i] = make_uint2(kDeadCand, 0);
}

__global__ void k_cands_finalize(Counters* c, uint32_t cand_cap) {
    const unsigned long long r = c->cand_reserved;
    if (r > cand_cap) atomicOr(&c->overflow, 2u);
    if (r > c->max_cand) c->max_cand = r;
    c->cands += r;
    c->n_cand = static_cast<uint32_t>(r < cand_cap ? r : cand_cap);
}

// ---------------------------------------------------------------------------------------------
// 5. per-guide segments: the scan counts each guide's candidates; their exclusive prefix gives
// every guide a segment of the hit buffer large enough for all of them, which the resolve pass
// fills from its start with the candidates that survive the ownership rule
struct LoadQhits {
    const uint32_t* p;
    __device__ uint32_t operator()(uint64_t i) const { return p[i]; }
};
// p[n] receives the total: element i also writes its inclusive prefix to p[i + 1] (the same
// value element i + 1 writes as its exclusive prefix)
struct StoreQoff {
    uint32_t* p;
    __device__ void operator()(uint64_t i, uint32_t ex, uint32_t inc) const {
        p[i] = ex;
        p[i + 1] = inc;
    }
};

// ---------------------------------------------------------------------------------------------
// 7. scoring of one guide's hits in the reference's visiting order
__device__ __forceinline__ uint64_t order_key(const uint4& r) {
    return (static_cast<uint64_t>(r.y) << 32) | r.x;  // slice, then list position
}

struct Contribution {
    double mit, cfd;
    uint32_t occ;
    int dist;  // mismatches between the guide and the site
};

// MIT (ISSLScoringModule.cpp:294-298) and CFD (:301-363) contributions of one site.
__device__ __forceinline__ Contribution contribution(const Tables& T, const ScoreParams& P, uint64_t q,
                                                     uint64_t sig, uint32_t occ) {
    const uint64_t mism = fold64(q ^ sig);
    const int dist = __popcll(mism);
    const uint32_t m20 = compress_even40(mism);
    Contribution c;
    c.occ = occ;
    c.mit = 0.0;
    c.cfd = 0.0;
    c.dist = dist;
    if (P.calc_mit && dist > 0 && dist <= kMaxDist) {  // the table holds 1..4 mismatches
        uint32_t rank = 0, i = 0, mm = m20;
        while (mm) {
            const int p = __ffs(mm) - 1;
            rank += T.binom[p][++i];
            mm &= mm - 1;
        }
        const uint32_t base = i == 1 ? 0u : i == 2 ? 20u : i == 3 ? 210u : 1350u;
        c.mit = __dmul_rn(T.mit[base + rank], static_cast<double>(occ));
    }
    if (P.calc_cfd) {
        double s = 1.0;
        if (dist > 0) {
            s = T.cfd_pam[0xA];  // PAM NGG
            uint32_t mm = m20;
            while (mm) {  // ascending positions, as the reference's pos loop multiplies
                const int p = __ffs(mm) - 1;
                const uint32_t qb = static_cast<uint32_t>(q >> (2 * p)) & 3u;
                const uint32_t ob = static_cast<uint32_t>(sig >> (2 * p)) & 3u;
                s = __dmul_rn(s, T.cfd_pos[(p << 4) | (qb << 2) | (ob ^ 3u)]);
                mm &= mm - 1;
            }
        }
        c.cfd = __dmul_rn(s, static_cast<double>(occ));
    }
    return c;
}

// 6. One thread per candidate (many independent random reads in flight). The list entry gives the
// site id, its occurrences and (8-byte entries) its residual code, from which the signature is
// rebuilt; with 4-byte entries the signature is a second read. The site's mismatch positions
// against the guide then settle the ownership rule (a site reached in slice s is counted only if
// no earlier slice has all its positions matching, the reference's toggle bitset of :252-258):
// avoid[p] holds the slices that do not contain position p, so the slices whose positions all
// match the site are the AND of avoid[] over its (at most four) mismatch positions. An owned site's
// MIT and CFD contributions are computed here, where the reads leave the arithmetic units idle, and
// its record is written to the next free slot of its guide's segment, so the scorers read only
// contiguous data.
__global__ void __launch_bounds__(256, 8)
    k_cand_resolve(const uint2* __restrict__ cands, Counters* c, IndexView ix, const uint64_t* __restrict__ qsig,
                   const uint32_t* __restrict__ qoff, uint32_t* __restrict__ qfill, const Tables* __restrict__ tables,
                   HitRec* __restrict__ seg, const SetDesc* __restrict__ sets, const uint16_t* __restrict__ qset) {
    __shared__ SliceGeom g[kMaxSlices];
    __shared__ unsigned long long avoid[kSeqLen];
    for (int i = threadIdx.x; i < static_cast<int>(ix.n_slices); i += blockDim.x) g[i] = ix.geom[i];
    if (threadIdx.x < kSeqLen) {
        unsigned long long m = 0;
        for (uint32_t e = 0; e < ix.n_slices; e++)
            if (!((ix.geom[e].pmask >> threadIdx.x) & 1u)) m |= 1ull << e;
        avoid[threadIdx.x] = m;
    }
    __syncthreads();
    if (c->overflow) return;  // the host grows the buffers and reruns
    const Tables& T_ = *tables;
    ScoreParams both{};
    both.calc_mit = 1;
    both.calc_cfd = 1;
    const uint32_t n = c->n_cand;
    uint32_t owned_here = 0;
    // one candidate per thread and round, eight blocks per SM (the grid is one wave): at the
    // 300M-site workload two or four candidates per thread with five or four blocks were 4-6%
    // slower (random list-entry reads, the L2 atomics of the segment fill and the hit writes
    // are all latency-bound)
    constexpr int U = 1;
    const uint32_t T = gridDim.x * blockDim.x;
    for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += U * T) {
        uint2 r[U];
        uint64_t gq[U];
        uint2 e[U];
#pragma unroll
        for (int u = 0; u < U; u++) {
            const uint32_t i = i0 + u * T;
            r[u] = i < n ? cands[i] : make_uint2(kDeadCand, 0u);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (r[u].x == kDeadCand) continue;
            gq[u] = qsig[r[u].x & ((1u << kGuideBits) - 1u)];
            e[u] = load_entry(ix, r[u].x >> kGuideBits, r[u].y);
        }
#pragma unroll
        for (int u = 0; u < U; u++) {
            if (r[u].x == kDeadCand) continue;
            const uint32_t s = r[u].x >> kGuideBits;
            const uint32_t q = r[u].x & ((1u << kGuideBits) - 1u);
            const uint32_t id = entry_id(e[u].x, ix.id_bits);
            const uint64_t sig = ix.entry_words == 2 ? site_signature(gq[u], e[u].y, g[s]) : ix.sigs[id];
            const uint32_t mism20 = compress_even40(fold64(gq[u] ^ sig));
            const int dist = __popc(mism20);
            if (dist > kMaxDist) {
                // the scan found this site within the bound: a record that says otherwise does not
                // describe a site of the guide's bucket (counted; the call then fails)
                atomicAdd(reinterpret_cast<unsigned long long*>(&c->dropped), 1ull);
                continue;
            }
            // batch form: the scan kept candidates up to the largest bound of the batch's sets
            if (qset && dist > sets[qset[q]].P.max_dist) continue;
            unsigned long long reach = ~0ull;  // slices whose positions all match the site
            for (uint32_t mm = mism20; mm; mm &= mm - 1) reach &= avoid[__ffs(mm) - 1];
            if (reach & ((1ull << s) - 1ull)) continue;  // an earlier slice reaches this site
            const uint32_t occ = entry_occ(e[u].x, ix);
            const Contribution ct = contribution(T_, both, gq[u], sig, occ);
            const uint32_t slot = qoff[q] + atomicAdd(&qfill[q], 1u);
            seg[slot] = HitRec{make_uint4(r[u].y, s, id, occ), ct.mit, ct.cfd};
            owned_here++;
        }
    }
    for (int d = 16; d > 0; d >>= 1) owned_here += __shfl_xor_sync(0xffffffffu, owned_here, d);
    if ((threadIdx.x & 31) == 0 && owned_here) atomicAdd(&c->hit_total, owned_here);
}

__device__ __forceinline__ bool exit_test(const ScoreParams& P, double mit, double cfd) {
    const double M = P.maximum_sum;  // :366-395
    switch (P.method) {
        case ISSL_METHOD_MIT_AND_CFD: return mit > M && cfd > M;
        case ISSL_METHOD_MIT_OR_CFD: return mit > M || cfd > M;
        case ISSL_METHOD_AVG_MIT_CFD: return ((mit + cfd) / 2.0) > M;
        case ISSL_METHOD_MIT: return mit > M;
        default: return cfd > M;
    }
}

// The accept rule on the sums where scoring stopped (:404-459).
__device__ __forceinline__ bool rejects(const ScoreParams& P, double tot_mit, double tot_cfd) {
    const double t = P.threshold;
    const double m = 10000.0 / (100.0 + tot_mit), c = 10000.0 / (100.0 + tot_cfd);  // :407-448
    switch (P.method) {
        case ISSL_METHOD_MIT_AND_CFD: return m < t && c < t;
        case ISSL_METHOD_MIT_OR_CFD: return m < t || c < t;
        case ISSL_METHOD_AVG_MIT_CFD: return (m + c) / 2 < t;
        case ISSL_METHOD_MIT: return m < t;
        default: return c < t;
    }
}

__device__ __forceinline__ void finalise(const ScoreParams& P, double tot_mit, double tot_cfd, uint64_t count,
                                         uint64_t q_index, double* out_mit, double* out_cfd, char* out_code,
                                         uint64_t* out_count) {
    const bool reject = rejects(P, tot_mit, tot_cfd);
    const double m = P.method == ISSL_METHOD_CFD ? -1.0 : 10000.0 / (100.0 + tot_mit);
    const double c = P.method == ISSL_METHOD_MIT ? -1.0 : 10000.0 / (100.0 + tot_cfd);
    if (out_mit) out_mit[q_index] = m;
    if (out_cfd) out_cfd[q_index] = c;
    out_code[q_index] = reject ? ISSL_CODE_REJECTED : ISSL_CODE_ACCEPTED;
    if (out_count) out_count[q_index] = count;
}

// Decisions within the reference's rounding. The reference adds a guide's contributions one at a
// time in double precision, in slice order then list order (:294-296, :362), tests its early exit
// after every addition (:366-395) and applies the accept rule to the sums where it stopped. The
// scorers below add the same contributions (the same rounded products) exactly, so an exact total
// S differs from the reference's running sum over the same hits only by the reference's own
// rounding: a sum of k non-negative terms rounded after every addition lies within (k - 1) u S
// of the exact sum (u = 2^-53; Higham, Accuracy and Stability of Numerical Algorithms, 2nd ed.,
// section 4.2). The exit tests and the accept rules are monotone in both sums, so a decision
// taken at both ends of that interval is the reference's when the two agree. When they do not
// (a threshold within a few ulps of one of the guide's running sums) the guide goes to
// k_replay, which repeats the reference's additions one by one.
struct Span {
    double lo, hi;
};
// terms bounds the number of non-zero additions (the occurrence sum: a site with no occurrences
// adds an exact zero); the 8 extra ulps cover the rounding of the exact total to a double and of
// this computation
__device__ __forceinline__ Span ref_span(double s, uint64_t terms) {
    const double w = s * (static_cast<double>(terms + 8) * 0x1p-52);
    return Span{fmax(s - w, 0.0), s + w};
}
// a guide whose exact running totals reach (m, c) without the exit test firing: does the
// reference certainly not fire either, and (last) does it certainly take the same decision?
__device__ __forceinline__ bool settled_without_exit(const ScoreParams& P, double m, double c, uint64_t terms,
                                                     bool last) {
    const Span sm = ref_span(m, terms), sc = ref_span(c, terms);
    if (exit_test(P, sm.hi, sc.hi)) return false;
    return !last || rejects(P, sm.lo, sc.lo) == rejects(P, sm.hi, sc.hi);
}
// a guide whose exact totals first fire the exit test at a hit, (pm, pc) before it and (m, c)
// with it: does the reference certainly stop at the same hit and take the same decision?
__device__ __forceinline__ bool settled_at_exit(const ScoreParams& P, double pm, double pc, double m, double c,
                                                uint64_t terms) {
    const Span bm = ref_span(pm, terms), bc = ref_span(pc, terms);
    const Span sm = ref_span(m, terms), sc = ref_span(c, terms);
    return !exit_test(P, bm.hi, bc.hi) && exit_test(P, sm.lo, sc.lo) &&
           rejects(P, sm.lo, sc.lo) == rejects(P, sm.hi, sc.hi);
}

__device__ __forceinline__ uint64_t warp_incl_sum_u64(uint64_t v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint64_t o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

struct Acc;

struct ScoreArgs {
    IndexView ix;
    const uint64_t* qsig;
    HitRec* seg;
    const uint32_t* qoff;    // each guide's hit segment: start, and hits written
    const uint32_t* qfill;
    const Tables* tables;
    Counters* counters;
    uint32_t* big;
    uint32_t* exitq;
    uint32_t* replay;        // guides left to k_replay
    uint32_t* bitmap;
    uint64_t n;
    const uint32_t* d_n;     // batch form: guide count on the device
    ScoreParams P;           // plain form: one parameter set for every guide
    const SetDesc* sets;     // batch form: per-set parameters, guide qi belongs to set qset[qi]
    const uint16_t* qset;
    double* out_mit;
    double* out_cfd;
    char* out_code;
    uint64_t* out_count;
    // slice waves: the guides of this wave, the guides that go on to the next one, and the
    // running totals carried between waves
    const uint32_t* active;  // nullptr: every guide (first wave)
    const uint32_t* d_nact;
    uint32_t* next_active;
    uint32_t* d_nnext;
    Acc* acc;
    int first_wave, last_wave;
};

__device__ __forceinline__ ScoreParams params_of(const ScoreArgs& a, uint64_t qi) {
    return a.qset ? a.sets[a.qset[qi]].P : a.P;
}

// Exact sums. Every contribution (MIT value x occurrences, CFD product x occurrences) lies in
// [6e-6, 2^33) and has no bit below 2^-84, so it converts exactly to a 128-bit fixed point
// value hi * 2^-20 + lo * 2^-84. Integer sums are exact and independent of the order of the
// additions: the totals are deterministic, need no sort, and are at least as accurate as the
// reference's sequential double sums (they are rounded once, when converted back).
struct Fx {
    uint64_t hi, lo;
};
__device__ __forceinline__ Fx fx_from(double c) {
    const double s = c * 1048576.0;  // 2^20
    const double h = floor(s);
    return Fx{static_cast<uint64_t>(h), __double2ull_rz((s - h) * 18446744073709551616.0)};  // x 2^64
}
__device__ __forceinline__ Fx fx_add(Fx a, Fx b) {
    Fx r;
    r.lo = a.lo + b.lo;
    r.hi = a.hi + b.hi + (r.lo < a.lo ? 1ull : 0ull);
    return r;
}
__device__ __forceinline__ Fx fx_sub(Fx a, Fx b) {
    Fx r;
    r.lo = a.lo - b.lo;
    r.hi = a.hi - b.hi - (a.lo < b.lo ? 1ull : 0ull);
    return r;
}
__device__ __forceinline__ double fx_double(Fx a) {
    return static_cast<double>(a.hi) * 9.5367431640625e-07 + static_cast<double>(a.lo) * 5.169878828456423e-26;
}
__device__ __forceinline__ Fx fx_shfl_up(Fx a, int d) {
    return Fx{__shfl_up_sync(0xffffffffu, a.hi, d), __shfl_up_sync(0xffffffffu, a.lo, d)};
}
__device__ __forceinline__ Fx fx_shfl_xor(Fx a, int d) {
    return Fx{__shfl_xor_sync(0xffffffffu, a.hi, d), __shfl_xor_sync(0xffffffffu, a.lo, d)};
}
__device__ __forceinline__ Fx fx_warp_incl(Fx v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const Fx o = fx_shfl_up(v, d);
        if (lane >= d) v = fx_add(o, v);
    }
    return v;
}
__device__ __forceinline__ Fx fx_warp_sum(Fx v) {
#pragma unroll
    for (int d = 16; d > 0; d >>= 1) v = fx_add(v, fx_shfl_xor(v, d));
    return v;
}

struct FxContribution {
    Fx mit, cfd;
    uint64_t occ;
};

// running totals of a guide carried from one slice wave to the next
struct Acc {
    Fx mit, cfd;
    uint64_t occ;
};

// a grouped hit's contributions under the guide's method (contribution() with its flags)
__device__ __forceinline__ FxContribution fx_contribution(const ScoreParams& P, const HitRec& h) {
    return FxContribution{fx_from(P.calc_mit ? h.mit : 0.0), fx_from(P.calc_cfd ? h.cfd : 0.0), h.r.w};
}

constexpr int kWarpSort = 1024;  // exiting guides with more hits are ordered by a whole block

// Warp per guide, pass 1: every hit's contribution added exactly. If the method's test does not
// fire on the totals it never fires on a prefix (contributions are >= 0 and the tests are
// monotone), so the totals are the reference's result and no ordering is needed; guides whose
// test fires go to the ordered scorers.
__global__ void __launch_bounds__(256) k_score_sum(ScoreArgs a) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (blockIdx.x == 0 && threadIdx.x == 0) a.counters->hits += a.counters->hit_total;
    if (a.counters->overflow) return;  // rerun follows
    const uint64_t gw = blockIdx.x * 8ull + warp, nw = gridDim.x * 8ull;
    const uint64_t n = a.d_nact ? *a.d_nact : guide_count(a.d_n, a.n);
    for (uint64_t i = gw; i < n; i += nw) {
        const uint64_t qi = a.active ? a.active[i] : i;
        const ScoreParams P = params_of(a, qi);
        const uint32_t h0 = a.qoff[qi], L = a.qfill[qi];
        const HitRec* seg = a.seg + h0;
        Fx tm{0, 0}, tc{0, 0};
        uint64_t tn = 0;
        auto add_hit = [&](const HitRec& hr) {
            const FxContribution c = fx_contribution(P, hr);
            tm = fx_add(tm, c.mit);
            tc = fx_add(tc, c.cfd);
            tn += c.occ;
        };
        // four hits per lane in flight, then the rest one at a time
        uint32_t j = lane;
        for (; j + 96 < L; j += 128) {
            const HitRec h0 = seg[j], h1 = seg[j + 32], h2 = seg[j + 64], h3 = seg[j + 96];
            add_hit(h0);
            add_hit(h1);
            add_hit(h2);
            add_hit(h3);
        }
        for (; j < L; j += 32) add_hit(seg[j]);
        tm = fx_warp_sum(tm);
        tc = fx_warp_sum(tc);
        for (int d = 16; d > 0; d >>= 1) tn += __shfl_xor_sync(0xffffffffu, tn, d);
        if (!a.first_wave) {
            const Acc pr = a.acc[qi];
            tm = fx_add(tm, pr.mit);
            tc = fx_add(tc, pr.cfd);
            tn += pr.occ;
        }
        const double dm = fx_double(tm), dc = fx_double(tc);
        if (exit_test(P, dm, dc)) {
            if (lane == 0) {
                if (L <= static_cast<uint32_t>(kWarpSort))
                    a.exitq[atomicAdd(&a.counters->n_exit, 1u)] = static_cast<uint32_t>(qi);
                else
                    a.big[atomicAdd(&a.counters->n_big, 1u)] = static_cast<uint32_t>(qi);
            }
            continue;
        }
        // within the reference's rounding of the exit test or (last wave) of the accept rule
        if (!settled_without_exit(P, dm, dc, tn, a.last_wave)) {
            if (lane == 0) a.replay[atomicAdd(&a.counters->n_replay, 1u)] = static_cast<uint32_t>(qi);
            continue;
        }
        if (P.want_distinct)
            for (uint32_t j = lane; j < L; j += 32) {
                const uint32_t id = seg[j].r.z;
                atomicOr(&a.bitmap[id >> 5], 1u << (id & 31));
            }
        if (lane == 0) {
            if (a.last_wave) {
                finalise(P, dm, dc, tn, qi, a.out_mit, a.out_cfd, a.out_code, a.out_count);
            } else {
                a.acc[qi] = Acc{tm, tc, tn};
                a.next_active[atomicAdd(a.d_nnext, 1u)] = static_cast<uint32_t>(qi);
            }
        }
    }
}

// Warp per guide whose test fires (at most kWarpSort hits). The reference visits hits by slice,
// then list position. The hits are first bucketed by slice (counting sort). Within a slice the
// order of the additions does not change exact totals, so lane t adds up slice t's hits, and one
// warp scan over the slice totals gives the running totals at every slice end; the first slice
// whose end fires the test is the one the reference stops in (the totals only grow, and a slice
// without hits repeats the test of the slice before it, which did not fire). Only that slice's
// hits are ordered by list position (a bitonic network whose comparators all point the same way;
// missing elements act as +infinity) to find the exact hit where the reference stops. Scores and
// counts are those at that hit. An exit slice with more than kOrdKeys hits goes to the block
// scorer.
constexpr int kOrdKeys = 256;
struct OrderedSmem {
    uint64_t keys[kOrdKeys];
    uint16_t idx[kWarpSort];
    uint32_t cnt[kMaxSlices + 1];
    uint32_t cur[kMaxSlices];
};

__device__ __forceinline__ uint32_t warp_incl_sum_u32(uint32_t v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

__global__ void __launch_bounds__(256, 3) k_score_ordered(ScoreArgs a) {
    extern __shared__ __align__(16) uint8_t s_raw[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    OrderedSmem& W = reinterpret_cast<OrderedSmem*>(s_raw)[warp];
    if (a.counters->overflow) return;  // rerun follows
    const uint32_t S = a.ix.n_slices;
    const uint32_t n_exit = a.counters->n_exit;
    const uint32_t gw = blockIdx.x * 8 + warp, nw = gridDim.x * 8;
    for (uint32_t e = gw; e < n_exit; e += nw) {
        const uint64_t qi = a.exitq[e];
        const ScoreParams P = params_of(a, qi);
        Fx rm{0, 0}, rc{0, 0};  // totals of the earlier waves
        uint64_t rn = 0;
        if (!a.first_wave) {
            const Acc pr = a.acc[qi];
            rm = pr.mit;
            rc = pr.cfd;
            rn = pr.occ;
        }
        const uint32_t h0 = a.qoff[qi], L = a.qfill[qi];
        const HitRec* seg = a.seg + h0;
        // counting sort of the hits by slice (four slice reads in flight per lane)
        for (uint32_t t = lane; t <= S; t += 32) W.cnt[t] = 0;
        __syncwarp();
        for (uint32_t i = lane; i < L; i += 128) {
            uint32_t y[4];
#pragma unroll
            for (int u = 0; u < 4; u++) y[u] = i + 32 * u < L ? seg[i + 32 * u].r.y : kEmpty;
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (y[u] != kEmpty) atomicAdd(&W.cnt[y[u]], 1u);
        }
        __syncwarp();
        uint32_t before = 0;  // hits in the slices of the earlier rounds
        for (uint32_t t0 = 0; t0 < S; t0 += 32) {
            const uint32_t t = t0 + lane;
            const uint32_t v = t < S ? W.cnt[t] : 0u;
            const uint32_t inc = warp_incl_sum_u32(v, lane);
            if (t < S) W.cnt[t] = W.cur[t] = before + inc - v;
            before += __shfl_sync(0xffffffffu, inc, 31);
        }
        if (lane == 0) W.cnt[S] = before;
        __syncwarp();
        for (uint32_t i = lane; i < L; i += 128) {
            uint32_t y[4];
#pragma unroll
            for (int u = 0; u < 4; u++) y[u] = i + 32 * u < L ? seg[i + 32 * u].r.y : kEmpty;
#pragma unroll
            for (int u = 0; u < 4; u++)
                if (y[u] != kEmpty) W.idx[atomicAdd(&W.cur[y[u]], 1u)] = static_cast<uint16_t>(i + 32 * u);
        }
        __syncwarp();
        // running totals at the slice ends, 32 slices per round; bm/bc/bn: the totals before the
        // exit slice
        Fx cm = rm, cc = rc, bm = rm, bc = rc;
        uint64_t cn = rn, bn = rn;
        int exit_sl = -1;
        for (uint32_t t0 = 0; t0 < S && exit_sl < 0; t0 += 32) {
            const uint32_t t = t0 + lane;
            // slice t's exact totals (four hits in flight)
            Fx sm{0, 0}, sc{0, 0};
            uint64_t so = 0;
            if (t < S) {
                const uint32_t j1 = W.cnt[t + 1];
                for (uint32_t j = W.cnt[t]; j < j1; j += 4) {
                    double hm[4], hc[4];
                    uint32_t ho[4];
#pragma unroll
                    for (int u = 0; u < 4; u++)
                        if (j + u < j1) {
                            const HitRec* hp = seg + W.idx[j + u];
                            hm[u] = hp->mit;
                            hc[u] = hp->cfd;
                            ho[u] = hp->r.w;
                        }
#pragma unroll
                    for (int u = 0; u < 4; u++)
                        if (j + u < j1) {
                            sm = fx_add(sm, fx_from(P.calc_mit ? hm[u] : 0.0));
                            sc = fx_add(sc, fx_from(P.calc_cfd ? hc[u] : 0.0));
                            so += ho[u];
                        }
                }
            }
            const Fx im = fx_add(fx_warp_incl(sm, lane), cm);
            const Fx ic = fx_add(fx_warp_incl(sc, lane), cc);
            const uint64_t in = warp_incl_sum_u64(so, lane) + cn;
            const unsigned fires = __ballot_sync(0xffffffffu, t < S && exit_test(P, fx_double(im), fx_double(ic)));
            if (fires) {
                const int f = __ffs(fires) - 1, pl = f > 0 ? f - 1 : 0;
                const Fx pm{__shfl_sync(0xffffffffu, im.hi, pl), __shfl_sync(0xffffffffu, im.lo, pl)};
                const Fx pc{__shfl_sync(0xffffffffu, ic.hi, pl), __shfl_sync(0xffffffffu, ic.lo, pl)};
                const uint64_t pn = __shfl_sync(0xffffffffu, in, pl);
                exit_sl = static_cast<int>(t0) + f;
                bm = f > 0 ? pm : cm;
                bc = f > 0 ? pc : cc;
                bn = f > 0 ? pn : cn;
            }
            cm = Fx{__shfl_sync(0xffffffffu, im.hi, 31), __shfl_sync(0xffffffffu, im.lo, 31)};
            cc = Fx{__shfl_sync(0xffffffffu, ic.hi, 31), __shfl_sync(0xffffffffu, ic.lo, 31)};
            cn = __shfl_sync(0xffffffffu, in, 31);
        }
        // the exit slice's hits as (list position, hit) keys
        const uint32_t b0 = exit_sl >= 0 ? W.cnt[exit_sl] : 0u;
        const uint32_t ns = exit_sl >= 0 ? W.cnt[exit_sl + 1] - b0 : 0u;
        if (ns <= static_cast<uint32_t>(kOrdKeys))
            for (uint32_t j = lane; j < ns; j += 32) {
                const uint32_t i = W.idx[b0 + j];
                W.keys[j] = (static_cast<uint64_t>(seg[i].r.x) << 10) | i;
            }
        if (ns == 0) {
            // no slice end fires (k_score_sum fired on the same exact totals, so this does not
            // happen): the one-by-one rescoring settles it
            if (lane == 0) a.replay[atomicAdd(&a.counters->n_replay, 1u)] = static_cast<uint32_t>(qi);
            __syncwarp();
            continue;
        }
        if (ns > static_cast<uint32_t>(kOrdKeys)) {
            // more hits in the exit slice than the warp orders: the block scorer takes the guide
            if (lane == 0) a.big[atomicAdd(&a.counters->n_big, 1u)] = static_cast<uint32_t>(qi);
            __syncwarp();
            continue;
        }
        rm = bm;
        rc = bc;
        rn = bn;
        // the test fires inside this slice: order its hits by list position
        uint32_t P2 = 1;
        while (P2 < ns) P2 <<= 1;
        for (uint32_t j = ns + lane; j < P2; j += 32) W.keys[j] = ~0ull;
        __syncwarp();
        for (uint32_t k = 2; k <= P2; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = lane; i < P2; i += 32) {
                    // first stage of each merge compares mirrored pairs, later stages i / i+j
                    const uint32_t partner = (j == (k >> 1)) ? (i ^ (k - 1)) : (i ^ j);
                    if (partner > i) {
                        const uint64_t x = W.keys[i], y = W.keys[partner];
                        if (x > y) {
                            W.keys[i] = y;
                            W.keys[partner] = x;
                        }
                    }
                }
                __syncwarp();
            }
        }
        // the hit where the exact totals fire: its totals (rm, rc, rn) and those before it (pm, pc)
        Fx pm = rm, pc = rc;
        uint32_t stop = ns;
        for (uint32_t c0 = 0; c0 < ns && stop == ns; c0 += 32) {
            const uint32_t t = c0 + lane;
            FxContribution c{{0, 0}, {0, 0}, 0};
            if (t < ns) c = fx_contribution(P, seg[W.keys[t] & 1023u]);
            const Fx im = fx_add(fx_warp_incl(c.mit, lane), rm);
            const Fx ic = fx_add(fx_warp_incl(c.cfd, lane), rc);
            const uint64_t in = warp_incl_sum_u64(c.occ, lane) + rn;
            const bool ex = t < ns && exit_test(P, fx_double(im), fx_double(ic));
            const unsigned em = __ballot_sync(0xffffffffu, ex);
            const int last = em ? __ffs(em) - 1 : (ns - c0 >= 32 ? 31 : static_cast<int>(ns - c0 - 1));
            const Fx em_ = fx_sub(im, c.mit), ec_ = fx_sub(ic, c.cfd);
            if (em) {
                pm = Fx{__shfl_sync(0xffffffffu, em_.hi, last), __shfl_sync(0xffffffffu, em_.lo, last)};
                pc = Fx{__shfl_sync(0xffffffffu, ec_.hi, last), __shfl_sync(0xffffffffu, ec_.lo, last)};
                stop = c0 + last;
            }
            rm = Fx{__shfl_sync(0xffffffffu, im.hi, last), __shfl_sync(0xffffffffu, im.lo, last)};
            rc = Fx{__shfl_sync(0xffffffffu, ic.hi, last), __shfl_sync(0xffffffffu, ic.lo, last)};
            rn = __shfl_sync(0xffffffffu, in, last);
        }
        const double dm = fx_double(rm), dc = fx_double(rc);
        if (stop == ns || !settled_at_exit(P, fx_double(pm), fx_double(pc), dm, dc, rn)) {
            if (lane == 0) a.replay[atomicAdd(&a.counters->n_replay, 1u)] = static_cast<uint32_t>(qi);
            __syncwarp();
            continue;
        }
        if (P.want_distinct) {  // the sites of the slices before the exit slice, then up to the stop
            for (uint32_t j = lane; j < b0; j += 32) {
                const uint32_t id = seg[W.idx[j]].r.z;
                atomicOr(&a.bitmap[id >> 5], 1u << (id & 31));
            }
            for (uint32_t j = lane; j <= stop; j += 32) {
                const uint32_t id = seg[W.keys[j] & 1023u].r.z;
                atomicOr(&a.bitmap[id >> 5], 1u << (id & 31));
            }
        }
        if (lane == 0) finalise(P, dm, dc, rn, qi, a.out_mit, a.out_cfd, a.out_code, a.out_count);
        __syncwarp();
    }
}

// Block per guide whose test fires and that has more than kWarpSort hits: up to kBlockHits hits
// are sorted in shared memory, larger segments in place in global memory, then the ordered
// accumulation runs with exact block-wide prefix sums.
constexpr int kBlockHits = 8192;
constexpr int kBlockIdxBits = 13;

__global__ void __launch_bounds__(256) k_score_block(ScoreArgs a) {
    extern __shared__ __align__(16) uint64_t s_bkeys[];  // kBlockHits keys
    __shared__ Fx s_wm[8], s_wc[8];
    __shared__ uint64_t s_wn[8];
    __shared__ int s_first;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (a.counters->overflow) return;  // rerun follows
    const uint32_t n_big = a.counters->n_big;
    for (uint32_t b = blockIdx.x; b < n_big; b += gridDim.x) {
        const uint64_t qi = a.big[b];
        const ScoreParams P = params_of(a, qi);
        Fx run_m{0, 0}, run_c{0, 0};  // totals of the earlier waves
        uint64_t run_n = 0;
        if (!a.first_wave) {
            const Acc pr = a.acc[qi];
            run_m = pr.mit;
            run_c = pr.cfd;
            run_n = pr.occ;
        }
        const uint32_t h0 = a.qoff[qi], L = a.qfill[qi];
        HitRec* seg = a.seg + h0;
        uint32_t P2 = 1;
        while (P2 < L) P2 <<= 1;
        const bool in_smem = L <= static_cast<uint32_t>(kBlockHits);
        if (in_smem) {
            for (uint32_t i = threadIdx.x; i < P2; i += blockDim.x)
                s_bkeys[i] = i < L ? (order_key(seg[i].r) << kBlockIdxBits) | i : ~0ull;
            __syncthreads();
        }
        for (uint32_t k = 2; k <= P2; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < P2; i += blockDim.x) {
                    const uint32_t partner = (j == (k >> 1)) ? (i ^ (k - 1)) : (i ^ j);
                    if (partner <= i) continue;
                    if (in_smem) {
                        const uint64_t x = s_bkeys[i], y = s_bkeys[partner];
                        if (x > y) {
                            s_bkeys[i] = y;
                            s_bkeys[partner] = x;
                        }
                    } else if (partner < L) {
                        const HitRec x = seg[i], y = seg[partner];
                        if (order_key(x.r) > order_key(y.r)) {
                            seg[i] = y;
                            seg[partner] = x;
                        }
                    }
                }
                __syncthreads();
            }
        }
        // sorted position of the hit where the exact totals fire, and the totals before it
        uint32_t stop = L;
        Fx pre_m = run_m, pre_c = run_c;
        for (uint32_t c0 = 0; c0 < L && stop == L; c0 += blockDim.x) {
            const uint32_t t = c0 + threadIdx.x;
            FxContribution c{{0, 0}, {0, 0}, 0};
            if (t < L) {
                const uint32_t h = in_smem ? static_cast<uint32_t>(s_bkeys[t] & ((1u << kBlockIdxBits) - 1)) : t;
                c = fx_contribution(P, seg[h]);
            }
            Fx im = fx_warp_incl(c.mit, lane), ic = fx_warp_incl(c.cfd, lane);
            uint64_t in = warp_incl_sum_u64(c.occ, lane);
            if (lane == 31) {
                s_wm[warp] = im;
                s_wc[warp] = ic;
                s_wn[warp] = in;
            }
            if (threadIdx.x == 0) s_first = 0x7fffffff;
            __syncthreads();
            Fx pm = run_m, pc = run_c;
            uint64_t pn = run_n;
            for (int w = 0; w < warp; w++) {
                pm = fx_add(pm, s_wm[w]);
                pc = fx_add(pc, s_wc[w]);
                pn += s_wn[w];
            }
            im = fx_add(im, pm);
            ic = fx_add(ic, pc);
            in += pn;
            if (t < L && exit_test(P, fx_double(im), fx_double(ic))) atomicMin(&s_first, static_cast<int>(threadIdx.x));
            __syncthreads();
            const int first = s_first;
            const uint32_t in_chunk = L - c0 < blockDim.x ? L - c0 : blockDim.x;
            const int last = first != 0x7fffffff ? first : static_cast<int>(in_chunk) - 1;
            __syncthreads();
            if (static_cast<int>(threadIdx.x) == last) {
                s_wm[0] = im;
                s_wc[0] = ic;
                s_wn[0] = in;
                s_wm[1] = fx_sub(im, c.mit);
                s_wc[1] = fx_sub(ic, c.cfd);
            }
            __syncthreads();
            run_m = s_wm[0];
            run_c = s_wc[0];
            run_n = s_wn[0];
            if (first != 0x7fffffff) {
                pre_m = s_wm[1];
                pre_c = s_wc[1];
                stop = c0 + static_cast<uint32_t>(first);
            }
            __syncthreads();
        }
        const double dm = fx_double(run_m), dc = fx_double(run_c);
        if (stop == L || !settled_at_exit(P, fx_double(pre_m), fx_double(pre_c), dm, dc, run_n)) {
            // within the reference's rounding (or, which does not happen, no hit fires)
            if (threadIdx.x == 0) a.replay[atomicAdd(&a.counters->n_replay, 1u)] = static_cast<uint32_t>(qi);
            __syncthreads();
            continue;
        }
        if (P.want_distinct)
            for (uint32_t t = threadIdx.x; t <= stop; t += blockDim.x) {
                const uint32_t h = in_smem ? static_cast<uint32_t>(s_bkeys[t] & ((1u << kBlockIdxBits) - 1)) : t;
                const uint32_t id = seg[h].r.z;
                atomicOr(&a.bitmap[id >> 5], 1u << (id & 31));
            }
        if (threadIdx.x == 0) finalise(P, dm, dc, run_n, qi, a.out_mit, a.out_cfd, a.out_code, a.out_count);
        __syncthreads();
    }
}

// Warp per guide that the exact totals cannot settle (see settled_at_exit): the reference's
// additions repeated one at a time, in its order -- slices in order, each bucket in list order,
// sites an earlier slice reached skipped (the ownership rule; the reference's toggle bitset,
// :252-258) -- with its early-exit test after every addition (:366-395), straight from the index.
// Such guides are rare (a threshold within a few ulps of one of their running sums), so this
// favours plainness over speed: the lanes compare 32 blocks of a bucket at once, then the warp
// walks their owned sites in list order, every lane doing the same additions.
__global__ void __launch_bounds__(256) k_replay(ScoreArgs a, IndexView v) {
    __shared__ SliceGeom g[kMaxSlices];
    for (int i = threadIdx.x; i < static_cast<int>(v.n_slices); i += blockDim.x) g[i] = v.geom[i];
    __syncthreads();
    if (a.counters->overflow) return;  // rerun follows
    const int lane = threadIdx.x & 31;
    const uint32_t n = a.counters->n_replay;
    const Tables& T = *a.tables;
    for (uint32_t e = blockIdx.x * 8u + (threadIdx.x >> 5); e < n; e += gridDim.x * 8u) {
        const uint64_t qi = a.replay[e];
        const ScoreParams P = params_of(a, qi);
        const uint64_t q = a.qsig[qi];
        double tm = 0.0, tc = 0.0;
        uint64_t cnt = 0;
        bool stop = false;
        for (uint32_t s = 0; s < v.n_slices && !stop; s++) {
            const SliceGeom& G = g[s];
            const uint64_t gb = G.bbase + slice_key(q, G), base = static_cast<uint64_t>(s) * v.n_sites;
            const uint64_t e0 = v.offsets[gb] - base, e1 = v.offsets[gb + 1] - base;
            if (e1 <= e0) continue;
            const uint32_t rq = slice_residual(q, G);
            for (uint64_t b0 = e0 / 32; b0 <= (e1 - 1) / 32 && !stop; b0 += 32) {
                const uint64_t b = b0 + lane;
                uint32_t own = 0;
                if (b <= (e1 - 1) / 32) {
                    const uint32_t* blk = v.rbits + (G.wbase + b * G.wpb - v.rbits_base);
                    uint32_t mm[kSeqLen];  // mismatch word of each residual position
                    uint32_t c0 = 0, c1 = 0, c2 = 0, c3 = 0;  // saturating bit-sliced count
                    for (int p = 0; p < G.rwidth; p++) {
                        const uint32_t q0 = 0u - ((rq >> (2 * p)) & 1u), q1 = 0u - ((rq >> (2 * p + 1)) & 1u);
                        const uint32_t m = (blk[2 * p] ^ q0) | (blk[2 * p + 1] ^ q1);
                        mm[p] = m;
                        const uint32_t k0 = c0 & m;
                        c0 ^= m;
                        const uint32_t k1 = c1 & k0;
                        c1 ^= k0;
                        const uint32_t k2 = c2 & k1;
                        c2 ^= k1;
                        c3 |= k2;
                    }
                    const int64_t lo = static_cast<int64_t>(e0) - static_cast<int64_t>(32 * b);
                    const int64_t hi = static_cast<int64_t>(e1) - static_cast<int64_t>(32 * b);
                    const uint32_t valid = (hi >= 32 ? 0xFFFFFFFFu : ((1u << hi) - 1u)) & (lo <= 0 ? 0xFFFFFFFFu : ~((1u << lo) - 1u));
                    uint32_t cb = bs::within(bs::Count{c0, c1, c2, c3}, P.max_dist) & valid;
                    while (cb) {
                        const int k = __ffs(cb) - 1;
                        cb &= cb - 1;
                        uint32_t mism20 = 0;
                        for (int p = 0; p < G.rwidth; p++)
                            if ((mm[p] >> k) & 1u) mism20 |= 1u << G.rpos[p];
                        bool owned = true;
                        for (uint32_t t = 0; t < s && owned; t++) owned = (mism20 & g[t].pmask) != 0;
                        if (owned) own |= 1u << k;
                    }
                }
                for (int l = 0; l < 32 && !stop; l++) {
                    uint32_t ob = __shfl_sync(0xffffffffu, own, l);
                    while (ob && !stop) {
                        const int k = __ffs(ob) - 1;
                        ob &= ob - 1;
                        const uint32_t pos = static_cast<uint32_t>(32 * (b0 + l) + k);
                        uint32_t id, occ;
                        uint64_t sig;
                        load_site(v, s, pos, q, G, id, occ, sig);
                        const Contribution c = contribution(T, P, q, sig, occ);
                        if (c.dist > P.max_dist) continue;  // not scored (:292)
                        tm = __dadd_rn(tm, c.mit);
                        tc = __dadd_rn(tc, c.cfd);
                        cnt += occ;
                        if (P.want_distinct && lane == 0) atomicOr(&a.bitmap[id >> 5], 1u << (id & 31));
                        stop = exit_test(P, tm, tc);
                    }
                }
            }
        }
        if (lane == 0) finalise(P, tm, tc, cnt, qi, a.out_mit, a.out_cfd, a.out_code, a.out_count);
        __syncwarp();
    }
}

// Distinct sites: the population count of the site bitmap (16-byte reads, four in flight per
// thread; the allocation is 256-byte aligned, the last words < 4 are read one at a time).
__global__ void k_popcount(const uint32_t* __restrict__ bm, uint64_t words, Counters* c) {
    uint64_t acc = 0;
    const uint4* v = reinterpret_cast<const uint4*>(bm);
    const uint64_t nv = words / 4, T = static_cast<uint64_t>(gridDim.x) * blockDim.x;
    uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    for (; i + 3 * T < nv; i += 4 * T) {
        const uint4 a = v[i], b = v[i + T], d = v[i + 2 * T], e = v[i + 3 * T];
        acc += __popc(a.x) + __popc(a.y) + __popc(a.z) + __popc(a.w) + __popc(b.x) + __popc(b.y) + __popc(b.z) +
               __popc(b.w) + __popc(d.x) + __popc(d.y) + __popc(d.z) + __popc(d.w) + __popc(e.x) + __popc(e.y) +
               __popc(e.z) + __popc(e.w);
    }
    for (; i < nv; i += T) {
        const uint4 a = v[i];
        acc += __popc(a.x) + __popc(a.y) + __popc(a.z) + __popc(a.w);
    }
    const uint64_t t = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x;
    if (t < words - nv * 4) acc += __popc(bm[nv * 4 + t]);
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, d);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(reinterpret_cast<unsigned long long*>(&c->distinct), acc);
}

__global__ void k_copy_distinct(const Counters* c, uint64_t* out) { *out = c->distinct; }

// ---------------------------------------------------------------------------------------------
// host orchestration
const void* scan_kernel(int rw) {
    switch (rw) {
        case 12: return reinterpret_cast<const void*>(&k_scan<12>);
        case 10: return reinterpret_cast<const void*>(&k_scan<10>);
        case 16: return reinterpret_cast<const void*>(&k_scan<16>);
        default: return reinterpret_cast<const void*>(&k_scan<0>);
    }
}

int sm_count(int device) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    return v > 0 ? v : 148;
}

// The penalty tables as the kernels read them: MIT by subset rank, CFD position and PAM penalties,
// and the binomial coefficients of the MIT rank. Every device copy is made from this one image.
const Tables& host_tables() {
    static const Tables h = [] {
        Tables t;
        const auto& mit = mit_rank_table();
        std::memcpy(t.mit, mit.data(), sizeof t.mit);
        std::memcpy(t.cfd_pos, cfd_pos_table(), sizeof t.cfd_pos);
        std::memcpy(t.cfd_pam, cfd_pam_table(), sizeof t.cfd_pam);
        for (int p = 0; p < 20; p++)
            for (int i = 0; i < 5; i++) {
                uint64_t r = (i <= p) ? 1 : 0;
                for (int k = 1; k <= i && i <= p; k++) r = r * (p - i + k) / k;
                t.binom[p][i] = static_cast<uint32_t>(r);
            }
        return t;
    }();
    return h;
}

void init_tables(Workspace& ws, cudaStream_t st) {
    ws.tables.reserve(1);
    ISSL_CUDA(cudaMemcpyAsync(ws.tables.p, &host_tables(), sizeof(Tables), cudaMemcpyHostToDevice, st));
    ISSL_CUDA(cudaStreamSynchronize(st));
}

uint32_t max_wpb_of(const issl_index* ix) {
    uint32_t m = 4;
    for (auto& g : ix->geom) m = std::max<uint32_t>(m, g.wpb);
    return m;
}

// A workspace holds every per-call buffer of the pipeline. The index keeps one for the plain
// entry points; batch contexts and server slots own theirs, so calls on different workspaces
// can run concurrently against the same resident index.
std::unique_ptr<Workspace> new_workspace(issl_index* ix) {
    auto ws = std::make_unique<Workspace>();
    ws->device = ix->device;
    ISSL_CUDA(cudaStreamCreateWithFlags(&ws->own_stream, cudaStreamNonBlocking));
    ISSL_CUDA(cudaStreamCreateWithFlags(&ws->cap_stream, cudaStreamNonBlocking));
    for (auto& e : ws->ev) ISSL_CUDA(cudaEventCreate(&e));
    // one residual width for every slice (the usual case) selects a specialised scan
    ws->scan_rw = ix->geom.empty() ? 0 : ix->geom[0].rwidth;
    for (auto& g : ix->geom)
        if (g.rwidth != ws->scan_rw) ws->scan_rw = 0;
    if (ws->scan_rw != 12 && ws->scan_rw != 10 && ws->scan_rw != 16) ws->scan_rw = 0;
    const int smem_max = static_cast<int>(kScanWarps * warp_layout(max_wpb_of(ix), kMaxStages).bytes);
    ISSL_CUDA(cudaFuncSetAttribute(scan_kernel(ws->scan_rw), cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max));
    ISSL_CUDA(cudaFuncSetAttribute(k_score_block, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(kBlockHits * sizeof(uint64_t))));
    ISSL_CUDA(cudaFuncSetAttribute(k_score_ordered, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   static_cast<int>(8 * sizeof(OrderedSmem))));
    ws->counters.reserve(1);
    ws->scan64.reserve(kScanBlocks + 4);
    ws->scan32.reserve(kScanBlocks + 4);
    init_tables(*ws, ws->own_stream);
    return ws;
}

Workspace& workspace(issl_index* ix) {
    if (!ix->ws) ix->ws = new_workspace(ix);
    return *ix->ws;
}

// Configures the scan for the index's current tuning (staging depth -> shared memory layout,
// blocks per SM -> persistent grid).
void apply_tuning(issl_index* ix, Workspace& ws) {
    if (ws.tuning_version == ix->tuning_version) return;
    const issl_tuning& t = ix->tuning;
    ws.scan_layout = warp_layout(max_wpb_of(ix), t.stages);
    ws.scan_smem = static_cast<int>(kScanWarps * ws.scan_layout.bytes);
    int per_sm = 0;
    ISSL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, scan_kernel(ws.scan_rw), kScanWarps * 32,
                                                            ws.scan_smem));
    per_sm = std::max(per_sm, 1);
    if (t.blocks_per_sm) per_sm = std::min<int>(per_sm, static_cast<int>(t.blocks_per_sm));
    ws.scan_blocks = sm_count(ix->device) * per_sm;
    ws.tuning_version = ix->tuning_version;
}

// A failed allocation leaves some buffers released: forget every capacity so that the next call
// reallocates what is missing (and re-zeroes the counters that must start at zero). (Freeing the
// large buffers outright here made calls at the edge of device memory reallocate tens of GB on
// every call: 956 instead of 634 ms on the 500M-site capacity workload.)
template <class F>
void with_alloc_guard(Workspace& ws, F&& f) {
    try {
        f();
    } catch (...) {
        ws.q_cap = ws.unit_cap = ws.cand_cap = 0;
        ws.g_cap = 0;
        ws.zero_state_ok = false;
        ws.epoch++;
        throw;
    }
}

// Slice waves of a call: the first `first_wave` slices, then the rest (one wave when first_wave
// is 0 or covers every slice). The reference visits slices in order and stops a guide at the hit
// where its test fires; a guide whose test fires within the first wave never probes the later
// slices, which bounds the work and memory of guides with thousands of hits. A host-list index
// further cuts each wave into groups of at most window_slices slices, one device window each.
std::vector<std::pair<uint32_t, uint32_t>> slice_waves(const issl_index* ix) {
    const uint32_t S = static_cast<uint32_t>(ix->n_slices), fw = ix->tuning.first_wave;
    std::vector<std::pair<uint32_t, uint32_t>> w;
    if (fw > 0 && fw < S)
        w = {{0u, fw}, {fw, S}};
    else
        w = {{0u, S}};
    if (!ix->host_lists) return w;
    const uint32_t W = std::max<uint32_t>(ix->window_slices, 1);
    std::vector<std::pair<uint32_t, uint32_t>> out;
    for (const auto& p : w)
        for (uint32_t s = p.first; s < p.second; s += W) out.push_back({s, std::min(p.second, s + W)});
    return out;
}

// The part of the bit-sliced array a window of slices [s0, s1) takes: from word wb0 (the slice's
// first word rounded down to 16 bytes, as the scan's copies are) for `words` words.
void window_rbits(const issl_index* ix, uint32_t s0, uint32_t s1, uint64_t* wb0, uint64_t* words) {
    const uint64_t end = s1 < ix->n_slices ? ix->geom[s1].wbase : bitsliced_words(ix->geom, ix->n_sites);
    *wb0 = ix->geom[s0].wbase & ~3ull;
    *words = end - *wb0;
}

// Device words a window needs, over the waves of a call: entries, and bit-sliced codes plus 8
// words for the scan's 16-byte-rounded copies at the window's end.
void window_capacity(const issl_index* ix, uint64_t* id_words, uint64_t* code_words) {
    *id_words = *code_words = 0;
    if (!ix->host_lists) return;
    for (const auto& p : slice_waves(ix)) {
        uint64_t wb0, words;
        window_rbits(ix, p.first, p.second, &wb0, &words);
        *id_words = std::max<uint64_t>(*id_words, (p.second - p.first) * ix->n_sites * ix->entry_words);
        *code_words = std::max<uint64_t>(*code_words, words + 8);
    }
}

void ensure_capacity_impl(issl_index* ix, Workspace& ws, size_t n, bool batch, cudaStream_t st);

void ensure_capacity(issl_index* ix, Workspace& ws, size_t n, bool batch, cudaStream_t st) {
    try {
        with_alloc_guard(ws, [&] { ensure_capacity_impl(ix, ws, n, batch, st); });
    } catch (const Error& e) {
        // a capacity floor the device cannot hold is dropped; the call then sizes for itself
        if (e.code != ISSL_ERR_NOMEM || (!ws.q_floor && !ws.cand_floor)) throw;
        ws.q_floor = ws.cand_floor = 0;
        with_alloc_guard(ws, [&] { ensure_capacity_impl(ix, ws, n, batch, st); });
    }
}

void ensure_capacity_impl(issl_index* ix, Workspace& ws, size_t n, bool batch, cudaStream_t st) {
    const uint64_t S = ix->n_slices, G = ix->n_buckets;
    n = std::max<size_t>(n, ws.q_floor);
    apply_tuning(ix, ws);
    if (ix->host_lists) {
        if (!ws.copy_stream) {
            ISSL_CUDA(cudaStreamCreateWithFlags(&ws.copy_stream, cudaStreamNonBlocking));
            for (cudaEvent_t* e : {&ws.win_start, &ws.win_ready[0], &ws.win_ready[1], &ws.win_free[0], &ws.win_free[1]})
                ISSL_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        }
        uint64_t idw, cw;
        window_capacity(ix, &idw, &cw);
        for (int b = 0; b < 2; b++) {
            if (ws.win_ids[b].n < idw || ws.win_rbits[b].n < cw) ws.epoch++;
            ws.win_ids[b].reserve(idw);
            ws.win_rbits[b].reserve(cw);
        }
    } else {
        for (int b = 0; b < 2; b++) {
            ws.win_ids[b].release();
            ws.win_rbits[b].release();
        }
    }
    if (ws.g_cap < G + 1) {
        ws.bucket_cnt.reserve(G + 1);
        ws.bucket_qstart.reserve(G + 1);
        ws.bucket_ustart.reserve(G + 1);
        ISSL_CUDA(cudaMemsetAsync(ws.bucket_cnt.p, 0, (G + 1) * 4, st));
        ws.g_cap = G + 1;
        ws.epoch++;
    }
    if (ws.q_cap < n || !ws.qcand.p) {
        const size_t cap = std::max<size_t>(n, 1024);
        ws.qsig.reserve(cap);
        ws.probe_gb.reserve(cap * S);
        ws.probe_qr.reserve(cap * S + 2);
        ws.qcand.reserve(cap + 1);
        ws.qoff.reserve(cap + 1);
        ws.qfill.reserve(cap + 1);
        ws.big.reserve(cap);
        ws.exitq.reserve(cap);
        ws.replayq.reserve(cap);
        ws.out_mit.reserve(cap);
        ws.out_cfd.reserve(cap);
        ws.out_code.reserve(cap);
        ws.out_count.reserve(cap);
        ws.out_distinct.reserve(1);
        ws.active[0].reserve(cap);
        ws.active[1].reserve(cap);
        ws.acc.reserve(cap * 5);
        if (ws.qset.p) ws.qset.reserve(cap);
        ws.q_cap = cap;
        ws.epoch++;
    }
    if (batch && !ws.qset.p) {
        ws.qset.reserve(ws.q_cap);
        ws.epoch++;
    }
    if (!ws.zero_state_ok) {
        ISSL_CUDA(cudaMemsetAsync(ws.bucket_cnt.p, 0, (G + 1) * 4, st));
        ws.zero_state_ok = true;
    }
    // first guesses: ~2.5 units per probe with 1024-entry units (more with smaller ones) plus
    // headroom; hits grow on demand
    uint32_t min_chunk = kChunk;
    for (uint32_t c : ix->tuning.chunk) min_chunk = std::min(min_chunk, c);
    const size_t want_units = std::max<size_t>(ws.unit_cap, n * S * 3 * (kChunk / min_chunk) + 4096);
    if (ws.unit_cap < want_units) {
        ws.units.reserve(want_units);
        ws.unit_cap = want_units;
        ws.epoch++;
    }
    // candidates: the density recent runs needed (64 per guide at first) plus one slab of slack
    // per scan warp; grown by at least half when it grows (every reallocation synchronises the
    // device, which stalls concurrent work); grown on demand after an overflow
    size_t want_cands = static_cast<size_t>(static_cast<double>(n) * ws.cand_density * 1.1) + 65536 +
                        static_cast<size_t>(ws.scan_blocks) * kScanWarps * kCandSlab;
    want_cands = std::min(std::max<size_t>(want_cands, ws.cand_floor), kMaxCandSlots);
    if (ws.cand_cap < want_cands) {
        want_cands = std::min(std::max<size_t>(want_cands, ws.cand_cap + ws.cand_cap / 2), kMaxCandSlots);
        ws.cands.reserve(want_cands);
        ws.seg.reserve(want_cands);
        ws.cand_cap = want_cands;
        ws.epoch++;
    }
}

}  // namespace

// The allocations of ensure_capacity as a formula: a fixed part, bytes per guide and bytes per
// candidate slot (candidate record, grouped hit record).
void workspace_model(const issl_index* ix, uint64_t* fixed, uint64_t* per_guide, uint64_t* per_candidate) {
    const uint64_t S = ix->n_slices, G = ix->n_buckets;
    uint32_t min_chunk = kChunk;
    for (uint32_t c : ix->tuning.chunk) min_chunk = std::min(min_chunk, c);
    const uint64_t slab_slack = 148ull * 16 * kScanWarps * kCandSlab;  // one slab per scan warp, at most
    *per_candidate = kCandSlotBytes;
    *fixed = 12 * (G + 1) + sizeof(Tables) + sizeof(Counters) + (kScanBlocks + 4) * 12 + 4096 * sizeof(UnitDesc) +
             (65536 + slab_slack) * *per_candidate;
    // qsig, probe lists, hit counts and offsets, exit and replay queues, outputs, set map, wave
    // lists and running totals; scan units
    *per_guide = 8 + 12 * S + 6 * 4 + (8 + 8 + 1 + 8) + 2 + 2 * 4 + 5 * 8 +
                 sizeof(UnitDesc) * 3 * S * (kChunk / min_chunk);
    uint64_t idw, cw;  // the two slice windows of a host-list index
    window_capacity(ix, &idw, &cw);
    *fixed += 2 * 4 * (idw + cw);
}

namespace {

ScoreParams make_params(int method, double threshold, int max_dist, bool want_distinct) {
    ISSL_REQUIRE(method >= ISSL_METHOD_MIT && method <= ISSL_METHOD_AVG_MIT_CFD, ISSL_ERR_ARG,
                 "Scoring method is not valid.");
    ISSL_REQUIRE(max_dist >= 0 && max_dist <= kMaxDist, ISSL_ERR_ARG,
                 "max_dist must be 0..4 (the MIT table covers at most four mismatches)");
    ScoreParams P;
    P.method = method;
    P.calc_mit = method != ISSL_METHOD_CFD;
    P.calc_cfd = method != ISSL_METHOD_MIT;
    P.max_dist = max_dist;
    P.threshold = threshold;
    P.maximum_sum = (10000.0 - threshold * 100) / threshold;
    P.want_distinct = want_distinct ? 1 : 0;
    P.pad = 0;
    return P;
}

inline unsigned grid_for(uint64_t n, unsigned threads, unsigned cap) {
    uint64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return static_cast<unsigned>(b);
}

// One pipeline run. Plain form: n guides, one parameter set P, sizes known on the host.
// Batch form: up to n (the capacity) guides, the count and the set table read on the device
// from `hdr` / `sets`, so that the enqueued work can be captured once and replayed.
struct RunSpec {
    const uint64_t* qsig = nullptr;
    uint64_t n = 0;
    ScoreParams P{};
    const BatchHeader* hdr = nullptr;
    const SetDesc* sets = nullptr;
    double* mit = nullptr;
    double* cfd = nullptr;
    char* code = nullptr;
    uint64_t* count = nullptr;
    bool events = true;  // record the timing events (not inside a graph capture)
    // distinct-site count over several runs (guide chunks): clear the bitmap in the first, count
    // it in the last
    bool distinct_first = true, distinct_last = true;
};

__global__ void k_expand_sets(const BatchHeader* __restrict__ hdr, const SetDesc* __restrict__ sets,
                              uint16_t* __restrict__ qset) {
    const uint32_t n = hdr->n, ns = hdr->n_sets;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = ns - 1;  // last set whose begin <= i
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (sets[mid].begin <= i) lo = mid;
            else hi = mid - 1;
        }
        qset[i] = static_cast<uint16_t>(lo);
    }
}

// Enqueues the whole pipeline. Returns the number of kernels it launched.
uint64_t enqueue_pipeline(issl_index* ix, Workspace& ws, const RunSpec& R, cudaStream_t st) {
    const IndexView v0 = ix->view();
    const bool staged = ix->host_lists;
    const uint64_t S = ix->n_slices, G = ix->n_buckets, n = R.n;
    const bool batch = R.hdr != nullptr;
    const uint32_t* d_n = batch ? &R.hdr->n : nullptr;
    const uint16_t* qset = batch ? ws.qset.p : nullptr;
    const int sms = sm_count(ix->device);
    const issl_tuning& tn = ix->tuning;
    const ChunkClasses cc{{tn.chunk[0], tn.chunk[1], tn.chunk[2]}};
    Counters* C = ws.counters.p;
    uint64_t k = 0;
    ISSL_CUDA(cudaMemsetAsync(C, 0, sizeof(Counters), st));
    const uint64_t* off = ix->offsets.p;
    if (R.events) ISSL_CUDA(cudaEventRecord(ws.ev[0], st));
    if (batch) {
        k_expand_sets<<<grid_for(n, 256, sms * 8), 256, 0, st>>>(R.hdr, R.sets, ws.qset.p);
        k++;
    }
    if (R.P.want_distinct && R.distinct_first)
        ISSL_CUDA(cudaMemsetAsync(ws.bitmap.p, 0, (ix->n_sites / 32 + 1) * 4, st));
    const auto waves = slice_waves(ix);
    ws.staged = 0;
    // host-list index: the copy stream starts after everything already queued on st (the last
    // call's waves may still read the windows)
    if (staged) {
        ISSL_CUDA(cudaEventRecord(ws.win_start, st));
    }
    for (size_t w = 0; w < waves.size(); w++) {
        const bool first = w == 0, last = w + 1 == waves.size();
        const uint32_t s0 = waves[w].first, s1 = waves[w].second, cur = w & 1u, nxt = cur ^ 1u;
        IndexView v = v0;
        const int wb = static_cast<int>(w & 1u);  // device window of this wave (host-list index)
        if (staged) {
            // stage the wave's slices: entries and bit-sliced codes, on the copy stream, once the
            // window is free (its previous wave's resolve pass has run)
            const uint64_t N = ix->n_sites, ew = ix->entry_words;
            uint64_t wbase0, words;
            window_rbits(ix, s0, s1, &wbase0, &words);
            cudaStream_t cs = ws.copy_stream;
            ISSL_CUDA(cudaStreamWaitEvent(cs, w < 2 ? ws.win_start : ws.win_free[wb], 0));
            ISSL_CUDA(cudaMemcpyAsync(ws.win_ids[wb].p, ix->h_ids.p + s0 * N * ew, (s1 - s0) * N * ew * 4,
                                      cudaMemcpyHostToDevice, cs));
            ISSL_CUDA(cudaMemcpyAsync(ws.win_rbits[wb].p, ix->h_rbits.p + wbase0, words * 4, cudaMemcpyHostToDevice, cs));
            ISSL_CUDA(cudaEventRecord(ws.win_ready[wb], cs));
            ws.staged += ((s1 - s0) * N * ew + words) * 4;
            v.ids = ws.win_ids[wb].p;
            v.ids_base = static_cast<uint64_t>(s0) * N;
            v.rbits = ws.win_rbits[wb].p;
            v.rbits_base = wbase0;
        }
        if (!first) ISSL_CUDA(cudaMemsetAsync(C, 0, kWaveCounterBytes, st));
        ISSL_CUDA(cudaMemsetAsync(ws.qcand.p, 0, (n + 1) * 4, st));
        ISSL_CUDA(cudaMemsetAsync(ws.qfill.p, 0, (n + 1) * 4, st));
        if (!last) ISSL_CUDA(cudaMemsetAsync(&C->act_n[nxt], 0, 4, st));
        const WaveProbes wp{first ? nullptr : ws.active[cur].p, first ? nullptr : &C->act_n[cur], d_n, n, s0, s1 - s0};
        const uint64_t g0 = ix->geom[s0].bbase, g1 = s1 < S ? ix->geom[s1].bbase : G;
        const unsigned pgrid = grid_for(n * (s1 - s0), 256, sms * 16);
        k_probe_count<<<pgrid, 256, 0, st>>>(v, R.qsig, wp, ws.probe_gb.p, ws.bucket_cnt.p, off);
        device_scan<uint64_t, OpSum>(BucketLoad{ws.bucket_cnt.p, off, ix->n_sites, cc, g0},
                                     BucketStore{ws.bucket_qstart.p, ws.bucket_ustart.p, g0},
                                     nullptr, g1 - g0, ws.scan64.p, &C->bucket_total, st);
        k_units_finalize<<<1, 1, 0, st>>>(C, ws.unit_cap);
        k_expand_units<<<sms * 8, 256, 0, st>>>(ws.bucket_cnt.p, off, ws.bucket_qstart.p, ws.bucket_ustart.p, g0, g1,
                                                ix->n_sites, 1.0 / static_cast<double>(ix->n_sites), cc,
                                                ix->d_geom.p, C, ws.units.p);
        k_probe_scatter<<<pgrid, 256, 0, st>>>(v, R.qsig, wp, ws.probe_gb.p, ws.bucket_cnt.p, ws.bucket_qstart.p,
                                               ws.probe_qr.p);
        k += 7;
        ScanArgs sa;
        sa.rbits = v.rbits;
        sa.rbits_base = v.rbits_base;
        sa.geom = ix->d_geom.p;
        sa.units = ws.units.p;
        sa.probe_qr = ws.probe_qr.p;
        sa.counters = C;
        sa.cands = ws.cands.p;
        sa.qcand = ws.qcand.p;
        sa.n_slices = static_cast<uint32_t>(S);
        sa.cand_cap = static_cast<uint32_t>(std::min<size_t>(ws.cand_cap, 0xFFFFFFFFull));
        sa.max_dist = R.P.max_dist;
        sa.hdr = R.hdr;
        sa.L = ws.scan_layout;
        if (staged) ISSL_CUDA(cudaStreamWaitEvent(st, ws.win_ready[wb], 0));
        if (R.events) ISSL_CUDA(cudaEventRecord(ws.ev[2 + 2 * w], st));
        switch (ws.scan_rw) {
            case 12: k_scan<12><<<ws.scan_blocks, kScanWarps * 32, ws.scan_smem, st>>>(sa); break;
            case 10: k_scan<10><<<ws.scan_blocks, kScanWarps * 32, ws.scan_smem, st>>>(sa); break;
            case 16: k_scan<16><<<ws.scan_blocks, kScanWarps * 32, ws.scan_smem, st>>>(sa); break;
            default: k_scan<0><<<ws.scan_blocks, kScanWarps * 32, ws.scan_smem, st>>>(sa); break;
        }
        if (R.events) ISSL_CUDA(cudaEventRecord(ws.ev[3 + 2 * w], st));
        k_cands_finalize<<<1, 1, 0, st>>>(C, sa.cand_cap);
        // each guide's segment of the hit buffer: the exclusive prefix of its candidate count
        device_scan<uint32_t, OpSum>(LoadQhits{ws.qcand.p}, StoreQoff{ws.qoff.p}, d_n, n, ws.scan32.p, nullptr, st);
        k_cand_resolve<<<sms * 8, 256, 0, st>>>(ws.cands.p, C, v, R.qsig, ws.qoff.p, ws.qfill.p, ws.tables.p, ws.seg.p,
                                                R.sets, qset);
        if (staged) ISSL_CUDA(cudaEventRecord(ws.win_free[wb], st));  // the last reader of the window
        k += 6;
        ScoreArgs a;
        a.ix = v;
        a.qsig = R.qsig;
        a.seg = ws.seg.p;
        a.exitq = ws.exitq.p;
        a.replay = ws.replayq.p;
        a.qoff = ws.qoff.p;
        a.qfill = ws.qfill.p;
        a.tables = ws.tables.p;
        a.counters = C;
        a.big = ws.big.p;
        a.bitmap = ws.bitmap.p;
        a.n = n;
        a.d_n = d_n;
        a.P = R.P;
        a.sets = R.sets;
        a.qset = qset;
        a.out_mit = R.mit;
        a.out_cfd = R.cfd;
        a.out_code = R.code;
        a.out_count = R.count;
        a.active = wp.active;
        a.d_nact = wp.d_nact;
        a.next_active = ws.active[nxt].p;
        a.d_nnext = &C->act_n[nxt];
        a.acc = reinterpret_cast<Acc*>(ws.acc.p);
        a.first_wave = first;
        a.last_wave = last;
        k_score_sum<<<grid_for(n, 8, sms * 8), 256, 0, st>>>(a);
        k_score_ordered<<<sms * 3, 256, 8 * sizeof(OrderedSmem), st>>>(a);
        k_score_block<<<sms * 2, 256, kBlockHits * sizeof(uint64_t), st>>>(a);
        k += 3;
        if (last) {
            // guides the exact totals do not settle, rescored one addition at a time from the
            // whole index (a host-list index: its lists read in place from page-locked host memory)
            IndexView vr = v0;
            if (staged) {
                void* d_ids = nullptr;
                void* d_rbits = nullptr;
                ISSL_CUDA(cudaHostGetDevicePointer(&d_ids, ix->h_ids.p, 0));
                ISSL_CUDA(cudaHostGetDevicePointer(&d_rbits, ix->h_rbits.p, 0));
                vr.ids = static_cast<const uint32_t*>(d_ids);
                vr.rbits = static_cast<const uint32_t*>(d_rbits);
            }
            k_replay<<<sms, 256, 0, st>>>(a, vr);
            k++;
        }
    }
    if (R.P.want_distinct && R.distinct_last) {
        k_popcount<<<sms * 4, 256, 0, st>>>(ws.bitmap.p, ix->n_sites / 32 + 1, C);
        k++;
    }
    if (R.events) ISSL_CUDA(cudaEventRecord(ws.ev[1], st));
    ISSL_CUDA(cudaGetLastError());
    return k;
}

// Reads the counters after a pipeline run; returns false (and grows capacities) on overflow.
bool check_and_grow(Workspace& ws, cudaStream_t st) {
    Counters c;
    ISSL_CUDA(cudaMemcpyAsync(&c, ws.counters.p, sizeof c, cudaMemcpyDeviceToHost, st));
    ISSL_CUDA(cudaStreamSynchronize(st));
    ws.last = c;
    if (c.overflow & 4u) {
        ws.zero_state_ok = false;
        throw Error(ISSL_ERR_TIMEOUT, "scan: an asynchronous copy did not complete within the wait limit");
    }
    if (c.dropped) {
        // a grouped hit farther than four mismatches from its guide: a candidate record that does
        // not describe a site of the guide's bucket. Never silently: the call's results are void.
        ws.zero_state_ok = false;
        throw Error(ISSL_ERR_INTERNAL, "scoring: " + std::to_string(c.dropped) +
                                           " candidate sites were farther than 4 mismatches from their guide");
    }
    const uint64_t units = c.max_units;
    bool ok = true;
    with_alloc_guard(ws, [&] {
        if (units > ws.unit_cap) {
            ws.units.reserve(units + units / 8 + 1024);
            ws.unit_cap = units + units / 8 + 1024;
            ok = false;
        }
        if (c.max_cand > ws.cand_cap || (c.overflow & 2u)) {
            const size_t cap = static_cast<size_t>(c.max_cand) + c.max_cand / 4 + 65536;
            // beyond 32-bit slot numbers: report it like a failed allocation, so that the caller
            // splits the guides into chunks (run_scoring / run_batch_chunked)
            ISSL_REQUIRE(cap <= kMaxCandSlots, ISSL_ERR_NOMEM,
                         "more than 2^32 candidate sites in one slice wave for these guides");
            ws.cands.reserve(cap);
            ws.seg.reserve(cap);
            ws.cand_cap = cap;
            ok = false;
        }
    });
    if (!ok) {
        ws.zero_state_ok = false;  // counters of the aborted run are not drained
        ws.epoch++;
    }
    return ok;
}

void fill_stats(const Workspace& ws, float scan_ms, float total_ms, uint64_t launches, issl_score_stats& s) {
    s.scan_ms = scan_ms;
    s.total_ms = total_ms;
    s.probes = ws.last.probes;
    s.units = ws.last.units;
    s.hits = ws.last.hits;
    s.buckets_scanned = ws.last.buckets;
    s.entries_scanned = ws.last.entries;
    // bytes the scan must move: the bit-sliced blocks it copies, 16 per unit descriptor, 8 per
    // guide of a unit (index + residual), 8 per candidate slot written
    s.scan_bytes = ws.last.rbytes + 16 * s.units + 8 * s.probes + 8 * ws.last.cands;
    s.launches = launches;
    for (int i = 0; i < 3; i++) s.class_probes[i] = ws.last.class_probes[i];
    s.candidates = ws.last.cands;
    s.staged_bytes = ws.staged;
    s.dropped_hits = ws.last.dropped;
    s.replayed = ws.last.n_replay;
    s.runs = 1;
}

issl_score_stats run_stats(issl_index* ix, Workspace& ws) {
    float scan = 0.f, total = 0.f;
    const size_t waves = slice_waves(ix).size();
    for (size_t w = 0; w < waves; w++) {
        float t = 0.f;
        cudaEventElapsedTime(&t, ws.ev[2 + 2 * w], ws.ev[3 + 2 * w]);
        scan += t;
    }
    cudaEventElapsedTime(&total, ws.ev[0], ws.ev[1]);
    issl_score_stats s{};
    fill_stats(ws, scan, total, ws.launches, s);
    ws.launches = 0;
    return s;
}

void add_stats(issl_score_stats& a, const issl_score_stats& b) {
    a.scan_ms += b.scan_ms;
    a.total_ms += b.total_ms;
    a.probes += b.probes;
    a.buckets_scanned += b.buckets_scanned;
    a.entries_scanned += b.entries_scanned;
    a.units += b.units;
    a.hits += b.hits;
    a.scan_bytes += b.scan_bytes;
    a.launches += b.launches;
    for (int i = 0; i < 3; i++) a.class_probes[i] += b.class_probes[i];
    a.candidates += b.candidates;
    a.staged_bytes += b.staged_bytes;
    a.dropped_hits += b.dropped_hits;
    a.replayed += b.replayed;
    a.runs += b.runs;
}

// One pipeline run over n guides, growing the workspace and rerunning on overflow.
issl_score_stats run_once(issl_index* ix, Workspace& ws, RunSpec R, uint64_t* d_distinct, cudaStream_t st) {
    for (int attempt = 0; attempt < 4; attempt++) {
        ensure_capacity(ix, ws, R.n, false, st);
        ws.launches += enqueue_pipeline(ix, ws, R, st);
        if (d_distinct && R.distinct_last) {
            k_copy_distinct<<<1, 1, 0, st>>>(ws.counters.p, d_distinct);
            ws.launches++;
        }
        if (check_and_grow(ws, st)) {
            issl_score_stats s = run_stats(ix, ws);
            s.runs = attempt + 1;  // with the runs that overflowed and were repeated
            return s;
        }
    }
    throw Error(ISSL_ERR_NOMEM, "scoring workspace kept overflowing");
}

// Remembers the candidate density of a run of k guides that needed `cands` slots: a size-weighted
// average over recent runs (halved at every run), at least 64 per guide.
void learn_density(Workspace& ws, uint64_t k, double cands) {
    if (!k) return;
    ws.cand_seen = 0.5 * ws.cand_seen + cands;
    ws.guides_seen = 0.5 * ws.guides_seen + static_cast<double>(k);
    ws.cand_density = std::max(64.0, ws.cand_seen / ws.guides_seen);
}
void learn_density(Workspace& ws, uint64_t k) { learn_density(ws, k, static_cast<double>(ws.last.max_cand)); }

// After a run of k guides that needed more candidate slots than the device can hold: the chunk
// of guides whose candidates fit in the buffers held plus about 3/4 of the free memory, at the
// demand the failed run measured (its candidate counter keeps counting past the buffer), never
// more than half of k.
uint64_t shrunk_chunk(Workspace& ws, uint64_t k) {
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const double per_slot = kCandSlotBytes;
    // the candidate and hit buffers the workspace already holds count as affordable too (a failed
    // growth leaves them allocated, so the free memory alone would shrink the chunk too far)
    const double held = static_cast<double>(ws.cands.bytes() + ws.seg.bytes());
    const double afford = std::min((0.75 * static_cast<double>(free_b) + held) / per_slot,
                                   static_cast<double>(kMaxCandSlots));
    const double demand = static_cast<double>(std::max<uint64_t>(ws.last.max_cand, 1));
    learn_density(ws, k, demand);  // size the next run from what this one needed
    uint64_t c = static_cast<uint64_t>(static_cast<double>(k) * std::min(0.5, afford / demand));
    return std::max<uint64_t>(c, 1);
}

// Guides per pipeline run: all of them, unless their candidates (at the density earlier runs
// measured) would not fit in about 3/4 of the free memory plus the buffers already held, or
// ISSL_MAX_GUIDES_PER_RUN caps it.
uint64_t initial_chunk(const Workspace& ws, uint64_t n) {
    uint64_t c = n;
    if (const char* e = std::getenv("ISSL_MAX_GUIDES_PER_RUN")) {
        const long long v = std::atoll(e);
        if (v > 0 && static_cast<uint64_t>(v) < c) c = static_cast<uint64_t>(v);
    }
    // the usual case: the buffers already held fit the call, no need to ask the driver (the query
    // is slow and would stall concurrent work)
    const double need = static_cast<double>(c) * ws.cand_density * 1.1;
    if (need <= static_cast<double>(ws.cand_cap)) return c;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) {
        const double per_slot = kCandSlotBytes;
        const double held = static_cast<double>(ws.cands.bytes() + ws.seg.bytes());
        const double afford = std::min((0.75 * static_cast<double>(free_b) + held) / per_slot,
                                       static_cast<double>(kMaxCandSlots));
        const double fit = afford / (ws.cand_density * 1.1);
        if (fit < static_cast<double>(c)) c = std::max<uint64_t>(static_cast<uint64_t>(fit), 1);
    }
    return c;
}

// The next chunk of the `left` guides still to score when a run may take at most `most`: the
// remainder cut into equal pieces (chunks of a split call take about the same time and memory, and
// no small last chunk streams the lists for a handful of guides).
uint64_t balanced_chunk(uint64_t most, uint64_t left) {
    most = std::max<uint64_t>(most, 1);
    const uint64_t pieces = (left + most - 1) / most;
    return (left + pieces - 1) / pieces;
}

// Scores the guides in one run, or, when the device cannot hold the workspace a run needs (the
// candidates of many promiscuous guides), in consecutive chunks of guides, halving the chunk
// until it fits. Results do not depend on the split.
void run_scoring(issl_index* ix, const uint64_t* d_qsig_in, uint64_t n, const ScoreParams& P, double* d_mit,
                 double* d_cfd, char* d_code, uint64_t* d_count, uint64_t* d_distinct, cudaStream_t st) {
    Workspace& ws = workspace(ix);
    if (P.want_distinct) ws.bitmap.reserve(ix->n_sites / 32 + 1);
    issl_score_stats sum{};
    uint64_t chunk = initial_chunk(ws, n), done = 0;
    while (done < n) {
        const uint64_t k = balanced_chunk(chunk, n - done);
        RunSpec R;
        R.qsig = d_qsig_in + done;
        R.n = k;
        R.P = P;
        R.mit = d_mit ? d_mit + done : nullptr;
        R.cfd = d_cfd ? d_cfd + done : nullptr;
        R.code = d_code + done;
        R.count = d_count ? d_count + done : nullptr;
        R.distinct_first = done == 0;
        R.distinct_last = done + k == n;
        try {
            add_stats(sum, run_once(ix, ws, R, d_distinct, st));
        } catch (const Error& e) {
            if (e.code != ISSL_ERR_NOMEM || k == 1) throw;
            chunk = shrunk_chunk(ws, k);
            continue;
        }
        learn_density(ws, k);
        done += k;
    }
    ix->stats = sum;
}

}  // namespace
}  // namespace issl

// ---------------------------------------------------------------------------------------------
// batch contexts
struct issl_batch {
    issl_index* ix = nullptr;
    std::unique_ptr<issl::Workspace> ws;
    issl_score_stats stats{};
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ~issl_batch() {
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }
};

void issl::batch_set_capacity_floor(issl_batch* b, uint64_t guides, uint64_t budget_bytes) {
    uint64_t fixed = 0, per_guide = 0, per_cand = 0;
    workspace_model(b->ix, &fixed, &per_guide, &per_cand);
    const uint64_t used = fixed + guides * per_guide;
    b->ws->q_floor = guides;
    // at most 4096 candidates per guide: a small server on a large device does not take it all
    const uint64_t room = budget_bytes > used ? (budget_bytes - used) / per_cand : 0;
    b->ws->cand_floor = std::min<uint64_t>({room, guides * 4096, kMaxCandSlots});
}

namespace issl {
namespace {

constexpr size_t kMaxSets = 65535;

// Scores ws.qsig[0..n) split into the given sets; results land in ws.out_*.
void run_batch(issl_batch* b, uint64_t n, const issl_guide_set* sets, size_t n_sets, cudaStream_t st) {
    issl_index* ix = b->ix;
    Workspace& ws = *b->ws;
    // the set table, staged in pinned memory so that its upload is an ordinary async copy
    const size_t table_bytes = sizeof(BatchHeader) + n_sets * sizeof(SetDesc);
    if (ws.sets_cap < n_sets) {
        const size_t cap = std::max<size_t>(n_sets, 256);
        ISSL_CUDA(cudaStreamSynchronize(st));
        if (ws.h_batch) cudaFreeHost(ws.h_batch);
        ws.h_batch = nullptr;
        ISSL_CUDA(cudaHostAlloc(reinterpret_cast<void**>(&ws.h_batch), sizeof(BatchHeader) + cap * sizeof(SetDesc),
                                cudaHostAllocDefault));
        ws.batch.reserve(sizeof(BatchHeader) + cap * sizeof(SetDesc));
        ws.sets_cap = cap;
        ws.epoch++;
    }
    BatchHeader h{};
    h.n = static_cast<uint32_t>(n);
    h.n_sets = static_cast<uint32_t>(n_sets);
    h.max_dist = 0;
    SetDesc* hs = reinterpret_cast<SetDesc*>(ws.h_batch + sizeof(BatchHeader));
    uint64_t begin = 0;
    for (size_t i = 0; i < n_sets; i++) {
        hs[i].P = make_params(sets[i].method, sets[i].threshold, sets[i].max_dist, false);
        hs[i].begin = static_cast<uint32_t>(begin);
        hs[i].count = static_cast<uint32_t>(sets[i].count);
        begin += sets[i].count;
        h.max_dist = std::max(h.max_dist, sets[i].max_dist);
    }
    std::memcpy(ws.h_batch, &h, sizeof h);
    const BatchHeader* d_hdr = reinterpret_cast<const BatchHeader*>(ws.batch.p);
    const SetDesc* d_sets = reinterpret_cast<const SetDesc*>(ws.batch.p + sizeof(BatchHeader));
    for (int attempt = 0; attempt < 4; attempt++) {
        ensure_capacity(ix, ws, n, true, st);
        // the graph covers every batch up to the capacities it was captured with
        if (!ws.graph || ws.graph_epoch != ws.epoch || ws.graph_tuning != ix->tuning_version) {
            if (ws.graph) cudaGraphExecDestroy(ws.graph);
            ws.graph = nullptr;
            ISSL_CUDA(cudaStreamSynchronize(st));
            RunSpec R;
            R.qsig = ws.qsig.p;
            R.n = ws.q_cap;
            R.P = make_params(ISSL_METHOD_MIT_AND_CFD, 50.0, kMaxDist, false);
            R.hdr = d_hdr;
            R.sets = d_sets;
            R.mit = ws.out_mit.p;
            R.cfd = ws.out_cfd.p;
            R.code = ws.out_code.p;
            R.count = ws.out_count.p;
            R.events = false;
            cudaGraph_t g = nullptr;
            ISSL_CUDA(cudaStreamBeginCapture(ws.cap_stream, cudaStreamCaptureModeThreadLocal));
            uint64_t k = 0;
            try {
                k = enqueue_pipeline(ix, ws, R, ws.cap_stream);
            } catch (...) {
                cudaStreamEndCapture(ws.cap_stream, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            ISSL_CUDA(cudaStreamEndCapture(ws.cap_stream, &g));
            const cudaError_t e = cudaGraphInstantiate(&ws.graph, g, 0);
            cudaGraphDestroy(g);
            ISSL_CUDA(e);
            ws.graph_epoch = ws.epoch;
            ws.graph_tuning = ix->tuning_version;
            ws.graph_kernels = k;
        }
        ISSL_CUDA(cudaMemcpyAsync(ws.batch.p, ws.h_batch, table_bytes, cudaMemcpyHostToDevice, st));
        ISSL_CUDA(cudaEventRecord(b->ev0, st));
        ISSL_CUDA(cudaGraphLaunch(ws.graph, st));
        ISSL_CUDA(cudaEventRecord(b->ev1, st));
        if (check_and_grow(ws, st)) {
            float total = 0.f;
            cudaEventElapsedTime(&total, b->ev0, b->ev1);
            fill_stats(ws, 0.f, total, ws.graph_kernels, b->stats);
            b->stats.runs = attempt + 1;
            return;
        }
    }
    throw Error(ISSL_ERR_NOMEM, "scoring workspace kept overflowing");
}

// Scores a batch in consecutive chunks of guides (one chunk unless the device cannot hold the
// workspace the whole batch needs; then the chunk is halved until it fits). load(offset, k) puts
// the chunk's signatures into the workspace, store(offset, k) hands its results out.
template <class Load, class Store>
void run_batch_chunked(issl_batch* b, uint64_t n, const issl_guide_set* sets, size_t n_sets, cudaStream_t st,
                       Load load, Store store) {
    Workspace& ws = *b->ws;
    issl_score_stats sum{};
    uint64_t chunk = initial_chunk(ws, n), done = 0;
    while (done < n) {
        const uint64_t k = balanced_chunk(chunk, n - done);
        std::vector<issl_guide_set> sub;  // the sets, cut to [done, done + k)
        uint64_t pos = 0;
        for (size_t i = 0; i < n_sets; i++) {
            const uint64_t lo = std::max(pos, done), hi = std::min(pos + sets[i].count, done + k);
            if (hi > lo) {
                issl_guide_set t = sets[i];
                t.count = hi - lo;
                sub.push_back(t);
            }
            pos += sets[i].count;
        }
        try {
            ensure_capacity(b->ix, ws, k, true, st);
            load(done, k);
            run_batch(b, k, sub.data(), sub.size(), st);
            store(done, k);
        } catch (const Error& e) {
            if (e.code != ISSL_ERR_NOMEM || k == 1) throw;
            chunk = shrunk_chunk(ws, k);
            continue;
        }
        add_stats(sum, b->stats);
        learn_density(ws, k);
        done += k;
    }
    b->stats = sum;
}

void check_sets(uint64_t n, const issl_guide_set* sets, size_t n_sets) {
    ISSL_REQUIRE(n_sets >= 1 && n_sets <= kMaxSets, ISSL_ERR_ARG, "a batch holds 1..65535 guide sets");
    ISSL_REQUIRE(sets, ISSL_ERR_ARG, "issl_batch_score: null set table");
    uint64_t total = 0;
    for (size_t i = 0; i < n_sets; i++) {
        make_params(sets[i].method, sets[i].threshold, sets[i].max_dist, false);  // validates
        total += sets[i].count;
    }
    ISSL_REQUIRE(total == n, ISSL_ERR_ARG, "the set counts must add up to the number of guides");
}

}  // namespace
}  // namespace issl

using issl::guarded;

extern "C" {

int issl_score_device(issl_index* ix, const uint64_t* d_sigs, size_t n, int method, double threshold, int max_dist,
                      double* d_mit, double* d_cfd, char* d_code, uint64_t* d_count, uint64_t* d_distinct,
                      void* stream) {
    return guarded([&] {
        ISSL_REQUIRE(ix && (d_sigs || n == 0) && d_code, ISSL_ERR_ARG, "issl_score_device: null argument");
        const issl::ScoreParams P = issl::make_params(method, threshold, max_dist, d_distinct != nullptr);
        ISSL_CUDA(cudaSetDevice(ix->device));
        issl::Workspace& ws = issl::workspace(ix);
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ws.own_stream;
        if (n == 0) {
            if (d_distinct) ISSL_CUDA(cudaMemsetAsync(d_distinct, 0, 8, st));
            return;
        }
        ISSL_REQUIRE(n < (1ull << issl::kGuideBits) && n * ix->n_slices < 0xFFFFFFFFull, ISSL_ERR_ARG,
                     "too many guides in one call (at most 2^26 and 2^32 guide-slice pairs)");
        issl::run_scoring(ix, d_sigs, n, P, d_mit, d_cfd, d_code, d_count, d_distinct, st);
    });
}

static int score_host_common(issl_index* ix, const char* seqs, size_t stride, const uint64_t* sigs, size_t n,
                             int method, double threshold, int max_dist, double* mit, double* cfd, char* code,
                             uint64_t* count, uint64_t* distinct) {
    return guarded([&] {
        ISSL_REQUIRE(ix && code && (n == 0 || seqs || sigs), ISSL_ERR_ARG, "issl_score: null argument");
        if (seqs) ISSL_REQUIRE(stride >= static_cast<size_t>(issl::kSeqLen), ISSL_ERR_ARG,
                               "issl_score: stride shorter than 20 characters");
        const issl::ScoreParams P = issl::make_params(method, threshold, max_dist, distinct != nullptr);
        ISSL_CUDA(cudaSetDevice(ix->device));
        issl::Workspace& ws = issl::workspace(ix);
        cudaStream_t st = ws.own_stream;
        if (n == 0) {
            if (distinct) *distinct = 0;
            return;
        }
        ISSL_REQUIRE(n < (1ull << issl::kGuideBits) && n * ix->n_slices < 0xFFFFFFFFull, ISSL_ERR_ARG,
                     "too many guides in one call (at most 2^26 and 2^32 guide-slice pairs)");
        issl::ensure_capacity(ix, ws, n, false, st);
        if (seqs) {
            const size_t bytes = (n - 1) * stride + issl::kSeqLen;
            if (ws.ascii_cap < bytes) {
                ws.ascii.reserve(bytes);
                ws.ascii_cap = bytes;
            }
            ISSL_CUDA(cudaMemcpyAsync(ws.ascii.p, seqs, bytes, cudaMemcpyHostToDevice, st));
            issl::k_encode_ascii<<<issl::grid_for(n, 256, 148 * 8), 256, 0, st>>>(ws.ascii.p, stride, n, ws.qsig.p);
            ws.launches++;
        } else {
            ISSL_CUDA(cudaMemcpyAsync(ws.qsig.p, sigs, n * 8, cudaMemcpyHostToDevice, st));
        }
        issl::run_scoring(ix, ws.qsig.p, n, P, ws.out_mit.p, ws.out_cfd.p, ws.out_code.p, ws.out_count.p,
                          distinct ? ws.out_distinct.p : nullptr, st);
        if (mit) ISSL_CUDA(cudaMemcpyAsync(mit, ws.out_mit.p, n * 8, cudaMemcpyDeviceToHost, st));
        if (cfd) ISSL_CUDA(cudaMemcpyAsync(cfd, ws.out_cfd.p, n * 8, cudaMemcpyDeviceToHost, st));
        ISSL_CUDA(cudaMemcpyAsync(code, ws.out_code.p, n, cudaMemcpyDeviceToHost, st));
        if (count) ISSL_CUDA(cudaMemcpyAsync(count, ws.out_count.p, n * 8, cudaMemcpyDeviceToHost, st));
        if (distinct) ISSL_CUDA(cudaMemcpyAsync(distinct, ws.out_distinct.p, 8, cudaMemcpyDeviceToHost, st));
        ISSL_CUDA(cudaStreamSynchronize(st));
    });
}

int issl_score(issl_index* ix, const char* seqs, size_t stride, size_t n, int method, double threshold, int max_dist,
               double* mit, double* cfd, char* code, uint64_t* count, uint64_t* distinct) {
    return score_host_common(ix, seqs, stride, nullptr, n, method, threshold, max_dist, mit, cfd, code, count,
                             distinct);
}

int issl_score_sigs(issl_index* ix, const uint64_t* sigs, size_t n, int method, double threshold, int max_dist,
                    double* mit, double* cfd, char* code, uint64_t* count, uint64_t* distinct) {
    return score_host_common(ix, nullptr, 0, sigs, n, method, threshold, max_dist, mit, cfd, code, count, distinct);
}

int issl_workspace_bytes(const issl_index* ix, uint64_t n, double candidates_per_guide, uint64_t* bytes) {
    return guarded([&] {
        ISSL_REQUIRE(ix && bytes && candidates_per_guide >= 0, ISSL_ERR_ARG, "issl_workspace_bytes: bad argument");
        uint64_t fixed, per_guide, per_candidate;
        issl::workspace_model(ix, &fixed, &per_guide, &per_candidate);
        *bytes = fixed + n * per_guide +
                 static_cast<uint64_t>(static_cast<double>(n) * candidates_per_guide) * per_candidate;
    });
}

int issl_index_trim(issl_index* ix) {
    return guarded([&] {
        ISSL_REQUIRE(ix, ISSL_ERR_ARG, "issl_index_trim: null argument");
        ISSL_CUDA(cudaSetDevice(ix->device));
        if (ix->ws) ISSL_CUDA(cudaStreamSynchronize(ix->ws->own_stream));
        ix->ws.reset();
    });
}

int issl_index_set_list_placement(issl_index* ix, uint32_t window_slices) {
    return guarded([&] {
        ISSL_REQUIRE(ix, ISSL_ERR_ARG, "issl_index_set_list_placement: null argument");
        ISSL_REQUIRE(window_slices <= static_cast<uint32_t>(issl::kMaxSlices), ISSL_ERR_ARG,
                     "issl_index_set_list_placement: window_slices must be 0..64");
        ISSL_CUDA(cudaSetDevice(ix->device));
        ISSL_CUDA(cudaDeviceSynchronize());  // nothing may be reading the lists while they move
        const uint64_t idw = ix->n_slices * ix->n_sites * ix->entry_words, rw = issl::rbits_words(ix);
        if (window_slices && !ix->host_lists) {
            ix->h_ids.reserve(idw);
            ix->h_rbits.reserve(rw);
            ISSL_CUDA(cudaMemcpy(ix->h_ids.p, ix->ids.p, idw * 4, cudaMemcpyDeviceToHost));
            ISSL_CUDA(cudaMemcpy(ix->h_rbits.p, ix->rbits.p, rw * 4, cudaMemcpyDeviceToHost));
            ix->ids.release();
            ix->rbits.release();
            ix->host_lists = true;
        } else if (!window_slices && ix->host_lists) {
            try {
                ix->ids.reserve(idw);
                ix->rbits.reserve(rw);
            } catch (...) {
                ix->ids.release();
                ix->rbits.release();
                throw;
            }
            ISSL_CUDA(cudaMemcpy(ix->ids.p, ix->h_ids.p, idw * 4, cudaMemcpyHostToDevice));
            ISSL_CUDA(cudaMemcpy(ix->rbits.p, ix->h_rbits.p, rw * 4, cudaMemcpyHostToDevice));
            ix->h_ids.release();
            ix->h_rbits.release();
            ix->host_lists = false;
        }
        ix->window_slices = window_slices;
        ix->ws.reset();
        ix->tuning_version++;  // batch contexts and server slots re-capture their graphs
    });
}

int issl_get_tuning(const issl_index* ix, issl_tuning* out) {
    return guarded([&] {
        ISSL_REQUIRE(ix && out, ISSL_ERR_ARG, "issl_get_tuning: null argument");
        *out = ix->tuning;
    });
}

int issl_set_tuning(issl_index* ix, const issl_tuning* t) {
    return guarded([&] {
        ISSL_REQUIRE(ix && t, ISSL_ERR_ARG, "issl_set_tuning: null argument");
        for (uint32_t c : t->chunk)
            ISSL_REQUIRE(c == 256 || c == 512 || c == 1024, ISSL_ERR_ARG, "tuning: unit sizes are 256, 512 or 1024");
        ISSL_REQUIRE(t->stages >= 2 && t->stages <= static_cast<uint32_t>(issl::kMaxStages), ISSL_ERR_ARG,
                     "tuning: stages must be 2..4");
        ISSL_REQUIRE(t->blocks_per_sm <= 32, ISSL_ERR_ARG, "tuning: blocks_per_sm must be 0..32");
        ISSL_REQUIRE(t->first_wave <= static_cast<uint32_t>(issl::kMaxSlices), ISSL_ERR_ARG,
                     "tuning: first_wave must be 0..64");
        ix->tuning = *t;
        ix->tuning_version++;
    });
}

int issl_batch_create(issl_index* ix, issl_batch** out) {
    return guarded([&] {
        ISSL_REQUIRE(ix && out, ISSL_ERR_ARG, "issl_batch_create: null argument");
        *out = nullptr;
        ISSL_CUDA(cudaSetDevice(ix->device));
        auto b = std::make_unique<issl_batch>();
        b->ix = ix;
        b->ws = issl::new_workspace(ix);
        ISSL_CUDA(cudaEventCreate(&b->ev0));
        ISSL_CUDA(cudaEventCreate(&b->ev1));
        *out = b.release();
    });
}

void issl_batch_destroy(issl_batch* b) {
    if (!b) return;
    cudaSetDevice(b->ix->device);
    delete b;
}

int issl_batch_score(issl_batch* b, const uint64_t* d_sigs, size_t n, const issl_guide_set* sets, size_t n_sets,
                     double* d_mit, double* d_cfd, char* d_code, uint64_t* d_count, void* stream) {
    return guarded([&] {
        ISSL_REQUIRE(b && (d_sigs || n == 0) && d_code, ISSL_ERR_ARG, "issl_batch_score: null argument");
        issl::check_sets(n, sets, n_sets);
        if (n == 0) return;
        ISSL_REQUIRE(n < (1ull << issl::kGuideBits) && n * b->ix->n_slices < 0xFFFFFFFFull, ISSL_ERR_ARG,
                     "too many guides in one batch (at most 2^26 and 2^32 guide-slice pairs)");
        ISSL_CUDA(cudaSetDevice(b->ix->device));
        issl::Workspace& ws = *b->ws;
        cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : ws.own_stream;
        const auto D2D = cudaMemcpyDeviceToDevice;
        issl::run_batch_chunked(
            b, n, sets, n_sets, st,
            [&](uint64_t o, uint64_t k) { ISSL_CUDA(cudaMemcpyAsync(ws.qsig.p, d_sigs + o, k * 8, D2D, st)); },
            [&](uint64_t o, uint64_t k) {
                if (d_mit) ISSL_CUDA(cudaMemcpyAsync(d_mit + o, ws.out_mit.p, k * 8, D2D, st));
                if (d_cfd) ISSL_CUDA(cudaMemcpyAsync(d_cfd + o, ws.out_cfd.p, k * 8, D2D, st));
                ISSL_CUDA(cudaMemcpyAsync(d_code + o, ws.out_code.p, k, D2D, st));
                if (d_count) ISSL_CUDA(cudaMemcpyAsync(d_count + o, ws.out_count.p, k * 8, D2D, st));
            });
        ISSL_CUDA(cudaStreamSynchronize(st));
    });
}

int issl_batch_score_host(issl_batch* b, const uint64_t* sigs, size_t n, const issl_guide_set* sets, size_t n_sets,
                          double* mit, double* cfd, char* code, uint64_t* count) {
    return guarded([&] {
        ISSL_REQUIRE(b && (sigs || n == 0) && code, ISSL_ERR_ARG, "issl_batch_score_host: null argument");
        issl::check_sets(n, sets, n_sets);
        if (n == 0) return;
        ISSL_REQUIRE(n < (1ull << issl::kGuideBits) && n * b->ix->n_slices < 0xFFFFFFFFull, ISSL_ERR_ARG,
                     "too many guides in one batch (at most 2^26 and 2^32 guide-slice pairs)");
        ISSL_CUDA(cudaSetDevice(b->ix->device));
        issl::Workspace& ws = *b->ws;
        cudaStream_t st = ws.own_stream;
        const auto D2H = cudaMemcpyDeviceToHost;
        issl::run_batch_chunked(
            b, n, sets, n_sets, st,
            [&](uint64_t o, uint64_t k) {
                ISSL_CUDA(cudaMemcpyAsync(ws.qsig.p, sigs + o, k * 8, cudaMemcpyHostToDevice, st));
            },
            [&](uint64_t o, uint64_t k) {
                if (mit) ISSL_CUDA(cudaMemcpyAsync(mit + o, ws.out_mit.p, k * 8, D2H, st));
                if (cfd) ISSL_CUDA(cudaMemcpyAsync(cfd + o, ws.out_cfd.p, k * 8, D2H, st));
                ISSL_CUDA(cudaMemcpyAsync(code + o, ws.out_code.p, k, D2H, st));
                if (count) ISSL_CUDA(cudaMemcpyAsync(count + o, ws.out_count.p, k * 8, D2H, st));
            });
        ISSL_CUDA(cudaStreamSynchronize(st));
    });
}

int issl_batch_stats(const issl_batch* b, issl_score_stats* out) {
    return guarded([&] {
        ISSL_REQUIRE(b && out, ISSL_ERR_ARG, "issl_batch_stats: null argument");
        *out = b->stats;
    });
}

int issl_last_stats(const issl_index* ix, issl_score_stats* out) {
    return guarded([&] {
        ISSL_REQUIRE(ix && out, ISSL_ERR_ARG, "issl_last_stats: null argument");
        *out = ix->stats;
    });
}

}  // extern "C"

// =============================================================================================
// Allocation-free scoring.
//
// Some callers cannot allocate device memory when they score: hosts that hand all device memory
// to their own pool allocator (a framework's caching allocator, a fixed arena on a shared GPU)
// and forbid stray cudaMalloc calls, and latency-bound services that allow no allocation after
// start-up. The regular entry points grow a per-index workspace on demand;
// issl_score_device_static instead runs one kernel whose only scratch is the file-scope array
// below, fixed at library load.
//
// One block scores one guide at a time (grid-stride over the guides): for every slice it walks
// the guide's bucket block by block with the bit-sliced comparison, applies the ownership rule
// to each candidate, stores the owned hits of the guide in its block's slice of g_static_hits,
// sorts them in shared memory in the order the reference visits them, and adds their MIT and
// CFD contributions one at a time in that order with the reference's early exit.
// =============================================================================================
namespace issl {
namespace {

constexpr int kStaticBlocks = 148;                       // scoring blocks (one per B200 SM)
constexpr int kStaticThreads = 256;
constexpr uint32_t kStaticHits = ISSL_STATIC_MAX_HITS;   // owned hits per guide
constexpr uint32_t kStaticIdxBits = 12;                  // log2(kStaticHits)
static_assert((1u << kStaticIdxBits) == kStaticHits, "hit index bits");

// 148 blocks x 4096 hits x 16 bytes = 9.7 MB, held by every GPU that loads the library
static __device__ __align__(256) uint4 g_static_hits[kStaticBlocks * kStaticHits];
// [0]: a guide had more than kStaticHits owned hits (cleared by every call)
static __device__ __align__(256) uint32_t g_static_status[4];
static __device__ __align__(256) Tables g_static_tables;

struct StaticArgs {
    IndexView ix;
    const uint64_t* qsig;
    uint64_t n;
    ScoreParams P;
    const Tables* tables;
    uint4* hits;
    uint32_t* status;
    double* out_mit;
    double* out_cfd;
    char* out_code;
    uint64_t* out_count;
};

// Bit-sliced comparison of one block (32 list positions) of slice s with the guide; owned hits
// are appended to the block's hit area.
template <int RW>
__device__ __forceinline__ void static_block(const StaticArgs& a, const SliceGeom* geom, uint32_t s, uint64_t b,
                                             uint32_t e0, uint32_t e1, const uint32_t* qm, uint4* hits,
                                             uint32_t* cnt) {
    const SliceGeom& g = geom[s];
    const uint32_t* blk = a.ix.rbits + g.wbase + b * g.wpb;
    uint32_t mm[RW];
#pragma unroll
    for (int p = 0; p < RW; p++) mm[p] = (blk[2 * p] ^ qm[2 * p]) | (blk[2 * p + 1] ^ qm[2 * p + 1]);
    // the bucket's positions in this block (list positions can exceed 2^31: 64-bit differences)
    const int64_t lo = max(static_cast<int64_t>(e0) - static_cast<int64_t>(32 * b), int64_t{0});
    const int64_t hi = min(static_cast<int64_t>(e1) - static_cast<int64_t>(32 * b), int64_t{32});
    const uint32_t valid = (hi >= 32 ? 0xFFFFFFFFu : ((1u << hi) - 1u)) & ~((1u << lo) - 1u);
    uint32_t cbits = bs::within(bs::count_mismatches<RW>(mm), a.P.max_dist) & valid;
    while (cbits) {
        const int e = __ffs(cbits) - 1;
        cbits &= cbits - 1;
        uint32_t rm = 0, mism20 = 0;
#pragma unroll
        for (int p = 0; p < RW; p++) rm |= ((mm[p] >> e) & 1u) << p;
        for (uint32_t t = rm; t; t &= t - 1) mism20 |= 1u << g.rpos[__ffs(t) - 1];
        bool own = true;
        for (uint32_t t = 0; t < s; t++)
            if ((mism20 & geom[t].pmask) == 0) {
                own = false;  // an earlier slice reaches this site
                break;
            }
        if (!own) continue;
        const uint32_t pos = static_cast<uint32_t>(32 * b) + e;
        const uint32_t slot = atomicAdd(cnt, 1u);
        if (slot < kStaticHits) hits[slot] = make_uint4(pos, s, rm, 0u);
    }
}

__global__ void __launch_bounds__(kStaticThreads) k_score_static(StaticArgs a) {
    __shared__ uint64_t s_keys[kStaticHits];
    __shared__ SliceGeom s_geom[kMaxSlices];
    __shared__ uint32_t s_qm[32];
    __shared__ uint32_t s_cnt;
    __shared__ double s_cm[kStaticThreads], s_cc[kStaticThreads];
    __shared__ uint32_t s_co[kStaticThreads];
    __shared__ int s_stop;
    for (int i = threadIdx.x; i < static_cast<int>(a.ix.n_slices); i += blockDim.x) s_geom[i] = a.ix.geom[i];
    __syncthreads();
    const Tables& T = *a.tables;
    uint4* hits = a.hits + static_cast<size_t>(blockIdx.x) * kStaticHits;
    for (uint64_t qi = blockIdx.x; qi < a.n; qi += gridDim.x) {
        const uint64_t q = a.qsig[qi];
        if (threadIdx.x == 0) s_cnt = 0;
        __syncthreads();
        for (uint32_t s = 0; s < a.ix.n_slices; s++) {
            const SliceGeom& g = s_geom[s];
            const uint32_t gb = g.bbase + slice_key(q, g);
            const uint64_t base = static_cast<uint64_t>(s) * a.ix.n_sites;
            const uint32_t e0 = static_cast<uint32_t>(a.ix.offsets[gb] - base);
            const uint32_t e1 = static_cast<uint32_t>(a.ix.offsets[gb + 1] - base);
            const uint32_t rq = slice_residual(q, g);
            if (threadIdx.x < 2u * g.rwidth) s_qm[threadIdx.x] = 0u - ((rq >> threadIdx.x) & 1u);
            __syncthreads();
            if (e1 > e0) {
                for (uint64_t b = e0 / 32 + threadIdx.x; b <= (e1 - 1) / 32; b += blockDim.x) {
                    switch (g.rwidth) {
                        case 12: static_block<12>(a, s_geom, s, b, e0, e1, s_qm, hits, &s_cnt); break;
                        case 10: static_block<10>(a, s_geom, s, b, e0, e1, s_qm, hits, &s_cnt); break;
                        case 16: static_block<16>(a, s_geom, s, b, e0, e1, s_qm, hits, &s_cnt); break;
                        case 15: static_block<15>(a, s_geom, s, b, e0, e1, s_qm, hits, &s_cnt); break;
                        case 14: static_block<14>(a, s_geom, s, b, e0, e1, s_qm, hits, &s_cnt); break;
                        case 13: static_block<13>(a, s_geom, s, b, e0, e1, s_qm, hits, &s_cnt); break;
                        case 11: static_block<11>(a, s_geom, s, b, e0, e1, s_qm, hits, &s_cnt); break;
                        case 9: static_block<9>(a, s_geom, s, b, e0, e1, s_qm, hits, &s_cnt); break;
                        case 8: static_block<8>(a, s_geom, s, b, e0, e1, s_qm, hits, &s_cnt); break;
                        default: static_block<7>(a, s_geom, s, b, e0, e1, s_qm, hits, &s_cnt); break;
                    }
                }
            }
            __syncthreads();  // s_qm is rewritten for the next slice
        }
        const uint32_t L = s_cnt;
        if (L > kStaticHits) {
            if (threadIdx.x == 0) atomicOr(&a.status[0], 1u);
            __syncthreads();
            continue;
        }
        // the reference's visiting order: slice, then list position
        uint32_t P2 = 1;
        while (P2 < L) P2 <<= 1;
        for (uint32_t i = threadIdx.x; i < P2; i += blockDim.x)
            s_keys[i] = i < L ? (((static_cast<uint64_t>(hits[i].y) << 32) | hits[i].x) << kStaticIdxBits) | i : ~0ull;
        __syncthreads();
        for (uint32_t k = 2; k <= P2; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < P2; i += blockDim.x) {
                    const uint32_t partner = (j == (k >> 1)) ? (i ^ (k - 1)) : (i ^ j);
                    if (partner > i) {
                        const uint64_t x = s_keys[i], y = s_keys[partner];
                        if (x > y) {
                            s_keys[i] = y;
                            s_keys[partner] = x;
                        }
                    }
                }
                __syncthreads();
            }
        }
        // the reference's additions, one at a time in that order (thread 0), with its early-exit
        // test after each (:366-395); the block computes the contributions 256 at a time
        double run_mit = 0.0, run_cfd = 0.0;
        uint64_t run_cnt = 0;
        bool stopped = false;
        for (uint32_t c0 = 0; c0 < L && !stopped; c0 += blockDim.x) {
            const uint32_t t = c0 + threadIdx.x;
            if (t < L) {
                const uint4 r = hits[s_keys[t] & (kStaticHits - 1)];
                uint32_t id, occ;
                uint64_t sig;
                load_site(a.ix, r.y, r.x, q, s_geom[r.y], id, occ, sig);
                const Contribution c = contribution(T, a.P, q, sig, occ);
                s_cm[threadIdx.x] = c.mit;
                s_cc[threadIdx.x] = c.cfd;
                s_co[threadIdx.x] = occ;
            }
            __syncthreads();
            if (threadIdx.x == 0) {
                const uint32_t m = L - c0 < blockDim.x ? L - c0 : blockDim.x;
                for (uint32_t i = 0; i < m && !stopped; i++) {
                    run_mit = __dadd_rn(run_mit, s_cm[i]);
                    run_cfd = __dadd_rn(run_cfd, s_cc[i]);
                    run_cnt += s_co[i];
                    stopped = exit_test(a.P, run_mit, run_cfd);
                }
                s_stop = stopped;
            }
            __syncthreads();
            stopped = s_stop != 0;
            __syncthreads();
        }
        if (threadIdx.x == 0)
            finalise(a.P, run_mit, run_cfd, run_cnt, qi, a.out_mit, a.out_cfd, a.out_code, a.out_count);
        __syncthreads();
    }
}

// Device addresses of the static scratch, looked up once per device with that device current.
struct StaticScratch {
    bool ready = false;
    uint4* hits = nullptr;
    uint32_t* status = nullptr;
    Tables* tables = nullptr;
};
std::mutex g_static_mu;
StaticScratch g_static[64];

StaticScratch& static_scratch(int device) {
    ISSL_REQUIRE(device >= 0 && device < 64, ISSL_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lock(g_static_mu);
    StaticScratch& sc = g_static[device];
    if (!sc.ready) {
        // the host-side names of the arrays are stand-ins, not device addresses
        ISSL_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&sc.hits), g_static_hits));
        ISSL_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&sc.status), g_static_status));
        ISSL_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&sc.tables), g_static_tables));
        ISSL_CUDA(cudaMemcpy(sc.tables, &host_tables(), sizeof(Tables), cudaMemcpyHostToDevice));
        sc.ready = true;
    }
    return sc;
}

}  // namespace
}  // namespace issl

extern "C" int issl_score_device_static(issl_index* ix, const uint64_t* d_sigs, size_t n, int method,
                                        double threshold, int max_dist, double* d_mit, double* d_cfd, char* d_code,
                                        uint64_t* d_count, void* stream) {
    return issl::guarded([&] {
        ISSL_REQUIRE(ix && (d_sigs || n == 0) && d_code, ISSL_ERR_ARG, "issl_score_device_static: null argument");
        ISSL_REQUIRE(!ix->host_lists, ISSL_ERR_UNSUPPORTED,
                     "issl_score_device_static: the index keeps its lists in host memory (issl_open_mapped)");
        ISSL_REQUIRE(n <= ISSL_STATIC_MAX_GUIDES, ISSL_ERR_ARG,
                     "issl_score_device_static: at most " + std::to_string(ISSL_STATIC_MAX_GUIDES) +
                         " guides per call");
        const issl::ScoreParams P = issl::make_params(method, threshold, max_dist, false);
        ISSL_CUDA(cudaSetDevice(ix->device));
        issl::StaticScratch& sc = issl::static_scratch(ix->device);
        if (n == 0) return;
        cudaStream_t st = static_cast<cudaStream_t>(stream);
        ISSL_CUDA(cudaMemsetAsync(sc.status, 0, sizeof(uint32_t), st));
        issl::StaticArgs a;
        a.ix = ix->view();
        a.qsig = d_sigs;
        a.n = n;
        a.P = P;
        a.tables = sc.tables;
        a.hits = sc.hits;
        a.status = sc.status;
        a.out_mit = d_mit;
        a.out_cfd = d_cfd;
        a.out_code = d_code;
        a.out_count = d_count;
        issl::k_score_static<<<issl::kStaticBlocks, issl::kStaticThreads, 0, st>>>(a);
        ISSL_CUDA(cudaGetLastError());
        uint32_t status = 0;
        ISSL_CUDA(cudaMemcpyAsync(&status, sc.status, sizeof status, cudaMemcpyDeviceToHost, st));
        ISSL_CUDA(cudaStreamSynchronize(st));
        ISSL_REQUIRE(status == 0, ISSL_ERR_UNSUPPORTED,
                     "issl_score_device_static: a guide has more than " + std::to_string(ISSL_STATIC_MAX_HITS) +
                         " off-target hits; score it with issl_score_device");
    });
}
