// ISSL scoring on the GPU: the hot path of lib/ISSLScoringModule.cpp:206-462 and
// ISSLScoreOfftargets/ISSLScoreOfftargets.cpp:308-505.
//
// Pipeline (one stream, no host round trip; sizes produced on the device are read on the device):
//   1 probe_count   every (guide, slice) pair -> its global bucket; count probes per bucket
//   2 bucket scan   exclusive scan over all buckets of (scan units, probes): per-bucket probe
//                   slot ranges, and unit descriptors -- a unit is (bucket chunk of kChunk
//                   entries) x (up to kGroup guides probing that bucket), so guides sharing a
//                   bucket read its entries once and heavy buckets split into many units
//   3 probe_scatter guides grouped by bucket, with each guide's residual code for that slice
//   4 scan          stream the residual codes of every unit with 128-bit loads; a candidate is
//                   an entry whose residual differs from the guide's in <= max_dist bases.
//                   Candidates are kept only in the first slice that reaches them (ownership
//                   rule, replacing the per-guide toggle bitset of :252-258): site reached in
//                   slice s is counted iff no earlier slice s' has all its positions matching
//   5 hit offsets   per-guide hit counts -> segment offsets
//   6 hit_scatter   hits grouped per guide
//   7 score         per guide: order its hits as the reference visits them (slice, then list
//                   position), accumulate MIT / CFD in FP64 with warp prefix sums, stop at the
//                   first hit where the reference's early-exit test fires (:366-395), finalise
//                   the scores and accept code (:404-459)
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <vector>

#include "device_util.cuh"
#include "issl_internal.cuh"
#include "scan.cuh"

namespace issl {

constexpr int kChunk = 512;        // entries per scan unit
constexpr int kGroup = 32;         // guides per scan unit
constexpr int kWarpHits = 256;     // guides with more hits are scored by a whole block
constexpr int kScanWarps = 8;      // warps per scan block
constexpr int kHitBuf = 64;        // per-warp staging of hits before one global reservation
constexpr uint32_t kEmpty = 0xFFFFFFFFu;

struct UnitDesc {   // 16 bytes
    uint64_t cb;    // first global entry (s * N + list position)
    uint32_t qbeg;  // first probe slot of the unit's guides
    uint16_t len;   // entries in the unit (<= kChunk)
    uint8_t qn;     // guides in the unit (<= kGroup)
    uint8_t s;      // slice
};

struct Counters {
    uint64_t bucket_total;  // hi: units, lo: probes into non-empty buckets
    uint32_t n_units;       // min(units, capacity)
    uint32_t n_hits;        // owned hits appended (may exceed capacity -> overflow)
    uint32_t hit_total;     // sum of per-guide hits (scan total)
    uint32_t n_big;         // guides deferred to the block scorer
    uint32_t overflow;      // 1: units, 2: hits
    uint32_t pad;
    uint64_t distinct;
    uint64_t buckets;       // distinct buckets probed
    uint64_t entries;       // entries streamed by the scan
};

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
};

}  // namespace issl

struct issl::Workspace {
    int device = 0;
    cudaStream_t own_stream = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    size_t q_cap = 0, unit_cap = 0, hit_cap = 0;
    uint64_t g_cap = 0;
    int scan_blocks = 0;
    bool zero_state_ok = false;  // bucket_cnt / qhits are all zero between calls
    DevBuf<uint64_t> qsig;
    DevBuf<char> ascii;
    size_t ascii_cap = 0;
    DevBuf<uint32_t> probe_gb, probe_q, probe_rq;
    DevBuf<uint32_t> bucket_cnt, bucket_qstart;
    DevBuf<UnitDesc> units;
    DevBuf<uint4> hits, seg;
    DevBuf<uint32_t> qhits, qhoff, big;
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
    ~Workspace() {
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
        if (own_stream) cudaStreamDestroy(own_stream);
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

__global__ void k_probe_count(IndexView ix, const uint64_t* __restrict__ qsig, uint64_t n,
                              uint32_t* __restrict__ probe_gb, uint32_t* __restrict__ bucket_cnt,
                              const uint64_t* __restrict__ off) {
    __shared__ SliceGeom g[kMaxSlices];
    for (int i = threadIdx.x; i < static_cast<int>(ix.n_slices); i += blockDim.x) g[i] = ix.geom[i];
    __syncthreads();
    const uint64_t S = ix.n_slices, total = n * S;
    for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < total;
         p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t q = p / S;
        const uint32_t s = static_cast<uint32_t>(p - q * S);
        const uint32_t gb = g[s].bbase + slice_key(qsig[q], g[s]);
        const bool nonempty = off[gb + 1] > off[gb];
        probe_gb[p] = nonempty ? gb : kEmpty;
        if (nonempty) atomicAdd(&bucket_cnt[gb], 1u);
    }
}

// 2. bucket scan: value = (units << 32) | probes
struct BucketLoad {
    const uint32_t* cnt;
    const uint64_t* off;
    __device__ uint64_t operator()(uint64_t g) const {
        const uint32_t c = cnt[g];
        if (!c) return 0;
        const uint64_t size = off[g + 1] - off[g];
        const uint64_t units = ((size + kChunk - 1) / kChunk) * ((c + kGroup - 1) / kGroup);
        return (units << 32) | c;
    }
};

struct BucketStore {
    const uint32_t* cnt;
    const uint64_t* off;
    uint32_t* qstart;
    UnitDesc* units;
    uint64_t unit_cap;
    uint64_t n_sites;
    __device__ void operator()(uint64_t g, uint64_t ex, uint64_t inc) const {
        qstart[g] = static_cast<uint32_t>(ex);
        const uint32_t c = static_cast<uint32_t>(inc) - static_cast<uint32_t>(ex);
        if (!c) return;
        const uint64_t u0 = ex >> 32, u1 = inc >> 32;
        const uint64_t e0 = off[g], e1 = off[g + 1];
        const uint32_t s = static_cast<uint32_t>(e0 / n_sites);
        const uint32_t ng = (c + kGroup - 1) / kGroup;
        uint64_t u = u0;
        for (uint64_t cb = e0; cb < e1 && u < u1; cb += kChunk) {
            const uint16_t len = static_cast<uint16_t>(e1 - cb < kChunk ? e1 - cb : kChunk);
            for (uint32_t j = 0; j < ng; j++, u++) {
                if (u >= unit_cap) return;
                UnitDesc d;
                d.cb = cb;
                d.qbeg = static_cast<uint32_t>(ex) + j * kGroup;
                d.len = len;
                d.qn = static_cast<uint8_t>(c - j * kGroup < kGroup ? c - j * kGroup : kGroup);
                d.s = static_cast<uint8_t>(s);
                units[u] = d;
            }
        }
    }
};

// work counters for the roofline: distinct buckets scanned and entries streamed (a bucket's
// entries are read once per group of up to kGroup guides)
__global__ void k_bucket_stats(const uint32_t* __restrict__ cnt, const uint64_t* __restrict__ off, uint64_t G,
                               Counters* c) {
    uint64_t buckets = 0, entries = 0;
    for (uint64_t g = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; g < G;
         g += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t k = cnt[g];
        if (!k) continue;
        buckets++;
        entries += (off[g + 1] - off[g]) * ((k + kGroup - 1) / kGroup);
    }
    for (int d = 16; d > 0; d >>= 1) {
        buckets += __shfl_down_sync(0xffffffffu, buckets, d);
        entries += __shfl_down_sync(0xffffffffu, entries, d);
    }
    if ((threadIdx.x & 31) == 0 && buckets) {
        atomicAdd(reinterpret_cast<unsigned long long*>(&c->buckets), buckets);
        atomicAdd(reinterpret_cast<unsigned long long*>(&c->entries), entries);
    }
}

__global__ void k_units_finalize(Counters* c, uint64_t unit_cap) {
    const uint64_t u = c->bucket_total >> 32;
    c->n_units = static_cast<uint32_t>(u < unit_cap ? u : unit_cap);
    if (u > unit_cap) atomicOr(&c->overflow, 1u);
}

// 3. guides grouped by bucket, with their residual codes
__global__ void k_probe_scatter(IndexView ix, const uint64_t* __restrict__ qsig, uint64_t n,
                                const uint32_t* __restrict__ probe_gb, uint32_t* __restrict__ bucket_cnt,
                                const uint32_t* __restrict__ qstart, uint32_t* __restrict__ probe_q,
                                uint32_t* __restrict__ probe_rq) {
    __shared__ SliceGeom g[kMaxSlices];
    for (int i = threadIdx.x; i < static_cast<int>(ix.n_slices); i += blockDim.x) g[i] = ix.geom[i];
    __syncthreads();
    const uint64_t S = ix.n_slices, total = n * S;
    for (uint64_t p = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; p < total;
         p += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint32_t gb = probe_gb[p];
        if (gb == kEmpty) continue;
        const uint64_t q = p / S;
        const uint32_t s = static_cast<uint32_t>(p - q * S);
        // the decrement leaves bucket_cnt all zero for the next call
        const uint32_t slot = qstart[gb] + atomicSub(&bucket_cnt[gb], 1u) - 1u;
        probe_q[slot] = static_cast<uint32_t>(q);
        probe_rq[slot] = slice_residual(qsig[q], g[s]);
    }
}

// ---------------------------------------------------------------------------------------------
// 4. the scan
struct ScanArgs {
    const uint32_t* resid;
    const SliceGeom* geom;
    const UnitDesc* units;
    const uint32_t* probe_q;
    const uint32_t* probe_rq;
    Counters* counters;
    uint4* hits;
    uint32_t* qhits;
    uint64_t n_sites;
    uint32_t hit_cap;
    uint32_t n_slices;
    int max_dist;
};

__device__ __forceinline__ uint4 ld_resid4(const uint32_t* p) {
    return __ldg(reinterpret_cast<const uint4*>(p));
}

__global__ void __launch_bounds__(kScanWarps * 32) k_scan(ScanArgs a) {
    __shared__ uint32_t s_pmask[kMaxSlices];
    __shared__ uint8_t s_rpos[kMaxSlices][kSeqLen];
    __shared__ uint4 s_buf[kScanWarps][kHitBuf];
    for (int i = threadIdx.x; i < static_cast<int>(a.n_slices); i += blockDim.x) {
        s_pmask[i] = a.geom[i].pmask;
        for (int j = 0; j < kSeqLen; j++) s_rpos[i][j] = a.geom[i].rpos[j];
    }
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    const uint32_t n_units = a.counters->n_units;
    const uint32_t gwarp = blockIdx.x * kScanWarps + warp;
    const uint32_t nwarps = gridDim.x * kScanWarps;
    uint32_t buffered = 0;
    uint4* buf = s_buf[warp];

    auto flush = [&]() {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(&a.counters->n_hits, buffered);
        base = __shfl_sync(0xffffffffu, base, 0);
        for (uint32_t i = lane; i < buffered; i += 32)
            if (base + i < a.hit_cap) a.hits[base + i] = buf[i];
        __syncwarp();
        buffered = 0;
    };

    for (uint32_t u = gwarp; u < n_units; u += nwarps) {
        const UnitDesc d = a.units[u];
        const uint32_t s = d.s;
        uint32_t q = 0, rq = 0;
        if (lane < d.qn) {
            q = a.probe_q[d.qbeg + lane];
            rq = a.probe_rq[d.qbeg + lane];
        }
        const uint64_t cb = d.cb, ce = d.cb + d.len;
        const uint64_t a0 = cb & ~3ull;
        // issue every load of the unit before using any (kChunk / 128 + 1 vectors per lane)
        constexpr int kVec = kChunk / 128 + 1;
        uint4 v[kVec];
#pragma unroll
        for (int it = 0; it < kVec; it++) {
            const uint64_t base = a0 + static_cast<uint64_t>(it) * 128 + 4 * lane;
            v[it] = base < ce ? ld_resid4(a.resid + base) : make_uint4(0, 0, 0, 0);
        }
        const uint64_t slice_base = static_cast<uint64_t>(s) * a.n_sites;
        for (int k = 0; k < d.qn; k++) {
            const uint32_t rqk = __shfl_sync(0xffffffffu, rq, k);
            const uint32_t qk = __shfl_sync(0xffffffffu, q, k);
#pragma unroll
            for (int it = 0; it < kVec; it++) {
                const uint64_t base = a0 + static_cast<uint64_t>(it) * 128 + 4 * lane;
                const uint32_t r4[4] = {v[it].x, v[it].y, v[it].z, v[it].w};
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const uint32_t m = fold32(r4[e] ^ rqk);
                    const uint64_t idx = base + e;
                    const bool cand = __popc(m) <= a.max_dist && idx >= cb && idx < ce;
                    const unsigned cm = __ballot_sync(0xffffffffu, cand);
                    if (cm == 0) continue;
                    bool own = false;
                    if (cand) {
                        // mismatch positions of the whole site: residual mismatches only (the
                        // slice positions match by construction)
                        uint32_t mism20 = 0, mm = m;
                        while (mm) {
                            const int b = __ffs(mm) - 1;
                            mism20 |= 1u << s_rpos[s][b >> 1];
                            mm &= mm - 1;
                        }
                        own = true;
                        for (uint32_t t = 0; t < s; t++)
                            if ((mism20 & s_pmask[t]) == 0) {
                                own = false;
                                break;
                            }
                    }
                    const unsigned om = __ballot_sync(0xffffffffu, own);
                    if (om == 0) continue;
                    if (buffered + 32 > kHitBuf) flush();
                    if (own) {
                        buf[buffered + __popc(om & lt)] =
                            make_uint4(qk, static_cast<uint32_t>(idx - slice_base), s, r4[e]);
                        atomicAdd(&a.qhits[qk], 1u);
                    }
                    __syncwarp();
                    buffered += __popc(om);
                }
            }
        }
    }
    if (buffered) flush();
}

// ---------------------------------------------------------------------------------------------
// 5/6. hits grouped per guide
struct LoadQhits {
    const uint32_t* p;
    __device__ uint32_t operator()(uint64_t i) const { return p[i]; }
};
struct StoreQoff {
    uint32_t* p;
    __device__ void operator()(uint64_t i, uint32_t ex, uint32_t) const { p[i] = ex; }
};

__global__ void k_hit_scatter(const uint4* __restrict__ hits, const Counters* c, uint32_t hit_cap,
                              uint32_t* __restrict__ qhits, const uint32_t* __restrict__ qhoff,
                              const uint32_t* __restrict__ ids, uint64_t n_sites, uint4* __restrict__ seg) {
    // on overflow the per-guide offsets count hits that were not stored: skip, the host reruns
    if (c->n_hits > hit_cap || c->overflow) return;
    const uint32_t n = c->n_hits;
    for (uint32_t h = blockIdx.x * blockDim.x + threadIdx.x; h < n; h += gridDim.x * blockDim.x) {
        const uint4 r = hits[h];
        const uint32_t q = r.x;
        const uint32_t slot = qhoff[q] + atomicSub(&qhits[q], 1u) - 1u;
        // seg record: (list position, slice, residual code, site id)
        seg[slot] = make_uint4(r.y, r.z, r.w, ids[static_cast<uint64_t>(r.z) * n_sites + r.y]);
    }
}

// ---------------------------------------------------------------------------------------------
// 7. scoring of one guide's hits in the reference's visiting order
__device__ __forceinline__ uint64_t order_key(const uint4& r) {
    return (static_cast<uint64_t>(r.y) << 32) | r.x;  // slice, then list position
}

__device__ __forceinline__ uint64_t site_signature(uint64_t q, const SliceGeom& g, uint32_t r) {
    uint64_t sig = 0;
    for (int j = 0; j < g.width; j++) sig |= q & (3ull << (2 * g.pos[j]));
    for (int j = 0; j < g.rwidth; j++) sig |= static_cast<uint64_t>((r >> (2 * j)) & 3u) << (2 * g.rpos[j]);
    return sig;
}

struct Contribution {
    double mit, cfd;
    uint32_t occ;
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
    if (P.calc_mit && dist > 0) {
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

__device__ __forceinline__ void finalise(const ScoreParams& P, double tot_mit, double tot_cfd, uint64_t count,
                                         uint64_t q_index, double* out_mit, double* out_cfd, char* out_code,
                                         uint64_t* out_count) {
    const double t = P.threshold;
    double m = 10000.0 / (100.0 + tot_mit), c = 10000.0 / (100.0 + tot_cfd);  // :407-448
    bool reject;
    switch (P.method) {
        case ISSL_METHOD_MIT_AND_CFD: reject = m < t && c < t; break;
        case ISSL_METHOD_MIT_OR_CFD: reject = m < t || c < t; break;
        case ISSL_METHOD_AVG_MIT_CFD: reject = (m + c) / 2 < t; break;
        case ISSL_METHOD_MIT: reject = m < t; c = -1; break;
        default: reject = c < t; m = -1; break;
    }
    if (out_mit) out_mit[q_index] = m;
    if (out_cfd) out_cfd[q_index] = c;
    out_code[q_index] = reject ? ISSL_CODE_REJECTED : ISSL_CODE_ACCEPTED;
    if (out_count) out_count[q_index] = count;
}

__device__ __forceinline__ double warp_incl_sum(double v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const double o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += o;
    }
    return v;
}
__device__ __forceinline__ uint64_t warp_incl_sum_u64(uint64_t v, int lane) {
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint64_t o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += o;
    }
    return v;
}

struct ScoreArgs {
    uint32_t hit_cap;
    IndexView ix;
    const uint64_t* qsig;
    uint4* seg;
    const uint32_t* qhoff;
    const Tables* tables;
    Counters* counters;
    uint32_t* big;
    uint32_t* bitmap;
    uint64_t n;
    ScoreParams P;
    double* out_mit;
    double* out_cfd;
    char* out_code;
    uint64_t* out_count;
};

// Warp per guide; hits (<= kWarpHits) sorted in shared memory by a bitonic network whose
// comparators all point the same way, so missing elements past L act as +infinity.
__global__ void __launch_bounds__(256) k_score_warp(ScoreArgs a) {
    __shared__ uint64_t s_keys[8][kWarpHits];
    __shared__ SliceGeom s_geom[kMaxSlices];
    for (int i = threadIdx.x; i < static_cast<int>(a.ix.n_slices); i += blockDim.x) s_geom[i] = a.ix.geom[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    uint64_t* keys = s_keys[warp];
    const Tables& T = *a.tables;
    if (a.counters->n_hits > a.hit_cap || a.counters->overflow) return;  // rerun follows
    const uint64_t gw = blockIdx.x * 8ull + warp, nw = gridDim.x * 8ull;
    for (uint64_t qi = gw; qi < a.n; qi += nw) {
        const uint32_t h0 = a.qhoff[qi], L = a.qhoff[qi + 1] - h0;
        if (L > static_cast<uint32_t>(kWarpHits)) {
            if (lane == 0) a.big[atomicAdd(&a.counters->n_big, 1u)] = static_cast<uint32_t>(qi);
            continue;
        }
        const uint64_t q = a.qsig[qi];
        const uint4* seg = a.seg + h0;
        uint32_t P2 = 1;
        while (P2 < L) P2 <<= 1;
        for (uint32_t i = lane; i < P2; i += 32)
            keys[i] = i < L ? (order_key(seg[i]) << 8) | i : ~0ull;
        __syncwarp();
        for (uint32_t k = 2; k <= P2; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = lane; i < P2; i += 32) {
                    // first stage of each merge compares mirrored pairs, later stages i / i+j
                    const uint32_t partner = (j == (k >> 1)) ? (i ^ (k - 1)) : (i ^ j);
                    if (partner > i) {
                        const uint64_t x = keys[i], y = keys[partner];
                        if (x > y) {
                            keys[i] = y;
                            keys[partner] = x;
                        }
                    }
                }
                __syncwarp();
            }
        }
        double run_mit = 0.0, run_cfd = 0.0;
        uint64_t run_cnt = 0;
        bool stopped = false;
        for (uint32_t c0 = 0; c0 < L && !stopped; c0 += 32) {
            const uint32_t t = c0 + lane;
            Contribution c{0.0, 0.0, 0};
            uint32_t id = 0;
            if (t < L) {
                const uint4 r = seg[keys[t] & 0xFF];
                const SliceGeom& g = s_geom[r.y];
                id = r.w;
                c = contribution(T, a.P, q, site_signature(q, g, r.z), a.ix.occ[id]);
            }
            const double im = warp_incl_sum(c.mit, lane) + run_mit;
            const double ic = warp_incl_sum(c.cfd, lane) + run_cfd;
            const uint64_t in = warp_incl_sum_u64(c.occ, lane) + run_cnt;
            const bool ex = t < L && exit_test(a.P, im, ic);
            const unsigned em = __ballot_sync(0xffffffffu, ex);
            const int last = em ? __ffs(em) - 1 : (L - c0 >= 32 ? 31 : static_cast<int>(L - c0 - 1));
            if (a.P.want_distinct && t < L && lane <= last) atomicOr(&a.bitmap[id >> 5], 1u << (id & 31));
            run_mit = __shfl_sync(0xffffffffu, im, last);
            run_cfd = __shfl_sync(0xffffffffu, ic, last);
            run_cnt = __shfl_sync(0xffffffffu, in, last);
            stopped = em != 0;
        }
        if (lane == 0)
            finalise(a.P, run_mit, run_cfd, run_cnt, qi, a.out_mit, a.out_cfd, a.out_code, a.out_count);
        __syncwarp();
    }
}

// Block per guide with more than kWarpHits hits: bitonic sort of the segment in global memory
// (in place), then the same ordered accumulation with block-wide prefix sums.
__global__ void __launch_bounds__(256) k_score_block(ScoreArgs a) {
    __shared__ SliceGeom s_geom[kMaxSlices];
    __shared__ double s_wm[8], s_wc[8];
    __shared__ uint64_t s_wn[8];
    __shared__ int s_first;
    for (int i = threadIdx.x; i < static_cast<int>(a.ix.n_slices); i += blockDim.x) s_geom[i] = a.ix.geom[i];
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const Tables& T = *a.tables;
    if (a.counters->n_hits > a.hit_cap || a.counters->overflow) return;  // rerun follows
    const uint32_t n_big = a.counters->n_big;
    for (uint32_t b = blockIdx.x; b < n_big; b += gridDim.x) {
        const uint64_t qi = a.big[b];
        const uint32_t h0 = a.qhoff[qi], L = a.qhoff[qi + 1] - h0;
        uint4* seg = a.seg + h0;
        const uint64_t q = a.qsig[qi];
        uint32_t P2 = 1;
        while (P2 < L) P2 <<= 1;
        for (uint32_t k = 2; k <= P2; k <<= 1) {
            for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                for (uint32_t i = threadIdx.x; i < P2; i += blockDim.x) {
                    const uint32_t partner = (j == (k >> 1)) ? (i ^ (k - 1)) : (i ^ j);
                    if (partner > i && partner < L) {
                        const uint4 x = seg[i], y = seg[partner];
                        if (order_key(x) > order_key(y)) {
                            seg[i] = y;
                            seg[partner] = x;
                        }
                    }
                }
                __syncthreads();
            }
        }
        double run_mit = 0.0, run_cfd = 0.0;
        uint64_t run_cnt = 0;
        bool stopped = false;
        for (uint32_t c0 = 0; c0 < L && !stopped; c0 += blockDim.x) {
            const uint32_t t = c0 + threadIdx.x;
            Contribution c{0.0, 0.0, 0};
            uint32_t id = 0;
            if (t < L) {
                const uint4 r = seg[t];
                id = r.w;
                c = contribution(T, a.P, q, site_signature(q, s_geom[r.y], r.z), a.ix.occ[id]);
            }
            double im = warp_incl_sum(c.mit, lane), ic = warp_incl_sum(c.cfd, lane);
            uint64_t in = warp_incl_sum_u64(c.occ, lane);
            if (lane == 31) {
                s_wm[warp] = im;
                s_wc[warp] = ic;
                s_wn[warp] = in;
            }
            if (threadIdx.x == 0) s_first = 0x7fffffff;
            __syncthreads();
            double pm = run_mit, pc = run_cfd;
            uint64_t pn = run_cnt;
            for (int w = 0; w < warp; w++) {
                pm += s_wm[w];
                pc += s_wc[w];
                pn += s_wn[w];
            }
            im += pm;
            ic += pc;
            in += pn;
            if (t < L && exit_test(a.P, im, ic)) atomicMin(&s_first, static_cast<int>(threadIdx.x));
            __syncthreads();
            const int first = s_first;
            const uint32_t in_chunk = L - c0 < blockDim.x ? L - c0 : blockDim.x;
            const int last = first != 0x7fffffff ? first : static_cast<int>(in_chunk) - 1;
            if (a.P.want_distinct && t < L && static_cast<int>(threadIdx.x) <= last)
                atomicOr(&a.bitmap[id >> 5], 1u << (id & 31));
            __syncthreads();
            if (static_cast<int>(threadIdx.x) == last) {
                s_wm[0] = im;
                s_wc[0] = ic;
                s_wn[0] = in;
            }
            __syncthreads();
            run_mit = s_wm[0];
            run_cfd = s_wc[0];
            run_cnt = s_wn[0];
            stopped = first != 0x7fffffff;
            __syncthreads();
        }
        if (threadIdx.x == 0)
            finalise(a.P, run_mit, run_cfd, run_cnt, qi, a.out_mit, a.out_cfd, a.out_code, a.out_count);
        __syncthreads();
    }
}

__global__ void k_popcount(const uint32_t* __restrict__ bm, uint64_t words, Counters* c) {
    uint64_t acc = 0;
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < words;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        acc += __popc(bm[i]);
    for (int d = 16; d > 0; d >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, d);
    if ((threadIdx.x & 31) == 0 && acc) atomicAdd(reinterpret_cast<unsigned long long*>(&c->distinct), acc);
}

__global__ void k_copy_distinct(const Counters* c, uint64_t* out) { *out = c->distinct; }

// ---------------------------------------------------------------------------------------------
// host orchestration
int sm_count(int device) {
    int v = 0;
    cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device);
    return v > 0 ? v : 148;
}

void init_tables(Workspace& ws, cudaStream_t st) {
    Tables h;
    const auto& mit = mit_rank_table();
    std::memcpy(h.mit, mit.data(), sizeof h.mit);
    std::memcpy(h.cfd_pos, cfd_pos_table(), sizeof h.cfd_pos);
    std::memcpy(h.cfd_pam, cfd_pam_table(), sizeof h.cfd_pam);
    for (int p = 0; p < 20; p++)
        for (int i = 0; i < 5; i++) {
            uint64_t r = (i <= p) ? 1 : 0;
            for (int t = 1; t <= i && i <= p; t++) r = r * (p - i + t) / t;
            h.binom[p][i] = static_cast<uint32_t>(r);
        }
    ws.tables.reserve(1);
    ISSL_CUDA(cudaMemcpyAsync(ws.tables.p, &h, sizeof h, cudaMemcpyHostToDevice, st));
    ISSL_CUDA(cudaStreamSynchronize(st));
}

Workspace& workspace(issl_index* ix) {
    if (!ix->ws) {
        auto ws = std::make_unique<Workspace>();
        ws->device = ix->device;
        ISSL_CUDA(cudaStreamCreateWithFlags(&ws->own_stream, cudaStreamNonBlocking));
        for (auto& e : ws->ev) ISSL_CUDA(cudaEventCreate(&e));
        int per_sm = 0;
        ISSL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_scan, kScanWarps * 32, 0));
        ws->scan_blocks = sm_count(ix->device) * std::max(per_sm, 1);
        ws->counters.reserve(1);
        ws->scan64.reserve(kScanBlocks + 4);
        ws->scan32.reserve(kScanBlocks + 4);
        init_tables(*ws, ws->own_stream);
        ix->ws = std::move(ws);
    }
    return *ix->ws;
}

void ensure_capacity(issl_index* ix, Workspace& ws, size_t n, cudaStream_t st) {
    const uint64_t S = ix->n_slices, G = ix->n_buckets;
    if (ws.g_cap < G + 1) {
        ws.bucket_cnt.reserve(G + 1);
        ws.bucket_qstart.reserve(G + 1);
        ISSL_CUDA(cudaMemsetAsync(ws.bucket_cnt.p, 0, (G + 1) * 4, st));
        ws.g_cap = G + 1;
    }
    if (ws.q_cap < n || !ws.qhits.p) {
        const size_t cap = std::max<size_t>(n, 1024);
        ws.qsig.reserve(cap);
        ws.probe_gb.reserve(cap * S);
        ws.probe_q.reserve(cap * S);
        ws.probe_rq.reserve(cap * S);
        ws.qhits.reserve(cap + 1);
        ws.qhoff.reserve(cap + 1);
        ws.big.reserve(cap);
        ws.out_mit.reserve(cap);
        ws.out_cfd.reserve(cap);
        ws.out_code.reserve(cap);
        ws.out_count.reserve(cap);
        ws.out_distinct.reserve(1);
        ISSL_CUDA(cudaMemsetAsync(ws.qhits.p, 0, (cap + 1) * 4, st));
        ws.q_cap = cap;
    }
    if (!ws.zero_state_ok) {
        ISSL_CUDA(cudaMemsetAsync(ws.bucket_cnt.p, 0, (G + 1) * 4, st));
        ISSL_CUDA(cudaMemsetAsync(ws.qhits.p, 0, (ws.q_cap + 1) * 4, st));
        ws.zero_state_ok = true;
    }
    // first guesses: ~2.5 units per probe plus headroom; hits grow on demand
    const size_t want_units = std::max<size_t>(ws.unit_cap, n * S * 3 + 4096);
    if (ws.unit_cap < want_units) {
        ws.units.reserve(want_units);
        ws.unit_cap = want_units;
    }
    const size_t want_hits = std::max<size_t>(ws.hit_cap, n * 64 + 65536);
    if (ws.hit_cap < want_hits) {
        ws.hits.reserve(want_hits);
        ws.seg.reserve(want_hits);
        ws.hit_cap = want_hits;
    }
}

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
    return P;
}

inline unsigned grid_for(uint64_t n, unsigned threads, unsigned cap) {
    uint64_t b = (n + threads - 1) / threads;
    if (b < 1) b = 1;
    if (b > cap) b = cap;
    return static_cast<unsigned>(b);
}

// Enqueues the whole pipeline for n guides whose signatures are in ws.qsig (or d_qsig).
void enqueue_pipeline(issl_index* ix, Workspace& ws, const uint64_t* d_qsig, uint64_t n, const ScoreParams& P,
                      double* d_mit, double* d_cfd, char* d_code, uint64_t* d_count, cudaStream_t st) {
    const IndexView v = ix->view();
    const uint64_t S = ix->n_slices, G = ix->n_buckets;
    const int sms = sm_count(ix->device);
    ISSL_CUDA(cudaMemsetAsync(ws.counters.p, 0, sizeof(Counters), st));
    const uint64_t* off = ix->offsets.p;
    ISSL_CUDA(cudaEventRecord(ws.ev[0], st));
    k_probe_count<<<grid_for(n * S, 256, sms * 16), 256, 0, st>>>(v, d_qsig, n, ws.probe_gb.p, ws.bucket_cnt.p, off);
    device_scan<uint64_t, OpSum>(BucketLoad{ws.bucket_cnt.p, off},
                                 BucketStore{ws.bucket_cnt.p, off, ws.bucket_qstart.p, ws.units.p, ws.unit_cap,
                                             ix->n_sites},
                                 nullptr, G, ws.scan64.p, &ws.counters.p->bucket_total, st);
    k_units_finalize<<<1, 1, 0, st>>>(ws.counters.p, ws.unit_cap);
    k_bucket_stats<<<sms * 4, 256, 0, st>>>(ws.bucket_cnt.p, off, G, ws.counters.p);
    k_probe_scatter<<<grid_for(n * S, 256, sms * 16), 256, 0, st>>>(v, d_qsig, n, ws.probe_gb.p, ws.bucket_cnt.p,
                                                                     ws.bucket_qstart.p, ws.probe_q.p, ws.probe_rq.p);
    ScanArgs sa;
    sa.resid = ix->resid.p;
    sa.geom = ix->d_geom.p;
    sa.units = ws.units.p;
    sa.probe_q = ws.probe_q.p;
    sa.probe_rq = ws.probe_rq.p;
    sa.counters = ws.counters.p;
    sa.hits = ws.hits.p;
    sa.qhits = ws.qhits.p;
    sa.n_sites = ix->n_sites;
    sa.hit_cap = static_cast<uint32_t>(std::min<size_t>(ws.hit_cap, 0xFFFFFFFFull));
    sa.n_slices = static_cast<uint32_t>(S);
    sa.max_dist = P.max_dist;
    ISSL_CUDA(cudaEventRecord(ws.ev[1], st));
    k_scan<<<ws.scan_blocks, kScanWarps * 32, 0, st>>>(sa);
    ISSL_CUDA(cudaEventRecord(ws.ev[2], st));
    device_scan<uint32_t, OpSum>(LoadQhits{ws.qhits.p}, StoreQoff{ws.qhoff.p}, nullptr, n, ws.scan32.p,
                                 ws.qhoff.p + n, st);
    k_hit_scatter<<<sms * 8, 256, 0, st>>>(ws.hits.p, ws.counters.p, sa.hit_cap, ws.qhits.p, ws.qhoff.p, ix->ids.p,
                                           ix->n_sites, ws.seg.p);
    if (P.want_distinct) ISSL_CUDA(cudaMemsetAsync(ws.bitmap.p, 0, (ix->n_sites / 32 + 1) * 4, st));
    ScoreArgs a;
    a.hit_cap = sa.hit_cap;
    a.ix = v;
    a.qsig = d_qsig;
    a.seg = ws.seg.p;
    a.qhoff = ws.qhoff.p;
    a.tables = ws.tables.p;
    a.counters = ws.counters.p;
    a.big = ws.big.p;
    a.bitmap = ws.bitmap.p;
    a.n = n;
    a.P = P;
    a.out_mit = d_mit;
    a.out_cfd = d_cfd;
    a.out_code = d_code;
    a.out_count = d_count;
    k_score_warp<<<grid_for(n, 8, sms * 8), 256, 0, st>>>(a);
    k_score_block<<<sms * 2, 256, 0, st>>>(a);
    if (P.want_distinct) k_popcount<<<sms * 4, 256, 0, st>>>(ws.bitmap.p, ix->n_sites / 32 + 1, ws.counters.p);
    ISSL_CUDA(cudaEventRecord(ws.ev[3], st));
    ISSL_CUDA(cudaGetLastError());
    // probe_count, 3 bucket-scan, units_finalize, bucket_stats, probe_scatter, scan, 3 hit-offset
    // scan, hit_scatter, score_warp, score_block (+ popcount for distinct counts)
    ws.launches += 14 + (P.want_distinct ? 1 : 0);
}

// Reads the counters after a pipeline run; returns false (and grows capacities) on overflow.
bool check_and_grow(issl_index* ix, Workspace& ws, cudaStream_t st) {
    Counters c;
    ISSL_CUDA(cudaMemcpyAsync(&c, ws.counters.p, sizeof c, cudaMemcpyDeviceToHost, st));
    ISSL_CUDA(cudaStreamSynchronize(st));
    ws.last = c;
    const uint64_t units = c.bucket_total >> 32;
    bool ok = true;
    if (units > ws.unit_cap) {
        ws.units.reserve(units + units / 8 + 1024);
        ws.unit_cap = units + units / 8 + 1024;
        ok = false;
    }
    if (c.n_hits > ws.hit_cap) {
        const size_t cap = static_cast<size_t>(c.n_hits) + c.n_hits / 4 + 65536;
        ISSL_REQUIRE(cap < 0xFFFFFFFFull, ISSL_ERR_UNSUPPORTED, "more than 2^32 hits in one call; split the guides");
        ws.hits.reserve(cap);
        ws.seg.reserve(cap);
        ws.hit_cap = cap;
        ok = false;
    }
    if (!ok) ws.zero_state_ok = false;  // counters of the aborted run are not drained
    return ok;
}

void record_stats(issl_index* ix, Workspace& ws, uint64_t n) {
    float scan = 0.f, total = 0.f;
    cudaEventElapsedTime(&scan, ws.ev[1], ws.ev[2]);
    cudaEventElapsedTime(&total, ws.ev[0], ws.ev[3]);
    issl_score_stats& s = ix->stats;
    s.scan_ms = scan;
    s.total_ms = total;
    s.probes = static_cast<uint64_t>(ws.last.bucket_total & 0xFFFFFFFFull);
    s.units = ws.last.bucket_total >> 32;
    s.hits = ws.last.n_hits;
    s.buckets_scanned = ws.last.buckets;
    s.entries_scanned = ws.last.entries;
    // bytes the scan must move: 4 per residual streamed, 16 per unit descriptor, 8 per guide of
    // a unit (slot + residual), 16 per hit written
    s.scan_bytes = 4 * s.entries_scanned + 16 * s.units + 8 * s.probes + 16 * s.hits;
    s.launches = ws.launches;
    ws.launches = 0;
    (void)n;
}

void run_scoring(issl_index* ix, const uint64_t* d_qsig_in, uint64_t n, const ScoreParams& P, double* d_mit,
                 double* d_cfd, char* d_code, uint64_t* d_count, uint64_t* d_distinct, cudaStream_t st,
                 bool sync_and_check) {
    Workspace& ws = workspace(ix);
    if (P.want_distinct) ws.bitmap.reserve(ix->n_sites / 32 + 1);
    for (int attempt = 0; attempt < 4; attempt++) {
        ensure_capacity(ix, ws, n, st);
        enqueue_pipeline(ix, ws, d_qsig_in, n, P, d_mit, d_cfd, d_code, d_count, st);
        if (d_distinct) {
            k_copy_distinct<<<1, 1, 0, st>>>(ws.counters.p, d_distinct);
            ws.launches++;
        }
        if (!sync_and_check) {
            // device-buffer path: one check per call keeps the workspace honest
        }
        if (check_and_grow(ix, ws, st)) {
            record_stats(ix, ws, n);
            return;
        }
    }
    throw Error(ISSL_ERR_NOMEM, "scoring workspace kept overflowing");
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
        ISSL_REQUIRE(n < (1ull << 31) && n * ix->n_slices < 0xFFFFFFFFull, ISSL_ERR_ARG,
                     "too many guides in one call");
        issl::run_scoring(ix, d_sigs, n, P, d_mit, d_cfd, d_code, d_count, d_distinct, st, true);
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
        ISSL_REQUIRE(n < (1ull << 31) && n * ix->n_slices < 0xFFFFFFFFull, ISSL_ERR_ARG,
                     "too many guides in one call");
        issl::ensure_capacity(ix, ws, n, st);
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
                          distinct ? ws.out_distinct.p : nullptr, st, true);
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

int issl_last_stats(const issl_index* ix, issl_score_stats* out) {
    return guarded([&] {
        ISSL_REQUIRE(ix && out, ISSL_ERR_ARG, "issl_last_stats: null argument");
        *out = ix->stats;
    });
}

}  // extern "C"
