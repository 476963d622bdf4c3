// Seeded synthetic workloads generated on the device: distinct 20-nt sites (i.i.d. with GC 41%
// plus repeat-seed families with Poisson substitutions), occurrence counts, query guides, and the
// resident index built from them. Every draw is a counter-based splitmix64 hash of
// (seed, stream, counter), so a spec always yields the same workload.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "device_util.cuh"
#include "issl_internal.cuh"
#include "scan.cuh"

namespace issl {
namespace {

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
__device__ __forceinline__ uint64_t draw(uint64_t seed, uint64_t stream, uint64_t i) {
    return mix64(mix64(seed * 0x100000001B3ull + stream * 0x9E3779B1ull) + i * 0xD1B54A32D192ED03ull);
}
__device__ __forceinline__ double unif(uint64_t h) { return static_cast<double>(h >> 11) * (1.0 / 9007199254740992.0); }

// GC 41%: P(A) = P(T) = 0.295, P(C) = P(G) = 0.205
__device__ __forceinline__ uint64_t gc41(double u) { return u < 0.295 ? 0u : u < 0.5 ? 1u : u < 0.705 ? 2u : 3u; }

__device__ uint64_t random_site(uint64_t seed, uint64_t stream, uint64_t i) {
    uint64_t s = 0;
    for (int j = 0; j < kSeqLen; j++) s |= gc41(unif(draw(seed, stream, i * 32 + j))) << (2 * j);
    return s;
}

// k substitutions at distinct uniform positions, each to a different base
__device__ uint64_t mutate(uint64_t sig, int k, uint64_t seed, uint64_t stream, uint64_t i) {
    uint32_t used = 0;
    uint64_t c = 0;
    for (int t = 0; t < k; t++) {
        int p = static_cast<int>(draw(seed, stream, i * 64 + c++) % kSeqLen);
        for (int tries = 0; (used >> p & 1u) && tries < 256; tries++)
            p = static_cast<int>(draw(seed, stream, i * 64 + c++) % kSeqLen);
        while (used >> p & 1u) p = (p + 1) % kSeqLen;  // k <= 20 leaves a free position
        used |= 1u << p;
        const uint64_t b = (sig >> (2 * p)) & 3u;
        const uint64_t nb = (b + 1 + draw(seed, stream + 1, i * 64 + t) % 3) & 3u;
        sig = (sig & ~(3ull << (2 * p))) | (nb << (2 * p));
    }
    return sig;
}

__device__ int poisson(double lam, double u) {
    double p = exp(-lam), c = p;
    int k = 0;
    while (u > c && k < kSeqLen) {
        k++;
        p *= lam / k;
        c += p;
    }
    return k;
}

enum : uint64_t { kStSeed = 1, kStRepPick = 3, kStRepSubs = 4, kStRepMut = 5, kStIid = 8, kStOcc = 10,
                  kStQPick = 11, kStQSubs = 12, kStQMut = 13, kStQRand = 15, kStQRep = 16, kStQRepMut = 17,
                  kStShuffle = 19 };

__global__ void k_gen_seeds(uint64_t seed, uint64_t n, uint64_t* out) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        out[i] = random_site(seed, kStSeed, i);
}

// pool[0, n_rep): repeat copies; pool[n_rep, n): i.i.d. sites
__global__ void k_gen_pool(uint64_t seed, const uint64_t* seeds, uint64_t n_seeds, uint64_t n_rep, double lam,
                           uint64_t n, uint64_t* pool) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (i < n_rep) {
            const uint64_t src = seeds[draw(seed, kStRepPick, i) % n_seeds];
            pool[i] = mutate(src, poisson(lam, unif(draw(seed, kStRepSubs, i))), seed, kStRepMut, i);
        } else {
            pool[i] = random_site(seed, kStIid, i);
        }
    }
}

__global__ void k_iota_copy(const uint64_t* in, uint64_t n, uint64_t* keys, uint32_t* vals) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        keys[i] = in[i];
        vals[i] = static_cast<uint32_t>(i);
    }
}

// keep[idx] = 1 for the first (lowest index) copy of every distinct signature
__global__ void k_mark_first(const uint64_t* sorted, const uint32_t* idx, uint64_t n, uint32_t* keep) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        keep[idx[i]] = (i == 0 || sorted[i] != sorted[i - 1]) ? 1u : 0u;
}

struct LoadKeep {
    const uint32_t* k;
    __device__ uint32_t operator()(uint64_t i) const { return k[i]; }
};
struct StoreCompact {
    const uint32_t* keep;
    const uint64_t* in;
    uint64_t* out;
    uint64_t limit;
    __device__ void operator()(uint64_t i, uint32_t ex, uint32_t) const {
        if (keep[i] && ex < limit) out[ex] = in[i];
    }
};

__global__ void k_occurrences(uint64_t seed, uint64_t n, uint32_t* occ) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const double u = unif(draw(seed, kStOcc, i));
        const double fails = floor(log1p(-u) / log(0.1));  // Geometric(p = 0.9) failures
        occ[i] = static_cast<uint32_t>(fmin(1.0 + fails, 255.0));
    }
}

// copied queries: a site with 0..4 substitutions (planted: the exact site, the mutant goes to out_mut)
__global__ void k_gen_copied(uint64_t seed, const uint64_t* sites, uint64_t n_sites, uint64_t n, int planted,
                             uint64_t* q_out, uint64_t* mut_out) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        const uint64_t src = sites[draw(seed, kStQPick, i) % n_sites];
        const uint64_t mut = mutate(src, static_cast<int>(draw(seed, kStQSubs, i) % 5), seed, kStQMut, i);
        if (planted) {
            q_out[i] = src;
            mut_out[i] = mut;
        } else {
            q_out[i] = mut;
        }
    }
}

__global__ void k_gen_other_queries(uint64_t seed, const uint64_t* seeds, uint64_t n_seeds, uint64_t n_rep,
                                    uint64_t n, uint64_t* q_out) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        if (i < n_rep) {
            const uint64_t src = seeds[draw(seed, kStQRep, i) % n_seeds];
            q_out[i] = mutate(src, static_cast<int>(draw(seed, kStQRep + 100, i) % 3), seed, kStQRepMut, i);
        } else {
            q_out[i] = random_site(seed, kStQRand, i);
        }
    }
}

__global__ void k_shuffle_keys(uint64_t seed, uint64_t n, uint64_t* keys, uint32_t* vals) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x) {
        keys[i] = draw(seed, kStShuffle, i);
        vals[i] = static_cast<uint32_t>(i);
    }
}

__global__ void k_gather(const uint64_t* in, const uint32_t* perm, uint64_t n, uint64_t* out) {
    for (uint64_t i = blockIdx.x * static_cast<uint64_t>(blockDim.x) + threadIdx.x; i < n;
         i += static_cast<uint64_t>(gridDim.x) * blockDim.x)
        out[i] = in[perm[i]];
}

inline unsigned grid(uint64_t n) {
    uint64_t b = (n + 255) / 256;
    return static_cast<unsigned>(std::max<uint64_t>(1, std::min<uint64_t>(b, 148ull * 32)));
}

// First `limit` distinct values of `in` (first occurrence order); returns how many were written.
uint64_t dedup_first(const uint64_t* in, uint64_t n, uint64_t* out, uint64_t limit, cudaStream_t st) {
    DevBuf<uint64_t> k1, k2;
    DevBuf<uint32_t> v1, v2, keep, scan_tmp, total;
    DevBuf<uint8_t> temp;
    k1.reserve(n);
    k2.reserve(n);
    v1.reserve(n);
    v2.reserve(n);
    keep.reserve(n);
    scan_tmp.reserve(kScanBlocks + 4);
    total.reserve(1);
    const size_t tb = radix_sort_temp_bytes(n, true);
    temp.reserve(tb);
    k_iota_copy<<<grid(n), 256, 0, st>>>(in, n, k1.p, v1.p);
    uint64_t* ko;
    uint32_t* vo;
    radix_sort_pairs_u64(k1.p, v1.p, k2.p, v2.p, n, 40, temp.p, tb, st, &ko, &vo);
    k_mark_first<<<grid(n), 256, 0, st>>>(ko, vo, n, keep.p);
    device_scan<uint32_t, OpSum>(LoadKeep{keep.p}, StoreCompact{keep.p, in, out, limit}, nullptr, n, scan_tmp.p,
                                 total.p, st);
    uint32_t t = 0;
    ISSL_CUDA(cudaMemcpyAsync(&t, total.p, 4, cudaMemcpyDeviceToHost, st));
    ISSL_CUDA(cudaStreamSynchronize(st));
    return std::min<uint64_t>(t, limit);
}

}  // namespace
}  // namespace issl

extern "C" int issl_synth(const issl_synth_spec* spec, int device, issl_index** out, uint64_t* queries) {
    using namespace issl;
    return guarded([&] {
        ISSL_REQUIRE(spec && out && spec->slice_masks && (queries || spec->n_queries == 0), ISSL_ERR_ARG,
                     "issl_synth: null argument");
        ISSL_REQUIRE(spec->n_sites >= 16 && spec->n_sites < (1ull << 31), ISSL_ERR_ARG,
                     "issl_synth: n_sites must be 16..2^31");
        ISSL_REQUIRE(spec->repeat_frac >= 0 && spec->repeat_frac <= 1 && spec->copied_frac >= 0 &&
                         spec->repeat_query_frac >= 0 && spec->copied_frac + spec->repeat_query_frac <= 1,
                     ISSL_ERR_ARG, "issl_synth: fractions out of range");
        *out = nullptr;
        ISSL_CUDA(cudaSetDevice(device));
        cudaStream_t st;
        ISSL_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
        struct G {
            cudaStream_t s;
            ~G() { cudaStreamDestroy(s); }
        } guard{st};
        const uint64_t seed = spec->seed;
        const uint64_t N = spec->n_sites, Q = spec->n_queries;
        const uint64_t n_seeds = std::max<uint64_t>(spec->n_repeat_seeds, 1);
        const uint64_t n_rep = static_cast<uint64_t>(std::llround(static_cast<double>(N) * spec->repeat_frac));
        const uint64_t n_copied = static_cast<uint64_t>(std::llround(static_cast<double>(Q) * spec->copied_frac));
        const uint64_t n_repq = static_cast<uint64_t>(std::llround(static_cast<double>(Q) * spec->repeat_query_frac));
        const bool planted = spec->planted_into_sites != 0;
        const uint64_t extra = n_rep / 2 + N / 64 + 4096;
        const uint64_t n_pool = N + extra;

        DevBuf<uint64_t> seeds, pool, sites, qbuf;
        seeds.reserve(n_seeds);
        k_gen_seeds<<<grid(n_seeds), 256, 0, st>>>(seed, n_seeds, seeds.p);
        pool.reserve(n_pool);
        k_gen_pool<<<grid(n_pool), 256, 0, st>>>(seed, seeds.p, n_seeds, n_rep, spec->repeat_lambda, n_pool, pool.p);
        sites.reserve(N);
        qbuf.reserve(std::max<uint64_t>(Q, 1));
        uint64_t got;
        if (planted && n_copied) {
            // queries copy sites of the first part; their 0-4 substitution mutants join the sites
            const uint64_t base_n = N - std::min(n_copied, N / 2);
            got = dedup_first(pool.p, n_pool, sites.p, base_n, st);
            ISSL_REQUIRE(got == base_n, ISSL_ERR_ARG, "issl_synth: not enough distinct sites");
            DevBuf<uint64_t> mut, pool2;
            mut.reserve(n_copied);
            k_gen_copied<<<grid(n_copied), 256, 0, st>>>(seed, sites.p, base_n, n_copied, 1, qbuf.p, mut.p);
            pool2.reserve(base_n + n_copied + n_pool);
            ISSL_CUDA(cudaMemcpyAsync(pool2.p, sites.p, base_n * 8, cudaMemcpyDeviceToDevice, st));
            ISSL_CUDA(cudaMemcpyAsync(pool2.p + base_n, mut.p, n_copied * 8, cudaMemcpyDeviceToDevice, st));
            ISSL_CUDA(cudaMemcpyAsync(pool2.p + base_n + n_copied, pool.p, n_pool * 8, cudaMemcpyDeviceToDevice, st));
            got = dedup_first(pool2.p, base_n + n_copied + n_pool, sites.p, N, st);
        } else {
            got = dedup_first(pool.p, n_pool, sites.p, N, st);
            if (n_copied)
                k_gen_copied<<<grid(n_copied), 256, 0, st>>>(seed, sites.p, N, n_copied, 0, qbuf.p, nullptr);
        }
        ISSL_REQUIRE(got == N, ISSL_ERR_ARG, "issl_synth: not enough distinct sites were generated");
        if (Q > n_copied)
            k_gen_other_queries<<<grid(Q - n_copied), 256, 0, st>>>(seed, seeds.p, n_seeds, n_repq, Q - n_copied,
                                                                    qbuf.p + n_copied);
        pool.release();
        // shuffle the query classes together
        if (Q > 1) {
            DevBuf<uint64_t> k1, k2, qs;
            DevBuf<uint32_t> v1, v2;
            DevBuf<uint8_t> temp;
            k1.reserve(Q);
            k2.reserve(Q);
            v1.reserve(Q);
            v2.reserve(Q);
            qs.reserve(Q);
            const size_t tb = radix_sort_temp_bytes(Q, true);
            temp.reserve(tb);
            k_shuffle_keys<<<grid(Q), 256, 0, st>>>(seed, Q, k1.p, v1.p);
            uint64_t* ko;
            uint32_t* vo;
            radix_sort_pairs_u64(k1.p, v1.p, k2.p, v2.p, Q, 64, temp.p, tb, st, &ko, &vo);
            k_gather<<<grid(Q), 256, 0, st>>>(qbuf.p, vo, Q, qs.p);
            ISSL_CUDA(cudaMemcpyAsync(queries, qs.p, Q * 8, cudaMemcpyDeviceToHost, st));
            ISSL_CUDA(cudaStreamSynchronize(st));
        } else if (Q == 1) {
            ISSL_CUDA(cudaMemcpyAsync(queries, qbuf.p, 8, cudaMemcpyDeviceToHost, st));
        }
        auto ix = std::make_unique<issl_index>();
        ix->device = device;
        ix->n_sites = N;
        ix->seq_len = kSeqLen;
        ix->n_slices = spec->n_slices;
        ix->masks.assign(spec->slice_masks, spec->slice_masks + spec->n_slices);
        ix->occ.reserve(N);
        k_occurrences<<<grid(N), 256, 0, st>>>(seed, N, ix->occ.p);
        ix->sigs.reserve(N);
        ISSL_CUDA(cudaMemcpyAsync(ix->sigs.p, sites.p, N * 8, cudaMemcpyDeviceToDevice, st));
        sites.release();
        ISSL_CUDA(cudaGetLastError());
        build_from_device_sites(ix.get(), ix->sigs.p, ix->occ.p, st);
        ISSL_CUDA(cudaStreamSynchronize(st));
        *out = ix.release();
    });
}
