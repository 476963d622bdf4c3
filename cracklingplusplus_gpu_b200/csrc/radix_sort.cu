// Stable LSD radix sort of (key, value) pairs, 8-bit digits, for the device index builder (or of
// keys alone when the value pointers are null).
//
// Per pass: (1) each block histograms the digit over its tile, written digit-major so that
// (2) one exclusive scan yields every (digit, block) output offset, then (3) each block
// re-reads its tile and scatters it. Stability inside a block comes from processing the tile
// in rounds of 32 consecutive items per warp: __match_any_sync groups the lanes holding the
// same digit, a lane's rank is the number of lower lanes in its group plus the warp's running
// count for that digit, and warps are combined in warp order.
#include <cuda_runtime.h>

#include "issl_internal.cuh"
#include "scan.cuh"

namespace issl {
namespace {

constexpr int kRsThreads = 256;               // 8 warps
constexpr int kRsWarps = kRsThreads / 32;
constexpr int kRsRounds = 8;                  // rounds of 32 items per warp per sub-tile
constexpr int kRsSub = kRsThreads * kRsRounds;  // 2048 items per sub-tile
constexpr int kRsSubTiles = 4;
constexpr int kRsTile = kRsSub * kRsSubTiles;   // 8192 items per block

template <class K>
__global__ void __launch_bounds__(kRsThreads) k_rs_upsweep(const K* keys, uint64_t n, int shift,
                                                          uint32_t* hist, uint32_t nblocks) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t lo = static_cast<uint64_t>(blockIdx.x) * kRsTile;
    const uint64_t hi = lo + kRsTile < n ? lo + kRsTile : n;
    for (uint64_t i = lo + threadIdx.x; i < hi; i += kRsThreads)
        atomicAdd(&h[static_cast<uint32_t>(keys[i] >> shift) & 255u], 1u);
    __syncthreads();
    hist[static_cast<uint64_t>(threadIdx.x) * nblocks + blockIdx.x] = h[threadIdx.x];
}

template <class K>
__global__ void __launch_bounds__(kRsThreads) k_rs_downsweep(const K* keys, const uint32_t* vals,
                                                            K* keys_out, uint32_t* vals_out,
                                                            uint64_t n, int shift,
                                                            const uint32_t* offs, uint32_t nblocks) {
    __shared__ uint32_t wcnt[kRsWarps][256];
    __shared__ uint32_t boff[256];
    __shared__ uint32_t stot[256];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    boff[threadIdx.x] = offs[static_cast<uint64_t>(threadIdx.x) * nblocks + blockIdx.x];
    const uint64_t blo = static_cast<uint64_t>(blockIdx.x) * kRsTile;
    for (int sub = 0; sub < kRsSubTiles; sub++) {
        const uint64_t sbase = blo + static_cast<uint64_t>(sub) * kRsSub;
        if (sbase >= n) break;
        for (int w = 0; w < kRsWarps; w++) wcnt[w][threadIdx.x] = 0;
        __syncthreads();
        K k[kRsRounds];
        uint32_t v[kRsRounds], d[kRsRounds], r[kRsRounds];
        const uint64_t wbase = sbase + static_cast<uint64_t>(warp) * 32 * kRsRounds;
#pragma unroll
        for (int j = 0; j < kRsRounds; j++) {
            const uint64_t i = wbase + j * 32 + lane;
            const bool ok = i < n;
            k[j] = ok ? keys[i] : K(0);
            v[j] = ok && vals ? vals[i] : 0u;
            d[j] = ok ? (static_cast<uint32_t>(k[j] >> shift) & 255u) : 256u;
        }
#pragma unroll
        for (int j = 0; j < kRsRounds; j++) {
            const unsigned peers = __match_any_sync(0xffffffffu, d[j]);
            const uint32_t before = d[j] < 256u ? wcnt[warp][d[j]] : 0u;
            __syncwarp();
            r[j] = before + __popc(peers & lt);
            if (d[j] < 256u && (peers & lt) == 0u) wcnt[warp][d[j]] = before + __popc(peers);
            __syncwarp();
        }
        __syncthreads();
        {
            uint32_t run = 0;
            for (int w = 0; w < kRsWarps; w++) {
                const uint32_t c = wcnt[w][threadIdx.x];
                wcnt[w][threadIdx.x] = run;
                run += c;
            }
            stot[threadIdx.x] = run;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kRsRounds; j++) {
            if (d[j] < 256u) {
                const uint32_t pos = boff[d[j]] + wcnt[warp][d[j]] + r[j];
                keys_out[pos] = k[j];
                if (vals_out) vals_out[pos] = v[j];
            }
        }
        __syncthreads();
        boff[threadIdx.x] += stot[threadIdx.x];
        __syncthreads();
    }
}

struct LoadU32 {
    const uint32_t* p;
    __device__ uint32_t operator()(uint64_t i) const { return p[i]; }
};
struct StoreExcl {
    uint32_t* p;
    __device__ void operator()(uint64_t i, uint32_t ex, uint32_t) const { p[i] = ex; }
};

template <class K>
void radix_sort_impl(K* keys, uint32_t* vals, K* keys_tmp, uint32_t* vals_tmp, size_t n, int bits,
                     void* temp, size_t temp_bytes, cudaStream_t st, K** keys_out, uint32_t** vals_out) {
    ISSL_REQUIRE(n < (1ull << 32), ISSL_ERR_UNSUPPORTED, "radix sort: more than 2^32 items");
    const uint32_t nblocks = static_cast<uint32_t>((n + kRsTile - 1) / kRsTile);
    const size_t need = (static_cast<size_t>(nblocks) * 256 + kScanBlocks + 8) * sizeof(uint32_t);
    ISSL_REQUIRE(temp_bytes >= need, ISSL_ERR_ARG, "radix sort: temp buffer too small");
    uint32_t* hist = static_cast<uint32_t*>(temp);
    uint32_t* scan_tmp = hist + static_cast<size_t>(nblocks) * 256;
    K* ka = keys;
    K* kb = keys_tmp;
    uint32_t* va = vals;
    uint32_t* vb = vals_tmp;
    for (int shift = 0; shift < bits && n > 0; shift += 8) {
        k_rs_upsweep<K><<<nblocks, kRsThreads, 0, st>>>(ka, n, shift, hist, nblocks);
        const uint64_t m = static_cast<uint64_t>(nblocks) * 256;
        device_scan<uint32_t, OpSum>(LoadU32{hist}, StoreExcl{hist}, nullptr, m, scan_tmp, nullptr, st);
        k_rs_downsweep<K><<<nblocks, kRsThreads, 0, st>>>(ka, va, kb, vb, n, shift, hist, nblocks);
        ISSL_CUDA(cudaGetLastError());
        K* t = ka;
        ka = kb;
        kb = t;
        uint32_t* u = va;
        va = vb;
        vb = u;
    }
    *keys_out = ka;
    *vals_out = va;
}

}  // namespace

size_t radix_sort_temp_bytes(size_t n, bool) {
    const size_t nblocks = (n + kRsTile - 1) / kRsTile;
    return (nblocks * 256 + kScanBlocks + 8) * sizeof(uint32_t);
}

void radix_sort_pairs_u32(uint32_t* keys, uint32_t* vals, uint32_t* keys_tmp, uint32_t* vals_tmp,
                          size_t n, int bits, void* temp, size_t temp_bytes, cudaStream_t st,
                          uint32_t** keys_out, uint32_t** vals_out) {
    radix_sort_impl<uint32_t>(keys, vals, keys_tmp, vals_tmp, n, bits, temp, temp_bytes, st, keys_out,
                              vals_out);
}

void radix_sort_pairs_u64(uint64_t* keys, uint32_t* vals, uint64_t* keys_tmp, uint32_t* vals_tmp,
                          size_t n, int bits, void* temp, size_t temp_bytes, cudaStream_t st,
                          uint64_t** keys_out, uint32_t** vals_out) {
    radix_sort_impl<uint64_t>(keys, vals, keys_tmp, vals_tmp, n, bits, temp, temp_bytes, st, keys_out,
                              vals_out);
}

}  // namespace issl
