// Device-wide scans with a fixed grid (reduce-then-scan, three launches).
//
// The element count may live in device memory (`d_n`), so a pipeline can chain scans whose
// sizes are produced by earlier kernels without a host round trip; the grid is fixed at
// kScanBlocks blocks, each owning one contiguous range of the input.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>

namespace issl {

constexpr int kScanBlocks = 296;    // 2 per SM on B200 (148 SMs)
constexpr int kScanThreads = 512;
constexpr int kScanItems = 4;       // consecutive items per thread per tile

struct OpSum {
    template <class T>
    __device__ __forceinline__ T operator()(T a, T b) const { return a + b; }
    template <class T>
    __device__ __forceinline__ static T identity() { return T(0); }
};
struct OpMax {
    template <class T>
    __device__ __forceinline__ T operator()(T a, T b) const { return a > b ? a : b; }
    template <class T>
    __device__ __forceinline__ static T identity() { return T(0); }
};

__device__ __forceinline__ uint64_t scan_count(const uint32_t* d_n, uint64_t n_host) {
    return d_n ? static_cast<uint64_t>(*d_n) : n_host;
}

__device__ __forceinline__ void scan_range(uint64_t n, uint64_t& lo, uint64_t& hi) {
    const uint64_t tile = static_cast<uint64_t>(kScanThreads) * kScanItems;
    uint64_t tiles = (n + tile - 1) / tile;
    uint64_t per = (tiles + gridDim.x - 1) / gridDim.x;
    lo = per * tile * blockIdx.x;
    hi = lo + per * tile;
    if (lo > n) lo = n;
    if (hi > n) hi = n;
}

// Block-wide inclusive scan of one value per thread; returns the inclusive prefix and writes
// the block total to *total.
template <class T, class Op>
__device__ __forceinline__ T block_inclusive(T v, Op op, T* smem_warp, T* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        T o = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v = op(o, v);
    }
    if (lane == 31) smem_warp[warp] = v;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        T w = lane < nw ? smem_warp[lane] : Op::template identity<T>();
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            T o = __shfl_up_sync(0xffffffffu, w, d);
            if (lane >= d) w = op(o, w);
        }
        if (lane < nw) smem_warp[lane] = w;
    }
    __syncthreads();
    if (warp > 0) v = op(smem_warp[warp - 1], v);
    *total = smem_warp[(blockDim.x >> 5) - 1];
    __syncthreads();
    return v;
}

template <class T, class Op, class Load>
__global__ void __launch_bounds__(kScanThreads) k_scan_reduce(Load load, const uint32_t* d_n,
                                                              uint64_t n_host, T* block_sums) {
    __shared__ T sw[32];
    Op op;
    uint64_t lo, hi;
    scan_range(scan_count(d_n, n_host), lo, hi);
    T acc = Op::template identity<T>();
    for (uint64_t i = lo + threadIdx.x; i < hi; i += blockDim.x) acc = op(acc, load(i));
    T total;
    block_inclusive<T, Op>(acc, op, sw, &total);
    if (threadIdx.x == 0) block_sums[blockIdx.x] = total;
}

template <class T, class Op>
__global__ void __launch_bounds__(1024) k_scan_top(T* block_sums, int nb, T* d_total) {
    __shared__ T sw[32];
    Op op;
    T v = threadIdx.x < nb ? block_sums[threadIdx.x] : Op::template identity<T>();
    T total;
    T inc = block_inclusive<T, Op>(v, op, sw, &total);
    if (threadIdx.x < nb) block_sums[threadIdx.x] = inc;  // inclusive per block
    if (threadIdx.x == 0 && d_total) *d_total = total;
}

// Store(i, exclusive, inclusive) receives both prefixes of element i.
template <class T, class Op, class Load, class Store>
__global__ void __launch_bounds__(kScanThreads) k_scan_down(Load load, Store store, const uint32_t* d_n,
                                                            uint64_t n_host, const T* block_incl) {
    __shared__ T sw[32];
    Op op;
    uint64_t lo, hi;
    scan_range(scan_count(d_n, n_host), lo, hi);
    T carry = blockIdx.x > 0 ? block_incl[blockIdx.x - 1] : Op::template identity<T>();
    const uint64_t tile = static_cast<uint64_t>(kScanThreads) * kScanItems;
    for (uint64_t t0 = lo; t0 < hi; t0 += tile) {
        T v[kScanItems];
        T run = Op::template identity<T>();
#pragma unroll
        for (int k = 0; k < kScanItems; k++) {
            uint64_t i = t0 + threadIdx.x * kScanItems + k;
            v[k] = i < hi ? load(i) : Op::template identity<T>();
            run = op(run, v[k]);
        }
        T total;
        T incl = block_inclusive<T, Op>(run, op, sw, &total);
        // exclusive prefix of this thread's first item within the block: the previous lane's
        // inclusive prefix, or the previous warp's total for lane 0
        T prev = __shfl_up_sync(0xffffffffu, incl, 1);
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        T before;
        if (lane > 0)
            before = prev;
        else
            before = warp > 0 ? sw[warp - 1] : Op::template identity<T>();
        T e = op(carry, before);
#pragma unroll
        for (int k = 0; k < kScanItems; k++) {
            uint64_t i = t0 + threadIdx.x * kScanItems + k;
            T inc_k = op(e, v[k]);
            if (i < hi) store(i, e, inc_k);
            e = inc_k;
        }
        carry = op(carry, total);
        __syncthreads();
    }
}

// Convenience driver. temp must hold kScanBlocks elements of T.
template <class T, class Op, class Load, class Store>
void device_scan(Load load, Store store, const uint32_t* d_n, uint64_t n_host, T* temp, T* d_total,
                 cudaStream_t st) {
    k_scan_reduce<T, Op, Load><<<kScanBlocks, kScanThreads, 0, st>>>(load, d_n, n_host, temp);
    k_scan_top<T, Op><<<1, 1024, 0, st>>>(temp, kScanBlocks, d_total);
    k_scan_down<T, Op, Load, Store><<<kScanBlocks, kScanThreads, 0, st>>>(load, store, d_n, n_host, temp);
}

}  // namespace issl
