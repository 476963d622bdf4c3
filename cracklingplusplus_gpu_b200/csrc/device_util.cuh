// Bit manipulation shared by the index builder and the scoring kernels.
#pragma once
#include <cstdint>

#include "issl_internal.cuh"

namespace issl {

// Slice key of a signature: the 2-bit bases at the slice positions, packed in ascending
// position order (ISSLScoringModule.cpp:235-239, ISSLCreateIndex.cpp:458-462).
__host__ __device__ __forceinline__ uint32_t slice_key(uint64_t sig, const SliceGeom& g) {
    uint32_t key = 0;
    for (int j = 0; j < g.width; j++) key |= static_cast<uint32_t>((sig >> (2 * g.pos[j])) & 3u) << (2 * j);
    return key;
}

// Residual code: the bases outside the slice packed the same way (at most 32 bits for
// slices of width >= 4).
__host__ __device__ __forceinline__ uint32_t slice_residual(uint64_t sig, const SliceGeom& g) {
    uint32_t r = 0;
    for (int j = 0; j < g.rwidth; j++) r |= static_cast<uint32_t>((sig >> (2 * g.rpos[j])) & 3u) << (2 * j);
    return r;
}

// Signature of a site in the bucket of guide q for slice g, from its residual code: the slice
// positions carry the guide's bases (that is what the bucket key means), the others the code.
__host__ __device__ __forceinline__ uint64_t site_signature(uint64_t q, uint32_t rcode, const SliceGeom& g) {
    uint64_t sig = 0;
    for (int j = 0; j < g.width; j++) sig |= q & (3ull << (2 * g.pos[j]));
    for (int j = 0; j < g.rwidth; j++) sig |= static_cast<uint64_t>((rcode >> (2 * j)) & 3u) << (2 * g.rpos[j]);
    return sig;
}

// Site of list position `pos` of slice s, found in the bucket of guide q: id, occurrences and
// signature. 8-byte entries (packed id, residual code) give everything in one read; 4-byte
// entries need the signature table too.
__device__ __forceinline__ void load_site(const IndexView& v, uint32_t s, uint32_t pos, uint64_t q, const SliceGeom& g,
                                          uint32_t& id, uint32_t& occ, uint64_t& sig) {
    const uint64_t j = static_cast<uint64_t>(s) * v.n_sites + pos - v.ids_base;
    if (v.entry_words == 2) {
        const uint2 e = reinterpret_cast<const uint2*>(v.ids)[j];
        id = entry_id(e.x, v.id_bits);
        occ = entry_occ(e.x, v);
        sig = site_signature(q, e.y, g);
    } else {
        const uint32_t e = v.ids[j];
        id = entry_id(e, v.id_bits);
        occ = entry_occ(e, v);
        sig = v.sigs[id];
    }
}

// The raw list entry of list position `pos` of slice s: the packed id (x) and, with 8-byte entries,
// the residual code (y; 0 with 4-byte entries).
__device__ __forceinline__ uint2 load_entry(const IndexView& v, uint32_t s, uint32_t pos) {
    const uint64_t j = static_cast<uint64_t>(s) * v.n_sites + pos - v.ids_base;
    if (v.entry_words == 2) return reinterpret_cast<const uint2*>(v.ids)[j];
    return make_uint2(v.ids[j], 0u);
}

// One bit per mismatching base pair, at the even bit of each 2-bit field. Equivalent to
// ((x & 0xAA..) >> 1) | (x & 0x55..) of ISSLScoringModule.cpp:287-289.
__host__ __device__ __forceinline__ uint64_t fold64(uint64_t x) {
    return (x | (x >> 1)) & 0x5555555555555555ull;
}
__host__ __device__ __forceinline__ uint32_t fold32(uint32_t x) { return (x | (x >> 1)) & 0x55555555u; }

// 32-bit even-bit mask -> 16-bit position mask.
__host__ __device__ __forceinline__ uint32_t compress_even32(uint32_t m) {
    m &= 0x55555555u;
    m = (m | (m >> 1)) & 0x33333333u;
    m = (m | (m >> 2)) & 0x0F0F0F0Fu;
    m = (m | (m >> 4)) & 0x00FF00FFu;
    m = (m | (m >> 8)) & 0x0000FFFFu;
    return m;
}

// 40-bit even-bit mismatch mask -> 20-bit position mask.
__host__ __device__ __forceinline__ uint32_t compress_even40(uint64_t m) {
    m &= 0x5555555555555555ull;
    m = (m | (m >> 1)) & 0x3333333333333333ull;
    m = (m | (m >> 2)) & 0x0F0F0F0F0F0F0F0Full;
    m = (m | (m >> 4)) & 0x00FF00FF00FF00FFull;
    m = (m | (m >> 8)) & 0x0000FFFF0000FFFFull;
    m = (m | (m >> 16)) & 0x00000000FFFFFFFFull;
    return static_cast<uint32_t>(m);
}

}  // namespace issl
