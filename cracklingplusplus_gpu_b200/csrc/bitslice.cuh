// Bit-sliced mismatch counting: 32 entries per lane at once.
//
// d[2p], d[2p+1] are the low / high bit planes of residual position p for the 32 entries of a
// block; q[2p], q[2p+1] are the guide's bits at that position spread to whole words (0 or ~0).
// Position p mismatches for entry e iff bit e of (d[2p] ^ q[2p]) | (d[2p+1] ^ q[2p+1]) is set.
// The per-entry mismatch counts are then summed as bit-sliced binary numbers with full adders
// (carry-save), and the result is compared with the distance bound. Everything is 32-bit
// logic (LOP3-friendly): about 2 operations per position plus ~2 per position for the adder tree.
#pragma once
#include <cstdint>

namespace issl {
namespace bs {

struct Count {  // bit-sliced count: c0 + 2 c1 + 4 c2, c3 = "8 or more"
    uint32_t c0, c1, c2, c3;
};

__device__ __forceinline__ void fa(uint32_t a, uint32_t b, uint32_t c, uint32_t& s, uint32_t& cy) {
    s = a ^ b ^ c;
    cy = (a & b) | (c & (a ^ b));
}
__device__ __forceinline__ void ha(uint32_t a, uint32_t b, uint32_t& s, uint32_t& cy) {
    s = a ^ b;
    cy = a & b;
}

// Wallace-style reductions for the slice widths in use (12, 10 and 16 residual positions).
__device__ __forceinline__ Count count12(const uint32_t* m) {
    uint32_t s0, s1, s2, s3, k0, k1, k2, k3, t0, j0, j1, u0, u1, l0, l1, l2;
    Count c;
    fa(m[0], m[1], m[2], s0, k0);
    fa(m[3], m[4], m[5], s1, k1);
    fa(m[6], m[7], m[8], s2, k2);
    fa(m[9], m[10], m[11], s3, k3);
    fa(s0, s1, s2, t0, j0);
    ha(t0, s3, c.c0, j1);
    fa(k0, k1, k2, u0, l0);
    fa(k3, j0, j1, u1, l1);
    ha(u0, u1, c.c1, l2);
    fa(l0, l1, l2, c.c2, c.c3);
    return c;
}

__device__ __forceinline__ Count count10(const uint32_t* m) {
    uint32_t s0, s1, s2, k0, k1, k2, t0, j0, j1, u0, l0, l1;
    Count c;
    fa(m[0], m[1], m[2], s0, k0);
    fa(m[3], m[4], m[5], s1, k1);
    fa(m[6], m[7], m[8], s2, k2);
    fa(s0, s1, s2, t0, j0);
    ha(t0, m[9], c.c0, j1);
    fa(k0, k1, k2, u0, l0);
    fa(u0, j0, j1, c.c1, l1);
    ha(l0, l1, c.c2, c.c3);
    return c;
}

__device__ __forceinline__ Count count16(const uint32_t* m) {
    uint32_t s[5], k[5], t0, t1, j0, j1, j2, u0, u1, u2, l0, l1, l2, l3, v0, z0, z1;
    Count c;
#pragma unroll
    for (int i = 0; i < 5; i++) fa(m[3 * i], m[3 * i + 1], m[3 * i + 2], s[i], k[i]);
    fa(s[0], s[1], s[2], t0, j0);
    fa(s[3], s[4], m[15], t1, j1);
    ha(t0, t1, c.c0, j2);
    fa(k[0], k[1], k[2], u0, l0);
    fa(k[3], k[4], j0, u1, l1);
    ha(j1, j2, u2, l2);
    fa(u0, u1, u2, c.c1, l3);
    fa(l0, l1, l2, v0, z0);
    ha(v0, l3, c.c2, z1);
    c.c3 = z0 | z1;
    return c;
}

// any number of positions: ripple-add each mismatch word into a saturating counter
template <int N>
__device__ __forceinline__ Count count_generic(const uint32_t* m) {
    Count c{0, 0, 0, 0};
#pragma unroll
    for (int i = 0; i < N; i++) {
        const uint32_t k0 = c.c0 & m[i];
        c.c0 ^= m[i];
        const uint32_t k1 = c.c1 & k0;
        c.c1 ^= k0;
        const uint32_t k2 = c.c2 & k1;
        c.c2 ^= k1;
        c.c3 |= k2;
    }
    return c;
}

template <int N>
__device__ __forceinline__ Count count_mismatches(const uint32_t* m) {
    if constexpr (N == 12) return count12(m);
    else if constexpr (N == 10) return count10(m);
    else if constexpr (N == 16) return count16(m);
    else return count_generic<N>(m);
}

// entries whose count is <= max_dist (0..4)
__device__ __forceinline__ uint32_t within(const Count& c, int max_dist) {
    switch (max_dist) {
        case 4: return ~c.c3 & ~(c.c2 & (c.c1 | c.c0));
        case 3: return ~(c.c3 | c.c2);
        case 2: return ~(c.c3 | c.c2) & ~(c.c1 & c.c0);
        case 1: return ~(c.c3 | c.c2 | c.c1);
        default: return ~(c.c3 | c.c2 | c.c1 | c.c0);
    }
}

}  // namespace bs
}  // namespace issl
