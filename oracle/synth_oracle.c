/*
 * Seeded synthetic workloads on the CPU -- TEST AND BENCHMARK INFRASTRUCTURE ONLY.
 *
 * A restatement, for the host, of the library's device generator (issl_synth): the same
 * counter-based splitmix64 draws per (seed, stream, counter), the same site pool (i.i.d. GC 41%
 * sites plus repeat-seed copies with Poisson substitutions), the same first-occurrence dedup, the
 * same occurrence counts and query classes and the same query shuffle. It lets the reference's
 * own binaries be timed on an index that no code of the library produced: ora_synth_write()
 * writes the index as a .issl file with the reference builder's layout (ISSLCreateIndex.cpp
 * :428-484; every slice's lists bucketed in ascending site id order, :450-484), slice by slice,
 * so the whole index is never held in memory.
 *
 * The only floating-point steps are the Poisson and geometric inverse CDFs (exp, log1p, log);
 * the host's libm and the device's may round those differently in the last place, which can
 * change a draw only when a uniform variate lies within an ulp of a CDF step.
 */
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "issl_oracle.h"

static inline uint64_t mix64(uint64_t z) {
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
static inline uint64_t draw(uint64_t seed, uint64_t stream, uint64_t i) {
    return mix64(mix64(seed * 0x100000001B3ull + stream * 0x9E3779B1ull) + i * 0xD1B54A32D192ED03ull);
}
static inline double unif(uint64_t h) { return (double)(h >> 11) * (1.0 / 9007199254740992.0); }
static inline uint64_t gc41(double u) { return u < 0.295 ? 0u : u < 0.5 ? 1u : u < 0.705 ? 2u : 3u; }

static uint64_t random_site(uint64_t seed, uint64_t stream, uint64_t i) {
    uint64_t s = 0;
    for (int j = 0; j < 20; j++) s |= gc41(unif(draw(seed, stream, i * 32 + j))) << (2 * j);
    return s;
}

static uint64_t mutate(uint64_t sig, int k, uint64_t seed, uint64_t stream, uint64_t i) {
    uint32_t used = 0;
    uint64_t c = 0;
    for (int t = 0; t < k; t++) {
        int p = (int)(draw(seed, stream, i * 64 + c++) % 20);
        for (int tries = 0; ((used >> p) & 1u) && tries < 256; tries++) p = (int)(draw(seed, stream, i * 64 + c++) % 20);
        while ((used >> p) & 1u) p = (p + 1) % 20;
        used |= 1u << p;
        const uint64_t b = (sig >> (2 * p)) & 3u;
        const uint64_t nb = (b + 1 + draw(seed, stream + 1, i * 64 + t) % 3) & 3u;
        sig = (sig & ~(3ull << (2 * p))) | (nb << (2 * p));
    }
    return sig;
}

static int poisson(double lam, double u) {
    double p = exp(-lam), c = p;
    int k = 0;
    while (u > c && k < 20) {
        k++;
        p *= lam / k;
        c += p;
    }
    return k;
}

enum { kStSeed = 1, kStRepPick = 3, kStRepSubs = 4, kStRepMut = 5, kStIid = 8, kStOcc = 10, kStQPick = 11,
       kStQSubs = 12, kStQMut = 13, kStQRand = 15, kStQRep = 16, kStQRepMut = 17, kStShuffle = 19 };

/* Parallel stable LSD radix sort of (key, index) pairs on the low `bits` bits of the keys. */
static int radix_pairs(uint64_t* keys, uint32_t* idx, uint64_t n, int bits) {
    uint64_t* k2 = malloc(8 * (n ? n : 1));
    uint32_t* i2 = malloc(4 * (n ? n : 1));
    if (!k2 || !i2) {
        free(k2);
        free(i2);
        return -1;
    }
    const int T = omp_get_max_threads();
    uint64_t* hist = calloc((size_t)T * 256, 8);
    uint64_t *ka = keys, *kb = k2;
    uint32_t *ia = idx, *ib = i2;
    for (int shift = 0; shift < bits; shift += 8) {
        memset(hist, 0, (size_t)T * 256 * 8);
#pragma omp parallel num_threads(T)
        {
            const int t = omp_get_thread_num();
            const uint64_t lo = n * t / T, hi = n * (t + 1) / T;
            uint64_t* h = hist + (size_t)t * 256;
            for (uint64_t i = lo; i < hi; i++) h[(ka[i] >> shift) & 255u]++;
#pragma omp barrier
#pragma omp single
            {
                uint64_t acc = 0;
                for (int d = 0; d < 256; d++)
                    for (int u = 0; u < T; u++) {
                        const uint64_t c = hist[(size_t)u * 256 + d];
                        hist[(size_t)u * 256 + d] = acc;
                        acc += c;
                    }
            }
            for (uint64_t i = lo; i < hi; i++) {
                const uint64_t pos = h[(ka[i] >> shift) & 255u]++;
                kb[pos] = ka[i];
                ib[pos] = ia[i];
            }
        }
        uint64_t* tk = ka;
        ka = kb;
        kb = tk;
        uint32_t* ti = ia;
        ia = ib;
        ib = ti;
    }
    if (ka != keys) {
        memcpy(keys, ka, 8 * n);
        memcpy(idx, ia, 4 * n);
    }
    free(hist);
    free(k2);
    free(i2);
    return 0;
}

/* First `limit` distinct values of in[0, n) in first-occurrence order; returns how many. */
static uint64_t dedup_first(const uint64_t* in, uint64_t n, uint64_t* out, uint64_t limit) {
    uint64_t* k = malloc(8 * (n ? n : 1));
    uint32_t* ix = malloc(4 * (n ? n : 1));
    uint8_t* keep = malloc(n ? n : 1);
    if (!k || !ix || !keep) {
        free(k);
        free(ix);
        free(keep);
        return 0;
    }
#pragma omp parallel for
    for (uint64_t i = 0; i < n; i++) {
        k[i] = in[i];
        ix[i] = (uint32_t)i;
    }
    radix_pairs(k, ix, n, 40);
#pragma omp parallel for
    for (uint64_t i = 0; i < n; i++) keep[ix[i]] = (i == 0 || k[i] != k[i - 1]) ? 1 : 0;
    uint64_t got = 0;
    for (uint64_t i = 0; i < n && got < limit; i++)
        if (keep[i]) out[got++] = in[i];
    free(k);
    free(ix);
    free(keep);
    return got;
}

int ora_synth(uint64_t seed, uint64_t n_sites, double repeat_frac, uint64_t n_repeat_seeds, double repeat_lambda,
              uint64_t n_queries, double copied_frac, double repeat_query_frac, int planted_into_sites,
              uint64_t* sites, uint32_t* occ, uint64_t* queries) {
    const uint64_t N = n_sites, Q = n_queries;
    const uint64_t n_seeds = n_repeat_seeds > 0 ? n_repeat_seeds : 1;
    const uint64_t n_rep = (uint64_t)llround((double)N * repeat_frac);
    const uint64_t n_copied = (uint64_t)llround((double)Q * copied_frac);
    const uint64_t n_repq = (uint64_t)llround((double)Q * repeat_query_frac);
    const uint64_t extra = n_rep / 2 + N / 64 + 4096;
    const uint64_t n_pool = N + extra;
    uint64_t* seeds = malloc(8 * n_seeds);
    uint64_t* pool = malloc(8 * n_pool);
    uint64_t* qbuf = malloc(8 * (Q ? Q : 1));
    if (!seeds || !pool || !qbuf) return -1;
    for (uint64_t i = 0; i < n_seeds; i++) seeds[i] = random_site(seed, kStSeed, i);
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < n_pool; i++) {
        if (i < n_rep) {
            const uint64_t src = seeds[draw(seed, kStRepPick, i) % n_seeds];
            pool[i] = mutate(src, poisson(repeat_lambda, unif(draw(seed, kStRepSubs, i))), seed, kStRepMut, i);
        } else {
            pool[i] = random_site(seed, kStIid, i);
        }
    }
    uint64_t got;
    if (planted_into_sites && n_copied) {
        const uint64_t base_n = N - (n_copied < N / 2 ? n_copied : N / 2);
        got = dedup_first(pool, n_pool, sites, base_n);
        if (got != base_n) return -2;
        uint64_t* pool2 = malloc(8 * (base_n + n_copied + n_pool));
        if (!pool2) return -1;
        memcpy(pool2, sites, 8 * base_n);
        for (uint64_t i = 0; i < n_copied; i++) {
            const uint64_t src = sites[draw(seed, kStQPick, i) % base_n];
            qbuf[i] = src;
            pool2[base_n + i] = mutate(src, (int)(draw(seed, kStQSubs, i) % 5), seed, kStQMut, i);
        }
        memcpy(pool2 + base_n + n_copied, pool, 8 * n_pool);
        got = dedup_first(pool2, base_n + n_copied + n_pool, sites, N);
        free(pool2);
    } else {
        got = dedup_first(pool, n_pool, sites, N);
        for (uint64_t i = 0; i < n_copied; i++) {
            const uint64_t src = sites[draw(seed, kStQPick, i) % N];
            qbuf[i] = mutate(src, (int)(draw(seed, kStQSubs, i) % 5), seed, kStQMut, i);
        }
    }
    if (got != N) return -2;
    for (uint64_t i = 0; i + n_copied < Q; i++) {
        if (i < n_repq) {
            const uint64_t src = seeds[draw(seed, kStQRep, i) % n_seeds];
            qbuf[n_copied + i] = mutate(src, (int)(draw(seed, kStQRep + 100, i) % 3), seed, kStQRepMut, i);
        } else {
            qbuf[n_copied + i] = random_site(seed, kStQRand, i);
        }
    }
    /* the query classes shuffled together: stable order of 64-bit random keys */
    if (Q > 1) {
        uint64_t* k = malloc(8 * Q);
        uint32_t* ix = malloc(4 * Q);
        for (uint64_t i = 0; i < Q; i++) {
            k[i] = draw(seed, kStShuffle, i);
            ix[i] = (uint32_t)i;
        }
        radix_pairs(k, ix, Q, 64);
        for (uint64_t i = 0; i < Q; i++) queries[i] = qbuf[ix[i]];
        free(k);
        free(ix);
    } else if (Q == 1) {
        queries[0] = qbuf[0];
    }
#pragma omp parallel for schedule(static)
    for (uint64_t i = 0; i < N; i++) {
        const double u = unif(draw(seed, kStOcc, i));
        const double fails = floor(log1p(-u) / log(0.1));
        occ[i] = (uint32_t)fmin(1.0 + fails, 255.0);
    }
    free(seeds);
    free(pool);
    free(qbuf);
    return 0;
}

static int mask_width(uint64_t mask, uint64_t seq_len, uint64_t* pos) {
    int w = 0;
    for (uint64_t j = 0; j < seq_len; j++)
        if (mask & (1ULL << j)) pos[w++] = j;
    return w;
}

int ora_write_built(const char* path, const uint64_t* sigs, const uint32_t* occ, uint64_t n_sites,
                    const uint64_t* slice_masks, uint64_t n_slices) {
    FILE* fp = fopen(path, "wb");
    if (!fp) return -1;
    const uint64_t N = n_sites, seq_len = 20;
    uint64_t hdr[3] = {N, seq_len, n_slices};
    int bad = fwrite(hdr, 8, 3, fp) != 3;
    bad |= fwrite(sigs, 8, N, fp) != N;
    bad |= fwrite(slice_masks, 8, n_slices, fp) != n_slices;
    const int T = omp_get_max_threads();
    uint32_t* keys = malloc(4 * (N ? N : 1));
    uint64_t* lists = malloc(8 * (N ? N : 1));
    for (uint64_t s = 0; s < n_slices && !bad; s++) {
        uint64_t pos[64];
        const int w = mask_width(slice_masks[s], seq_len, pos);
        const uint64_t nb = 1ULL << (2 * w);
        uint64_t* hist = calloc((size_t)T * nb, 8);
        uint64_t* sizes = calloc(nb, 8);
        if (!keys || !lists || !hist || !sizes) {
            bad = 1;
            free(hist);
            free(sizes);
            break;
        }
#pragma omp parallel num_threads(T)
        {
            const int t = omp_get_thread_num();
            const uint64_t lo = N * t / T, hi = N * (t + 1) / T;
            uint64_t* h = hist + (size_t)t * nb;
            for (uint64_t id = lo; id < hi; id++) {
                uint64_t key = 0;
                for (int j = 0; j < w; j++) key |= ((sigs[id] >> (pos[j] * 2)) & 3ULL) << (j * 2);
                keys[id] = (uint32_t)key;
                h[key]++;
            }
#pragma omp barrier
#pragma omp single
            {
                /* bucket b: threads' ids in ascending order, so each bucket lists ids ascending */
                uint64_t acc = 0;
                for (uint64_t b = 0; b < nb; b++) {
                    const uint64_t start = acc;
                    for (int u = 0; u < T; u++) {
                        const uint64_t c = hist[(size_t)u * nb + b];
                        hist[(size_t)u * nb + b] = acc;
                        acc += c;
                    }
                    sizes[b] = acc - start;
                }
            }
            for (uint64_t id = lo; id < hi; id++) lists[h[keys[id]]++] = ((uint64_t)occ[id] << 32) | id;
        }
        bad |= fwrite(sizes, 8, nb, fp) != nb;
        bad |= fwrite(lists, 8, N, fp) != N;
        free(hist);
        free(sizes);
    }
    free(keys);
    free(lists);
    bad |= fclose(fp) != 0;
    return bad ? -2 : 0;
}
