/*
 * CPU oracle for ISSL off-target scoring -- TEST INFRASTRUCTURE ONLY (see issl_oracle.h).
 * Compiled with -ffp-contract=off so every double operation happens in the order the
 * reference writes it. Nothing in the shipped library links or calls this file.
 */
#include "issl_oracle.h"

#include <omp.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------ */
/* Encoding: lib/ISSLScoringModule.cpp:10 (nucleotideIndex) and :469-476.                 */
/* The reference table has 85 entries (ASCII 0..84): 'C'=67 -> 1, 'G'=71 -> 2, 'T'=84 -> 3,
 * every other index -> 0. Characters above 84 index past the end of the reference table
 * (undefined behaviour there); here they encode as 0 like every other non-CGT character. */
static inline uint64_t nuc2bit(unsigned char c) {
    return c == 'C' ? 1u : c == 'G' ? 2u : c == 'T' ? 3u : 0u;
}

uint64_t ora_encode(const char* seq, uint64_t len) {
    uint64_t sig = 0;
    for (uint64_t j = 0; j < len; j++) sig |= nuc2bit((unsigned char)seq[j]) << (j * 2);
    return sig;
}

/* ------------------------------------------------------------------------------------ */
/* MIT local score: ISSLCreateIndex/ISSLCreateIndex.cpp:235-261.                           */
static const double kMitM[20] = {0.0,   0.0,   0.014, 0.0,   0.0,   0.395, 0.317,
                                 0.0,   0.389, 0.079, 0.445, 0.508, 0.613, 0.851,
                                 0.732, 0.828, 0.615, 0.804, 0.685, 0.583};

double ora_mit_local_score(const uint64_t* pos, uint64_t length) {
    double t1 = 1.0, t2, t3, d = 0.0;
    for (uint64_t i = 0; i < length; ++i) t1 = t1 * (1.0 - kMitM[pos[i]]);
    if (length == 1) {
        d = 19.0;
    } else {
        for (uint64_t i = 0; i < length - 1; ++i) d += (double)(pos[i + 1] - pos[i]);
        d = d / (double)(length - 1);
    }
    t2 = 1.0 / ((19.0 - d) / 19.0 * 4.0 + 1);
    t3 = 1.0 / (double)(length * length);
    return t1 * t2 * t3 * 100;
}

/* 2^20-entry table indexed by the 20-bit mismatch-position mask; NaN marks masks that the
 * reference map does not hold (more than four mismatches, or none). */
static double* g_mit20 = NULL;

static void build_mit20(void) {
    if (g_mit20) return;
    double* t = (double*)malloc(sizeof(double) << 20);
    for (uint32_t m = 0; m < (1u << 20); m++) {
        int k = __builtin_popcount(m);
        if (k < 1 || k > 4) {
            t[m] = __builtin_nan("");
            continue;
        }
        uint64_t p[4];
        int n = 0;
        for (uint64_t j = 0; j < 20; j++)
            if (m >> j & 1) p[n++] = j;
        t[m] = ora_mit_local_score(p, (uint64_t)n);
    }
    g_mit20 = t;
}

/* Mismatch mask with bits at even positions 2p (ISSLScoringModule.cpp:286-289) -> 20-bit
 * position mask. */
static inline uint32_t compress_even(uint64_t mism) {
    uint32_t m = 0;
    for (int p = 0; p < 20; p++) m |= (uint32_t)((mism >> (2 * p)) & 1u) << p;
    return m;
}

int ora_mit_table(uint64_t* masks_out, double* scores_out) {
    build_mit20();
    /* ascending order of the 64-bit mask equals ascending order of the 20-bit mask */
    int n = 0;
    for (uint32_t m = 0; m < (1u << 20); m++) {
        if (g_mit20[m] != g_mit20[m]) continue;
        if (masks_out) {
            uint64_t wide = 0;
            for (int p = 0; p < 20; p++) wide |= (uint64_t)((m >> p) & 1u) << (2 * p);
            masks_out[n] = wide;
        }
        if (scores_out) scores_out[n] = g_mit20[m];
        n++;
    }
    return n;
}

/* ------------------------------------------------------------------------------------ */
/* CFD tables (lib/otScorePenalties.cpp:6201-6546), installed by the caller.              */
static double g_cfd_pos[320];
static double g_cfd_pam[16];
static int g_cfd_set = 0;

void ora_set_cfd_tables(const double* pos320, const double* pam16) {
    memcpy(g_cfd_pos, pos320, sizeof g_cfd_pos);
    memcpy(g_cfd_pam, pam16, sizeof g_cfd_pam);
    g_cfd_set = 1;
}

/* CFD of one site, lib/ISSLScoringModule.cpp:308-361. */
static inline double cfd_score(uint64_t q, uint64_t sig, uint64_t dist) {
    if (dist == 0) return 1;
    double s = g_cfd_pam[0xA]; /* PAM NGG, :313 */
    for (uint64_t pos = 0; pos < 20; pos++) {
        uint64_t mask = pos << 4;
        uint64_t qi = ((q >> (pos * 2)) & 3ULL) << 2;
        uint64_t oi = (sig >> (pos * 2)) & 3ULL;
        mask = mask | qi | (oi ^ 3ULL);
        if (qi >> 2 != oi) s *= g_cfd_pos[mask];
    }
    return s;
}

/* ------------------------------------------------------------------------------------ */
/* Loader: lib/ISSLScoringModule.cpp:72-150.                                              */
static int read_exact(FILE* fp, void* dst, size_t sz, size_t n) {
    return fread(dst, sz, n, fp) == n ? 0 : -1;
}

int ora_load(const char* path, ora_index* out) {
    memset(out, 0, sizeof *out);
    FILE* fp = fopen(path, "rb");
    if (!fp) return -1;
    uint64_t hdr[3];
    if (read_exact(fp, hdr, 8, 3)) goto fail;
    out->n_sites = hdr[0];
    out->seq_len = hdr[1];
    out->n_slices = hdr[2];
    out->owns_memory = 1;
    out->sigs = (uint64_t*)malloc(8 * (out->n_sites ? out->n_sites : 1));
    out->slice_masks = (uint64_t*)malloc(8 * (out->n_slices ? out->n_slices : 1));
    if (out->n_sites && read_exact(fp, out->sigs, 8, out->n_sites)) goto fail;
    if (out->n_slices && read_exact(fp, out->slice_masks, 8, out->n_slices)) goto fail;
    uint64_t total = 0;
    for (uint64_t s = 0; s < out->n_slices; s++) {
        uint64_t w = (uint64_t)__builtin_popcountll(out->slice_masks[s] &
                                                    ((out->seq_len >= 64) ? ~0ULL : ((1ULL << out->seq_len) - 1)));
        total += 1ULL << (2 * w);
    }
    out->list_sizes = (uint64_t*)malloc(8 * (total ? total : 1));
    uint64_t n_entries = out->n_sites * out->n_slices;
    out->lists = (uint64_t*)malloc(8 * (n_entries ? n_entries : 1));
    uint64_t off = 0;
    for (uint64_t s = 0; s < out->n_slices; s++) {
        uint64_t w = (uint64_t)__builtin_popcountll(out->slice_masks[s] &
                                                    ((out->seq_len >= 64) ? ~0ULL : ((1ULL << out->seq_len) - 1)));
        uint64_t nb = 1ULL << (2 * w);
        if (read_exact(fp, out->list_sizes + off, 8, nb)) goto fail;
        if (out->n_sites && read_exact(fp, out->lists + s * out->n_sites, 8, out->n_sites)) goto fail;
        off += nb;
    }
    fclose(fp);
    return 0;
fail:
    fclose(fp);
    ora_free(out);
    return -2;
}

void ora_free(ora_index* idx) {
    if (idx->owns_memory) {
        free(idx->sigs);
        free(idx->slice_masks);
        free(idx->list_sizes);
        free(idx->lists);
    }
    memset(idx, 0, sizeof *idx);
}

/* ------------------------------------------------------------------------------------ */
/* Builder: ISSLCreateIndex/ISSLCreateIndex.cpp:450-484.                                  */
static int mask_positions(uint64_t mask, uint64_t seq_len, uint64_t* pos) {
    int w = 0;
    for (uint64_t j = 0; j < seq_len; j++)
        if (mask & (1ULL << j)) pos[w++] = j;
    return w;
}

int ora_build(const uint64_t* sigs, const uint32_t* occ, uint64_t n_sites,
              const uint64_t* slice_masks, uint64_t n_slices, uint64_t seq_len, ora_index* out) {
    memset(out, 0, sizeof *out);
    out->n_sites = n_sites;
    out->seq_len = seq_len;
    out->n_slices = n_slices;
    out->owns_memory = 1;
    out->sigs = (uint64_t*)malloc(8 * (n_sites ? n_sites : 1));
    memcpy(out->sigs, sigs, 8 * n_sites);
    out->slice_masks = (uint64_t*)malloc(8 * (n_slices ? n_slices : 1));
    memcpy(out->slice_masks, slice_masks, 8 * n_slices);
    uint64_t total = 0;
    uint64_t pos[64];
    for (uint64_t s = 0; s < n_slices; s++) total += 1ULL << (2 * mask_positions(slice_masks[s], seq_len, pos));
    out->list_sizes = (uint64_t*)calloc(total ? total : 1, 8);
    uint64_t n_entries = n_sites * n_slices;
    out->lists = (uint64_t*)malloc(8 * (n_entries ? n_entries : 1));
    uint64_t base = 0;
    for (uint64_t s = 0; s < n_slices; s++) {
        int w = mask_positions(slice_masks[s], seq_len, pos);
        uint64_t nb = 1ULL << (2 * w);
        uint64_t* sizes = out->list_sizes + base;
        uint64_t* keys = (uint64_t*)malloc(8 * (n_sites ? n_sites : 1));
        for (uint64_t id = 0; id < n_sites; id++) {
            uint64_t key = 0;
            for (int j = 0; j < w; j++) key |= ((sigs[id] >> (pos[j] * 2)) & 3ULL) << (j * 2);
            keys[id] = key;
            sizes[key]++;
        }
        uint64_t* cursor = (uint64_t*)malloc(8 * nb);
        uint64_t acc = 0;
        for (uint64_t b = 0; b < nb; b++) {
            cursor[b] = acc;
            acc += sizes[b];
        }
        uint64_t* dst = out->lists + s * n_sites;
        for (uint64_t id = 0; id < n_sites; id++)
            dst[cursor[keys[id]]++] = ((uint64_t)occ[id] << 32) | id;
        free(cursor);
        free(keys);
        base += nb;
    }
    return 0;
}

int ora_write(const char* path, const ora_index* idx) {
    FILE* fp = fopen(path, "wb");
    if (!fp) return -1;
    uint64_t hdr[3] = {idx->n_sites, idx->seq_len, idx->n_slices};
    int bad = fwrite(hdr, 8, 3, fp) != 3;
    bad |= fwrite(idx->sigs, 8, idx->n_sites, fp) != idx->n_sites;
    bad |= fwrite(idx->slice_masks, 8, idx->n_slices, fp) != idx->n_slices;
    uint64_t base = 0, pos[64];
    for (uint64_t s = 0; s < idx->n_slices; s++) {
        uint64_t nb = 1ULL << (2 * mask_positions(idx->slice_masks[s], idx->seq_len, pos));
        bad |= fwrite(idx->list_sizes + base, 8, nb, fp) != nb;
        bad |= fwrite(idx->lists + s * idx->n_sites, 8, idx->n_sites, fp) != idx->n_sites;
        base += nb;
    }
    bad |= fclose(fp) != 0;
    return bad ? -2 : 0;
}

/* ------------------------------------------------------------------------------------ */
/* Scoring: lib/ISSLScoringModule.cpp:154-462; count/distinct: ISSLScoreOfftargets.cpp. */
int ora_score(const ora_index* idx, const uint64_t* qsigs, uint64_t nq, int method,
              double threshold, int max_dist, int threads, double* tot_mit, double* tot_cfd,
              uint64_t* count, uint64_t* distinct) {
    build_mit20();
    const int calc_mit = method == ORA_MIT || method == ORA_AND || method == ORA_OR || method == ORA_AVG;
    const int calc_cfd = method == ORA_CFD || method == ORA_AND || method == ORA_OR || method == ORA_AVG;
    const uint64_t N = idx->n_sites, S = idx->n_slices;
    /* slice positions and per-slice bucket base, :100-122 and :181-198 */
    uint64_t(*pos)[64] = malloc(sizeof(uint64_t[64]) * (S ? S : 1));
    int* width = malloc(sizeof(int) * (S ? S : 1));
    uint64_t* size_base = malloc(8 * (S ? S : 1));
    uint64_t** list_start = malloc(sizeof(uint64_t*) * (S ? S : 1));
    uint64_t acc = 0;
    for (uint64_t s = 0; s < S; s++) {
        width[s] = mask_positions(idx->slice_masks[s], idx->seq_len, pos[s]);
        size_base[s] = acc;
        acc += 1ULL << (2 * width[s]);
    }
    /* prefix offsets per bucket so sliceLists[s][key] is O(1), :188-198 */
    uint64_t* bucket_off = malloc(8 * (acc ? acc : 1));
    for (uint64_t s = 0; s < S; s++) {
        uint64_t nb = 1ULL << (2 * width[s]);
        uint64_t o = 0;
        for (uint64_t b = 0; b < nb; b++) {
            bucket_off[size_base[s] + b] = o;
            o += idx->list_sizes[size_base[s] + b];
        }
        list_start[s] = idx->lists + s * N;
    }
    const uint64_t n_toggles = N / 64 + 1; /* :162 */
    uint64_t* seen = calloc(n_toggles, 8);  /* CLI :206 */
    const double maximum_sum = (10000.0 - threshold * 100) / threshold; /* :225 */
    int err = 0;
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel
    {
        uint64_t* toggles = calloc(n_toggles, 8);
        uint64_t* tail = toggles + n_toggles - 1; /* :209 */
#pragma omp for schedule(dynamic, 16)
        for (int64_t qi = 0; qi < (int64_t)nq; qi++) {
            const uint64_t q = qsigs[qi];
            double mit = 0.0, cfd = 0.0;
            uint64_t local_count = 0;
            int check_next = 1;
            for (uint64_t s = 0; s < S && check_next; s++) {
                uint64_t key = 0;
                for (int j = 0; j < width[s]; j++) key |= ((q >> (pos[s][j] * 2)) & 3ULL) << (j * 2);
                const uint64_t n_in = idx->list_sizes[size_base[s] + key];
                const uint64_t* lst = list_start[s] + bucket_off[size_base[s] + key];
                for (uint64_t j = 0; j < n_in; j++) {
                    const uint64_t e = lst[j];
                    const uint64_t id = e & 0xFFFFFFFFULL;
                    const uint32_t occ = (uint32_t)(e >> 32);
                    uint64_t* flag = tail - (id / 64); /* :254 */
                    if ((*flag >> (id % 64)) & 1ULL) continue;
                    *flag |= 1ULL << (id % 64);
                    const uint64_t x = q ^ idx->sigs[id];
                    const uint64_t mism = ((x & 0xAAAAAAAAAAAAAAAAULL) >> 1) | (x & 0x5555555555555555ULL);
                    const uint64_t dist = (uint64_t)__builtin_popcountll(mism);
                    if (dist > (uint64_t)max_dist) continue; /* :292 */
                    local_count += occ;                     /* CLI :371 */
                    __atomic_fetch_or(&seen[id / 64], 1ULL << (id % 64), __ATOMIC_RELAXED);
                    if (calc_mit && dist > 0) {
                        double v = g_mit20[compress_even(mism)];
                        if (v != v) {
#pragma omp atomic write
                            err = -1;
                            v = 0.0;
                        }
                        mit += v * (double)occ; /* :296 */
                    }
                    if (calc_cfd) cfd += cfd_score(q, idx->sigs[id], dist) * (double)occ; /* :362 */
                    int stop = 0; /* :366-395 */
                    if (method == ORA_AND) stop = mit > maximum_sum && cfd > maximum_sum;
                    if (method == ORA_OR) stop = mit > maximum_sum || cfd > maximum_sum;
                    if (method == ORA_AVG) stop = ((mit + cfd) / 2.0) > maximum_sum;
                    if (method == ORA_MIT) stop = mit > maximum_sum;
                    if (method == ORA_CFD) stop = cfd > maximum_sum;
                    if (stop) {
                        check_next = 0;
                        break;
                    }
                }
            }
            tot_mit[qi] = mit;
            tot_cfd[qi] = cfd;
            if (count) count[qi] = local_count;
            memset(toggles, 0, 8 * n_toggles); /* :461 */
        }
        free(toggles);
    }
    if (distinct) {
        uint64_t d = 0;
        for (uint64_t w = 0; w < n_toggles; w++) d += (uint64_t)__builtin_popcountll(seen[w]);
        *distinct = d;
    }
    free(seen);
    free(bucket_off);
    free(list_start);
    free(size_base);
    free(width);
    free(pos);
    return err;
}

/* The terms one guide's sums receive, in the order the reference adds them (slices in order,
 * each bucket in list order, sites seen in an earlier slice skipped; lib/ISSLScoringModule.cpp
 * :230-363) with no early exit: for every scored site (dist <= max_dist) its MIT term
 * (score * occurrences, 0 for an exact match, :294-298), its CFD term (:301-362) and its
 * occurrences. Returns the number of scored sites; at most cap are written. */
uint64_t ora_trace(const ora_index* idx, uint64_t q, int max_dist, double* mit_terms, double* cfd_terms,
                   uint32_t* occ_out, uint64_t cap) {
    build_mit20();
    const uint64_t N = idx->n_sites, S = idx->n_slices;
    uint64_t pos[64];
    uint64_t base = 0, n = 0;
    uint64_t* seen = calloc(N / 64 + 1, 8);
    for (uint64_t s = 0; s < S; s++) {
        const int w = mask_positions(idx->slice_masks[s], idx->seq_len, pos);
        uint64_t key = 0;
        for (int j = 0; j < w; j++) key |= ((q >> (pos[j] * 2)) & 3ULL) << (j * 2);
        uint64_t start = 0;
        for (uint64_t b = 0; b < key; b++) start += idx->list_sizes[base + b];
        const uint64_t* lst = idx->lists + s * N + start;
        for (uint64_t j = 0; j < idx->list_sizes[base + key]; j++) {
            const uint64_t id = lst[j] & 0xFFFFFFFFULL;
            const uint32_t occ = (uint32_t)(lst[j] >> 32);
            if ((seen[id / 64] >> (id % 64)) & 1ULL) continue;
            seen[id / 64] |= 1ULL << (id % 64);
            const uint64_t x = q ^ idx->sigs[id];
            const uint64_t mism = ((x & 0xAAAAAAAAAAAAAAAAULL) >> 1) | (x & 0x5555555555555555ULL);
            const uint64_t dist = (uint64_t)__builtin_popcountll(mism);
            if (dist > (uint64_t)max_dist) continue;
            if (n < cap) {
                mit_terms[n] = dist > 0 ? g_mit20[compress_even(mism)] * (double)occ : 0.0;
                cfd_terms[n] = cfd_score(q, idx->sigs[id], dist) * (double)occ;
                occ_out[n] = occ;
            }
            n++;
        }
        base += 1ULL << (2 * w);
    }
    free(seen);
    return n;
}

void ora_finalise(int method, double t, double tot_mit, double tot_cfd, double* mit_score,
                  double* cfd_score, char* code) {
    double m = 10000.0 / (100.0 + tot_mit), c = 10000.0 / (100.0 + tot_cfd);
    int reject = 0;
    switch (method) { /* :404-459 */
        case ORA_AND: reject = m < t && c < t; break;
        case ORA_OR: reject = m < t || c < t; break;
        case ORA_AVG: reject = (m + c) / 2 < t; break;
        case ORA_MIT: reject = m < t; c = -1; break;
        case ORA_CFD: reject = c < t; m = -1; break;
        default: break;
    }
    *mit_score = m;
    *cfd_score = c;
    *code = reject ? '0' : '1';
}

/* ------------------------------------------------------------------------------------ */
/* Brute force: the candidate set is every site within max_dist mismatches.               */
int ora_bruteforce(const uint64_t* sigs, const uint32_t* occ, uint64_t n_sites,
                   const uint64_t* qsigs, uint64_t nq, int max_dist, int threads,
                   double* sum_mit, double* sum_cfd, uint64_t* count) {
    build_mit20();
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 4)
    for (int64_t qi = 0; qi < (int64_t)nq; qi++) {
        const uint64_t q = qsigs[qi];
        double mit = 0.0, cfd = 0.0;
        uint64_t c = 0;
        for (uint64_t id = 0; id < n_sites; id++) {
            const uint64_t x = q ^ sigs[id];
            const uint64_t mism = ((x & 0xAAAAAAAAAAAAAAAAULL) >> 1) | (x & 0x5555555555555555ULL);
            const uint64_t dist = (uint64_t)__builtin_popcountll(mism);
            if (dist > (uint64_t)max_dist) continue;
            c += occ[id];
            if (dist > 0) mit += g_mit20[compress_even(mism)] * (double)occ[id];
            cfd += cfd_score(q, sigs[id], dist) * (double)occ[id];
        }
        sum_mit[qi] = mit;
        sum_cfd[qi] = cfd;
        count[qi] = c;
    }
    return 0;
}
