/*
 * issl_b200 -- B200-native ISSL off-target scoring behind a plain C ABI.
 *
 * The reference computes Crackling++'s specificity score on the CPU: it reads the .issl
 * index inside every ISSLScoringModule::run() call (lib/ISSLScoringModule.cpp:72-150),
 * then for each guide walks the guide's bucket in every slice, deduplicates sites with a
 * per-guide toggle bitset, and accumulates occurrence-weighted MIT and CFD penalties with
 * a threshold early exit (lib/ISSLScoringModule.cpp:206-462). This library keeps the index
 * resident in HBM across calls and runs the same computation as CUDA kernels for sm_100a.
 *
 * All entry points return an ISSL_* status (0 = success); on failure issl_last_error()
 * gives a message for the calling thread. No torch types, plain pointers and sizes only.
 */
#ifndef ISSL_B200_H
#define ISSL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes -------------------------------------------------------------------- */
#define ISSL_OK 0
#define ISSL_ERR_ARG (-1)         /* invalid argument (null pointer, bad method, size) */
#define ISSL_ERR_IO (-2)          /* file could not be opened / short read or write */
#define ISSL_ERR_FORMAT (-3)      /* malformed or unsupported .issl content */
#define ISSL_ERR_NOMEM (-4)       /* device or pinned host allocation failed */
#define ISSL_ERR_CUDA (-5)        /* CUDA runtime error (message has the CUDA text) */
#define ISSL_ERR_TIMEOUT (-6)     /* a bounded device wait gave up */
#define ISSL_ERR_UNSUPPORTED (-7) /* valid request this build does not implement */
#define ISSL_ERR_BUSY (-8)        /* admission refused: not enough device memory now */

/* ---- score methods: otScoreMethod, include/util.hpp:20 (same numbering) -------------- */
#define ISSL_METHOD_MIT 0
#define ISSL_METHOD_CFD 1
#define ISSL_METHOD_MIT_AND_CFD 2
#define ISSL_METHOD_MIT_OR_CFD 3
#define ISSL_METHOD_AVG_MIT_CFD 4

/* accept codes written per guide: CODE_ACCEPTED / CODE_REJECTED, lib/util.cpp:21-22 */
#define ISSL_CODE_ACCEPTED '1'
#define ISSL_CODE_REJECTED '0'

typedef struct issl_index issl_index;

typedef struct {
    uint64_t n_sites;         /* offtargetsCount */
    uint64_t seq_len;         /* seqLength (20) */
    uint64_t n_slices;        /* sliceCount */
    uint64_t n_buckets;       /* sum over slices of 4^width */
    uint64_t device_bytes;    /* HBM held by the resident index */
    int device;               /* CUDA ordinal holding the index */
    int min_width, max_width; /* slice widths (positions per slice) */
} issl_index_info;

/* Message for the last failing call on this thread ("" when none). */
const char* issl_last_error(void);

/* ---- index lifetime -------------------------------------------------------------------- */

/* Load a .issl file and keep it resident on `device`.
 * Replaces the per-call fread loader and bucket-pointer build of
 * lib/ISSLScoringModule.cpp:72-198 (same layout: header [N, seqLen, S], N signatures,
 * S slice masks, then per slice 4^w list sizes and N (occ<<32 | id) entries).
 * The file is streamed through pinned staging buffers; no full host copy is made. */
int issl_open(const char* path, int device, issl_index** out);

/* Same, from host arrays already in the file layout (list_sizes concatenated over slices,
 * lists = S*N entries). Used by embedders that hold the index in memory. */
int issl_open_arrays(const uint64_t* sigs, uint64_t n_sites, uint64_t seq_len,
                     const uint64_t* slice_masks, uint64_t n_slices, const uint64_t* list_sizes,
                     const uint64_t* lists, int device, issl_index** out);

/* Build the index on the GPU from distinct sites and their occurrence counts (the slice
 * bucketing of ISSLCreateIndex/ISSLCreateIndex.cpp:450-484: every site in ascending id order
 * lands in the bucket of its slice key). sigs are 2-bit packed 20-mers (base j at bits 2j). */
int issl_build(const uint64_t* sigs, const uint32_t* occ, uint64_t n_sites,
               const uint64_t* slice_masks, uint64_t n_slices, int device, issl_index** out);

int issl_close(issl_index* index);
int issl_index_get_info(const issl_index* index, issl_index_info* out);

/* Copy the index back to host in the reference's file layout (ISSLCreateIndex.cpp:428-484);
 * any output pointer may be NULL. Sizes: sigs N, masks S, list_sizes n_buckets, lists S*N. */
int issl_export(const issl_index* index, uint64_t* sigs, uint64_t* slice_masks,
                uint64_t* list_sizes, uint64_t* lists);
/* Write the index as a .issl file. */
int issl_save(const issl_index* index, const char* path);

/* ---- scoring (the hot path) ------------------------------------------------------------- */

/* Score n guides given as ASCII (first 20 characters at seqs + i*stride are used, as
 * sequenceToSignature(seq, 20) does at lib/ISSLScoringModule.cpp:219; C=1 G=2 T=3, any
 * other byte encodes as A=0). Host buffers. Per guide i:
 *   mit_score[i], cfd_score[i]: 10000/(100 + sum) at the point the reference would have
 *                 stopped (-1 for the score the method does not compute, :404-459)
 *   code[i]:      ISSL_CODE_ACCEPTED / ISSL_CODE_REJECTED by the method's rule
 *   count[i]:     sum of occurrences of the scored sites (ISSLScoreOfftargets.cpp:371)
 * distinct (optional): number of distinct sites scored over all guides (:375-377).
 * Any output pointer except code may be NULL. max_dist: 0..4 (the reference fixes 4).
 * One call takes at most 2^26 guides (and fewer than 2^32 guide-slice pairs). */
int issl_score(issl_index* index, const char* seqs, size_t stride, size_t n, int method,
               double threshold, int max_dist, double* mit_score, double* cfd_score, char* code,
               uint64_t* count, uint64_t* distinct);

/* Same from packed signatures in host memory. */
int issl_score_sigs(issl_index* index, const uint64_t* sigs, size_t n, int method,
                    double threshold, int max_dist, double* mit_score, double* cfd_score,
                    char* code, uint64_t* count, uint64_t* distinct);

/* Same with every buffer in device memory of the index's device, enqueued on `stream`
 * (a cudaStream_t; NULL = the library's own stream). Returns after enqueueing unless the
 * workspace must grow, in which case the call synchronises once and retries. */
int issl_score_device(issl_index* index, const uint64_t* d_sigs, size_t n, int method,
                      double threshold, int max_dist, double* d_mit_score, double* d_cfd_score,
                      char* d_code, uint64_t* d_count, uint64_t* d_distinct, void* stream);

/* Allocation-free scoring. No counterpart in the reference, which scores on the CPU.
 *
 * For callers that cannot allocate device memory while they score: code running during CUDA
 * graph capture, hosts whose device memory belongs to their own pool allocator, services that
 * allow no allocation after start-up. The regular entry points grow a per-index workspace on
 * demand; this one allocates nothing (no cudaMalloc, no cudaFree, no allocating library call).
 * Its only scratch is a fixed 9.7 MB array inside the library, which every GPU that loads the
 * library holds until the process exits.
 *
 * Same arguments and results as issl_score_device (minus the distinct count), buffers in device
 * memory of the index's device, enqueued on `stream` (NULL = the default stream); the call waits
 * for the kernel to finish. Limits: at most ISSL_STATIC_MAX_GUIDES guides per call (larger n is
 * rejected with ISSL_ERR_ARG) and at most ISSL_STATIC_MAX_HITS owned off-target hits per guide
 * (a guide beyond that makes the call fail with ISSL_ERR_UNSUPPORTED; its outputs are not set).
 * The first call on a device looks up the scratch address and uploads the penalty tables; make
 * that first call before any stream capture. Every call shares the one scratch array, so calls
 * that overlap on the GPU (concurrent streams or threads) race and must be serialised. */
#define ISSL_STATIC_MAX_GUIDES 1048576
#define ISSL_STATIC_MAX_HITS 4096
int issl_score_device_static(issl_index* index, const uint64_t* d_sigs, size_t n, int method,
                             double threshold, int max_dist, double* d_mit_score, double* d_cfd_score,
                             char* d_code, uint64_t* d_count, void* stream);

/* Kernel timing of the last issl_score* call on this index (device milliseconds of the scan
 * kernel and of the whole pipeline, taken with CUDA events on its stream) and its work
 * counters: probes, distinct buckets scanned, entries streamed, scan units, owned hits, the
 * bytes the scan kernel must move, and the number of kernels launched. */
typedef struct {
    double scan_ms, total_ms;
    uint64_t probes, buckets_scanned, entries_scanned, units, hits, scan_bytes;
    uint64_t launches;  /* kernels this library launched for the call */
} issl_score_stats;
int issl_last_stats(const issl_index* index, issl_score_stats* out);

/* ---- synthetic workloads (benchmarks and tests) ------------------------------------------ */
typedef struct {
    uint64_t seed;
    uint64_t n_sites;           /* distinct sites in the index */
    double repeat_frac;         /* share of sites that are repeat-seed copies (0.05) */
    uint64_t n_repeat_seeds;    /* 10000 */
    double repeat_lambda;       /* Poisson substitutions per repeat copy (2.0) */
    uint64_t n_queries;
    double copied_frac;         /* share of queries sampled from the sites (0.5) */
    double repeat_query_frac;   /* share of queries derived from repeat seeds */
    int planted_into_sites;     /* 1: queries are exact site copies and their 0-4 mutants join
                                   the site set; 0: queries carry the 0-4 mutations */
    const uint64_t* slice_masks;
    uint64_t n_slices;
} issl_synth_spec;

/* Generate sites + occurrences on the device (i.i.d. GC 41% plus repeat families, made
 * distinct, occurrences min(1+Geometric(0.9),255)), build the resident index, and write the
 * query signatures to host memory (n_queries entries). */
int issl_synth(const issl_synth_spec* spec, int device, issl_index** out, uint64_t* queries);

/* ---- tables (for verification) ------------------------------------------------------------ */
/* MIT local scores for every 1..4-mismatch mask in ascending mask order (6195 entries;
 * masks use bit 2p for position p) and the CFD position/PAM penalties. */
int issl_tables(uint64_t* mit_masks, double* mit_scores, double* cfd_pos320, double* cfd_pam16);

#ifdef __cplusplus
}
#endif
#endif
