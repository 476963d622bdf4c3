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
#define ISSL_ERR_INTERNAL (-9)    /* a consistency check of the pipeline failed; the call's
                                     outputs are not valid (message says which check) */

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
    int entry_bytes;          /* 8: list entries carry the residual code (one read per scored
                                 hit); 4: chosen when HBM is short (a second read for the
                                 signature). ISSL_ENTRY_BYTES=4|8 in the environment forces it */
    uint64_t host_bytes;      /* page-locked host memory holding the lists (issl_open_mapped) */
    int window_slices;        /* slices staged on the device at a time (0: lists resident) */
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

/* Load a .issl file for an index whose lists do not fit in HBM: replaces the memory-mapped
 * module (lib/ISSLScoringModuleMMF.cpp:73-128, selected by offTarget.memoryMapped), which scores
 * straight from a mapping of the file. Signatures, occurrence counts and bucket offsets are
 * resident on `device`; the list entries and bit-sliced residual codes are built on the device
 * slice by slice and kept in page-locked host memory. Every scoring call then streams them back
 * window_slices slices at a time (two device windows: the copy of the next window overlaps the
 * scan of the current one), so a call moves the whole lists over the host link once and large
 * guide batches amortise it. Results are identical to a resident index. Everything else works on
 * such an index except issl_score_device_static (ISSL_ERR_UNSUPPORTED). */
int issl_open_mapped(const char* path, int device, uint32_t window_slices, issl_index** out);

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

/* Every scoring entry point runs the pipeline over all its guides at once, or, when the device
 * cannot hold the workspace that needs (many guides with thousands of candidate sites), over
 * consecutive chunks of guides, halving the chunk until it fits; results do not depend on the
 * split. ISSL_MAX_GUIDES_PER_RUN=<n> in the environment caps the chunk from the start. */

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
 * For callers that cannot allocate device memory while they score: hosts whose device memory
 * belongs to their own pool allocator (a framework's caching allocator, a fixed arena on a shared
 * GPU) and forbid stray cudaMalloc calls, and services that allow no allocation after start-up.
 * The regular entry points grow a per-index workspace on demand; this one allocates nothing (no
 * cudaMalloc, no cudaFree, no allocating library call). Its only scratch is a fixed 9.7 MB array
 * inside the library, which every GPU that loads the library holds until the process exits.
 *
 * Same arguments and results as issl_score_device (minus the distinct count), buffers in device
 * memory of the index's device, enqueued on `stream` (NULL = the default stream); the call waits
 * for the kernel to finish, then reads the overflow flag. Each guide's sums are accumulated one
 * addition at a time in the reference's order, as the reference does. Limits: at most
 * ISSL_STATIC_MAX_GUIDES guides per call (larger n is rejected with ISSL_ERR_ARG) and at most
 * ISSL_STATIC_MAX_HITS owned off-target hits per guide
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
    uint64_t launches;          /* kernels this library launched for the call */
    uint64_t class_probes[3];   /* probes into buckets of < 64, 64..4095 and >= 4096 entries */
    uint64_t candidates;        /* candidate slots the scan wrote, before the ownership rule */
    uint64_t staged_bytes;      /* host-list index: list bytes copied from host memory */
    uint64_t dropped_hits;      /* candidate sites found farther than 4 mismatches from their guide:
                                   none by construction; any makes the call fail with
                                   ISSL_ERR_INTERNAL */
    uint64_t replayed;          /* guides whose decision lay within the reference's rounding of
                                   its running sums, rescored one addition at a time */
    uint64_t runs;              /* pipeline runs of the call: one per guide chunk, plus any run
                                   repeated after its buffers had to grow */
} issl_score_stats;

/* Frees the device memory of the index's own scoring workspace (the buffers the plain
 * issl_score* calls grow on demand); the next call re-creates it. The index stays resident.
 * No counterpart in the reference. */
int issl_index_trim(issl_index* index);

/* Moves an open index's list entries and bit-sliced codes between HBM and page-locked host
 * memory: window_slices > 0 keeps them in host memory and stages that many slices per device
 * window while scoring (what issl_open_mapped gives), 0 brings them back to HBM. The index must
 * be idle (no call on it, its batch contexts or its server in flight); batch contexts and
 * servers re-capture their graphs on their next call. No counterpart in the reference. */
int issl_index_set_list_placement(issl_index* index, uint32_t window_slices);

/* Modelled device bytes of one scoring workspace (the per-call buffers of issl_score*,
 * a batch context or a server slot) holding n guides, when the scan finds `candidates_per_guide`
 * candidate sites per guide (64 is the library's first guess). No counterpart in the reference.
 * The server admits requests by this footprint. */
int issl_workspace_bytes(const issl_index* index, uint64_t n, double candidates_per_guide, uint64_t* bytes);
int issl_last_stats(const issl_index* index, issl_score_stats* out);

/* ---- scan tuning and autotuning ------------------------------------------------------------
 * No counterpart in the reference (its CPU loop has no tiles). The scan streams each probed
 * bucket in units of up to 1024 list positions shared by up to 32 guides; `chunk` sets the unit
 * size per bucket-size class (smaller units spread a heavy bucket over more warps), `stages`
 * the depth of each warp's asynchronous copy ring, `blocks_per_sm` the persistent grid,
 * `first_wave` the slices scored in a first wave. Results do not depend on the tuning; only
 * speed and memory do. */
typedef struct {
    uint32_t chunk[3];       /* buckets of < 64, 64..4095, >= 4096 entries: 256, 512 or 1024 */
    uint32_t stages;         /* 2..4 (default 2: seven scan blocks fit an SM) */
    uint32_t blocks_per_sm;  /* 0 = as many as fit (default) */
    uint32_t first_wave;     /* slices scored before the rest (default 1; 0 = all in one wave):
                                guides whose early exit fires there never probe the later slices */
} issl_tuning;
int issl_get_tuning(const issl_index* index, issl_tuning* out);
int issl_set_tuning(issl_index* index, const issl_tuning* tuning);

typedef struct {
    double default_ms;       /* pipeline time with the tuning the index had */
    double best_ms;          /* pipeline time with the chosen tuning */
    uint32_t configs_timed;  /* tunings measured (0 when the result came from the cache) */
    uint32_t from_cache;
    uint64_t class_probes[3];/* bucket-size class histogram of the sample's probes */
} issl_tune_report;

/* Sweeps the tuning on a sample workload (d_sigs: n guides in device memory, scored with the
 * given method / threshold / max_dist), starting from the current tuning: staging depth first,
 * then the unit size of each bucket-size class that the sample's probes reach (heaviest class
 * first), then blocks per SM, then the first wave, keeping a change only when the pipeline gets
 * faster by more than 2%. The winner is applied to the index and, when cache_path is not NULL, appended there under
 * a key made of the GPU name, the index geometry and the sample size; a later call with the
 * same key reads it back without timing. */
int issl_autotune(issl_index* index, const uint64_t* d_sigs, size_t n, int method, double threshold,
                  int max_dist, const char* cache_path, issl_tuning* out, issl_tune_report* report);

/* ---- batched scoring -----------------------------------------------------------------------
 * No counterpart in the reference, which scores one query file per process. Many independent
 * guide sets, each with its own method, threshold and mismatch bound, are scored in one pass:
 * the whole pipeline is captured once into a CUDA graph and replayed for every batch that fits
 * its capacities (it is re-captured when a capacity grows or the tuning changes). Every guide
 * gets exactly the result issl_score_device gives it in a call of its own. */
typedef struct {
    uint64_t count;      /* guides in the set; sets follow each other in the signature array */
    int method;          /* ISSL_METHOD_* */
    int max_dist;        /* 0..4 */
    double threshold;
} issl_guide_set;

typedef struct issl_batch issl_batch;

/* A batch context: its own workspace and graph on the index's device (one per thread). */
int issl_batch_create(issl_index* index, issl_batch** out);
void issl_batch_destroy(issl_batch* batch);

/* Scores n guides (device memory, packed signatures) split into n_sets consecutive sets
 * (host array; counts sum to n; at most 65535 sets and 2^26 guides). Outputs are device
 * buffers of n entries (any may be NULL except d_code); counts are per guide as in issl_score.
 * Work is enqueued on `stream` (NULL = the batch's own stream); the call returns when the
 * results are in the output buffers. */
int issl_batch_score(issl_batch* batch, const uint64_t* d_sigs, size_t n, const issl_guide_set* sets,
                     size_t n_sets, double* d_mit_score, double* d_cfd_score, char* d_code,
                     uint64_t* d_count, void* stream);

/* Same with host buffers: signatures in, scores out. */
int issl_batch_score_host(issl_batch* batch, const uint64_t* sigs, size_t n, const issl_guide_set* sets,
                          size_t n_sets, double* mit_score, double* cfd_score, char* code, uint64_t* count);

/* Timing and counters of the last batch: total_ms is the graph replay (device time), launches
 * the kernels in the graph. */
int issl_batch_stats(const issl_batch* batch, issl_score_stats* out);

/* ---- serving ---------------------------------------------------------------------------------
 * No counterpart in the reference (a CLI run per query file). A request loop in front of the
 * resident index: guide-set requests (each with its own method / threshold / mismatch bound)
 * are queued as they arrive; each of n_slots worker slots, with its own workspace and captured
 * graph, repeatedly takes the waiting requests in arrival order and scores them together as one
 * batch. A batch is admitted while it stays within max_batch_guides and its device-memory
 * footprint (issl_workspace_bytes, with a candidates-per-guide estimate that grows with what
 * batches produced) stays within the slot's share of the device memory that was free at creation
 * minus headroom_bytes. Batches of different slots overlap on the GPU. Every request gets exactly
 * the result a call of its own gives. */
typedef struct {
    uint32_t n_slots;           /* batches on the GPU at once (0 = 3) */
    uint32_t max_wait_us;       /* a free slot waits this long for more arrivals before scoring (0) */
    uint64_t max_batch_guides;  /* guides per batch (0 = 131072); larger requests run in parts */
    uint64_t headroom_bytes;    /* device memory left free beside the index and the slots (0 = 16 GiB) */
} issl_server_config;

typedef struct {
    double queue_ms;            /* submit -> admitted into a batch */
    double service_ms;          /* admitted -> results ready */
    double latency_ms;          /* submit -> results ready */
    uint64_t batch_guides;      /* guides in the request's batch */
    uint32_t batch_requests;    /* requests in the request's batch */
    uint32_t slot;
} issl_request_info;

typedef struct {
    uint64_t requests, guides, batches;   /* completed since creation or the last reset */
    double p50_ms, p99_ms, max_ms;        /* request latency, submit -> results ready */
    double mean_batch_guides;
    uint32_t slots, peak_in_flight;       /* peak_in_flight: most batches on the GPU at once */
    uint64_t slot_budget_bytes, peak_batch_bytes;
} issl_server_summary;

typedef struct issl_server issl_server;

/* Starts the slots (NULL config = defaults). Fails with ISSL_ERR_NOMEM when the free device
 * memory minus the headroom cannot hold one slot's workspace. */
int issl_server_create(issl_index* index, const issl_server_config* config, issl_server** out);

/* Queues n guides (host memory, packed signatures; copied) as one request and returns its ticket
 * at once. A request above max_batch_guides, or whose modelled device footprint exceeds a slot's
 * share, is scored as consecutive parts (its ticket completes with the last one). ISSL_ERR_ARG
 * for a bad method / max_dist, ISSL_ERR_BUSY when not even one guide fits a slot. */
int issl_server_submit(issl_server* server, const uint64_t* sigs, size_t n, int method, double threshold,
                       int max_dist, uint64_t* ticket);

/* Waits up to timeout_ms (< 0: no limit) for the request and copies its n results (any output
 * may be NULL; info may be NULL). ISSL_ERR_TIMEOUT when not finished yet (the ticket stays
 * valid); otherwise the ticket is consumed. */
int issl_server_wait(issl_server* server, uint64_t ticket, int timeout_ms, double* mit_score,
                     double* cfd_score, char* code, uint64_t* count, issl_request_info* info);

/* Latency percentiles and counters of the completed requests; reset != 0 starts a new window. */
int issl_server_stats(issl_server* server, issl_server_summary* out, int reset);

/* Finishes every submitted request, then stops the slots and frees their workspaces. */
void issl_server_destroy(issl_server* server);

/* ---- off-target extraction -------------------------------------------------------------------
 * ExtractOfftargets (ExtractOfftargets/ExtractOfftargets.cpp:16-370) on the GPU. Inputs are files
 * or directories (every file in them): a file whose first line starts with '>' is FASTA (each
 * record's lines trimmed, upper-cased and joined), any other file holds one sequence per line.
 * Every site matching the reference's forward pattern [ACG][ACGT]{19}[ACGT][AG]G (its first 20
 * bases) or reverse pattern C[CT][ACGT][ACGT]{19}[TGC] (the first 20 bases of its reverse
 * complement) is found at every position, overlaps included. */

/* Writes every site, sorted, one 20-mer per line with duplicates kept: the reference's output
 * file, byte for byte. n_offtargets (may be NULL) receives the number of lines. */
int issl_extract_offtargets(const char* const* inputs, size_t n_inputs, const char* out_path, int device,
                            uint64_t* n_offtargets);

/* Extracts the sites and builds the resident index from them without a file in between: the
 * distinct sites in sorted order with their counts as occurrences, as ISSLCreateIndex reads the
 * sorted list (ISSLCreateIndex/ISSLCreateIndex.cpp:393-417), then issl_build's bucketing. */
int issl_build_from_sequences(const char* const* inputs, size_t n_inputs, const uint64_t* slice_masks,
                              uint64_t n_slices, int device, issl_index** out, uint64_t* n_offtargets);

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
