/*
 * CPU oracle for ISSL off-target scoring -- TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference's CPU algorithm, used by tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline leg as the checker. The shipped
 * library never links, loads or calls it. Every function cites the reference lines it
 * restates (paths relative to the reference project root).
 *
 * Parity pin: tests/test_oracle_pin.py checks this restatement against the reference's
 * own binaries (oracle/_ref, built from the reference sources by oracle/Makefile) and
 * against the golden vectors committed under tests/golden/ (penalty tables extracted from
 * lib/otScorePenalties.cpp, the MIT pairs embedded in the reference's legacy test index,
 * reference-generated indexes and reference-scored outputs).
 */
#ifndef ISSL_ORACLE_H
#define ISSL_ORACLE_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* otScoreMethod, include/util.hpp:20 */
enum { ORA_MIT = 0, ORA_CFD = 1, ORA_AND = 2, ORA_OR = 3, ORA_AVG = 4 };

/* An index in the reference's in-memory layout (lib/ISSLScoringModule.cpp:83-147). */
typedef struct {
    uint64_t n_sites;      /* offtargetsCount */
    uint64_t seq_len;      /* seqLength */
    uint64_t n_slices;     /* sliceCount */
    uint64_t* sigs;        /* offtargets[n_sites] */
    uint64_t* slice_masks; /* one position bitmask per slice */
    uint64_t* list_sizes;  /* allSlicelistSizes, concatenated over slices */
    uint64_t* lists;       /* allSignatures[n_slices * n_sites], (occ << 32) | id */
    int owns_memory;
} ora_index;

/* sequenceToSignature, lib/ISSLScoringModule.cpp:469-476 with nucleotideIndex :10 */
uint64_t ora_encode(const char* seq, uint64_t len);

/* calcMITLocalScore, ISSLCreateIndex/ISSLCreateIndex.cpp:235-261 (Hsu et al. 2013).
 * positions ascending, count 1..20. */
double ora_mit_local_score(const uint64_t* positions, uint64_t count);

/* Install the CFD tables (cfdPosPenalties[320], cfdPamPenalties[16] of
 * lib/otScorePenalties.cpp:6201-6546). The tests load them from the golden fixture. */
void ora_set_cfd_tables(const double* pos320, const double* pam16);

/* Builds the MIT table from the formula for every 1..4-mismatch mask; returns the number
 * of entries (6195) and writes (mask, score) pairs in ascending mask order when non-NULL. */
int ora_mit_table(uint64_t* masks_out, double* scores_out);

/* Reader for the .issl layout, lib/ISSLScoringModule.cpp:72-150. 0 on success. */
int ora_load(const char* path, ora_index* out);
void ora_free(ora_index* idx);

/* Index construction, ISSLCreateIndex/ISSLCreateIndex.cpp:450-484: per slice, bucket every
 * site in ascending id order by its slice key. Fills list_sizes and lists (allocated). */
int ora_build(const uint64_t* sigs, const uint32_t* occ, uint64_t n_sites,
              const uint64_t* slice_masks, uint64_t n_slices, uint64_t seq_len, ora_index* out);

/* Writer, ISSLCreateIndex/ISSLCreateIndex.cpp:428-484. 0 on success. */
int ora_write(const char* path, const ora_index* idx);

/* The scoring loop of lib/ISSLScoringModule.cpp:206-462 (and ISSLScoreOfftargets.cpp:308-505
 * for the count/distinct extras). For each query signature:
 *   tot_mit[q], tot_cfd[q]: the raw occurrence-weighted sums at the point scoring stopped
 *   count[q]: sum of occurrences of the dist<=max_dist sites scored (CLI :371)
 *   distinct: number of distinct site ids scored over all queries (CLI :375-377, :549-553)
 * max_dist: the reference hard-codes 4 (:292); values 0..4 are honoured here as a filter.
 * threads: OpenMP threads (0 = runtime default). Returns 0, or -1 if a mask is missing
 * from the MIT table (the reference's .at() would throw). */
int ora_score(const ora_index* idx, const uint64_t* query_sigs, uint64_t n_queries, int method,
              double threshold, int max_dist, int threads, double* tot_mit, double* tot_cfd,
              uint64_t* count, uint64_t* distinct);

/* The scored terms of one guide in the reference's adding order, without the early exit
 * (lib/ISSLScoringModule.cpp:230-363): MIT term, CFD term and occurrences per scored site.
 * Returns the number of scored sites (at most cap written). For deriving thresholds that sit
 * on the reference's own running sums. */
uint64_t ora_trace(const ora_index* idx, uint64_t query_sig, int max_dist, double* mit_terms,
                   double* cfd_terms, uint32_t* occ, uint64_t cap);

/* Synthetic workloads (synth_oracle.c): the library's seeded generator restated for the host.
 * sites[n_sites], occ[n_sites], queries[n_queries] receive the workload issl_synth generates for
 * the same spec. Returns 0, -1 (allocation) or -2 (not enough distinct sites). */
int ora_synth(uint64_t seed, uint64_t n_sites, double repeat_frac, uint64_t n_repeat_seeds,
              double repeat_lambda, uint64_t n_queries, double copied_frac, double repeat_query_frac,
              int planted_into_sites, uint64_t* sites, uint32_t* occ, uint64_t* queries);

/* Writes the .issl file of sites + occurrences bucketed by the slice masks (ISSLCreateIndex.cpp
 * :428-484 layout), one slice at a time (OpenMP). 0 on success. */
int ora_write_built(const char* path, const uint64_t* sigs, const uint32_t* occ, uint64_t n_sites,
                    const uint64_t* slice_masks, uint64_t n_slices);

/* Per-guide finalisation, lib/ISSLScoringModule.cpp:404-459: scores and the accept code
 * ('1' accepted / '0' rejected). For mit (cfd) the unused score is -1. */
void ora_finalise(int method, double threshold, double tot_mit, double tot_cfd, double* mit_score,
                  double* cfd_score, char* code);

/* Independent candidate-set check: for each query, every site with popcount of the folded
 * mismatch mask <= max_dist, found by a brute-force scan over all sites (no slices).
 * Writes per-query sums of occurrences and of MIT/CFD contributions (no early exit). */
int ora_bruteforce(const uint64_t* sigs, const uint32_t* occ, uint64_t n_sites,
                   const uint64_t* query_sigs, uint64_t n_queries, int max_dist, int threads,
                   double* sum_mit, double* sum_cfd, uint64_t* count);

#ifdef __cplusplus
}
#endif
#endif
