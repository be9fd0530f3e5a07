/*
 * CPU oracle for the SuperCountingBloom insert / query / spectrum path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the reference
 * crate `super-counting-bloom` 0.1.0 used as the checker for the CUDA
 * library.  Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline
 * leg load it; the product library never links or calls it.
 *
 * Parity status:
 *   - pinned: in-repo arithmetic of the reference (xorshift_u64, probe chain,
 *     block/shard/subblock mapping, s-mer ranges, saturation, deque minimum,
 *     .scb layout) and the known-answer counts of the reference's own tests
 *     (tests/golden/reference_known_answers.json).
 *   - parity unpinned: the arithmetic of the third-party crates that are not
 *     present anywhere on this machine (packed-seq 4.4.2 base encoding and
 *     bit order; simd-minimizers 2.3.1 / seq-hash 0.1.2 m-mer hash, canonical
 *     strand rule and tie-break).  Those are restated from the crates'
 *     published descriptions and isolated in ora_base_code(),
 *     ora_read_kmer(), ora_read_revcomp_kmer(), ora_mmer_hash() and
 *     ora_window_minimizer().
 */
#ifndef SCB_ORACLE_H
#define SCB_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct ora_config {
    uint64_t k, m, s, n_hashes;
    uint8_t counter_bits;           /* 8, 16 or 32 */
    uint8_t counter_slots_exponent;
    uint8_t block_slots_exponent;
    uint64_t threads, queue;
} ora_config;

typedef struct ora_layout {
    uint64_t shard_count, subblocks, block_slots, shard_mask;
    uint32_t shard_shift;
    uint64_t block_slots_mask, nb_blocks, block_mask, n_hashes;
} ora_layout;

typedef struct ora_report {
    uint64_t records_processed, total_windows, valid_kmers, positive_estimates, estimate_checksum;
} ora_report;

typedef struct ora_filter ora_filter;

/* config.rs:50-92 (+ filter.rs:96-100 power-of-two rule).  0 = ok, 1 = invalid. */
int ora_validate(const ora_config* cfg, char* msg, size_t cap);
int ora_layout_from_config(const ora_config* cfg, ora_layout* out);

/* filter.rs:629-635 */
uint64_t ora_xorshift_u64(uint64_t x);

/* packed-seq restatement: 2-bit code of an ASCII base (A=0, C=1, T=2, G=3). */
uint8_t ora_base_code(uint8_t ascii);
int ora_is_acgt(uint8_t ascii);                                   /* api.rs:929-931 */
uint64_t ora_read_kmer(const uint8_t* codes, size_t len, size_t pos);
uint64_t ora_read_revcomp_kmer(const uint8_t* codes, size_t len, size_t pos);
uint64_t ora_canonical_kmer(const uint8_t* codes, size_t len, size_t pos);   /* filter.rs:622-627 */

/* simd-minimizers restatement. */
uint32_t ora_mmer_hash(const uint8_t* codes, size_t pos, size_t m);
size_t ora_window_minimizer(const uint8_t* codes, const uint32_t* hashes, size_t i, size_t k, size_t m);
/* filter.rs:608-620: returns the number of super-k-mers; starts/minimizers must hold len-k+1 entries. */
size_t ora_super_kmers(const uint8_t* codes, size_t len, size_t k, size_t m, uint32_t* starts,
                       uint64_t* minimizers);

/* Filter lifecycle (filter.rs:118-145).  The counter table is kept in file order. */
ora_filter* ora_filter_new(const ora_config* cfg);
void ora_filter_free(ora_filter* f);
void ora_filter_clear(ora_filter* f);
void* ora_filter_table(ora_filter* f);
uint64_t ora_filter_table_bytes(const ora_filter* f);
uint64_t ora_filter_inserted_kmers(const ora_filter* f);
uint64_t ora_filter_inserted_smers(const ora_filter* f);
void ora_filter_set_inserted_kmers(ora_filter* f, uint64_t v);

/* filter.rs:199-237 on one ACGT run of 2-bit codes; returns inserted s-mers. */
uint64_t ora_insert_packed(ora_filter* f, const uint8_t* codes, size_t len);
/* filter.rs:337-369 + 462-508: len+1-k estimates (nothing when len < k). */
void ora_estimate_packed(const ora_filter* f, const uint8_t* codes, size_t len, uint64_t* out);

/* api.rs:676-726 per sequence; batch over concatenated sequences with n+1 offsets. */
void ora_insert_batch(ora_filter* f, const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                      uint64_t* inserted_kmers, uint64_t* inserted_smers);
/* api.rs:799-853: per sequence max(0, len+1-k) windows, concatenated; valid=0 means None. */
void ora_query_batch(const ora_filter* f, const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                     uint64_t* out, uint8_t* valid);
/* api.rs:273-327 reduction over the same windows. */
void ora_query_report(const ora_filter* f, const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                      ora_report* rep);
/* fastx.rs:255-308 + 392-410: histogram over distinct canonical k-mers of their estimates.
 * Returns the number of rows; rows are written when cap is large enough.  *distinct_keys and
 * *queried_kmers receive the map size and the number of queried windows.  *mismatches counts
 * repeated keys whose estimate differed from the first one seen (0 when the estimate is a
 * function of the canonical k-mer). */
uint64_t ora_spectrum_distinct(const ora_filter* f, const uint8_t* seqs, const uint64_t* offsets,
                               uint64_t n, uint64_t* values, uint64_t* counts, uint64_t cap,
                               uint64_t* distinct_keys, uint64_t* queried_kmers, uint64_t* mismatches);
/* filter.rs:267-275 */
uint64_t ora_counter_histogram(const ora_filter* f, uint64_t* values, uint64_t* counts, uint64_t cap);

/* api.rs:388-608 .scb writer / reader.  ora_load returns NULL and fills msg on failure. */
int ora_save(const ora_filter* f, const char* path);
ora_filter* ora_load(const char* path, char* msg, size_t cap);
const ora_config* ora_filter_config(const ora_filter* f);

/* Per-window minimizer positions over a batch, indexed by global byte position; positions
 * that start no valid window get UINT32_MAX.  Used to localise GPU mismatches. */
void ora_batch_window_minimizers(const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                                 uint64_t k, uint64_t m, uint32_t* out);

/* Workload statistics over a batch: super-k-mers, s-mers, and distinct 32-byte sectors of
 * the counter block touched by each super-k-mer's probes (summed). */
void ora_batch_sector_stats(const ora_config* cfg, const uint8_t* seqs, const uint64_t* offsets,
                            uint64_t n, uint64_t* super_kmers, uint64_t* smers, uint64_t* sectors);

/* Multi-threaded port with the reference's structure (scb_cpu_port.cpp): one producer feeding
 * `threads` workers through a bounded queue of `queue` records; counters guarded by one mutex
 * per shard (filter.rs:57-65, 220-222; api.rs:621-666; fastx.rs:310-369).  Builds into `f` and
 * then stream-queries the same records.  Timings in seconds. */
int ora_port_build_and_stream_query(ora_filter* f, const uint8_t* seqs, const uint64_t* offsets,
                                    uint64_t n, uint64_t threads, uint64_t queue,
                                    uint64_t* inserted_kmers, uint64_t* inserted_smers,
                                    ora_report* rep, double* build_s, double* query_s);

#ifdef __cplusplus
}
#endif

#endif
