/*
 * scb.h -- C ABI of the B200 (sm_100a) SuperCountingBloom library (libscb_b200.so).
 *
 * The entry points are what a GPU backend inside the reference crate's public API
 * (super-counting-bloom 0.1.0, src/api.rs) binds through `extern "C"`: plain pointers and
 * sizes, no Rust, no torch types.  Each declaration cites the reference interface it replaces.
 *
 * Conventions
 *   - Sequences are passed as one concatenated byte buffer `seqs` plus `n_seqs + 1` offsets
 *     (sequence i is seqs[offsets[i] .. offsets[i+1])), exactly the records the reference's
 *     workers receive (src/api.rs:621-674).  Bytes other than A/C/G/T (either case) split a
 *     sequence into runs; runs shorter than k are skipped (src/api.rs:676-726, 929-931).
 *   - `*_device` entry points take device pointers and a CUDA stream (cudaStream_t passed as
 *     void*); all others take host pointers (pinned or pageable) and return after the result
 *     is on the host.
 *   - Every function returns an scb_status; on failure scb_last_error() gives a thread-local
 *     message.  Status values map 1:1 onto SuperCountingBloomError (src/error.rs:4-12).
 *   - The library owns device memory; the caller owns host buffers.  No callbacks.
 *   - Query entry points on a frozen index are thread-safe (src/api.rs:278-286 runs them
 *     from several threads); insert entry points need a single writer (&mut self).
 */
#ifndef SCB_H
#define SCB_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* src/error.rs:4-12 */
typedef enum scb_status {
    SCB_OK = 0,
    SCB_ERR_INVALID_CONFIG = 1,       /* InvalidConfig(String) */
    SCB_ERR_FASTX_OPEN = 2,           /* FastxOpen { path, message } */
    SCB_ERR_INVALID_INDEX_FORMAT = 3, /* InvalidIndexFormat(String) */
    SCB_ERR_CHANNEL_CLOSED = 4,       /* ChannelClosed(String) */
    SCB_ERR_WORKER_PANIC = 5,         /* WorkerPanic(&'static str) */
    SCB_ERR_INTERNAL_STATE = 6,       /* InternalState(String): CUDA errors, device status words */
    SCB_ERR_IO = 7                    /* Io { path, message } */
} scb_status;

/* src/config.rs:20-31 (SuperCountingBloomConfig); counter_bits is CounterBits::as_u8. */
typedef struct scb_config {
    uint64_t k;
    uint64_t m;
    uint64_t s;
    uint64_t n_hashes;
    uint8_t counter_bits;           /* 8, 16 or 32 */
    uint8_t counter_slots_exponent; /* total counters = 2^counter_slots_exponent */
    uint8_t block_slots_exponent;   /* counters per block = 2^block_slots_exponent */
    uint64_t threads;               /* carried into .scb (src/api.rs:478) */
    uint64_t queue;                 /* carried into .scb (src/api.rs:479) */
} scb_config;

/* src/api.rs:20-27 (QueryFastaReport); also the stream-query statistics of
 * src/fastx.rs:74-79 (queried_kmers = valid_kmers). */
typedef struct scb_report {
    uint64_t records_processed;
    uint64_t total_windows;
    uint64_t valid_kmers;
    uint64_t positive_estimates;
    uint64_t estimate_checksum; /* wrapping sum of the estimates */
} scb_report;

/* Device-side work statistics of a batch (super-k-mers, s-mers, distinct 32-byte sectors of
 * the counter blocks touched per super-k-mer); used to state algorithmic bytes. */
typedef struct scb_stats {
    uint64_t windows;
    uint64_t super_kmers;
    uint64_t smers;
    uint64_t sectors;
} scb_stats;

/* Insert / query kernel strategies (selected by the autotuner unless set). */
typedef enum scb_strategy {
    SCB_STRATEGY_AUTO = 0,
    SCB_STRATEGY_PLAIN = 1,  /* one launch per stage, per-window arrays in HBM, direct atomics */
    SCB_STRATEGY_FUSED = 2,  /* one persistent tile kernel over a device work queue */
    SCB_STRATEGY_STAGED = 3, /* fused tiles, one warp per super-k-mer staging its block deltas */
    SCB_STRATEGY_GROUPED = 4 /* super-k-mers bucketed by block, blocks applied in shared memory */
} scb_strategy;

typedef struct scb_ctx scb_ctx;

/* Thread-local text of the last failure on this thread ("" if none). */
const char* scb_last_error(void);
/* Library version string. */
const char* scb_version(void);

/* src/config.rs:33-47 (Default).  threads is set to the host's core count. */
scb_status scb_config_default(scb_config* cfg);
/* src/config.rs:50-92 + src/filter.rs:96-100 (number of blocks a power of two). */
scb_status scb_config_validate(const scb_config* cfg);

/* SuperCountingBloomBuilder::new (src/api.rs:101-121): validates, allocates the counter table
 * on device 0 (or the current device) in .scb file order and zeroes it. */
scb_status scb_create(const scb_config* cfg, scb_ctx** out);
/* Drop of builder / index: frees all device memory of the context. */
void scb_destroy(scb_ctx* ctx);

/* SuperCountingBloomBuilder::add_sequence / add_fasta's per-record insert
 * (src/api.rs:123-158, 621-726, filter.rs:199-237).  Adds the batch's k-mer windows and
 * inserted s-mers to the context totals and returns this batch's counts. */
scb_status scb_insert_batch(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n_seqs,
                            uint64_t* inserted_kmers, uint64_t* inserted_smers);
scb_status scb_insert_batch_device(scb_ctx* ctx, const uint8_t* d_seqs, const uint64_t* d_offsets,
                                   uint64_t n_seqs, uint64_t n_bytes, void* stream,
                                   uint64_t* inserted_kmers, uint64_t* inserted_smers);

/* SuperCountingBloomBuilder::into_index (src/api.rs:160-177).  After freezing, inserts fail
 * with SCB_ERR_INTERNAL_STATE and queries are allowed. */
scb_status scb_freeze(scb_ctx* ctx);
/* SuperCountingBloomBuilder::{inserted_kmers, inserted_smers}, SuperCountingBloomIndex::
 * {inserted_kmers, config} (src/api.rs:179-207, 225-231). */
scb_status scb_get_counts(const scb_ctx* ctx, uint64_t* inserted_kmers, uint64_t* inserted_smers);
scb_status scb_get_config(const scb_ctx* ctx, scb_config* cfg);
/* SuperCountingBloomBuilder::set_threads (src/api.rs:187-195): only the value carried into .scb. */
scb_status scb_set_threads(scb_ctx* ctx, uint64_t threads);

/* SuperCountingBloomIndex::estimate_sequence_abundances for each sequence
 * (src/api.rs:250-262, 799-853).  Sequence i contributes max(0, len_i + 1 - k) windows,
 * written consecutively; valid[w] = 0 marks a window with a non-ACGT base (None). */
scb_status scb_query_batch(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n_seqs,
                           uint64_t* abundances, uint8_t* valid);
scb_status scb_query_batch_device(scb_ctx* ctx, const uint8_t* d_seqs, const uint64_t* d_offsets,
                                  uint64_t n_seqs, uint64_t n_bytes, void* stream, uint64_t* d_abundances,
                                  uint8_t* d_valid);
/* Number of windows scb_query_batch writes for these offsets. */
uint64_t scb_count_windows(const scb_ctx* ctx, const uint64_t* offsets, uint64_t n_seqs);
/* AddReport::records_indexed of add_fasta (src/api.rs:640-642): records with at least one run of
 * k A/C/G/T bases (either case), i.e. records that insert at least one k-mer.  Host-side scan that
 * stops at each record's first such run. */
uint64_t scb_records_indexed(const scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n_seqs);

/* SuperCountingBloomIndex::query_fasta's reduction (src/api.rs:273-327): records, windows,
 * valid k-mers, positive estimates and the wrapping checksum, without per-window output. */
scb_status scb_query_report(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n_seqs,
                            scb_report* report);
scb_status scb_query_report_device(scb_ctx* ctx, const uint8_t* d_seqs, const uint64_t* d_offsets,
                                   uint64_t n_seqs, uint64_t n_bytes, void* stream, scb_report* report);

/* No counterpart in the reference.  scb_query_report_device without any device allocation, for
 * callers that cannot call cudaMalloc while they run: real-time serving threads that keep the
 * allocator's latency and its device-wide synchronisation out of the request path, and hosts
 * that hand the library a fixed device-memory budget at start-up and account for every byte.  Its
 * scratch is one static device array of about 16 MiB that every GPU loading this library holds
 * until the process exits; batches are limited to 32 MiB of sequence bytes (larger ones fail
 * with SCB_ERR_INTERNAL_STATE before any work).  The first call on a device looks up the array's
 * device address with that device current and keeps it for the life of the process, so a
 * process that resets the device (cudaDeviceReset) must not call this entry point afterwards.
 * The call ends by reading the report back and synchronising the stream.  All calls share the
 * array (each clears what it reads), so calls whose GPU work overlaps race: serialise them. */
scb_status scb_query_report_device_noalloc(scb_ctx* ctx, const uint8_t* d_seqs, const uint64_t* d_offsets,
                                           uint64_t n_seqs, uint64_t n_bytes, void* stream, scb_report* report);

/* stream_estimates_from_fastx (src/fastx.rs:107-131, 172-204, 206-253, 310-369) on in-memory
 * records: builds from the records, freezes, then stream-queries the same records.  The
 * records are copied to the device once and kept resident between the two passes. */
scb_status scb_build_and_stream_query_device(scb_ctx* ctx, const uint8_t* d_seqs, const uint64_t* d_offsets,
                                             uint64_t n_seqs, uint64_t n_bytes, void* stream,
                                             uint64_t* inserted_kmers, uint64_t* inserted_smers,
                                             scb_report* report);
scb_status scb_build_and_stream_query(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets,
                                      uint64_t n_seqs, uint64_t* inserted_kmers, uint64_t* inserted_smers,
                                      scb_report* report);

/* estimate_distinct_kmers + spectrum_from_estimates (src/fastx.rs:255-308, 392-410): the
 * histogram over distinct canonical k-mers of their estimates, rows sorted by value.  Call
 * with values == NULL to get the row count in *n_rows; then call again with capacity >= rows.
 * *distinct_keys = number of distinct canonical k-mers, *queried_kmers = windows queried. */
scb_status scb_spectrum_distinct(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n_seqs,
                                 uint64_t* values, uint64_t* counts, uint64_t capacity, uint64_t* n_rows,
                                 uint64_t* distinct_keys, uint64_t* queried_kmers);

/* SuperCountingBloomIndex::counter_histogram (src/api.rs:329-335, filter.rs:267-275): value ->
 * number of counters, rows sorted by value.  Same two-call convention as above. */
scb_status scb_counter_histogram(scb_ctx* ctx, uint64_t* values, uint64_t* counts, uint64_t capacity,
                                 uint64_t* n_rows);

/* SuperCountingBloomIndex::save / load (src/api.rs:233-248, 388-608): the .scb file, byte
 * identical to the reference's writer.  scb_load creates a frozen context. */
scb_status scb_save(const scb_ctx* ctx, const char* path);
scb_status scb_load(const char* path, scb_ctx** out);
/* Raw counter table in file order (little-endian), for callers that do their own I/O
 * (src/filter.rs:575-605). bytes must equal 2^counter_slots_exponent * counter_bits / 8. */
uint64_t scb_table_bytes(const scb_ctx* ctx);
scb_status scb_table_download(const scb_ctx* ctx, void* host, uint64_t bytes);
/* The same bytes in pieces: table bytes [offset, offset + bytes) (write_counter_data streams
 * shard by shard, src/filter.rs:575-580), so a caller can save or compare a table of up to
 * 16 GiB without holding it whole in host memory. */
scb_status scb_table_download_range(const scb_ctx* ctx, uint64_t offset, void* host, uint64_t bytes);
scb_status scb_table_upload(scb_ctx* ctx, const void* host, uint64_t bytes, uint64_t inserted_kmers);

/* Strategy control and workload statistics. */
scb_status scb_set_strategy(scb_ctx* ctx, scb_strategy insert_strategy, scb_strategy query_strategy);
scb_status scb_get_strategy(const scb_ctx* ctx, scb_strategy* insert_strategy, scb_strategy* query_strategy);
scb_status scb_batch_stats(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n_seqs,
                           scb_stats* stats);
/* Per-window chosen minimizer position, indexed by byte position of the batch (UINT32_MAX where
 * no valid window starts): exposes kernel (b) alone for localising mismatches. */
scb_status scb_debug_window_minimizers(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets,
                                       uint64_t n_seqs, uint32_t* out);
/* Number of kernels this library launched since load (all contexts). */
uint64_t scb_kernel_launches(void);

/* Per-stage device times (CUDA events on the launching stream), accumulated over batches
 * since timing was enabled: pack = kernel (a) plus sequence starts; insert / query = the
 * insert or query kernels of the active strategy (plain: the per-window stage included). */
typedef struct scb_timings {
    double pack_ms;
    double insert_ms;
    double query_ms;
    uint64_t batches;
    /* grouped strategy breakdown (part of insert_ms / query_ms) */
    double cut_ms;          /* kernel (b): records + bucket counts */
    double bucket_ms;       /* bucket offsets, scatter, work items */
    double apply_insert_ms; /* shared-memory insert apply kernel */
    double apply_query_ms;  /* shared-memory query apply kernel */
} scb_timings;
scb_status scb_set_timing(scb_ctx* ctx, int enable); /* enabling also clears the totals */
scb_status scb_get_timings(const scb_ctx* ctx, scb_timings* out);

/* CUDA graphs per batch shape (no counterpart in the reference).  A batch of the fused or
 * grouped strategy (scb_insert_batch[_device], scb_query_report[_device],
 * scb_build_and_stream_query[_device]) replays a graph captured for its shape class: batch
 * kind, byte capacity (the batch's bytes rounded up to four steps per octave, at least 64 KiB),
 * sequence capacity (a power of two, at least 256) and strategies.  The batch's sizes and input
 * pointers reach the kernels through a device parameter block, so one capture serves every
 * batch of its class.  A replay whose super-k-mer records outgrow the class's record slots
 * applies nothing and the batch is redone eagerly.  Results are identical either way.
 * Default on; enable = 0 runs every batch eagerly (the plain strategy always does). */
scb_status scb_set_graphs(scb_ctx* ctx, int enable);
/* Graph captures, replays, and replays redone eagerly (record overflow or failed capture). */
scb_status scb_graph_stats(const scb_ctx* ctx, uint64_t* captures, uint64_t* replays, uint64_t* fallbacks);

/* Build + stream query in one apply pass (no counterpart in the reference, whose stream query
 * runs after the whole build, src/fastx.rs:172-204).  With the grouped strategy for both passes,
 * every super-k-mer record of a batch that maps to a counter bucket is in that bucket's one work
 * item, so once the item commits its deltas its blocks hold their final counters: the same pass
 * then answers those records' windows from shared memory, and only buckets split over several
 * items (or with more than 8192 s-mers) go through a second, query-only pass.  Results are
 * identical to a separate query after the build.  Default on; enable = 0 runs the insert and the
 * query as two passes (the comparison point). */
scb_status scb_set_fused_build(scb_ctx* ctx, int enable);

/* Host scb_build_and_stream_query in pieces (no counterpart in the reference; the reference's
 * parser thread feeds its workers the same way, src/api.rs:621-674).  A batch of at least two
 * pieces is split into pieces of whole sequences of at most piece_bytes (0: 512 MiB; raised so
 * that a batch has at most about 32 pieces), the first piece_bytes / 2.2 and each next 1.3x
 * larger, so the first copy, which nothing overlaps, is
 * short; piece p + 1 is copied to the device while piece p is inserted, every piece keeps its super-k-mer records
 * for its query after the last insert, so the copy overlaps the work.  Applies with graphs on and
 * the grouped strategy; results are identical to one batch. */
scb_status scb_set_piece_bytes(scb_ctx* ctx, uint64_t piece_bytes);

/* Host packing of those pieces (performance setting, no reference counterpart; on by default):
 * the host packs each piece into the device's 2-bit code and validity layout on all host
 * threads, into pinned staging, and copies 3 bits per base instead of the 8-bit letters; piece
 * p + 1 is packed while the GPU works on piece p.  enable = 0 copies the letters and packs on the
 * device.  Results are identical either way. */
scb_status scb_set_host_pack(scb_ctx* ctx, int enable);

/* Bytes the host entry points of this context have copied to the device since it was created
 * (sequences or their packed form, offsets); no reference counterpart, a measurement aid. */
scb_status scb_h2d_bytes(scb_ctx* ctx, uint64_t* bytes);

/* Host FASTA/FASTQ reader (replaces the reference's parser thread feeding the workers,
 * src/api.rs:621-674, with its record rules, src/api.rs:893-915): reads a plain or gzip file in
 * one pass into concatenated sequences with n_records + 1 offsets (the layout of
 * scb_insert_batch) and the records' header lines.  Host memory only; no GPU needed.  The
 * pointers stay valid until scb_fastx_free.  A file that cannot be opened fails with
 * SCB_ERR_FASTX_OPEN. */
typedef struct scb_fastx scb_fastx;
scb_status scb_fastx_read(const char* path, scb_fastx** out);
scb_status scb_fastx_sequences(const scb_fastx* f, const uint8_t** seqs, const uint64_t** offsets,
                               uint64_t* n_records);
scb_status scb_fastx_headers(const scb_fastx* f, const uint8_t** headers, const uint64_t** header_offsets);
void scb_fastx_free(scb_fastx* f);

/* ---------------------------------------------------------------------------------------
 * Serving: a request loop over a frozen, device-resident index (no counterpart in the
 * reference, whose queries run per call; this batches SuperCountingBloomIndex::
 * estimate_sequence_abundances requests, src/api.rs:250-262, as they arrive).
 * Requests are split into pieces of whole sequences; pending pieces are packed into batches
 * of at most max_batch_bytes / max_batch_seqs and run on one of several slots (streams with
 * their own device buffers) as soon as a slot is free, so batches overlap on the GPU.  The
 * number of slots is min(max_inflight, memory_budget_bytes / bytes of one slot): the budget
 * admits work.  Results are bit-identical to scb_query_batch on the same request.
 * --------------------------------------------------------------------------------------- */
typedef struct scb_server scb_server;
typedef struct scb_server_config {
    uint64_t memory_budget_bytes; /* device bytes for in-flight batches (0: max_inflight slots) */
    uint64_t max_batch_bytes;     /* sequence bytes per batch (default 64 MiB, at most 1 GiB) */
    uint64_t max_batch_seqs;      /* sequences per batch (default max_batch_bytes / 64) */
    uint32_t max_inflight;        /* batches on the GPU at once (default 4) */
    uint32_t reserved;
    /* distinct k-mers the whole-stream spectrum can hold (0: no spectrum).  The server keeps a
     * device set of twice that many (rounded up to a power of two) 8-byte keys beside the slots,
     * outside memory_budget_bytes; every batch also adds its windows' canonical k-mers to it. */
    uint64_t spectrum_keys;
} scb_server_config;
typedef struct scb_request_stats {
    double queue_ms;   /* submit -> first piece launched */
    double service_ms; /* first piece launched -> results written */
    double total_ms;   /* submit -> results written */
    uint64_t windows;
} scb_request_stats;
typedef struct scb_server_summary {
    uint64_t requests; /* completed since the last reset */
    uint64_t windows;
    uint64_t batches;
    double p50_ms, p99_ms, mean_ms, max_ms; /* submit -> results written */
    double span_s;                          /* first submit -> last completion */
    uint32_t slots;
    uint32_t reserved;
} scb_server_summary;
scb_status scb_server_create(scb_ctx* index, const scb_server_config* cfg, scb_server** out);
/* Queues a request; host buffers stay owned by the caller and must stay valid until
 * scb_server_wait(ticket) returns.  Outputs are laid out as for scb_query_batch. */
scb_status scb_server_submit(scb_server* s, const uint8_t* seqs, const uint64_t* offsets, uint64_t n_seqs,
                             uint64_t* abundances, uint8_t* valid, uint64_t* ticket);
scb_status scb_server_wait(scb_server* s, uint64_t ticket, scb_request_stats* stats);
scb_status scb_server_get_summary(scb_server* s, scb_server_summary* out);
/* Clears the latency statistics and the whole-stream spectrum (call it with no request in flight). */
scb_status scb_server_reset_stats(scb_server* s);
/* The whole stream's distinct-k-mer spectrum: estimate_distinct_kmers + spectrum_from_estimates
 * (src/fastx.rs:255-308, 392-410) over every sequence the server answered since it was created or
 * last reset: value -> number of distinct canonical k-mers with that estimate, rows sorted by
 * value, same two-call convention as scb_spectrum_distinct.  Waits for the batches in flight.
 * Needs spectrum_keys > 0; a stream with more distinct k-mers than the set holds fails with
 * SCB_ERR_INTERNAL_STATE (device status word 2). */
scb_status scb_server_spectrum(scb_server* s, uint64_t* values, uint64_t* counts, uint64_t capacity,
                               uint64_t* n_rows, uint64_t* distinct_keys, uint64_t* queried_kmers);
/* Graphs captured (one per slot and shape class) and batches replayed through them.  A server
 * uses graphs when its index context had them on at scb_server_create (scb_set_graphs). */
scb_status scb_server_graph_stats(scb_server* s, uint64_t* captures, uint64_t* replays);
/* Drains in-flight batches, then frees the server (not the index). */
void scb_server_destroy(scb_server* s);

/* ---------------------------------------------------------------------------------------
 * Autotuner (no counterpart in the reference).  Measures, on a sample of the caller's reads and
 * a scratch table of the same geometry (the context's own table is not touched), the insert and
 * query strategies for small and large batches (shared-memory staging of grouped blocks versus
 * direct CAS atomics versus the plain pipeline), the grouped pipeline's records per bucket and
 * apply CTA width (warps per work item), and the batch size of host calls (reads per batch).
 * The result applies to the context's SCB_STRATEGY_AUTO and to every context created later in
 * the process with the same (counter_bits, block_slots_exponent, counter_slots_exponent, k, m,
 * s, n_hashes).  Results never change counters or estimates, only speed.
 * --------------------------------------------------------------------------------------- */
typedef struct scb_tuning {
    uint64_t small_batch_bytes; /* batches below this use the *_small strategies */
    int32_t insert_small, insert_large, query_small, query_large; /* scb_strategy values */
    uint32_t bucket_records;  /* grouped: target super-k-mer records per bucket */
    uint32_t apply_threads;   /* grouped: threads per apply CTA */
    uint64_t host_batch_bytes; /* sequence bytes per device batch of a host call */
    double insert_ms, query_ms; /* best times on the sample */
    uint32_t candidates;       /* configurations measured */
    uint32_t reserved;
} scb_tuning;
scb_status scb_autotune(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n_seqs,
                        scb_tuning* out);
scb_status scb_get_tuning(const scb_ctx* ctx, scb_tuning* out);

/* Clears the counter table and the insert totals and makes the context a builder again
 * (SuperCountingBloomBuilder::new on the existing allocation). */
scb_status scb_reset(scb_ctx* ctx);

#ifdef __cplusplus
}
#endif

#endif /* SCB_H */
