// Kernel launch interface shared by the C ABI implementation (scb_api.cu) and the kernels
// (scb_kernels.cu).  Host-only declarations; device code lives in scb_kernels.cu.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "scb_device.cuh"

namespace scb {

// Zero words kept after a batch's codes and bitmaps (reads that run past the last base).
constexpr uint64_t kPadWords = 16;

// Tile geometry of the fused kernels: windows per tile and threads per CTA.
constexpr int kTileWindows = 1024;
constexpr int kTileThreads = 256;

enum TileMode : int {
    kModeInsert = 0,       // (b)+(c)+(d): cut, hash, saturating insert
    kModeReport = 1,       // (b)+(c)+(e): query, reduce to the QueryFastaReport fields
    kModeAbund = 2,        // (b)+(c)+(e): query, per-window abundances
    kModeDistinct = 3,     // (b)+(c)+(e)+(f): query, distinct-k-mer set and histogram
    kModeStats = 4,        // super-k-mer / s-mer / sector counts
    kModeDebugMin = 5,     // (b) only: chosen minimizer position per window
    kModeMaterialize = 6,  // (b) for the plain pipeline: per-window block id + end flag in HBM
    kModeInsertStaged = 7, // (b)+(c)+(d) with one warp per super-k-mer staging block deltas
    kModeCut = 8,          // (b) for the grouped pipeline: one record per super-k-mer + bucket counts
    kModeBuild = 9,        // grouped apply of a build + stream query: insert a bucket's records, commit,
                           // then answer the same records' query from the committed shared-memory block
    kModeSpectrum = 10,    // grouped distinct-k-mer spectrum: a bucket's windows' estimates from its staged
                           // blocks, their canonical k-mers deduplicated in shared memory
    kModeAbundDistinct = 11  // kModeAbund and kModeDistinct from one estimate per window (a serving batch
                             // that also feeds the whole-stream spectrum)
};

// Sizes and input pointers of one batch, in device memory: a graph captured for a shape class
// reads them at replay, so one graph serves every batch of its class.
struct BatchParams {
    uint64_t n_bytes;
    uint64_t n_seqs;
    const uint8_t* ascii;
    const uint64_t* offsets;
};

// Grouped pipeline: super-k-mer records bucketed by counter block.
// Overflow record: key = block id, val = first window position | windows << 32.
// Sorted record:   val = first window position | windows << 32 | block-in-bucket << 38.
// Record bases:    the super-k-mer's 2-bit codes from its first window's first base, 64 bases
//                  (at most w + k - 1 <= 63 are its own) in one 16-byte entry per record, slot for
//                  slot beside the overflow list and the sorted records.
constexpr uint32_t kRecWindowsShift = 32;
constexpr uint32_t kRecLocalShift = 38;
constexpr uint32_t kItemRecords = 4096;    // records per work item (heavier buckets are split)
constexpr uint32_t kApplyChunk = 256;      // records staged in shared memory at a time (<= CTA width)
constexpr uint32_t kMaxBucketSlots = 16384;  // counters of one bucket held in shared memory
constexpr uint32_t kApplyMaxThreads = 512;
// s-mers of one work item whose probe slots a build apply keeps between its insert and its query,
// in its CTA's region of a small global scratch that stays in L2 (items with more are deferred to
// the query kernel)
constexpr uint32_t kKeptSmers = 8192;
// CTAs per SM the kept scratch has room for (2048 threads of 256-thread CTAs)
constexpr uint32_t kKeptCtasPerSm = 8;
// spectrum apply: largest shared-memory key set of a work item (items with more than half as
// many windows use the global set) and the estimates histogrammed in shared memory per CTA
constexpr uint32_t kSpecSet = 8192;
constexpr uint32_t kSpecBins = 1024;

struct GroupArgs {
    DevGeom g;
    const uint32_t* codes;
    uint64_t n_code_words;
    void* table;
    uint32_t* status;
    unsigned long long* cnt;
    const unsigned long long* recs;  // sorted records
    const uint4* sbases;             // their bases, slot for slot
    const uint4* items;              // {bucket, first record, records, exclusive}
    const unsigned long long* n_items;
    unsigned int* work_counter;
    uint32_t bucket_shift;
    uint32_t apply_threads;  // CTA width of the apply kernel: 256 (default) or 512
    // record slots the cut reserved and the capacity it had: when the count exceeds the capacity
    // (a graph replay whose records outgrew its class) the apply does nothing and the host redoes
    // the batch with room for every record
    const unsigned long long* rec_count;
    uint64_t rec_cap;
    // probe slots of every s-mer (n_hashes <= 4 bucket-cell indices, 16-bit lanes),
    // written by an insert and read back by a query of the same records, which then skips the
    // hashing.  item_base[i] = first entry of work item i, kNoProbes when the array was full (that
    // item's query hashes again).  probes = nullptr: hash in every pass.
    unsigned long long* probes;
    unsigned long long* item_base;
    unsigned long long* probe_count;
    uint64_t probe_cap;
    // build apply (kModeBuild): the report counters of the items it answers itself, and the list
    // of items it leaves to the query kernel (split buckets, items of more than kKeptSmers
    // s-mers) with their probe-slot bases; dcount counts them
    unsigned long long* qcnt;
    uint4* ditems;
    unsigned long long* ditem_base;
    unsigned long long* dcount;
    unsigned long long* kept;  // kKeptSmers probe words per CTA, for kept_ctas CTAs
    uint32_t kept_ctas;
    uint32_t pad0_;
    // spectrum apply (kModeSpectrum): the global key set for items that cannot deduplicate in
    // shared memory, the dense histogram [0, hist_dense) and the overflow list of larger values
    unsigned long long* set_keys;
    uint64_t set_mask;
    unsigned long long* hist;
    uint32_t hist_dense;
    uint32_t pad_;
    unsigned long long* ovf;
    uint64_t ovf_cap;
};
constexpr unsigned long long kNoProbes = ~0ull;

// Slots of the per-launch 64-bit counter array.
enum CounterSlot : int {
    kCntWindows = 0,
    kCntSmers = 1,
    kCntValid = 2,
    kCntPositive = 3,
    kCntChecksum = 4,
    kCntSuperKmers = 5,
    kCntSectors = 6,
    kCntDistinct = 7,
    kCntOverflow = 8,
    kCntRecords = 9,
    kCntTotalWindows = 10,
    kCntSlots = 16
};

struct TileArgs {
    DevGeom g;
    const uint32_t* codes;     // 2-bit codes (+ >= 4 zero words of padding)
    const uint32_t* valid;     // valid bitmap (+ >= 4 zero words of padding)
    const uint32_t* seqstart;  // sequence-start bitmap (+ padding)
    uint64_t n_bytes;
    uint64_t n_code_words;     // readable words (including padding)
    uint64_t n_bit_words;
    uint32_t n_tiles;
    uint32_t pad_;
    void* table;
    uint32_t* status;
    unsigned long long* cnt;   // kCntSlots counters
    unsigned int* tile_counter;
    // per-window abundances (kModeAbund)
    const uint64_t* offsets;
    uint64_t n_seqs;
    const uint64_t* woff;      // first output window of each sequence
    unsigned long long* out;
    uint8_t* out_valid;
    // distinct-k-mer spectrum (kModeDistinct)
    unsigned long long* set_keys;
    uint64_t set_mask;
    unsigned long long* hist;  // dense bins [0, hist_dense)
    uint32_t hist_dense;
    uint32_t pad2_;
    unsigned long long* ovf;   // values >= hist_dense of newly seen keys
    uint64_t ovf_cap;
    // plain pipeline (kModeMaterialize) and debug output
    uint32_t* wblock;
    uint8_t* wend;
    uint32_t* dbg;
    // grouped pipeline (kModeCut): records go to their bucket's region of bucket_cap slots in
    // sorted (bucket_hist counts them per bucket), the rest to the overflow list rec_key / rec_val
    // of rec_cap entries (rec_count counts them)
    uint32_t* rec_key;
    unsigned long long* rec_val;
    unsigned long long* rec_count;
    uint64_t rec_cap;
    unsigned long long* bucket_hist;
    uint32_t bucket_shift;
    uint32_t pad3_;
    unsigned long long* sorted;
    uint64_t bucket_cap;
    uint4* sbases;     // bases of the records in sorted, slot for slot
    uint4* rec_bases;  // bases of the overflow records
    // when set, n_bytes / n_seqs / offsets come from here at run time (graph replays) and the
    // fields above give the capacity of the batch's shape class
    const BatchParams* dyn;
};

// Kernel launches; each counts itself in the library-wide launch counter.
void launch_pack(const uint8_t* ascii, uint64_t n_bytes, uint32_t* codes, uint32_t* valid, cudaStream_t st);
// Graph-replayable forms: the batch's sizes and input pointers come from a BatchParams block in
// device memory; grids are fixed (grid-stride loops over the batch), so one capture serves any
// batch that fits the buffers.  The out / out_valid buffers of launch_clear_dyn need 16-byte
// alignment and room for n_bytes rounded up to 16.
void launch_set_params(BatchParams* bp, const BatchParams& v, cudaStream_t st);
void launch_pack_dyn(const BatchParams* bp, uint32_t* codes, uint32_t* valid, int sm_count, cudaStream_t st);
void launch_clear_dyn(const BatchParams* bp, uint32_t* seqstart, unsigned long long* out, uint8_t* out_valid,
                      int sm_count, cudaStream_t st);
void launch_seqstart_dyn(const BatchParams* bp, uint32_t* seqstart, int sm_count, cudaStream_t st);
void launch_seq_windows_dyn(const BatchParams* bp, uint32_t k, unsigned long long* cnt, int sm_count,
                            cudaStream_t st);
void launch_seqstart(const uint64_t* offsets, uint64_t n_seqs, uint64_t n_bytes, uint32_t* seqstart,
                     cudaStream_t st);
void launch_seq_windows(const uint64_t* offsets, uint64_t n_seqs, uint32_t k, unsigned long long* cnt,
                        uint64_t* woff_or_null, cudaStream_t st);
void launch_scan_inplace(uint64_t* data, uint64_t n, uint64_t* scratch, cudaStream_t st);
void launch_tiles(int mode, const TileArgs& a, int grid, cudaStream_t st);
int tile_grid(int mode, int bits, int sm_count, uint32_t n_tiles);
void launch_plain_insert(const TileArgs& a, cudaStream_t st);
void launch_plain_query(int mode, const TileArgs& a, cudaStream_t st);
void launch_counter_hist(const void* table, uint64_t slots, int bits, unsigned long long* hist, uint32_t dense,
                         unsigned long long* ovf, uint64_t ovf_cap, unsigned long long* ovf_count, cudaStream_t st);
void launch_fill_u32(uint32_t* p, uint32_t v, uint64_t n, cudaStream_t st);
// grouped pipeline
void launch_scatter(const uint32_t* rec_key, const unsigned long long* rec_val, const uint4* rec_bases,
                    const unsigned long long* rec_count, uint64_t rec_cap, uint32_t bucket_shift,
                    unsigned long long* cursor, uint64_t base, unsigned long long* sorted, uint4* sbases,
                    cudaStream_t st);
void launch_item_counts(const unsigned long long* counts, uint64_t n_buckets, uint64_t bucket_cap, uint64_t* item_count,
                        uint64_t* ovf_count, const unsigned long long* rec_count, uint64_t rec_cap, cudaStream_t st);
void launch_item_write(const unsigned long long* counts, uint64_t bucket_cap, const uint64_t* item_off,
                       const uint64_t* ovf_off, uint64_t ovf_base, uint64_t n_buckets, uint4* items,
                       cudaStream_t st);
void launch_apply(int mode, const GroupArgs& a, int block_slots, uint32_t bucket_blocks, int sm_count,
                  uint64_t max_items, cudaStream_t st);
void launch_shared_item_windows(const uint4* items, const unsigned long long* n_items, const unsigned long long* recs,
                                unsigned long long* out, cudaStream_t st);

uint64_t kernel_launch_count();
void note_launch();
void note_launches(uint64_t n);  // kernels of one graph replay
// Counts this thread's launches into *counter instead (a graph being recorded); nullptr ends it.
void record_launches_into(uint64_t* counter);

}  // namespace scb
