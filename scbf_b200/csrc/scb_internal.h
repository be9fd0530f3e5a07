// Internal host-side types shared by the C ABI (scb_api.cu) and the serving loop (scb_server.cu):
// error reporting, device buffers, the per-context staging lane and the context itself.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/scb.h"
#include "scb_kernels.cuh"

namespace scb {

// Thread-local text of the last failure (scb_last_error).
inline std::string& last_error_slot() {
    thread_local std::string s;
    return s;
}

inline scb_status fail(scb_status st, const std::string& msg) {
    last_error_slot() = msg;
    return st;
}

inline const char* kind_prefix(scb_status st) {
    switch (st) {
        case SCB_ERR_INVALID_CONFIG: return "invalid config: ";
        case SCB_ERR_INVALID_INDEX_FORMAT: return "invalid index format: ";
        case SCB_ERR_INTERNAL_STATE: return "internal state error: ";
        case SCB_ERR_IO: return "I/O error for ";
        default: return "";
    }
}

inline scb_status fail_kind(scb_status st, const std::string& msg) {
    return fail(st, std::string(kind_prefix(st)) + msg);
}

#define SCB_CUDA(call)                                                                                    \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) {                                                                          \
            return ::scb::fail_kind(SCB_ERR_INTERNAL_STATE, std::string(#call) + ": " + cudaGetErrorString(e_)); \
        }                                                                                                 \
    } while (0)

#define SCB_TRY(expr)                \
    do {                             \
        scb_status s_ = (expr);      \
        if (s_ != SCB_OK) return s_; \
    } while (0)

// Grow-only device buffer.
struct DevBuf {
    void* p = nullptr;
    size_t cap = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
    scb_status ensure(size_t bytes) {
        if (bytes <= cap) return SCB_OK;
        if (p) {
            cudaFree(p);
            p = nullptr;
            cap = 0;
        }
        size_t want = std::max<size_t>(bytes, 256);
        cudaError_t e = cudaMalloc(&p, want);
        if (e != cudaSuccess) {
            p = nullptr;
            return fail_kind(SCB_ERR_INTERNAL_STATE,
                             "device allocation of " + std::to_string(want) + " bytes failed: " + cudaGetErrorString(e));
        }
        cap = want;
        return SCB_OK;
    }
    template <typename T>
    T* as() const {
        return reinterpret_cast<T*>(p);
    }
};

// Largest batch the kernels index with 32-bit positions.
constexpr uint64_t kMaxBatchBytes = (1ull << 31);

// Prepared grouped batch of a lane: sorted records and work items for the lane's current codes.
struct GroupedState {
    bool valid = false;
    bool probes_written = false;  // the insert apply stored every s-mer's probe slots
    bool built = false;           // a build apply answered its items' queries and listed the rest
    uint64_t probe_cap = 0;
    uint32_t shift = 0;
    uint64_t n_buckets = 0, max_items = 0, produced = 0;
    GroupArgs ga{};
};

// Timing events of a lane: which spans the current batch recorded (read_counters adds them up).
enum TimedSpan : uint32_t {
    kSpanPack = 1,          // ev 0 -> 1
    kSpanInsert = 2,        // ev 2 -> 3
    kSpanCut = 4,           // ev 4 -> 5 cut, 5 -> 6 bucketing
    kSpanApplyInsert = 8,   // ev 7 -> 8
    kSpanQuery = 16,        // ev 9 -> 10
    kSpanApplyQuery = 32,   // ev 11 -> 12
};
constexpr int kLaneEvents = 13;

// Byte class of a grouped graph: bytes rounded up to four steps per octave (at least 64 KiB).
inline uint64_t class_bytes(uint64_t n) {
    if (n <= (64u << 10)) return 64u << 10;
    const uint32_t e = 63u - (uint32_t)__builtin_clzll(n - 1);  // 2^e <= n - 1 < 2^(e + 1)
    const uint64_t step = 1ull << (e - 2);
    return ((n + step - 1) / step) * step;
}

// Kinds of batch a lane runs, eagerly or as a replay of a captured graph.
// kBatchInsertKeep inserts and keeps the batch's records and probe slots in its lane, and
// kBatchReportKept queries them after the table is complete (a build + stream query split into
// pieces, each on its own lane).
enum BatchKind : int {
    kBatchInsert = 1,
    kBatchReport = 2,
    kBatchBuildStream = 3,
    kBatchInsertKeep = 4,
    kBatchReportKept = 5
};
inline bool kind_inserts(int kind) { return kind == kBatchInsert || kind == kBatchBuildStream || kind == kBatchInsertKeep; }
inline bool kind_queries(int kind) { return kind == kBatchReport || kind == kBatchBuildStream || kind == kBatchReportKept; }

// Shape class of a graph: batch kind, strategies, byte capacity and the grouped pipeline's
// sizes, plus a signature of the lane buffers the graph's nodes point at.
struct GraphKey {
    int kind = 0, s_ins = 0, s_query = 0;
    uint64_t cap_bytes = 0, rec_cap = 0, bucket_cap = 0, max_items = 0, n_buckets = 0, probe_cap = 0;
    uint32_t shift = 0, apply_threads = 0;
    bool fused = false;  // a grouped build + stream query in one build apply (plus deferred items)
    bool prepacked = false;  // the batch's codes and bitmap came packed from the host
    uint64_t sig = 0;
    bool operator==(const GraphKey& o) const {
        return kind == o.kind && s_ins == o.s_ins && s_query == o.s_query && fused == o.fused &&
               prepacked == o.prepacked &&
               cap_bytes == o.cap_bytes && rec_cap == o.rec_cap && bucket_cap == o.bucket_cap &&
               probe_cap == o.probe_cap &&
               max_items == o.max_items && n_buckets == o.n_buckets && shift == o.shift &&
               apply_threads == o.apply_threads && sig == o.sig;
    }
};

struct GraphEntry {
    GraphKey key;
    cudaGraphExec_t exec = nullptr;
    uint64_t launches = 0;  // kernels per replay
    uint64_t last_use = 0;
};

// Derived per-batch arrays (codes, bitmaps, window offsets, plain-pipeline arrays, counters).
struct Lane {
    DevBuf ascii, offsets, codes, valid, seqstart, woff, scan, wblock, wend, cnt, cnt2, tiles, params;
    // grouped pipeline: records, bucket offsets / cursors, work items
    DevBuf rec_key, rec_val, rec_sorted, bhist, bcursor, icount, items, gscan, rec_count;
    DevBuf rec_bases, rec_sbases;  // 16-byte base entries of the overflow and the sorted records
    // probe slots kept from a grouped insert for the query of the same records (build + stream)
    DevBuf probes, item_base;
    // items a build apply leaves to the query kernel, with their probe-slot bases (the count is
    // rec_count[2])
    DevBuf ditems, ditem_base;
    DevBuf kept;  // the build apply's per-CTA probe words (kKeptSmers per CTA)
    // a host per-window query's outputs: u64 estimates, validity bytes, and the estimates narrowed
    // to the counters' width for the copy to the host
    DevBuf qout, qvalid, qnarrow;
    bool want_probes = false;
    bool want_build = false;  // the grouped insert of this batch is a build apply
    bool want_spectrum = false;  // buckets sized for the spectrum apply
    // codes and valid hold the batch already (packed on the host and copied), so the batch skips
    // the device packing kernel
    bool prepacked = false;
    cudaStream_t stream = nullptr;
    GroupedState gs;
    cudaEvent_t ev[kLaneEvents] = {};
    uint32_t spans = 0;
    // captured graphs of this lane by shape class and the record capacity learned from
    // overflowing replays
    std::vector<GraphEntry> graphs;
    uint64_t rec_hint = 0;
    bool recording = false;  // a stream capture of this lane is in progress
    // records and probe slots kept by a kBatchInsertKeep replay of this key for kBatchReportKept
    bool kept_graph = false;
    GraphKey kept_key;
    uint64_t graph_clock = 0, captures = 0, replays = 0, graph_fallbacks = 0;
    ~Lane() {
        for (auto& g : graphs) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
        }
        for (auto& e : ev) {
            if (e) cudaEventDestroy(e);
        }
        if (stream) cudaStreamDestroy(stream);
    }
};

// Choices of the autotuner (scb_autotune) for one geometry; defaults until tuned.
struct Tuning {
    bool valid = false;
    uint64_t small_bytes = 0;  // batches below this many bytes use the *_small strategies
    scb_strategy insert_small = SCB_STRATEGY_FUSED, insert_large = SCB_STRATEGY_GROUPED;
    scb_strategy query_small = SCB_STRATEGY_FUSED, query_large = SCB_STRATEGY_GROUPED;
    uint32_t bucket_records = 512;  // grouped: target super-k-mer records per bucket
    uint32_t apply_threads = 256;   // grouped: CTA width of the apply kernel
    uint64_t host_batch_bytes = kMaxBatchBytes - 64;  // sequence bytes per batch of a host call
};

// Narrows u64 per-window estimates to `width` (2 or 4) bytes each for a copy to the host: the
// first n entries, or bp->n_bytes of them when bp is given (graph replays).
void launch_narrow_out(const BatchParams* bp, uint64_t n, const unsigned long long* out, void* outn, uint32_t width,
                       int sm_count, cudaStream_t st);

// Packs n sequence bytes on the host into the device layout of kernel (a) (codes: 16 bases per
// 32-bit word; valid: 32 bases per word; kPadWords zero words after each), on up to `threads`
// threads (scb_hostpack.cpp).
void host_pack(const uint8_t* ascii, uint64_t n, uint32_t* codes, uint32_t* valid, unsigned threads);

}  // namespace scb

struct scb_ctx {
    scb_config cfg{};
    scb::DevGeom g{};
    // FrozenFilterLayout (filter.rs:77-116)
    uint64_t shard_count = 0, subblocks = 0, block_slots = 0, shard_mask = 0, block_slots_mask = 0, nb_blocks = 0,
             block_mask = 0;
    uint32_t shard_shift = 0;
    int device = 0;
    int sm_count = 148;
    void* table = nullptr;
    uint64_t table_bytes = 0;
    uint32_t* status = nullptr;
    bool frozen = false;
    uint64_t inserted_kmers = 0, inserted_smers = 0;
    scb_strategy insert_strategy = SCB_STRATEGY_AUTO, query_strategy = SCB_STRATEGY_AUTO;
    scb::Tuning tuning;
    scb::Lane lane;
    // a host build + stream query in pieces: one lane per piece, uploads on their own stream
    std::vector<std::unique_ptr<scb::Lane>> piece_lanes;
    cudaStream_t copy_stream = nullptr;
    std::vector<cudaEvent_t> piece_events;
    uint64_t piece_bytes = 0;  // 0: the default
    // host packing of the pieces (scb_set_host_pack): two pinned staging areas, each the codes and
    // valid words of the largest piece, reused once the copy that read them (stage_free) is done
    bool host_pack = true;
    uint32_t* stage_codes[2] = {nullptr, nullptr};
    uint32_t* stage_valid[2] = {nullptr, nullptr};
    uint64_t stage_groups = 0;
    cudaEvent_t stage_free[2] = {nullptr, nullptr};
    uint64_t h2d_bytes = 0;  // bytes the host entry points copied to the device (scb_h2d_bytes)
    // the distinct-k-mer spectrum's key set, dense histogram and overflow list (grown as needed)
    scb::DevBuf spec_set, spec_hist, spec_ovf;
    // pinned staging of a host per-window query's narrowed estimates and validity bytes
    uint8_t* q_stage = nullptr;
    uint64_t q_stage_bytes = 0;
    bool timing = false;
    bool graphs = true;  // replay batches through graphs captured per shape class
    bool fused_build = true;  // a grouped build + stream query answers exclusive buckets in its insert
    scb_timings times{};
    std::mutex mu;
    ~scb_ctx() {
        if (copy_stream) cudaStreamSynchronize(copy_stream);
        if (lane.stream) cudaStreamSynchronize(lane.stream);
        if (q_stage) cudaFreeHost(q_stage);
        for (int i = 0; i < 2; i++) {
            if (stage_codes[i]) cudaFreeHost(stage_codes[i]);
            if (stage_valid[i]) cudaFreeHost(stage_valid[i]);
            if (stage_free[i]) cudaEventDestroy(stage_free[i]);
        }
        for (auto e : piece_events) cudaEventDestroy(e);
        if (copy_stream) cudaStreamDestroy(copy_stream);
        piece_lanes.clear();
        if (table) cudaFree(table);
        if (status) cudaFree(status);
    }
};
