// Internal host-side types shared by the C ABI (scb_api.cu) and the serving loop (scb_server.cu):
// error reporting, device buffers, the per-context staging lane and the context itself.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <string>

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
constexpr uint64_t kPadWords = 16;

// Prepared grouped batch of a lane: sorted records and work items for the lane's current codes.
struct GroupedState {
    bool valid = false;
    uint32_t shift = 0;
    uint64_t n_buckets = 0, max_items = 0, produced = 0;
    GroupArgs ga{};
};

// Derived per-batch arrays (codes, bitmaps, window offsets, plain-pipeline arrays, counters).
struct Lane {
    DevBuf ascii, offsets, codes, valid, seqstart, woff, scan, wblock, wend, cnt, tiles;
    // grouped pipeline: records, bucket offsets / cursors, work items
    DevBuf rec_key, rec_val, rec_sorted, bhist, bcursor, icount, items, gscan, rec_count;
    cudaStream_t stream = nullptr;
    GroupedState gs;
    // stage timing: [0,1] pack, [2,3] main stage (main_kind 1 = insert, 2 = query),
    // [4,5,6] grouped cut start / cut end / prepare end, [7,8] apply start / end
    cudaEvent_t ev[9] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    bool pack_timed = false;
    bool cut_timed = false;
    int main_kind = 0;
    int grouped_kind = 0;
    ~Lane() {
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
    bool timing = false;
    scb_timings times{};
    std::mutex mu;
    ~scb_ctx() {
        if (table) cudaFree(table);
        if (status) cudaFree(status);
    }
};
