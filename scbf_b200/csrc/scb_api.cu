// C ABI of the B200 SuperCountingBloom library: context lifecycle, batch staging, kernel
// pipelines per strategy, .scb save/load.  See include/scb.h for the contract of each entry.
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <memory>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <map>
#include <tuple>
#include <vector>

#include "../../include/scb.h"
#include "scb_internal.h"

using namespace scb;

namespace {

uint32_t log2u(uint64_t v) {
    uint32_t r = 0;
    while ((1ull << r) < v) r++;
    return r;
}

// config.rs:50-92 and filter.rs:96-100, with the reference's messages.
scb_status validate_config(const scb_config* c) {
    if (!c) return fail_kind(SCB_ERR_INVALID_CONFIG, "null config");
    if (c->k == 0 || c->k > 32) return fail_kind(SCB_ERR_INVALID_CONFIG, "k must be in 1..=32");
    if (c->m == 0 || c->m > c->k) return fail_kind(SCB_ERR_INVALID_CONFIG, "m must be in 1..=k");
    if (c->s == 0 || c->s > c->k || c->s > 32) return fail_kind(SCB_ERR_INVALID_CONFIG, "s must be in 1..=k and <= 32");
    if (c->k % 2 == 0) return fail_kind(SCB_ERR_INVALID_CONFIG, "canonical SIMD minimizers require odd k");
    if (c->n_hashes == 0) return fail_kind(SCB_ERR_INVALID_CONFIG, "n_hashes must be positive");
    if (c->block_slots_exponent >= c->counter_slots_exponent)
        return fail_kind(SCB_ERR_INVALID_CONFIG, "block_slots_exponent must be smaller than counter_slots_exponent");
    if (c->threads == 0) return fail_kind(SCB_ERR_INVALID_CONFIG, "threads must be positive");
    if (c->queue == 0) return fail_kind(SCB_ERR_INVALID_CONFIG, "queue must be positive");
    if (c->counter_bits != 8 && c->counter_bits != 16 && c->counter_bits != 32)
        return fail_kind(SCB_ERR_INVALID_CONFIG, "unsupported counter width");
    if (c->counter_slots_exponent >= 64) return fail_kind(SCB_ERR_INVALID_CONFIG, "counter_slots_exponent is too large");
    return SCB_OK;
}

// Device limits of this implementation (beyond the reference's rules).
scb_status device_limits(const scb_config* c) {
    if (c->counter_slots_exponent - c->block_slots_exponent > 32)
        return fail_kind(SCB_ERR_INVALID_CONFIG, "more than 2^32 blocks is beyond the device table limit");
    if (c->counter_slots_exponent > 37)
        return fail_kind(SCB_ERR_INVALID_CONFIG, "counter_slots_exponent above 37 exceeds device memory");
    return SCB_OK;
}

void fill_geometry(scb_ctx* ctx) {
    const scb_config& c = ctx->cfg;
    const uint64_t slots = 1ull << c.counter_slots_exponent;
    ctx->block_slots = 1ull << c.block_slots_exponent;
    ctx->nb_blocks = slots / ctx->block_slots;
    ctx->shard_count = std::min<uint64_t>(ctx->nb_blocks, 1024);
    ctx->subblocks = ctx->nb_blocks / ctx->shard_count;
    ctx->shard_mask = ctx->shard_count - 1;
    ctx->shard_shift = log2u(ctx->shard_count);
    ctx->block_slots_mask = ctx->block_slots - 1;
    ctx->block_mask = ctx->nb_blocks - 1;
    ctx->table_bytes = slots * (c.counter_bits / 8);
    DevGeom& g = ctx->g;
    g.k = (uint32_t)c.k;
    g.m = (uint32_t)c.m;
    g.s = (uint32_t)c.s;
    g.h = (uint32_t)c.n_hashes;
    g.w = (uint32_t)(c.k - c.m + 1);
    g.bits = c.counter_bits;
    g.block_log2 = c.block_slots_exponent;
    g.shard_shift = ctx->shard_shift;
    g.sub_log2 = log2u(ctx->subblocks);
    g.block_mask = ctx->block_mask;
    g.shard_mask = ctx->shard_mask;
    g.bs_mask = ctx->block_slots_mask;
}

scb_status check_offsets(const uint64_t* offsets, uint64_t n) {
    if (!offsets) return fail_kind(SCB_ERR_INTERNAL_STATE, "null offsets");
    // branch-free (vectorised) and, for millions of sequences, split over host threads: one
    // thread streams offsets at about 10 GB/s, which alone would cost ~10 ms per 13 M reads
    auto scan = [offsets](uint64_t a, uint64_t b) {
        uint64_t bad = 0;
        for (uint64_t i = a; i < b; i++) bad |= (uint64_t)(offsets[i + 1] < offsets[i]);
        return bad;
    };
    const uint64_t parts = n < (1u << 20) ? 1 : std::min<uint64_t>(8, std::max(1u, std::thread::hardware_concurrency()));
    uint64_t bad = 0;
    if (parts == 1) {
        bad = scan(0, n);
    } else {
        std::vector<uint64_t> res(parts, 0);
        std::vector<std::thread> th;
        for (uint64_t t = 0; t < parts; t++) {
            th.emplace_back([&, t] { res[t] = scan(n * t / parts, n * (t + 1) / parts); });
        }
        for (auto& x : th) x.join();
        for (uint64_t r : res) bad |= r;
    }
    if (bad) return fail_kind(SCB_ERR_INTERNAL_STATE, "offsets must be non-decreasing");
    return SCB_OK;
}

uint64_t windows_of(const uint64_t* offsets, uint64_t n, uint64_t k) {
    uint64_t w = 0;
    for (uint64_t i = 0; i < n; i++) {
        const uint64_t len = offsets[i + 1] - offsets[i];
        if (len >= k) w += len + 1 - k;
    }
    return w;
}

// A contiguous range of whole sequences processed as one device batch.
struct Chunk {
    uint64_t seq0, seq1;    // sequences [seq0, seq1)
    uint64_t byte0, byte1;  // bytes [byte0, byte1) of the caller's buffer
    uint64_t win0;          // first output window of the chunk
};

// Pieces of whole sequences for an upload pipeline: the first about cap / 1.3^3 bytes and each
// next 1.3x larger, up to cap, so the first copy (which no work overlaps) is short while later
// copies stay ahead of the work on the pieces before them; a tail under cap / 4 joins the piece
// before it.  One longer sequence goes alone.
uint64_t ramp_cap(uint64_t cap) { return std::max<uint64_t>(std::min<uint64_t>(cap, kMaxBatchBytes - 64), 1); }
double ramp_first(uint64_t cap) { return (double)ramp_cap(cap) / (1.3 * 1.3 * 1.3); }

scb_status plan_ramp(const uint64_t* offsets, uint64_t n, uint64_t cap, std::vector<Chunk>& out) {
    out.clear();
    const uint64_t end = offsets[n], lim = kMaxBatchBytes - 64;
    double size = ramp_first(cap);
    cap = ramp_cap(cap);
    uint64_t s = 0;
    while (s < n) {
        uint64_t want = (uint64_t)std::min<double>(size, (double)cap);
        const uint64_t left = end - offsets[s];
        if (left < want + cap / 4 && left <= lim) want = left;
        const uint64_t* hi = std::upper_bound(offsets + s + 1, offsets + n + 1, offsets[s] + want);
        uint64_t e = (uint64_t)(hi - offsets) - 1;  // last index with offsets[e] <= offsets[s] + want
        if (e <= s) e = s + 1;
        if (offsets[e] - offsets[s] > kMaxBatchBytes - 64)
            return fail_kind(SCB_ERR_INTERNAL_STATE, "a single sequence longer than 2 GiB is not supported");
        out.push_back(Chunk{s, e, offsets[s], offsets[e], 0});
        s = e;
        size *= 1.3;
    }
    return SCB_OK;
}

scb_status plan_chunks(const uint64_t* offsets, uint64_t n, uint64_t k, uint64_t cap, std::vector<Chunk>& out) {
    out.clear();
    uint64_t s = 0, win = 0;
    while (s < n) {
        uint64_t e = s;
        const uint64_t b0 = offsets[s];
        uint64_t w = 0;
        while (e < n && (e == s || offsets[e + 1] - b0 <= cap)) {
            const uint64_t len = offsets[e + 1] - offsets[e];
            w += len >= k ? len + 1 - k : 0;
            e++;
        }
        if (offsets[e] - b0 > kMaxBatchBytes - 64)
            return fail_kind(SCB_ERR_INTERNAL_STATE, "a single sequence longer than 2 GiB is not supported");
        out.push_back(Chunk{s, e, b0, offsets[e], win});
        win += w;
        s = e;
    }
    return SCB_OK;
}

__global__ void k_rebase(uint64_t* off, uint64_t n, uint64_t base) {
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) off[i] -= base;
}

// Narrows a batch's u64 estimates (out, cleared past the batch's windows) to `width` bytes each
// for the copy to the host: the first n entries, or the batch's byte count (an upper bound of its
// windows) from the parameter block on graph replays.
__global__ void k_narrow_out(const BatchParams* __restrict__ bp, uint64_t n, const unsigned long long* __restrict__ out,
                             void* __restrict__ outn, uint32_t width) {
    if (bp) n = bp->n_bytes;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const unsigned long long v = __ldcs(out + i);
        if (width == 2) {
            static_cast<uint16_t*>(outn)[i] = (uint16_t)v;
        } else {
            static_cast<uint32_t*>(outn)[i] = (uint32_t)v;
        }
    }
}

// Derived arrays of a batch of n_bytes (codes, bitmaps, counters).  The input buffers (ascii,
// offsets) are left alone: they may hold an uploaded batch.
scb_status ensure_lane_work(scb_ctx* ctx, Lane& L, uint64_t n_bytes) {
    if (!L.stream) SCB_CUDA(cudaStreamCreateWithFlags(&L.stream, cudaStreamNonBlocking));
    for (auto& e : L.ev) {
        if (!e) SCB_CUDA(cudaEventCreate(&e));
    }
    const uint64_t groups = (n_bytes + 31) / 32;
    SCB_TRY(L.codes.ensure((2 * groups + kPadWords) * 4));
    SCB_TRY(L.valid.ensure((groups + kPadWords) * 4));
    SCB_TRY(L.seqstart.ensure((groups + kPadWords) * 4));
    SCB_TRY(L.cnt.ensure(kCntSlots * 8));
    SCB_TRY(L.tiles.ensure(64));
    (void)ctx;
    return SCB_OK;
}

// Input buffers for an upload of n_bytes / n_seqs, plus the derived arrays.
scb_status ensure_lane(scb_ctx* ctx, Lane& L, uint64_t n_bytes, uint64_t n_seqs) {
    const uint64_t groups = (n_bytes + 31) / 32;
    SCB_TRY(L.ascii.ensure(groups * 32 + 64));
    SCB_TRY(L.offsets.ensure((n_seqs + 1) * 8));
    return ensure_lane_work(ctx, L, n_bytes);
}

// Records a lane timing event.  A graph always holds its events as event nodes (the external-
// record flag, valid only under capture), so every replay records them and one graph serves
// timed and untimed batches; read_counters reads them only while timing is on.
scb_status mark(const scb_ctx* ctx, Lane& L, int i, cudaStream_t st) {
    if (!ctx->timing && !L.recording) return SCB_OK;
    if (L.recording) {
        SCB_CUDA(cudaEventRecordWithFlags(L.ev[i], st, cudaEventRecordExternal));
    } else {
        SCB_CUDA(cudaEventRecord(L.ev[i], st));
    }
    return SCB_OK;
}

// Stages a device batch (ascii + rebased offsets already on the device in L) into codes,
// bitmaps and sequence starts, and fills the tile arguments.
scb_status prepare_batch(scb_ctx* ctx, Lane& L, const uint8_t* d_ascii, const uint64_t* d_offsets, uint64_t n_seqs,
                         uint64_t n_bytes, cudaStream_t st, TileArgs& a) {
    const uint64_t groups = (n_bytes + 31) / 32;
    L.gs.valid = false;
    SCB_TRY(mark(ctx, L, 0, st));
    if (!L.prepacked) {  // a prepacked lane's codes and bitmap hold the batch already
        SCB_CUDA(cudaMemsetAsync(L.codes.p, 0, (2 * groups + kPadWords) * 4, st));
        SCB_CUDA(cudaMemsetAsync(L.valid.p, 0, (groups + kPadWords) * 4, st));
        launch_pack(d_ascii, n_bytes, L.codes.as<uint32_t>(), L.valid.as<uint32_t>(), st);
    }
    SCB_CUDA(cudaMemsetAsync(L.seqstart.p, 0, (groups + kPadWords) * 4, st));
    launch_seqstart(d_offsets, n_seqs, n_bytes, L.seqstart.as<uint32_t>(), st);
    SCB_TRY(mark(ctx, L, 1, st));
    if (ctx->timing) L.spans |= kSpanPack;
    SCB_CUDA(cudaMemsetAsync(L.cnt.p, 0, kCntSlots * 8, st));
    std::memset(&a, 0, sizeof(a));
    a.g = ctx->g;
    a.codes = L.codes.as<uint32_t>();
    a.valid = L.valid.as<uint32_t>();
    a.seqstart = L.seqstart.as<uint32_t>();
    a.n_bytes = n_bytes;
    a.n_code_words = 2 * groups;
    a.n_bit_words = groups;
    a.n_tiles = (uint32_t)((n_bytes + kTileWindows - 1) / kTileWindows);
    a.table = ctx->table;
    a.status = ctx->status;
    a.cnt = L.cnt.as<unsigned long long>();
    a.tile_counter = L.tiles.as<unsigned int>();
    a.offsets = d_offsets;
    a.n_seqs = n_seqs;
    return SCB_OK;
}

bool grouped_supported(const scb_ctx* ctx) { return ctx->block_slots <= kMaxBucketSlots; }

// Expected super-k-mer records of a batch: about 2/(w+1) per window (random minimizers).
uint64_t records_estimate(const scb_ctx* ctx, uint64_t n_bytes) { return n_bytes * 2 / (ctx->g.w + 1) + 1; }

scb_strategy resolve(const scb_ctx* ctx, scb_strategy s, uint64_t n_bytes, bool insert) {
    if (s == SCB_STRATEGY_PLAIN || s == SCB_STRATEGY_FUSED) return s;
    if (s == SCB_STRATEGY_GROUPED) return grouped_supported(ctx) ? s : SCB_STRATEGY_FUSED;
    if (ctx->tuning.valid) {  // the autotuner's measured choice for this batch size
        const bool small = n_bytes < ctx->tuning.small_bytes;
        scb_strategy t = insert ? (small ? ctx->tuning.insert_small : ctx->tuning.insert_large)
                                : (small ? ctx->tuning.query_small : ctx->tuning.query_large);
        if (t == SCB_STRATEGY_GROUPED && !grouped_supported(ctx)) t = SCB_STRATEGY_FUSED;
        return t;
    }
    // untuned: grouping pays once a batch brings about one super-k-mer per two blocks
    if (grouped_supported(ctx) && records_estimate(ctx, n_bytes) >= ctx->nb_blocks / 2) return SCB_STRATEGY_GROUPED;
    return SCB_STRATEGY_FUSED;
}

scb_strategy resolve(scb_strategy s) { return s == SCB_STRATEGY_AUTO ? SCB_STRATEGY_FUSED : s; }

// Buckets of 2^shift consecutive blocks: about tuning.bucket_records (512 untuned) records per
// bucket, at most 4096 counters
// (or one block when blocks are larger) staged in shared memory.
uint32_t bucket_shift_for(const scb_ctx* ctx, uint64_t records, uint64_t target) {
    uint32_t shift = 0;
    while ((ctx->block_slots << (shift + 1)) <= 4096 && (1ull << (shift + 1)) <= ctx->nb_blocks &&
           records * (1ull << shift) / ctx->nb_blocks < target) {
        shift++;
    }
    return shift;
}

// Records per bucket of a build apply: a bucket's s-mers (about (w + 1) / 2 windows plus k - s
// per random super-k-mer) stay well inside the kept probe slots, so almost every bucket answers
// its own query.
uint64_t build_bucket_records(const scb_ctx* ctx) {
    const uint64_t per_record = (ctx->g.w + 1) / 2 + (ctx->g.k - ctx->g.s);
    return std::max<uint64_t>(kKeptSmers * 10 / (16 * std::max<uint64_t>(per_record, 1)), 1);
}

// Records per bucket of a spectrum apply: a bucket's windows (about (w + 1) / 2 per random
// super-k-mer) stay well below half the shared-memory key set.
uint64_t spectrum_bucket_records(const scb_ctx* ctx) {
    const uint64_t per_record = std::max<uint64_t>((ctx->g.w + 1) / 2, 1);
    return std::max<uint64_t>(kSpecSet / 2 * 10 / (14 * per_record), 1);
}

enum BucketTarget : int { kTargetTuned = 0, kTargetBuild = 1, kTargetSpectrum = 2 };

// Sizes of the grouped pipeline for a batch: bucket shift and count, record slots (the estimate
// with a quarter of slack, at least min_records, plus the unused tail of each CTA's last reserved
// chunk of 4096 slots) and the work-item bound for that many records.
// Sizes of the grouped pipeline for a batch: bucket shift and count; each bucket's region of
// bucket_cap record slots (1.5x the expected records per bucket plus 64, rounded to a 32-byte
// sector); the overflow list's capacity cap (records past their region: a quarter of the
// estimate plus 64 Ki, at least min_records); and the work-item bound.
struct GroupedSizes {
    uint32_t shift = 0;
    uint64_t n_buckets = 0, bucket_cap = 0, cap = 0, max_items = 0;
    uint64_t region() const { return n_buckets * bucket_cap; }
};

uint64_t items_bound(const GroupedSizes& z) {
    return z.n_buckets * ((z.bucket_cap + kItemRecords - 1) / kItemRecords) + std::min<uint64_t>(z.n_buckets, z.cap) +
           z.cap / kItemRecords + 1;
}

// Probe slots kept between the insert and the query of the same records: one 64-bit word per
// s-mer holds the bucket-cell indices of its n_hashes probes when there are at most four.  The capacity is the batch's bytes (an
// upper bound of its windows) plus k - s extra s-mers per estimated super-k-mer; items past it
// hash again in the query.
// (kept as four 16-bit lanes of bucket-cell indices; buckets hold at most 16384 counters)
bool probes_fit(const scb_ctx* ctx) { return ctx->g.h <= 4; }

// A build + stream query of one batch with the grouped strategy for both passes runs the build
// apply (kModeBuild) when probe slots fit and fusion is on.
bool build_fused(const scb_ctx* ctx, uint64_t n_bytes) {
    return ctx->fused_build && probes_fit(ctx) &&
           resolve(ctx, ctx->insert_strategy, n_bytes, true) == SCB_STRATEGY_GROUPED &&
           resolve(ctx, ctx->query_strategy, n_bytes, false) == SCB_STRATEGY_GROUPED;
}

// Build-apply buffers: the deferred-item list and the per-CTA kept probe words.
scb_status build_buffers(const scb_ctx* ctx, Lane& L, uint64_t max_items) {
    SCB_TRY(L.ditems.ensure(std::max<uint64_t>(max_items, 1) * 16));
    SCB_TRY(L.ditem_base.ensure(std::max<uint64_t>(max_items, 1) * 8));
    SCB_TRY(L.kept.ensure((uint64_t)ctx->sm_count * kKeptCtasPerSm * kKeptSmers * 8));
    return SCB_OK;
}

// Build-apply arguments: report counters into qcnt, deferred items into the lane's list.
scb_status attach_build(const scb_ctx* ctx, Lane& L, uint64_t max_items, unsigned long long* qcnt, GroupArgs& ga,
                        cudaStream_t st) {
    SCB_TRY(build_buffers(ctx, L, max_items));
    ga.kept = L.kept.as<unsigned long long>();
    ga.kept_ctas = (uint32_t)(ctx->sm_count * kKeptCtasPerSm);
    SCB_CUDA(cudaMemsetAsync(L.rec_count.as<unsigned long long>() + 2, 0, 8, st));
    ga.qcnt = qcnt;
    ga.ditems = L.ditems.as<uint4>();
    ga.ditem_base = L.ditem_base.as<unsigned long long>();
    ga.dcount = L.rec_count.as<unsigned long long>() + 2;
    return SCB_OK;
}

// The query kernel over the items a build apply left (attach_probes for the query first).
void attach_deferred(const Lane& L, GroupArgs& ga) {
    ga.items = L.ditems.as<uint4>();
    ga.n_items = L.rec_count.as<unsigned long long>() + 2;
    ga.item_base = L.ditem_base.as<unsigned long long>();
}

// In a build apply only the items it leaves to the query kernel (split buckets, items with more
// s-mers than the kept region) store probe words, a few percent of the s-mers: an eighth of the
// capacity suffices there (items past it hash again), which keeps 25 GB off the device at 2 Gbp.
uint64_t probe_capacity(const scb_ctx* ctx, uint64_t n_bytes, bool build) {
    const uint64_t all = n_bytes + records_estimate(ctx, n_bytes) * (ctx->g.k - ctx->g.s);
    return build ? all / 8 + 65536 : all;
}

// Turns on probe reuse in the apply arguments: the insert writes (and first clears the count),
// the query of the same prepared records reads.
scb_status attach_probes(Lane& L, int mode, uint64_t cap, GroupArgs& ga, cudaStream_t st) {
    if (mode == kModeInsert) SCB_CUDA(cudaMemsetAsync(L.rec_count.as<unsigned long long>() + 1, 0, 8, st));
    ga.probes = L.probes.as<unsigned long long>();
    ga.item_base = L.item_base.as<unsigned long long>();
    ga.probe_count = L.rec_count.as<unsigned long long>() + 1;
    ga.probe_cap = cap;
    return SCB_OK;
}

GroupedSizes grouped_sizes(const scb_ctx* ctx, uint64_t n_bytes, uint64_t min_records, int target = kTargetTuned) {
    GroupedSizes z;
    const uint64_t est = records_estimate(ctx, n_bytes);
    const uint64_t want = target == kTargetBuild      ? build_bucket_records(ctx)
                          : target == kTargetSpectrum ? spectrum_bucket_records(ctx)
                                                      : (uint64_t)ctx->tuning.bucket_records;
    z.shift = bucket_shift_for(ctx, est, want);
    z.n_buckets = ctx->nb_blocks >> z.shift;
    z.bucket_cap = ((est / z.n_buckets * 3 / 2 + 64) + 3) & ~3ull;
    z.cap = std::max<uint64_t>(est / 4 + 65536, min_records);
    z.max_items = items_bound(z);
    return z;
}

scb_status grouped_buffers(Lane& L, const GroupedSizes& z) {
    if (z.region() + z.cap >= (1ull << 32))
        return fail_kind(SCB_ERR_INTERNAL_STATE, "super-k-mer record slots beyond 2^32 for one batch");
    SCB_TRY(L.bhist.ensure((z.n_buckets + 1) * 8));
    SCB_TRY(L.bcursor.ensure((z.n_buckets + 1) * 8));
    SCB_TRY(L.icount.ensure((z.n_buckets + 1) * 8));
    SCB_TRY(L.gscan.ensure(((z.n_buckets + 1) / 1024 + 64) * 8 * 2));
    SCB_TRY(L.rec_count.ensure(64));
    SCB_TRY(L.rec_key.ensure(z.cap * 4));
    SCB_TRY(L.rec_val.ensure(z.cap * 8));
    SCB_TRY(L.rec_sorted.ensure((z.region() + z.cap) * 8));
    SCB_TRY(L.rec_bases.ensure(z.cap * 16));
    SCB_TRY(L.rec_sbases.ensure((z.region() + z.cap) * 16));
    SCB_TRY(L.items.ensure(z.max_items * 16));
    return SCB_OK;
}

// The cut kernel: one record per super-k-mer, into its bucket's region or the overflow list.
scb_status launch_cut(scb_ctx* ctx, Lane& L, TileArgs& a, const GroupedSizes& z, cudaStream_t st) {
    SCB_CUDA(cudaMemsetAsync(L.bhist.p, 0, (z.n_buckets + 1) * 8, st));
    SCB_CUDA(cudaMemsetAsync(L.rec_count.p, 0, 16, st));  // overflow records, probe slots
    a.rec_key = L.rec_key.as<uint32_t>();
    a.rec_val = L.rec_val.as<unsigned long long>();
    a.rec_count = L.rec_count.as<unsigned long long>();
    a.rec_cap = z.cap;
    a.bucket_hist = L.bhist.as<unsigned long long>();
    a.bucket_shift = z.shift;
    a.sorted = L.rec_sorted.as<unsigned long long>();
    a.sbases = L.rec_sbases.as<uint4>();
    a.rec_bases = L.rec_bases.as<uint4>();
    a.bucket_cap = z.bucket_cap;
    if (a.n_tiles == 0) return SCB_OK;
    SCB_CUDA(cudaMemsetAsync(L.tiles.p, 0, 4, st));
    launch_tiles(kModeCut, a, tile_grid(kModeCut, ctx->g.bits, ctx->sm_count, a.n_tiles), st);
    SCB_CUDA(cudaGetLastError());
    return SCB_OK;
}

// Work items over the bucket regions and the overflow records, which are first sorted into
// bucket order after the regions.  Every kernel here leaves the records alone when the overflow
// list ran out of room (more than z.cap entries).
scb_status launch_bucketing(scb_ctx* ctx, Lane& L, const GroupedSizes& z, cudaStream_t st) {
    (void)ctx;
    const unsigned long long* counts = L.bhist.as<unsigned long long>();
    uint64_t* ovf = reinterpret_cast<uint64_t*>(L.bcursor.p);
    launch_item_counts(counts, z.n_buckets, z.bucket_cap, L.icount.as<uint64_t>(), ovf,
                       L.rec_count.as<unsigned long long>(), z.cap, st);
    launch_scan_inplace(L.icount.as<uint64_t>(), z.n_buckets + 1, L.gscan.as<uint64_t>(), st);
    launch_scan_inplace(ovf, z.n_buckets + 1, L.gscan.as<uint64_t>(), st);
    launch_item_write(counts, z.bucket_cap, L.icount.as<uint64_t>(), ovf, z.region(), z.n_buckets,
                      L.items.as<uint4>(), st);
    // the overflow cursors start at the overflow offsets, which item_write has read
    launch_scatter(L.rec_key.as<uint32_t>(), L.rec_val.as<unsigned long long>(), L.rec_bases.as<uint4>(),
                   L.rec_count.as<unsigned long long>(), z.cap, z.shift, L.bcursor.as<unsigned long long>(),
                   z.region(), L.rec_sorted.as<unsigned long long>(), L.rec_sbases.as<uint4>(), st);
    SCB_CUDA(cudaGetLastError());
    return SCB_OK;
}

GroupArgs group_args(const scb_ctx* ctx, const Lane& L, const TileArgs& a, const GroupedSizes& z) {
    GroupArgs ga;
    std::memset(&ga, 0, sizeof(ga));
    ga.g = ctx->g;
    ga.codes = a.codes;
    ga.n_code_words = a.n_code_words;
    ga.table = ctx->table;
    ga.status = ctx->status;
    ga.recs = L.rec_sorted.as<unsigned long long>();
    ga.sbases = L.rec_sbases.as<uint4>();
    ga.items = L.items.as<uint4>();
    ga.n_items = reinterpret_cast<const unsigned long long*>(L.icount.as<uint64_t>() + z.n_buckets);
    ga.work_counter = L.tiles.as<unsigned int>() + 1;
    ga.bucket_shift = z.shift;
    ga.apply_threads = ctx->tuning.apply_threads;
    ga.rec_count = L.rec_count.as<unsigned long long>();
    ga.rec_cap = z.cap;
    return ga;
}

// The shared-memory apply kernel over prepared work items (insert or report), timed as its span.
scb_status launch_group_apply(scb_ctx* ctx, Lane& L, int mode, GroupArgs ga, unsigned long long* cnt,
                              uint64_t max_items, cudaStream_t st) {
    ga.cnt = cnt;
    const bool ins = mode == kModeInsert || mode == kModeBuild;  // the build apply is timed as the insert apply
    SCB_CUDA(cudaMemsetAsync(ga.work_counter, 0, 4, st));
    SCB_TRY(mark(ctx, L, ins ? 7 : 11, st));
    launch_apply(mode, ga, (int)ctx->cfg.block_slots_exponent, 1u << ga.bucket_shift, ctx->sm_count, max_items, st);
    SCB_CUDA(cudaGetLastError());
    SCB_TRY(mark(ctx, L, ins ? 8 : 12, st));
    if (ctx->timing) L.spans |= ins ? kSpanApplyInsert : kSpanApplyQuery;
    return SCB_OK;
}

scb_status run_tiles(scb_ctx* ctx, Lane& L, int mode, TileArgs& a, cudaStream_t st) {
    if (a.n_tiles == 0) return SCB_OK;
    SCB_CUDA(cudaMemsetAsync(L.tiles.p, 0, 4, st));
    const int grid = tile_grid(mode, ctx->g.bits, ctx->sm_count, a.n_tiles);
    launch_tiles(mode, a, grid, st);
    SCB_CUDA(cudaGetLastError());
    return SCB_OK;
}

// Plain pipeline stage (b): per-window block ids and end flags in HBM.
scb_status run_materialize(scb_ctx* ctx, Lane& L, TileArgs& a, cudaStream_t st) {
    SCB_TRY(L.wblock.ensure(std::max<uint64_t>(a.n_bytes, 1) * 4));
    SCB_TRY(L.wend.ensure(std::max<uint64_t>(a.n_bytes, 1)));
    a.wblock = L.wblock.as<uint32_t>();
    a.wend = L.wend.as<uint8_t>();
    return run_tiles(ctx, L, kModeMaterialize, a, st);
}

// Grouped pipeline, first half (eager): cut the batch into super-k-mer records, bucket them by
// block and build the work items.  The host reads the record count between the cut and the
// bucketing, so the second cut (rare) gets exactly the slots it needs.  The prepared records stay
// valid for the lane's current batch, so a query of the same reads (build then stream-query)
// reuses them.
scb_status grouped_prepare(scb_ctx* ctx, Lane& L, TileArgs& a, cudaStream_t st) {
    GroupedState& gs = L.gs;
    gs.valid = false;
    gs.built = false;
    GroupedSizes z = grouped_sizes(ctx, a.n_bytes, 0,
                                   L.want_build ? kTargetBuild : L.want_spectrum ? kTargetSpectrum : kTargetTuned);
    unsigned long long overflow = 0, records = 0;
    SCB_TRY(mark(ctx, L, 4, st));
    for (int attempt = 0; attempt < 2; attempt++) {
        SCB_TRY(grouped_buffers(L, z));
        if (attempt == 1) {  // the cut's own counters only (windows, s-mers, super-k-mers)
            SCB_CUDA(cudaMemsetAsync(a.cnt + kCntWindows, 0, 8, st));
            SCB_CUDA(cudaMemsetAsync(a.cnt + kCntSmers, 0, 8, st));
            SCB_CUDA(cudaMemsetAsync(a.cnt + kCntSuperKmers, 0, 8, st));
        }
        SCB_TRY(launch_cut(ctx, L, a, z, st));
        SCB_TRY(mark(ctx, L, 5, st));
        SCB_CUDA(cudaMemcpyAsync(&overflow, L.rec_count.p, 8, cudaMemcpyDeviceToHost, st));
        SCB_CUDA(cudaMemcpyAsync(&records, a.cnt + kCntSuperKmers, 8, cudaMemcpyDeviceToHost, st));
        SCB_CUDA(cudaStreamSynchronize(st));
        if (overflow <= z.cap) break;
        // more records past their bucket's region than the list held: the count is exact, so
        // a second cut with room for all of them suffices
        z.cap = overflow + 65536;
        z.max_items = items_bound(z);
    }
    if (overflow > z.cap) return fail_kind(SCB_ERR_INTERNAL_STATE, "super-k-mer record overflow");
    gs.produced = records;
    gs.shift = z.shift;
    gs.n_buckets = z.n_buckets;
    gs.max_items = records ? z.max_items : 0;
    if (records) SCB_TRY(launch_bucketing(ctx, L, z, st));
    gs.ga = group_args(ctx, L, a, z);
    gs.probes_written = false;
    gs.probe_cap = 0;
    if (L.want_probes && records) {
        gs.probe_cap = probe_capacity(ctx, a.n_bytes, L.want_build);
        SCB_TRY(L.probes.ensure(gs.probe_cap * 8));
        SCB_TRY(L.item_base.ensure(z.max_items * 8));
    }
    SCB_TRY(mark(ctx, L, 6, st));
    if (ctx->timing) L.spans |= kSpanCut;
    gs.valid = true;
    return SCB_OK;
}

// Grouped pipeline, second half: the shared-memory apply kernel over the prepared work items.
scb_status grouped_apply(scb_ctx* ctx, Lane& L, int mode, unsigned long long* cnt, cudaStream_t st) {
    GroupedState& gs = L.gs;
    if (!gs.valid) return fail_kind(SCB_ERR_INTERNAL_STATE, "no prepared super-k-mer records");
    if (gs.produced == 0) return SCB_OK;
    GroupArgs ga = gs.ga;
    if (gs.probe_cap && (mode == kModeInsert || gs.probes_written)) {
        SCB_TRY(attach_probes(L, mode, gs.probe_cap, ga, st));
        if (mode == kModeInsert) gs.probes_written = true;
    }
    int launch_mode = mode;
    if (mode == kModeInsert && L.want_build && gs.probe_cap) {
        // build + stream query: the insert answers the exclusive buckets' queries (report sums
        // into the lane's second counter array) and lists the other items for the query below
        SCB_TRY(attach_build(ctx, L, gs.max_items, L.cnt2.as<unsigned long long>(), ga, st));
        launch_mode = kModeBuild;
        gs.built = true;
    } else if (mode == kModeReport && gs.built) {
        attach_deferred(L, ga);
    }
    return launch_group_apply(ctx, L, launch_mode, ga, cnt, gs.max_items, st);
}

scb_status run_grouped(scb_ctx* ctx, Lane& L, int mode, TileArgs& a, cudaStream_t st) {
    if (a.n_tiles == 0) return SCB_OK;
    SCB_TRY(grouped_prepare(ctx, L, a, st));
    return grouped_apply(ctx, L, mode, a.cnt, st);
}

scb_status insert_stage(scb_ctx* ctx, Lane& L, TileArgs& a, cudaStream_t st) {
    const scb_strategy s = resolve(ctx, ctx->insert_strategy, a.n_bytes, true);
    if (s == SCB_STRATEGY_GROUPED) return run_grouped(ctx, L, kModeInsert, a, st);
    if (s == SCB_STRATEGY_PLAIN) {
        SCB_TRY(run_materialize(ctx, L, a, st));
        launch_plain_insert(a, st);
        SCB_CUDA(cudaGetLastError());
        return SCB_OK;
    }
    return run_tiles(ctx, L, kModeInsert, a, st);
}

scb_status query_stage(scb_ctx* ctx, Lane& L, int mode, TileArgs& a, cudaStream_t st) {
    const scb_strategy s = resolve(ctx, ctx->query_strategy, a.n_bytes, false);
    if (s == SCB_STRATEGY_GROUPED && mode == kModeReport) {
        // the lane's batch was already cut by a grouped insert of the same reads: reuse its records
        if (L.gs.valid) return grouped_apply(ctx, L, kModeReport, a.cnt, st);
        return run_grouped(ctx, L, kModeReport, a, st);
    }
    if (s == SCB_STRATEGY_PLAIN && (mode == kModeReport || mode == kModeAbund)) {
        SCB_TRY(run_materialize(ctx, L, a, st));
        launch_plain_query(mode, a, st);
        SCB_CUDA(cudaGetLastError());
        return SCB_OK;
    }
    return run_tiles(ctx, L, mode, a, st);
}

// The insert / query stage between two timing events when timing is on.
scb_status insert_device_batch(scb_ctx* ctx, Lane& L, TileArgs& a, cudaStream_t st) {
    SCB_TRY(mark(ctx, L, 2, st));
    SCB_TRY(insert_stage(ctx, L, a, st));
    SCB_TRY(mark(ctx, L, 3, st));
    if (ctx->timing) L.spans |= kSpanInsert;
    return SCB_OK;
}

scb_status query_device_batch(scb_ctx* ctx, Lane& L, int mode, TileArgs& a, cudaStream_t st) {
    SCB_TRY(mark(ctx, L, 9, st));
    SCB_TRY(query_stage(ctx, L, mode, a, st));
    SCB_TRY(mark(ctx, L, 10, st));
    if (ctx->timing) L.spans |= kSpanQuery;
    return SCB_OK;
}

scb_status read_counters(scb_ctx* ctx, Lane& L, cudaStream_t st, unsigned long long* host) {
    SCB_CUDA(cudaMemcpyAsync(host, L.cnt.p, kCntSlots * 8, cudaMemcpyDeviceToHost, st));
    uint32_t status = 0;
    SCB_CUDA(cudaMemcpyAsync(&status, ctx->status, 4, cudaMemcpyDeviceToHost, st));
    SCB_CUDA(cudaStreamSynchronize(st));
    if (ctx->timing && L.spans) {
        float ms = 0;
        auto span = [&](uint32_t bit, int e0, int e1, double& acc) {
            if ((L.spans & bit) && cudaEventElapsedTime(&ms, L.ev[e0], L.ev[e1]) == cudaSuccess) acc += ms;
        };
        span(kSpanPack, 0, 1, ctx->times.pack_ms);
        span(kSpanInsert, 2, 3, ctx->times.insert_ms);
        span(kSpanCut, 4, 5, ctx->times.cut_ms);
        span(kSpanCut, 5, 6, ctx->times.bucket_ms);
        span(kSpanApplyInsert, 7, 8, ctx->times.apply_insert_ms);
        span(kSpanQuery, 9, 10, ctx->times.query_ms);
        span(kSpanApplyQuery, 11, 12, ctx->times.apply_query_ms);
        if (L.spans & kSpanPack) ctx->times.batches++;
    }
    L.spans = 0;
    if (status) {
        return fail_kind(SCB_ERR_INTERNAL_STATE, "device status word 0x" + std::to_string(status) +
                                                     " (1=CAS retry limit, 2=distinct set full, 4=overflow list full)");
    }
    return SCB_OK;
}

// ---------------------------------------------------------------------------------------
// CUDA graphs per batch shape.  A batch of the persistent strategies (fused, grouped) replays
// a graph captured for its shape class: the batch kind, the strategies, and for the grouped
// pipeline the byte class (n rounded up to four steps per octave, at least 64 KiB) that sizes its
// record slots, buckets and work items.  The batch's own sizes and input pointers reach the
// kernels through a parameter block that a one-thread kernel writes just before the replay, and
// the other kernels' grids do not depend on the batch, so one graph serves every batch of its
// class and a replay has no host round trip between the cut and the apply.  A replay whose
// super-k-mer records outgrow the class's slots applies nothing (the bucketing and apply
// kernels check the count) and the batch is redone eagerly; the lane then captures with room
// for that many records.  The plain strategy stays one launch per stage, eagerly.
// ---------------------------------------------------------------------------------------
constexpr size_t kMaxGraphsPerLane = 8;

uint64_t lane_signature(const scb_ctx* ctx, const Lane& L) {
    const void* ptrs[] = {L.codes.p, L.valid.p, L.seqstart.p, L.cnt.p, L.cnt2.p, L.tiles.p, L.params.p,
                          L.rec_key.p, L.rec_val.p, L.rec_sorted.p, L.rec_bases.p, L.rec_sbases.p, L.bhist.p,
                          L.bcursor.p, L.icount.p,
                          L.items.p, L.gscan.p, L.rec_count.p, L.probes.p, L.item_base.p, L.ditems.p,
                          L.ditem_base.p, L.kept.p, ctx->table, ctx->status};
    uint64_t h = 0x243F6A8885A308D3ull;
    for (const void* q : ptrs) h = (h ^ (uint64_t)(uintptr_t)q) * 0x100000001B3ull + 0x9E3779B97F4A7C15ull;
    return h;
}

// The graph body: the whole batch of kind K on the capturing stream st.
scb_status record_batch(scb_ctx* ctx, Lane& L, const GraphKey& K, cudaStream_t st) {
    const BatchParams* bp = L.params.as<BatchParams>();
    const int sms = ctx->sm_count;
    // capacity of the graph: its class for the grouped pipeline, else the lane's buffers
    const uint64_t cap = K.cap_bytes;
    const uint64_t groups = (cap + 31) / 32;
    if (K.kind != kBatchReportKept) {  // a kept batch's codes are still in the lane
        SCB_TRY(mark(ctx, L, 0, st));
        launch_clear_dyn(bp, L.seqstart.as<uint32_t>(), nullptr, nullptr, sms, st);
        if (!K.prepacked) launch_pack_dyn(bp, L.codes.as<uint32_t>(), L.valid.as<uint32_t>(), sms, st);
        launch_seqstart_dyn(bp, L.seqstart.as<uint32_t>(), sms, st);
        SCB_TRY(mark(ctx, L, 1, st));
        SCB_CUDA(cudaMemsetAsync(L.cnt.p, 0, kCntSlots * 8, st));
    }
    TileArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = ctx->g;
    a.codes = L.codes.as<uint32_t>();
    a.valid = L.valid.as<uint32_t>();
    a.seqstart = L.seqstart.as<uint32_t>();
    a.n_bytes = cap;  // capacities: the kernels take the batch's sizes from bp
    a.n_code_words = 2 * groups;
    a.n_bit_words = groups;
    a.n_tiles = (uint32_t)((cap + kTileWindows - 1) / kTileWindows);  // grid size of the tile kernels
    a.table = ctx->table;
    a.status = ctx->status;
    a.cnt = L.cnt.as<unsigned long long>();
    a.tile_counter = L.tiles.as<unsigned int>();
    a.dyn = bp;
    GroupedSizes z;
    z.shift = K.shift;
    z.n_buckets = K.n_buckets;
    z.cap = K.rec_cap;
    z.bucket_cap = K.bucket_cap;
    z.max_items = K.max_items;
    bool cut = K.kind == kBatchReportKept;  // the insert's records are kept
    auto cut_and_bucket = [&]() -> scb_status {
        SCB_TRY(mark(ctx, L, 4, st));
        SCB_TRY(launch_cut(ctx, L, a, z, st));
        SCB_TRY(mark(ctx, L, 5, st));
        SCB_TRY(launch_bucketing(ctx, L, z, st));
        SCB_TRY(mark(ctx, L, 6, st));
        cut = true;
        return SCB_OK;
    };
    const bool fuse = K.fused && K.probe_cap;
    if (kind_inserts(K.kind)) {
        SCB_TRY(mark(ctx, L, 2, st));
        if (K.s_ins == SCB_STRATEGY_GROUPED) {
            SCB_TRY(cut_and_bucket());
            GroupArgs ga = group_args(ctx, L, a, z);
            if (K.probe_cap) SCB_TRY(attach_probes(L, kModeInsert, K.probe_cap, ga, st));
            int mode = kModeInsert;
            if (fuse) {  // report sums of the buckets the build apply answers itself
                SCB_CUDA(cudaMemsetAsync(L.cnt2.p, 0, kCntSlots * 8, st));
                SCB_TRY(attach_build(ctx, L, z.max_items, L.cnt2.as<unsigned long long>(), ga, st));
                mode = kModeBuild;
            }
            SCB_TRY(launch_group_apply(ctx, L, mode, ga, L.cnt.as<unsigned long long>(), z.max_items, st));
        } else {
            SCB_TRY(run_tiles(ctx, L, kModeInsert, a, st));
        }
        SCB_TRY(mark(ctx, L, 3, st));
    }
    if (kind_queries(K.kind)) {
        unsigned long long* qc = L.cnt.as<unsigned long long>();
        if (K.kind == kBatchBuildStream || K.kind == kBatchReportKept) {
            qc = L.cnt2.as<unsigned long long>();
            if (!fuse) SCB_CUDA(cudaMemsetAsync(qc, 0, kCntSlots * 8, st));
        }
        a.cnt = qc;
        SCB_TRY(mark(ctx, L, 9, st));
        launch_seq_windows_dyn(bp, ctx->g.k, qc, sms, st);
        if (K.s_query == SCB_STRATEGY_GROUPED) {
            if (!cut) SCB_TRY(cut_and_bucket());  // else: reuse the insert's records
            GroupArgs ga = group_args(ctx, L, a, z);
            if (K.probe_cap) SCB_TRY(attach_probes(L, kModeReport, K.probe_cap, ga, st));
            if (fuse) attach_deferred(L, ga);  // only the items the build apply left
            SCB_TRY(launch_group_apply(ctx, L, kModeReport, ga, qc, z.max_items, st));
        } else {
            SCB_TRY(run_tiles(ctx, L, kModeReport, a, st));
        }
        SCB_TRY(mark(ctx, L, 10, st));
    }
    return SCB_OK;
}

scb_status capture_batch(scb_ctx* ctx, Lane& L, const GraphKey& K, GraphEntry& out) {
    cudaStream_t cs = L.stream;
    uint64_t launches = 0;
    SCB_CUDA(cudaStreamBeginCapture(cs, cudaStreamCaptureModeRelaxed));
    record_launches_into(&launches);
    L.recording = true;
    const scb_status rs = record_batch(ctx, L, K, cs);
    L.recording = false;
    record_launches_into(nullptr);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(cs, &graph);
    L.spans = 0;
    if (rs != SCB_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        if (rs != SCB_OK) return rs;
        return fail_kind(SCB_ERR_INTERNAL_STATE, std::string("graph capture: ") + cudaGetErrorString(e));
    }
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
        cudaGetLastError();
        return fail_kind(SCB_ERR_INTERNAL_STATE, std::string("graph instantiate: ") + cudaGetErrorString(ei));
    }
    out.key = K;
    out.exec = exec;
    out.launches = launches;
    L.captures++;
    return SCB_OK;
}

// A graph launched for a batch, finished (counters read, record count checked) later.
struct GraphRun {
    bool launched = false;
    bool grouped = false;
    int kind = 0;
    GraphKey K;
};

// Keys, sizes, captures (first time) and launches the batch's graph on st without waiting for it;
// run.launched = false leaves the batch to the eager path (graphs off, plain strategy, empty
// batch, capture failure, kept records that came from the eager path).
scb_status graph_launch(scb_ctx* ctx, Lane& L, int kind, const uint8_t* d_ascii, const uint64_t* d_offsets,
                        uint64_t n, uint64_t n_bytes, cudaStream_t st, GraphRun& run) {
    run = GraphRun();
    run.kind = kind;
    if (n == 0 || n_bytes == 0) return SCB_OK;
    GraphKey K;
    if (kind == kBatchReportKept) {  // runs whenever the kept records came from a graph
        if (!L.kept_graph) return SCB_OK;
        K = L.kept_key;  // the kept insert's sizes and buffers
        K.kind = kBatchReportKept;
        K.s_ins = 0;
        K.s_query = SCB_STRATEGY_GROUPED;
    } else {
        if (!ctx->graphs) return SCB_OK;
        K.kind = kind;
        K.prepacked = L.prepacked;
        if (kind_inserts(kind)) K.s_ins = resolve(ctx, ctx->insert_strategy, n_bytes, true);
        if (kind_queries(kind)) K.s_query = resolve(ctx, ctx->query_strategy, n_bytes, false);
        if (K.s_ins == SCB_STRATEGY_PLAIN || K.s_query == SCB_STRATEGY_PLAIN) return SCB_OK;
        if (kind == kBatchInsertKeep && (K.s_ins != SCB_STRATEGY_GROUPED || !probes_fit(ctx))) return SCB_OK;
        // the grouped pipeline's record slots, buckets and work items are sized for a byte class;
        // the fused kernels take any batch that fits the lane's buffers (capacity: those buffers)
        const uint64_t cls = std::max(n_bytes, std::min(class_bytes(n_bytes), kMaxBatchBytes - 64));
        const bool grouped = K.s_ins == SCB_STRATEGY_GROUPED || K.s_query == SCB_STRATEGY_GROUPED;
        // lane buffers grow in class steps, so growing batches recapture rarely
        SCB_TRY(ensure_lane_work(ctx, L, cls));
        K.cap_bytes =
            grouped ? cls : std::min<uint64_t>(L.seqstart.cap / 4 - kPadWords, (kMaxBatchBytes - 64) / 32) * 32;
        SCB_TRY(L.params.ensure(sizeof(BatchParams)));
        SCB_TRY(L.cnt2.ensure(kCntSlots * 8));
        if (grouped) {
            K.fused = kind == kBatchBuildStream && build_fused(ctx, n_bytes);
            const GroupedSizes z = grouped_sizes(ctx, cls, L.rec_hint, K.fused ? kTargetBuild : kTargetTuned);
            K.shift = z.shift;
            K.n_buckets = z.n_buckets;
            K.rec_cap = z.cap;
            K.bucket_cap = z.bucket_cap;
            K.max_items = z.max_items;
            K.apply_threads = ctx->tuning.apply_threads;
            SCB_TRY(grouped_buffers(L, z));
            const bool keep = kind == kBatchInsertKeep ||
                              (kind == kBatchBuildStream && K.s_ins == SCB_STRATEGY_GROUPED &&
                               K.s_query == SCB_STRATEGY_GROUPED);
            if (keep && probes_fit(ctx)) {
                K.probe_cap = probe_capacity(ctx, cls, K.fused);
                SCB_TRY(L.probes.ensure(K.probe_cap * 8));
                SCB_TRY(L.item_base.ensure(z.max_items * 8));
            }
            if (K.fused) SCB_TRY(build_buffers(ctx, L, z.max_items));  // before the signature: the graph points at them
        }
        K.sig = lane_signature(ctx, L);
    }
    // graphs whose nodes point at buffers that have since been replaced are dropped
    for (size_t i = 0; i < L.graphs.size();) {
        if (L.graphs[i].key.sig != K.sig) {
            cudaGraphExecDestroy(L.graphs[i].exec);
            L.graphs.erase(L.graphs.begin() + (long)i);
        } else {
            i++;
        }
    }
    GraphEntry* ge = nullptr;
    for (auto& g : L.graphs) {
        if (g.key == K) ge = &g;
    }
    if (!ge) {
        GraphEntry fresh;
        if (capture_batch(ctx, L, K, fresh) != SCB_OK) {
            ctx->graphs = false;  // this context runs eagerly from now on
            L.graph_fallbacks++;
            return SCB_OK;
        }
        if (L.graphs.size() >= kMaxGraphsPerLane) {
            auto lru = std::min_element(L.graphs.begin(), L.graphs.end(), [](const GraphEntry& x, const GraphEntry& y) {
                return x.last_use < y.last_use;
            });
            cudaGraphExecDestroy(lru->exec);
            L.graphs.erase(lru);
        }
        L.graphs.push_back(fresh);
        ge = &L.graphs.back();
    }
    launch_set_params(L.params.as<BatchParams>(), BatchParams{n_bytes, n, d_ascii, d_offsets}, st);
    SCB_CUDA(cudaGraphLaunch(ge->exec, st));
    note_launches(ge->launches);
    ge->last_use = ++L.graph_clock;
    L.replays++;
    L.gs.valid = false;
    run.grouped = K.s_ins == SCB_STRATEGY_GROUPED || K.s_query == SCB_STRATEGY_GROUPED;
    if (kind == kBatchInsertKeep) {
        L.kept_graph = true;
        L.kept_key = K;
    }
    if (ctx->timing) {
        L.spans = kind == kBatchReportKept ? 0u : (uint32_t)kSpanPack;
        if (kind_inserts(kind)) L.spans |= kSpanInsert | (K.s_ins == SCB_STRATEGY_GROUPED ? kSpanApplyInsert : 0u);
        if (kind_queries(kind)) L.spans |= kSpanQuery | (K.s_query == SCB_STRATEGY_GROUPED ? kSpanApplyQuery : 0u);
        if (run.grouped && kind != kBatchReportKept) L.spans |= kSpanCut;
    }
    run.launched = true;
    run.K = K;
    return SCB_OK;
}

// Waits for a launched graph, reads its counters (c_ins: insert, c_q: query) and checks the
// record count; done = false: the replay applied nothing and the batch goes to the eager path.
scb_status graph_finish(scb_ctx* ctx, Lane& L, const GraphRun& run, cudaStream_t st, unsigned long long* c_ins,
                        unsigned long long* c_q, bool& done) {
    done = false;
    if (!run.launched) return SCB_OK;
    const int kind = run.kind;
    const bool check = run.grouped && kind_inserts(kind);
    unsigned long long produced = 0, scratch[kCntSlots];
    if (check) SCB_CUDA(cudaMemcpyAsync(&produced, L.rec_count.p, 8, cudaMemcpyDeviceToHost, st));
    if (kind == kBatchBuildStream || kind == kBatchReportKept) {
        SCB_CUDA(cudaMemcpyAsync(c_q, L.cnt2.p, kCntSlots * 8, cudaMemcpyDeviceToHost, st));
    }
    unsigned long long* main = kind == kBatchReport ? c_q : kind == kBatchReportKept ? scratch : c_ins;
    SCB_TRY(read_counters(ctx, L, st, main));
    if (check && produced > run.K.rec_cap) {
        // nothing was applied: redo the batch eagerly and capture with room for these records
        L.rec_hint = produced + produced / 4;
        L.graph_fallbacks++;
        if (kind == kBatchInsertKeep) L.kept_graph = false;
        return SCB_OK;
    }
    done = true;
    return SCB_OK;
}

scb_status graph_batch(scb_ctx* ctx, Lane& L, int kind, const uint8_t* d_ascii, const uint64_t* d_offsets, uint64_t n,
                       uint64_t n_bytes, cudaStream_t st, unsigned long long* c_ins, unsigned long long* c_q,
                       bool& done) {
    GraphRun run;
    SCB_TRY(graph_launch(ctx, L, kind, d_ascii, d_offsets, n, n_bytes, st, run));
    return graph_finish(ctx, L, run, st, c_ins, c_q, done);
}

// One device batch of the given kind: a graph replay when possible, else the eager pipeline.
// c_ins receives the insert's counters (kinds insert, build+stream), c_q the query's.
scb_status run_batch(scb_ctx* ctx, Lane& L, int kind, const uint8_t* d_ascii, const uint64_t* d_offsets, uint64_t n,
                     uint64_t n_bytes, cudaStream_t st, unsigned long long* c_ins, unsigned long long* c_q) {
    bool done = false;
    SCB_TRY(graph_batch(ctx, L, kind, d_ascii, d_offsets, n, n_bytes, st, c_ins, c_q, done));
    if (done) return SCB_OK;
    if (kind == kBatchReportKept) {  // query the records an eager insert kept in this lane
        if (!L.gs.valid) return fail_kind(SCB_ERR_INTERNAL_STATE, "no kept super-k-mer records for this batch");
        TileArgs a;
        std::memset(&a, 0, sizeof(a));
        a.g = ctx->g;
        a.n_bytes = n_bytes;
        a.cnt = L.cnt.as<unsigned long long>();
        SCB_CUDA(cudaMemsetAsync(L.cnt.p, 0, kCntSlots * 8, st));
        launch_seq_windows(d_offsets, n, ctx->g.k, a.cnt, nullptr, st);
        SCB_TRY(query_device_batch(ctx, L, kModeReport, a, st));
        return read_counters(ctx, L, st, c_q);
    }
    SCB_TRY(ensure_lane_work(ctx, L, n_bytes));
    TileArgs a;
    SCB_TRY(prepare_batch(ctx, L, d_ascii, d_offsets, n, n_bytes, st, a));
    const bool fuse = kind == kBatchBuildStream && build_fused(ctx, n_bytes);
    if (kind_inserts(kind)) {
        // a grouped build + stream query keeps the insert's probe slots for the query
        L.want_probes = (kind == kBatchBuildStream || kind == kBatchInsertKeep) && probes_fit(ctx) &&
                        resolve(ctx, ctx->insert_strategy, n_bytes, true) == SCB_STRATEGY_GROUPED &&
                        (kind == kBatchInsertKeep ||
                         resolve(ctx, ctx->query_strategy, n_bytes, false) == SCB_STRATEGY_GROUPED);
        L.want_build = fuse;
        scb_status rs = SCB_OK;
        if (fuse) {
            rs = L.cnt2.ensure(kCntSlots * 8);
            if (rs == SCB_OK && cudaMemsetAsync(L.cnt2.p, 0, kCntSlots * 8, st) != cudaSuccess) {
                rs = fail_kind(SCB_ERR_INTERNAL_STATE, "clearing the report counters failed");
            }
        }
        if (rs == SCB_OK) rs = insert_device_batch(ctx, L, a, st);
        L.want_probes = false;
        L.want_build = false;
        SCB_TRY(rs);
        SCB_TRY(read_counters(ctx, L, st, c_ins));
        if (kind == kBatchInsertKeep) L.kept_graph = false;  // the lane's eager state holds the records
    }
    if (kind == kBatchBuildStream || kind == kBatchReport) {
        if (kind == kBatchBuildStream) SCB_CUDA(cudaMemsetAsync(L.cnt.p, 0, kCntSlots * 8, st));
        launch_seq_windows(d_offsets, n, ctx->g.k, a.cnt, nullptr, st);
        SCB_TRY(query_device_batch(ctx, L, kModeReport, a, st));
        SCB_TRY(read_counters(ctx, L, st, c_q));
        if (fuse && L.gs.built) {  // the report sums of the buckets the build apply answered
            unsigned long long c2[kCntSlots];
            SCB_CUDA(cudaMemcpyAsync(c2, L.cnt2.p, kCntSlots * 8, cudaMemcpyDeviceToHost, st));
            SCB_CUDA(cudaStreamSynchronize(st));
            for (int slot : {(int)kCntValid, (int)kCntPositive, (int)kCntChecksum}) c_q[slot] += c2[slot];
        }
    }
    return SCB_OK;
}

// Pinned staging for host packing of up to `groups` 32-byte groups: two areas, so the host packs
// piece (or slice) p + 1 while the copy of piece p reads the other.
static scb_status ensure_staging(scb_ctx* ctx, uint64_t groups) {
    for (int i = 0; i < 2; i++) {
        if (!ctx->stage_free[i]) SCB_CUDA(cudaEventCreateWithFlags(&ctx->stage_free[i], cudaEventDisableTiming));
    }
    if (groups <= ctx->stage_groups) return SCB_OK;
    for (int i = 0; i < 2; i++) SCB_CUDA(cudaEventSynchronize(ctx->stage_free[i]));  // copies still reading
    for (int i = 0; i < 2; i++) {
        if (ctx->stage_codes[i]) cudaFreeHost(ctx->stage_codes[i]);
        if (ctx->stage_valid[i]) cudaFreeHost(ctx->stage_valid[i]);
        ctx->stage_codes[i] = nullptr;
        ctx->stage_valid[i] = nullptr;
    }
    ctx->stage_groups = 0;
    for (int i = 0; i < 2; i++) {
        SCB_CUDA(cudaMallocHost((void**)&ctx->stage_codes[i], (2 * groups + kPadWords) * 4));
        SCB_CUDA(cudaMallocHost((void**)&ctx->stage_valid[i], (groups + kPadWords) * 4));
    }
    ctx->stage_groups = groups;
    return SCB_OK;
}

// Host packing of one upload: slices of kPackSlice bytes are packed on all host threads into the
// two staging areas in turn and copied to their place in the lane's codes and validity words (the
// padding words with the last slice), so slice i + 1 is packed while slice i copies.
constexpr uint64_t kPackSlice = 256ull << 20;  // a multiple of 32: slices end on whole groups
constexpr uint64_t kHostPackMin = 1ull << 20;  // smaller uploads copy the letters
scb_status host_pack_upload(scb_ctx* ctx, Lane& L, const uint8_t* src, uint64_t n_bytes, cudaStream_t st) {
    SCB_TRY(ensure_staging(ctx, (std::min(n_bytes, kPackSlice) + 31) / 32));
    const unsigned threads = std::max(1u, std::thread::hardware_concurrency());
    uint32_t* codes = L.codes.as<uint32_t>();
    uint32_t* valid = L.valid.as<uint32_t>();
    for (uint64_t off = 0, i = 0; off < n_bytes; off += kPackSlice, i++) {
        const uint64_t len = std::min(kPackSlice, n_bytes - off), g = (len + 31) / 32;
        const uint64_t pad = off + len == n_bytes ? kPadWords : 0;
        const int s = (int)(i & 1);
        SCB_CUDA(cudaEventSynchronize(ctx->stage_free[s]));  // the copy that last read this area
        host_pack(src + off, len, ctx->stage_codes[s], ctx->stage_valid[s], threads);
        SCB_CUDA(cudaMemcpyAsync(codes + off / 16, ctx->stage_codes[s], (2 * g + pad) * 4, cudaMemcpyHostToDevice, st));
        SCB_CUDA(cudaMemcpyAsync(valid + off / 32, ctx->stage_valid[s], (g + pad) * 4, cudaMemcpyHostToDevice, st));
        SCB_CUDA(cudaEventRecord(ctx->stage_free[s], st));
        ctx->h2d_bytes += (3 * g + 2 * pad) * 4;
    }
    return SCB_OK;
}

// Copies a host chunk into the lane and rebases its offsets.  Uploads of at least kHostPackMin
// bytes are packed on the host (3 bits per base cross PCIe, and pageable input needs no driver
// staging of the letters) unless scb_set_host_pack turned that off; the lane is then marked
// prepacked, so its batch skips the device packing.
scb_status upload_chunk(scb_ctx* ctx, Lane& L, const uint8_t* seqs, const uint64_t* offsets, const Chunk& c) {
    const uint64_t n_seqs = c.seq1 - c.seq0, n_bytes = c.byte1 - c.byte0;
    SCB_TRY(ensure_lane(ctx, L, n_bytes, n_seqs));
    cudaStream_t st = L.stream;
    L.prepacked = false;
    if (ctx->host_pack && n_bytes >= kHostPackMin) {
        // a graph of this batch sizes the lane's work buffers for its byte class: grow them before
        // the copy, so that no later growth drops the copied words
        SCB_TRY(ensure_lane_work(ctx, L, std::max(n_bytes, std::min(class_bytes(n_bytes), kMaxBatchBytes - 64))));
        SCB_TRY(host_pack_upload(ctx, L, seqs + c.byte0, n_bytes, st));
        L.prepacked = true;
    } else if (n_bytes) {
        SCB_CUDA(cudaMemcpyAsync(L.ascii.p, seqs + c.byte0, n_bytes, cudaMemcpyHostToDevice, st));
        ctx->h2d_bytes += n_bytes;
    }
    SCB_CUDA(cudaMemcpyAsync(L.offsets.p, offsets + c.seq0, (n_seqs + 1) * 8, cudaMemcpyHostToDevice, st));
    ctx->h2d_bytes += (n_seqs + 1) * 8;
    if (c.byte0) {
        k_rebase<<<(unsigned)((n_seqs + 1 + 255) / 256), 256, 0, st>>>(L.offsets.as<uint64_t>(), n_seqs + 1, c.byte0);
        note_launch();
    }
    return SCB_OK;
}

struct CtxLock {
    std::unique_lock<std::mutex> lk;
    explicit CtxLock(scb_ctx* c) : lk(c->mu) { cudaSetDevice(c->device); }
};

// Process-wide autotuner results, keyed by the geometry they were measured on.
using TuneKey = std::tuple<uint8_t, uint8_t, uint8_t, uint64_t, uint64_t, uint64_t, uint64_t>;
std::mutex g_tune_mu;
std::map<TuneKey, Tuning> g_tune_cache;

TuneKey tune_key(const scb_config& c) {
    return TuneKey(c.counter_bits, c.block_slots_exponent, c.counter_slots_exponent, c.k, c.m, c.s, c.n_hashes);
}

void lookup_tuning(scb_ctx* ctx) {
    std::lock_guard<std::mutex> lk(g_tune_mu);
    auto it = g_tune_cache.find(tune_key(ctx->cfg));
    if (it != g_tune_cache.end()) ctx->tuning = it->second;
}

scb_status alloc_ctx(const scb_config* cfg, scb_ctx** out) {
    SCB_TRY(validate_config(cfg));
    SCB_TRY(device_limits(cfg));
    int dev_count = 0;
    cudaError_t e = cudaGetDeviceCount(&dev_count);
    if (e != cudaSuccess || dev_count == 0) {
        return fail_kind(SCB_ERR_INTERNAL_STATE, std::string("no CUDA device available: ") +
                                                     (e != cudaSuccess ? cudaGetErrorString(e) : "0 devices"));
    }
    auto* ctx = new scb_ctx();
    ctx->cfg = *cfg;
    fill_geometry(ctx);
    cudaGetDevice(&ctx->device);
    cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, ctx->device);
    // whole 32-bit words: counters are updated through 32-bit CAS on their containing word
    e = cudaMalloc(&ctx->table, ((ctx->table_bytes + 255) / 256) * 256);
    if (e != cudaSuccess) {
        ctx->table = nullptr;
        delete ctx;
        return fail_kind(SCB_ERR_INTERNAL_STATE, "device allocation of the counter table failed: " +
                                                     std::string(cudaGetErrorString(e)));
    }
    e = cudaMalloc(&ctx->status, 64);
    if (e == cudaSuccess) e = cudaMemset(ctx->table, 0, ((ctx->table_bytes + 255) / 256) * 256);
    if (e == cudaSuccess) e = cudaMemset(ctx->status, 0, 64);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        delete ctx;
        return fail_kind(SCB_ERR_INTERNAL_STATE, std::string("device setup failed: ") + cudaGetErrorString(e));
    }
    lookup_tuning(ctx);
    *out = ctx;
    return SCB_OK;
}

// Host-pointer batch driver: uploads every chunk into the lane and runs fn(lane, chunk).
template <typename Fn>
scb_status for_each_upload(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n, Fn&& fn) {
    SCB_TRY(check_offsets(offsets, n));
    std::vector<Chunk> chunks;
    SCB_TRY(plan_chunks(offsets, n, ctx->cfg.k, ctx->tuning.host_batch_bytes, chunks));
    for (const Chunk& c : chunks) {
        Lane& L = ctx->lane;
        SCB_TRY(upload_chunk(ctx, L, seqs, offsets, c));
        SCB_TRY(fn(L, c));
    }
    return SCB_OK;
}

// Host-pointer batch driver: runs fn(lane, tile_args, chunk) on every staged chunk.
template <typename Fn>
scb_status for_each_chunk(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n, Fn&& fn) {
    SCB_TRY(check_offsets(offsets, n));
    std::vector<Chunk> chunks;
    SCB_TRY(plan_chunks(offsets, n, ctx->cfg.k, ctx->tuning.host_batch_bytes, chunks));
    for (const Chunk& c : chunks) {
        Lane& L = ctx->lane;
        SCB_TRY(upload_chunk(ctx, L, seqs, offsets, c));
        TileArgs a;
        SCB_TRY(prepare_batch(ctx, L, L.ascii.as<uint8_t>(), L.offsets.as<uint64_t>(), c.seq1 - c.seq0,
                              c.byte1 - c.byte0, L.stream, a));
        SCB_TRY(fn(L, a, c));
    }
    return SCB_OK;
}

}  // namespace

void scb::launch_narrow_out(const BatchParams* bp, uint64_t n, const unsigned long long* out, void* outn, uint32_t width,
                            int sm_count, cudaStream_t st) {
    k_narrow_out<<<(unsigned)(sm_count * 4), 256, 0, st>>>(bp, n, out, outn, width);
    note_launch();
}

// ---------------------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------------------
extern "C" {

const char* scb_last_error(void) { return last_error_slot().c_str(); }
const char* scb_version(void) { return "scb_b200 0.1.0 (sm_100a)"; }
uint64_t scb_kernel_launches(void) { return kernel_launch_count(); }

scb_status scb_config_default(scb_config* cfg) {
    if (!cfg) return fail_kind(SCB_ERR_INVALID_CONFIG, "null config");
    cfg->k = 31;
    cfg->m = 21;
    cfg->s = 25;
    cfg->n_hashes = 4;
    cfg->counter_bits = 16;
    cfg->counter_slots_exponent = 30;
    cfg->block_slots_exponent = 9;
    const unsigned hc = std::thread::hardware_concurrency();
    cfg->threads = hc ? hc : 1;
    cfg->queue = 4096;
    return SCB_OK;
}

scb_status scb_config_validate(const scb_config* cfg) { return validate_config(cfg); }

scb_status scb_create(const scb_config* cfg, scb_ctx** out) {
    if (!out) return fail_kind(SCB_ERR_INTERNAL_STATE, "null output pointer");
    *out = nullptr;
    return alloc_ctx(cfg, out);
}

void scb_destroy(scb_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    delete ctx;
}

scb_status scb_get_counts(const scb_ctx* ctx, uint64_t* kmers, uint64_t* smers) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    if (kmers) *kmers = ctx->inserted_kmers;
    if (smers) *smers = ctx->inserted_smers;
    return SCB_OK;
}

scb_status scb_get_config(const scb_ctx* ctx, scb_config* cfg) {
    if (!ctx || !cfg) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    *cfg = ctx->cfg;
    return SCB_OK;
}

scb_status scb_set_threads(scb_ctx* ctx, uint64_t threads) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    if (threads == 0) return fail_kind(SCB_ERR_INVALID_CONFIG, "threads must be positive");
    ctx->cfg.threads = threads;
    return SCB_OK;
}

// Waits for the context's own streams (not the device's other work: a server or another
// context on the same GPU keeps running).
static scb_status sync_ctx_streams(scb_ctx* ctx) {
    if (ctx->lane.stream) SCB_CUDA(cudaStreamSynchronize(ctx->lane.stream));
    for (auto& pl : ctx->piece_lanes) {
        if (pl->stream) SCB_CUDA(cudaStreamSynchronize(pl->stream));
    }
    if (ctx->copy_stream) SCB_CUDA(cudaStreamSynchronize(ctx->copy_stream));
    return SCB_OK;
}

scb_status scb_freeze(scb_ctx* ctx) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    CtxLock lk(ctx);
    SCB_TRY(sync_ctx_streams(ctx));
    ctx->frozen = true;
    return SCB_OK;
}

scb_status scb_set_strategy(scb_ctx* ctx, scb_strategy ins, scb_strategy q) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    ctx->insert_strategy = ins;
    ctx->query_strategy = q;
    return SCB_OK;
}

scb_status scb_get_strategy(const scb_ctx* ctx, scb_strategy* ins, scb_strategy* q) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    if (ins) *ins = resolve(ctx->insert_strategy);
    if (q) *q = resolve(ctx->query_strategy);
    return SCB_OK;
}

uint64_t scb_records_indexed(const scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n) {
    if (!ctx || !seqs || !offsets) return 0;
    static const auto acgt = [] {
        std::array<uint8_t, 256> t{};
        for (const char c : {'A', 'C', 'G', 'T', 'a', 'c', 'g', 't'}) t[(uint8_t)c] = 1;
        return t;
    }();
    const uint64_t k = ctx->cfg.k;
    uint64_t indexed = 0;
    for (uint64_t j = 0; j < n; j++) {
        uint64_t run = 0;
        for (uint64_t p = offsets[j]; p < offsets[j + 1]; p++) {
            run = acgt[seqs[p]] ? run + 1 : 0;
            if (run >= k) {
                indexed++;
                break;
            }
        }
    }
    return indexed;
}

uint64_t scb_count_windows(const scb_ctx* ctx, const uint64_t* offsets, uint64_t n) {
    if (!ctx || !offsets) return 0;
    return windows_of(offsets, n, ctx->cfg.k);
}

scb_status scb_insert_batch(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                            uint64_t* kmers, uint64_t* smers) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    CtxLock lk(ctx);
    if (ctx->frozen) return fail_kind(SCB_ERR_INTERNAL_STATE, "the index is frozen; inserts need a builder");
    uint64_t tk = 0, ts = 0;
    SCB_TRY(for_each_upload(ctx, seqs, offsets, n, [&](Lane& L, const Chunk& ch) -> scb_status {
        unsigned long long c[kCntSlots] = {};
        SCB_TRY(run_batch(ctx, L, kBatchInsert, L.ascii.as<uint8_t>(), L.offsets.as<uint64_t>(), ch.seq1 - ch.seq0,
                          ch.byte1 - ch.byte0, L.stream, c, nullptr));
        tk += c[kCntWindows];
        ts += c[kCntSmers];
        return SCB_OK;
    }));
    ctx->inserted_kmers += tk;
    ctx->inserted_smers += ts;
    if (kmers) *kmers = tk;
    if (smers) *smers = ts;
    return SCB_OK;
}

scb_status scb_insert_batch_device(scb_ctx* ctx, const uint8_t* d_seqs, const uint64_t* d_offsets, uint64_t n,
                                   uint64_t n_bytes, void* stream, uint64_t* kmers, uint64_t* smers) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    CtxLock lk(ctx);
    if (ctx->frozen) return fail_kind(SCB_ERR_INTERNAL_STATE, "the index is frozen; inserts need a builder");
    if (n_bytes > kMaxBatchBytes - 64) return fail_kind(SCB_ERR_INTERNAL_STATE, "device batch above 2 GiB");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    Lane& L = ctx->lane;
    L.prepacked = false;  // device input: the batch packs on the device
    unsigned long long c[kCntSlots] = {};
    SCB_TRY(run_batch(ctx, L, kBatchInsert, d_seqs, d_offsets, n, n_bytes, st, c, nullptr));
    ctx->inserted_kmers += c[kCntWindows];
    ctx->inserted_smers += c[kCntSmers];
    if (kmers) *kmers = c[kCntWindows];
    if (smers) *smers = c[kCntSmers];
    return SCB_OK;
}

static scb_status need_frozen(const scb_ctx* ctx) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    if (!ctx->frozen) return fail_kind(SCB_ERR_INTERNAL_STATE, "queries need a frozen index (into_index)");
    return SCB_OK;
}

scb_status scb_query_report(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                            scb_report* rep) {
    SCB_TRY(need_frozen(ctx));
    if (!rep) return fail_kind(SCB_ERR_INTERNAL_STATE, "null report");
    CtxLock lk(ctx);
    std::memset(rep, 0, sizeof(*rep));
    SCB_TRY(for_each_upload(ctx, seqs, offsets, n, [&](Lane& L, const Chunk& ch) -> scb_status {
        unsigned long long c[kCntSlots] = {};
        SCB_TRY(run_batch(ctx, L, kBatchReport, L.ascii.as<uint8_t>(), L.offsets.as<uint64_t>(), ch.seq1 - ch.seq0,
                          ch.byte1 - ch.byte0, L.stream, nullptr, c));
        rep->records_processed += c[kCntRecords];
        rep->total_windows += c[kCntTotalWindows];
        rep->valid_kmers += c[kCntValid];
        rep->positive_estimates += c[kCntPositive];
        rep->estimate_checksum += c[kCntChecksum];
        return SCB_OK;
    }));
    return SCB_OK;
}

scb_status scb_query_report_device(scb_ctx* ctx, const uint8_t* d_seqs, const uint64_t* d_offsets, uint64_t n,
                                   uint64_t n_bytes, void* stream, scb_report* rep) {
    SCB_TRY(need_frozen(ctx));
    if (!rep) return fail_kind(SCB_ERR_INTERNAL_STATE, "null report");
    CtxLock lk(ctx);
    if (n_bytes > kMaxBatchBytes - 64) return fail_kind(SCB_ERR_INTERNAL_STATE, "device batch above 2 GiB");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    Lane& L = ctx->lane;
    L.prepacked = false;  // device input: the batch packs on the device
    unsigned long long c[kCntSlots] = {};
    SCB_TRY(run_batch(ctx, L, kBatchReport, d_seqs, d_offsets, n, n_bytes, st, nullptr, c));
    rep->records_processed = c[kCntRecords];
    rep->total_windows = c[kCntTotalWindows];
    rep->valid_kmers = c[kCntValid];
    rep->positive_estimates = c[kCntPositive];
    rep->estimate_checksum = c[kCntChecksum];
    return SCB_OK;
}

// Per-window abundances of one device batch into d_out / d_valid (windows of the batch).
static scb_status abund_batch(scb_ctx* ctx, Lane& L, TileArgs& a, uint64_t n_seqs, cudaStream_t st,
                              unsigned long long* d_out, uint8_t* d_valid, uint64_t n_windows) {
    SCB_TRY(L.woff.ensure((n_seqs + 1) * 8));
    SCB_TRY(L.scan.ensure(((n_seqs + 1) / 1024 + 64) * 8 * 2));
    launch_seq_windows(a.offsets, n_seqs, ctx->g.k, a.cnt, L.woff.as<uint64_t>(), st);
    launch_scan_inplace(L.woff.as<uint64_t>(), n_seqs, L.scan.as<uint64_t>(), st);
    if (n_windows) {
        SCB_CUDA(cudaMemsetAsync(d_out, 0, n_windows * 8, st));
        SCB_CUDA(cudaMemsetAsync(d_valid, 0, n_windows, st));
    }
    a.woff = L.woff.as<uint64_t>();
    a.out = d_out;
    a.out_valid = d_valid;
    return query_device_batch(ctx, L, kModeAbund, a, st);
}

// Widens n estimates of `width` (2 or 4) bytes into u64, on the host's threads when n is large.
static void widen_estimates(uint64_t* dst, const uint8_t* src, uint64_t n, uint32_t width) {
    auto run = [&](uint64_t lo, uint64_t hi) {
        if (width == 2) {
            const uint16_t* s16 = reinterpret_cast<const uint16_t*>(src);
            for (uint64_t j = lo; j < hi; j++) dst[j] = s16[j];
        } else {
            const uint32_t* s32 = reinterpret_cast<const uint32_t*>(src);
            for (uint64_t j = lo; j < hi; j++) dst[j] = s32[j];
        }
    };
    const uint64_t parts = std::min<uint64_t>(std::max(1u, std::thread::hardware_concurrency()), n >> 19);
    if (parts <= 1) {
        run(0, n);
        return;
    }
    std::vector<std::thread> th;
    for (uint64_t t = 1; t < parts; t++) th.emplace_back(run, n * t / parts, n * (t + 1) / parts);
    run(0, n / parts);
    for (auto& x : th) x.join();
}

// The per-window estimates cross PCIe at the counters' width (2 bytes for 8- and 16-bit counters, 4
// for 32-bit ones) into pinned staging, and are widened into the caller's u64 buffer on the host.
scb_status scb_query_batch(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n, uint64_t* ab,
                           uint8_t* valid) {
    SCB_TRY(need_frozen(ctx));
    CtxLock lk(ctx);
    const uint32_t width = ctx->g.bits <= 16 ? 2u : 4u;
    SCB_TRY(for_each_chunk(ctx, seqs, offsets, n, [&](Lane& L, TileArgs& a, const Chunk& ch) -> scb_status {
        const uint64_t nw = windows_of(offsets + ch.seq0, ch.seq1 - ch.seq0, ctx->cfg.k);
        SCB_TRY(L.qout.ensure(std::max<uint64_t>(nw, 1) * 8));
        SCB_TRY(L.qvalid.ensure(std::max<uint64_t>(nw, 1)));
        SCB_TRY(L.qnarrow.ensure(std::max<uint64_t>(nw, 1) * width));
        SCB_TRY(abund_batch(ctx, L, a, ch.seq1 - ch.seq0, L.stream, L.qout.as<unsigned long long>(),
                            L.qvalid.as<uint8_t>(), nw));
        if (nw) {
            const uint64_t need = nw * (width + 1);
            if (need > ctx->q_stage_bytes) {
                SCB_CUDA(cudaStreamSynchronize(L.stream));
                if (ctx->q_stage) cudaFreeHost(ctx->q_stage);
                ctx->q_stage = nullptr;
                ctx->q_stage_bytes = 0;
                SCB_CUDA(cudaMallocHost((void**)&ctx->q_stage, need));
                ctx->q_stage_bytes = need;
            }
            launch_narrow_out(nullptr, nw, L.qout.as<unsigned long long>(), L.qnarrow.p, width, ctx->sm_count,
                              L.stream);
            SCB_CUDA(cudaMemcpyAsync(ctx->q_stage, L.qnarrow.p, nw * width, cudaMemcpyDeviceToHost, L.stream));
            SCB_CUDA(cudaMemcpyAsync(ctx->q_stage + nw * width, L.qvalid.p, nw, cudaMemcpyDeviceToHost, L.stream));
        }
        unsigned long long c[kCntSlots];
        SCB_TRY(read_counters(ctx, L, L.stream, c));  // waits for the copies
        if (nw) {
            widen_estimates(ab + ch.win0, ctx->q_stage, nw, width);
            std::memcpy(valid + ch.win0, ctx->q_stage + nw * width, nw);
        }
        return SCB_OK;
    }));
    return SCB_OK;
}

scb_status scb_query_batch_device(scb_ctx* ctx, const uint8_t* d_seqs, const uint64_t* d_offsets, uint64_t n,
                                  uint64_t n_bytes, void* stream, uint64_t* d_ab, uint8_t* d_valid) {
    SCB_TRY(need_frozen(ctx));
    CtxLock lk(ctx);
    if (n_bytes > kMaxBatchBytes - 64) return fail_kind(SCB_ERR_INTERNAL_STATE, "device batch above 2 GiB");
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    Lane& L = ctx->lane;
    L.prepacked = false;  // device input: the batch packs on the device
    SCB_TRY(ensure_lane_work(ctx, L, n_bytes));
    TileArgs a;
    SCB_TRY(prepare_batch(ctx, L, d_seqs, d_offsets, n, n_bytes, st, a));
    // window count: the scan's last element + last length is computed on the device; the
    // caller sized the outputs with scb_count_windows, so clear through the kernel writes only
    SCB_TRY(L.woff.ensure((n + 1) * 8));
    SCB_TRY(L.scan.ensure(((n + 1) / 1024 + 64) * 8 * 2));
    launch_seq_windows(d_offsets, n, ctx->g.k, a.cnt, L.woff.as<uint64_t>(), st);
    launch_scan_inplace(L.woff.as<uint64_t>(), n, L.scan.as<uint64_t>(), st);
    a.woff = L.woff.as<uint64_t>();
    a.out = reinterpret_cast<unsigned long long*>(d_ab);
    a.out_valid = d_valid;
    SCB_TRY(query_device_batch(ctx, L, kModeAbund, a, st));
    unsigned long long c[kCntSlots];
    return read_counters(ctx, L, st, c);
}

// Build from one staged batch, freeze, then stream-query the same staged batch.
static scb_status build_stream_batch(scb_ctx* ctx, Lane& L, const uint8_t* d_seqs, const uint64_t* d_offsets,
                                     uint64_t n, uint64_t n_bytes, cudaStream_t st, uint64_t* kmers,
                                     uint64_t* smers, scb_report* rep) {
    unsigned long long c1[kCntSlots] = {}, c2[kCntSlots] = {};
    const scb_status rs = run_batch(ctx, L, kBatchBuildStream, d_seqs, d_offsets, n, n_bytes, st, c1, c2);
    if (rs != SCB_OK) return rs;
    ctx->inserted_kmers += c1[kCntWindows];
    ctx->inserted_smers += c1[kCntSmers];
    ctx->frozen = true;
    if (kmers) *kmers = c1[kCntWindows];
    if (smers) *smers = c1[kCntSmers];
    rep->records_processed = c2[kCntRecords];
    rep->total_windows = c2[kCntTotalWindows];
    rep->valid_kmers = c2[kCntValid];
    rep->positive_estimates = c2[kCntPositive];
    rep->estimate_checksum = c2[kCntChecksum];
    return SCB_OK;
}

// Default largest piece of a host build + stream query (whole sequences; the first pieces are
// smaller, plan_ramp).
constexpr uint64_t kPieceBytes = 512ull << 20;


// Piece lanes, their upload events and the copy stream, for P pieces.
static scb_status ensure_pieces(scb_ctx* ctx, size_t P) {
    while (ctx->piece_lanes.size() < P) ctx->piece_lanes.push_back(std::make_unique<Lane>());
    while (ctx->piece_events.size() < P) {
        cudaEvent_t e;
        SCB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ctx->piece_events.push_back(e);
    }
    if (!ctx->copy_stream) SCB_CUDA(cudaStreamCreateWithFlags(&ctx->copy_stream, cudaStreamNonBlocking));
    return SCB_OK;
}

// Largest piece of a batch of `total` bytes: the setting (0: kPieceBytes), raised so that a batch
// has at most about kMaxPieces pieces (each piece has its own lane of device buffers).
constexpr uint64_t kMaxPieces = 32;
static uint64_t piece_bytes_for(const scb_ctx* ctx, uint64_t total) {
    const uint64_t pb = ctx->piece_bytes ? ctx->piece_bytes : kPieceBytes;
    return std::max<uint64_t>(pb, (total + kMaxPieces - 1) / kMaxPieces);
}

static bool pieces_apply(const scb_ctx* ctx, uint64_t total) {
    return ctx->graphs && probes_fit(ctx) && total / 2 >= piece_bytes_for(ctx, total);
}

// Starts the copy of the first piece's bytes (the ramp's first size, which needs no offsets) to
// the first piece lane, so that it runs while the host validates the offsets.  pre = the bytes
// in flight on the copy stream (0: none).  Reads only inside [offsets[0], offsets[n]).
static scb_status preload_first_piece(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                                      uint64_t& pre) {
    pre = 0;
    if (!seqs || !n || offsets[n] < offsets[0] || !pieces_apply(ctx, offsets[n] - offsets[0])) return SCB_OK;
    const uint64_t first = (uint64_t)ramp_first(piece_bytes_for(ctx, offsets[n] - offsets[0]));
    if (!first || first >= offsets[n] - offsets[0]) return SCB_OK;
    SCB_TRY(ensure_pieces(ctx, 1));
    Lane& L = *ctx->piece_lanes[0];
    SCB_TRY(L.ascii.ensure((first + 31) / 32 * 32 + 64));
    SCB_CUDA(cudaMemcpyAsync(L.ascii.p, seqs + offsets[0], first, cudaMemcpyHostToDevice, ctx->copy_stream));
    ctx->h2d_bytes += first;
    pre = first;
    return SCB_OK;
}

// Clears the prepacked mark of the piece lanes when a host build + stream query leaves.
struct PrepackedReset {
    scb_ctx* ctx;
    ~PrepackedReset() {
        for (auto& pl : ctx->piece_lanes) pl->prepacked = false;
    }
};

// Host build + stream query of a large batch in pieces, each in its own lane: piece p + 1 is
// copied to the device on the copy stream while piece p's insert graph runs, every piece keeps
// its super-k-mer records and probe slots, and after the last insert each piece's query runs on
// what it kept.  done = false: the batch is not split (small, graphs off, or a strategy other
// than grouped for some piece), and the caller runs it as one batch.
// pre = bytes of the first piece already being copied to the first piece lane (preload_first_piece).
static scb_status build_stream_pieces(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                                      uint64_t pre, uint64_t* kmers, uint64_t* smers, scb_report* rep, bool& done) {
    done = false;
    const uint64_t total = n ? offsets[n] - offsets[0] : 0;
    if (!pieces_apply(ctx, total)) return SCB_OK;
    const uint64_t piece_bytes = piece_bytes_for(ctx, total);
    std::vector<Chunk> pieces;
    SCB_TRY(plan_ramp(offsets, n, piece_bytes, pieces));
    if (pieces.size() < 2) return SCB_OK;
    for (const Chunk& c : pieces) {
        const uint64_t b = c.byte1 - c.byte0;
        if (resolve(ctx, ctx->insert_strategy, b, true) != SCB_STRATEGY_GROUPED ||
            resolve(ctx, ctx->query_strategy, b, false) != SCB_STRATEGY_GROUPED) {
            return SCB_OK;
        }
    }
    const size_t P = pieces.size();
    SCB_TRY(ensure_pieces(ctx, P));
    Lane& main = ctx->lane;
    SCB_TRY(ensure_lane_work(ctx, main, 0));  // its stream runs the pieces
    cudaStream_t cs = main.stream, xs = ctx->copy_stream;
    // pinned reads are copied asynchronously; pageable ones block the host per copy, which still
    // overlaps the GPU's work on the pieces already launched.  The first piece's bytes are already
    // on their way when it fits the preloaded size (a longer first sequence reallocates the
    // buffer, after the copy, and copies the piece again).
    // With host packing (the default) the host packs each piece after the first into the device
    // layout in a pinned staging area (all host threads) and copies 3 bits per base instead of the
    // 8-bit letters; it packs piece p + 1 while the GPU works on piece p.
    const bool hp = ctx->host_pack;
    PrepackedReset reset_marks{ctx};
    if (hp) {
        uint64_t max_groups = 0;
        for (const Chunk& c : pieces) max_groups = std::max<uint64_t>(max_groups, (c.byte1 - c.byte0 + 31) / 32);
        SCB_TRY(ensure_staging(ctx, max_groups));
    }
    const unsigned pack_threads = std::max(1u, std::thread::hardware_concurrency());
    auto upload = [&](size_t p) -> scb_status {
        const Chunk& c = pieces[p];
        Lane& L = *ctx->piece_lanes[p];
        const uint64_t ns = c.seq1 - c.seq0, nb = c.byte1 - c.byte0;
        SCB_TRY(ensure_lane(ctx, L, nb, ns));
        // the first piece goes as letters when they are already on their way (copied while the
        // offsets were validated, so the GPU starts without waiting for the host to pack it)
        if (hp && !(p == 0 && pre && nb <= pre)) {
            // the piece's graph sizes the lane's work buffers for its byte class: grow them before
            // the copy, so that no later growth drops the copied codes
            SCB_TRY(ensure_lane_work(ctx, L, std::max(nb, std::min(class_bytes(nb), kMaxBatchBytes - 64))));
            const uint64_t groups = (nb + 31) / 32;
            const int s = (int)(p & 1);
            SCB_CUDA(cudaEventSynchronize(ctx->stage_free[s]));  // the copy that last read this area
            host_pack(seqs + c.byte0, nb, ctx->stage_codes[s], ctx->stage_valid[s], pack_threads);
            SCB_CUDA(cudaMemcpyAsync(L.codes.p, ctx->stage_codes[s], (2 * groups + kPadWords) * 4,
                                     cudaMemcpyHostToDevice, xs));
            SCB_CUDA(cudaMemcpyAsync(L.valid.p, ctx->stage_valid[s], (groups + kPadWords) * 4, cudaMemcpyHostToDevice,
                                     xs));
            SCB_CUDA(cudaEventRecord(ctx->stage_free[s], xs));
            ctx->h2d_bytes += (3 * groups + 2 * kPadWords) * 4;
            L.prepacked = true;
        } else if (p != 0 || nb > pre) {
            SCB_CUDA(cudaMemcpyAsync(L.ascii.p, seqs + c.byte0, nb, cudaMemcpyHostToDevice, xs));
            ctx->h2d_bytes += nb;
        }
        SCB_CUDA(cudaMemcpyAsync(L.offsets.p, offsets + c.seq0, (ns + 1) * 8, cudaMemcpyHostToDevice, xs));
        ctx->h2d_bytes += (ns + 1) * 8;
        SCB_CUDA(cudaEventRecord(ctx->piece_events[p], xs));
        return SCB_OK;
    };
    std::vector<GraphRun> runs(P);
    SCB_TRY(upload(0));
    for (size_t p = 0; p < P; p++) {
        const Chunk& c = pieces[p];
        Lane& L = *ctx->piece_lanes[p];
        const uint64_t ns = c.seq1 - c.seq0, nb = c.byte1 - c.byte0;
        SCB_CUDA(cudaStreamWaitEvent(cs, ctx->piece_events[p], 0));
        if (c.byte0) {
            k_rebase<<<(unsigned)((ns + 1 + 255) / 256), 256, 0, cs>>>(L.offsets.as<uint64_t>(), ns + 1, c.byte0);
            note_launch();
        }
        SCB_TRY(graph_launch(ctx, L, kBatchInsertKeep, L.ascii.as<uint8_t>(), L.offsets.as<uint64_t>(), ns, nb, cs,
                             runs[p]));
        if (!runs[p].launched) {  // no graph: the eager insert (it waits for its own results)
            unsigned long long c_ins[kCntSlots] = {};
            SCB_TRY(run_batch(ctx, L, kBatchInsertKeep, L.ascii.as<uint8_t>(), L.offsets.as<uint64_t>(), ns, nb, cs,
                              c_ins, nullptr));
            ctx->inserted_kmers += c_ins[kCntWindows];
            ctx->inserted_smers += c_ins[kCntSmers];
            if (kmers) *kmers += c_ins[kCntWindows];
            if (smers) *smers += c_ins[kCntSmers];
        }
        if (p + 1 < P) SCB_TRY(upload(p + 1));
    }
    for (size_t p = 0; p < P; p++) {
        if (!runs[p].launched) continue;
        const Chunk& c = pieces[p];
        Lane& L = *ctx->piece_lanes[p];
        const uint64_t ns = c.seq1 - c.seq0, nb = c.byte1 - c.byte0;
        unsigned long long c_ins[kCntSlots] = {};
        bool ok = false;
        SCB_TRY(graph_finish(ctx, L, runs[p], cs, c_ins, nullptr, ok));
        if (!ok) {  // records outgrew the class: nothing was applied, insert it eagerly
            std::memset(c_ins, 0, sizeof(c_ins));
            SCB_TRY(run_batch(ctx, L, kBatchInsertKeep, L.ascii.as<uint8_t>(), L.offsets.as<uint64_t>(), ns, nb, cs,
                              c_ins, nullptr));
        }
        ctx->inserted_kmers += c_ins[kCntWindows];
        ctx->inserted_smers += c_ins[kCntSmers];
        if (kmers) *kmers += c_ins[kCntWindows];
        if (smers) *smers += c_ins[kCntSmers];
    }
    ctx->frozen = true;
    for (size_t p = 0; p < P; p++) {
        const Chunk& c = pieces[p];
        Lane& L = *ctx->piece_lanes[p];
        SCB_TRY(graph_launch(ctx, L, kBatchReportKept, L.ascii.as<uint8_t>(), L.offsets.as<uint64_t>(),
                             c.seq1 - c.seq0, c.byte1 - c.byte0, cs, runs[p]));
    }
    for (size_t p = 0; p < P; p++) {
        const Chunk& c = pieces[p];
        Lane& L = *ctx->piece_lanes[p];
        unsigned long long q[kCntSlots] = {};
        bool ok = false;
        SCB_TRY(graph_finish(ctx, L, runs[p], cs, nullptr, q, ok));
        if (!ok) {
            SCB_TRY(run_batch(ctx, L, kBatchReportKept, L.ascii.as<uint8_t>(), L.offsets.as<uint64_t>(),
                              c.seq1 - c.seq0, c.byte1 - c.byte0, cs, nullptr, q));
        }
        rep->records_processed += q[kCntRecords];
        rep->total_windows += q[kCntTotalWindows];
        rep->valid_kmers += q[kCntValid];
        rep->positive_estimates += q[kCntPositive];
        rep->estimate_checksum += q[kCntChecksum];
    }
    done = true;
    return SCB_OK;
}

scb_status scb_build_and_stream_query(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                                      uint64_t* kmers, uint64_t* smers, scb_report* rep) {
    if (!ctx || !rep) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    {
        CtxLock lk(ctx);
        if (ctx->frozen) return fail_kind(SCB_ERR_INTERNAL_STATE, "the index is frozen; inserts need a builder");
        if (!offsets) return fail_kind(SCB_ERR_INTERNAL_STATE, "null offsets");
        // the first piece's bytes copy while the offsets are validated; every return below
        // waits for that copy, which reads the caller's buffer
        uint64_t pre = 0;
        SCB_TRY(preload_first_piece(ctx, seqs, offsets, n, pre));
        const scb_status vs = check_offsets(offsets, n);
        if (vs != SCB_OK) {
            if (pre) cudaStreamSynchronize(ctx->copy_stream);
            return vs;
        }
        const uint64_t total = n ? offsets[n] - offsets[0] : 0;
        std::memset(rep, 0, sizeof(*rep));
        if (kmers) *kmers = 0;
        if (smers) *smers = 0;
        bool done = false;
        const scb_status ps = build_stream_pieces(ctx, seqs, offsets, n, pre, kmers, smers, rep, done);
        if (pre && (ps != SCB_OK || !done)) SCB_CUDA(cudaStreamSynchronize(ctx->copy_stream));
        SCB_TRY(ps);
        if (done) return SCB_OK;
        if (total <= kMaxBatchBytes - 64) {
            // one resident batch: copy once, insert, freeze, query the same staged codes (and,
            // with the grouped strategy, the same super-k-mer records)
            Lane& L = ctx->lane;
            Chunk c{0, n, n ? offsets[0] : 0, n ? offsets[n] : 0, 0};
            SCB_TRY(upload_chunk(ctx, L, seqs, offsets, c));
            return build_stream_batch(ctx, L, L.ascii.as<uint8_t>(), L.offsets.as<uint64_t>(), n, total, L.stream,
                                      kmers, smers, rep);
        }
    }
    SCB_TRY(scb_insert_batch(ctx, seqs, offsets, n, kmers, smers));
    SCB_TRY(scb_freeze(ctx));
    return scb_query_report(ctx, seqs, offsets, n, rep);
}

scb_status scb_build_and_stream_query_device(scb_ctx* ctx, const uint8_t* d_seqs, const uint64_t* d_offsets,
                                             uint64_t n, uint64_t n_bytes, void* stream, uint64_t* kmers,
                                             uint64_t* smers, scb_report* rep) {
    if (!ctx || !rep) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    CtxLock lk(ctx);
    if (ctx->frozen) return fail_kind(SCB_ERR_INTERNAL_STATE, "the index is frozen; inserts need a builder");
    if (n_bytes > kMaxBatchBytes - 64) return fail_kind(SCB_ERR_INTERNAL_STATE, "device batch above 2 GiB");
    Lane& L = ctx->lane;
    L.prepacked = false;  // device input: the batch packs on the device
    return build_stream_batch(ctx, L, d_seqs, d_offsets, n, n_bytes, reinterpret_cast<cudaStream_t>(stream), kmers,
                              smers, rep);
}

// Rows of a dense histogram plus an overflow list, sorted by value, zero counts dropped.
static void rows_from_hist(const std::vector<unsigned long long>& dense, std::vector<unsigned long long> ovf,
                           std::vector<std::pair<uint64_t, uint64_t>>& rows) {
    rows.clear();
    for (size_t v = 0; v < dense.size(); v++) {
        if (dense[v]) rows.emplace_back(v, dense[v]);
    }
    std::sort(ovf.begin(), ovf.end());
    for (size_t i = 0; i < ovf.size();) {
        size_t j = i;
        while (j < ovf.size() && ovf[j] == ovf[i]) j++;
        rows.emplace_back(ovf[i], j - i);
        i = j;
    }
}

static scb_status emit_rows(const std::vector<std::pair<uint64_t, uint64_t>>& rows, uint64_t* values, uint64_t* counts,
                            uint64_t cap, uint64_t* n_rows) {
    if (n_rows) *n_rows = rows.size();
    if (!values || !counts) return SCB_OK;
    if (cap < rows.size()) return fail_kind(SCB_ERR_INTERNAL_STATE, "row capacity too small");
    for (size_t i = 0; i < rows.size(); i++) {
        values[i] = rows[i].first;
        counts[i] = rows[i].second;
    }
    return SCB_OK;
}

scb_status scb_spectrum_distinct(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                                 uint64_t* values, uint64_t* counts, uint64_t capacity, uint64_t* n_rows,
                                 uint64_t* distinct_keys, uint64_t* queried_kmers) {
    SCB_TRY(need_frozen(ctx));
    CtxLock lk(ctx);
    SCB_TRY(check_offsets(offsets, n));
    // the context's buffers (grown, never freed per call: a free would synchronise the device)
    DevBuf& set = ctx->spec_set;
    DevBuf& hist = ctx->spec_hist;
    DevBuf& ovf = ctx->spec_ovf;
    const uint32_t dense = ctx->g.bits == 8 ? 256u : 65536u;
    SCB_TRY(hist.ensure((uint64_t)dense * 8));
    // the batch's window count bounds the overflow list (32-bit counters) and the tile kernel's key set
    uint64_t W = ~0ull;
    auto windows = [&]() {
        if (W == ~0ull) W = windows_of(offsets, n, ctx->cfg.k);
        return W;
    };
    const uint64_t ovf_cap = ctx->g.bits == 32 ? std::max<uint64_t>(windows(), 1) : 1;
    SCB_TRY(ovf.ensure(ovf_cap * 8));
    // the chunks run on the lane's stream, behind these clears
    SCB_TRY(ensure_lane_work(ctx, ctx->lane, 0));
    SCB_CUDA(cudaMemsetAsync(hist.p, 0, (uint64_t)dense * 8, ctx->lane.stream));
    // the global key set: twice the keys it can receive, at least 1024 slots, cleared on the
    // lane's stream
    uint64_t cap = 0;
    auto make_set = [&](uint64_t keys) -> scb_status {
        cap = 1024;
        while (cap < 2 * keys) cap <<= 1;
        SCB_TRY(set.ensure(cap * 8));
        SCB_CUDA(cudaMemsetAsync(set.p, 0xFF, cap * 8, ctx->lane.stream));
        return SCB_OK;
    };
    uint64_t distinct = 0, queried = 0, n_ovf = 0;
    // one device batch with the grouped strategy: the spectrum apply deduplicates each exclusive
    // bucket's keys in shared memory, so the global set only holds the keys of split buckets;
    // otherwise the tile kernel inserts every key into a set sized for all the windows
    std::vector<Chunk> plan;
    SCB_TRY(plan_chunks(offsets, n, ctx->cfg.k, ctx->tuning.host_batch_bytes, plan));
    const uint64_t total = n ? offsets[n] - offsets[0] : 0;
    const bool grouped = plan.size() == 1 && grouped_supported(ctx) &&
                         resolve(ctx, ctx->query_strategy, total, false) == SCB_STRATEGY_GROUPED;
    if (!grouped) SCB_TRY(make_set(windows()));
    SCB_TRY(for_each_chunk(ctx, seqs, offsets, n, [&](Lane& L, TileArgs& a, const Chunk&) -> scb_status {
        a.hist = hist.as<unsigned long long>();
        a.hist_dense = dense;
        a.ovf = ovf.as<unsigned long long>() + n_ovf;
        a.ovf_cap = ovf_cap - n_ovf;
        if (grouped) {
            SCB_TRY(mark(ctx, L, 9, L.stream));
            L.want_spectrum = true;
            const scb_status rs = grouped_prepare(ctx, L, a, L.stream);
            L.want_spectrum = false;
            SCB_TRY(rs);
            if (L.gs.produced) {
                // windows of the split buckets' items bound the global set
                unsigned long long* cnt = L.rec_count.as<unsigned long long>() + 3;
                unsigned long long shared_windows = 0;
                SCB_CUDA(cudaMemsetAsync(cnt, 0, 8, L.stream));
                launch_shared_item_windows(L.gs.ga.items, L.gs.ga.n_items, L.gs.ga.recs, cnt, L.stream);
                SCB_CUDA(cudaMemcpyAsync(&shared_windows, cnt, 8, cudaMemcpyDeviceToHost, L.stream));
                SCB_CUDA(cudaStreamSynchronize(L.stream));
                SCB_TRY(make_set(shared_windows));
                a.set_keys = set.as<unsigned long long>();
                a.set_mask = cap - 1;
                GroupArgs ga = L.gs.ga;
                ga.set_keys = a.set_keys;
                ga.set_mask = a.set_mask;
                ga.hist = a.hist;
                ga.hist_dense = a.hist_dense;
                ga.ovf = a.ovf;
                ga.ovf_cap = a.ovf_cap;
                SCB_TRY(launch_group_apply(ctx, L, kModeSpectrum, ga, a.cnt, L.gs.max_items, L.stream));
            }
            L.gs.valid = false;  // records bucketed for the spectrum, not for a later query
            SCB_TRY(mark(ctx, L, 10, L.stream));
            if (ctx->timing) L.spans |= kSpanQuery;
        } else {
            a.set_keys = set.as<unsigned long long>();
            a.set_mask = cap - 1;
            SCB_TRY(query_device_batch(ctx, L, kModeDistinct, a, L.stream));
        }
        unsigned long long c[kCntSlots];
        SCB_TRY(read_counters(ctx, L, L.stream, c));
        distinct += c[kCntDistinct];
        queried += c[kCntValid];
        n_ovf += c[kCntOverflow];
        return SCB_OK;
    }));
    std::vector<unsigned long long> h(dense), o(n_ovf);
    SCB_CUDA(cudaMemcpyAsync(h.data(), hist.p, (uint64_t)dense * 8, cudaMemcpyDeviceToHost, ctx->lane.stream));
    if (n_ovf) SCB_CUDA(cudaMemcpyAsync(o.data(), ovf.p, n_ovf * 8, cudaMemcpyDeviceToHost, ctx->lane.stream));
    SCB_CUDA(cudaStreamSynchronize(ctx->lane.stream));
    std::vector<std::pair<uint64_t, uint64_t>> rows;
    rows_from_hist(h, o, rows);
    if (distinct_keys) *distinct_keys = distinct;
    if (queried_kmers) *queried_kmers = queried;
    return emit_rows(rows, values, counts, capacity, n_rows);
}

scb_status scb_counter_histogram(scb_ctx* ctx, uint64_t* values, uint64_t* counts, uint64_t capacity,
                                 uint64_t* n_rows) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    CtxLock lk(ctx);
    const uint64_t slots = 1ull << ctx->cfg.counter_slots_exponent;
    const uint32_t dense = ctx->g.bits == 8 ? 256u : 65536u;
    const uint64_t ovf_cap = ctx->g.bits == 32 ? std::min<uint64_t>(slots, 1ull << 26) : 1;
    DevBuf hist, ovf, cnt;
    SCB_TRY(hist.ensure((uint64_t)dense * 8));
    SCB_TRY(ovf.ensure(ovf_cap * 8));
    SCB_TRY(cnt.ensure(8));
    SCB_CUDA(cudaMemset(hist.p, 0, (uint64_t)dense * 8));
    SCB_CUDA(cudaMemset(cnt.p, 0, 8));
    launch_counter_hist(ctx->table, slots, ctx->g.bits, hist.as<unsigned long long>(), dense,
                        ovf.as<unsigned long long>(), ovf_cap, cnt.as<unsigned long long>(), 0);
    SCB_CUDA(cudaGetLastError());
    unsigned long long n_ovf = 0;
    SCB_CUDA(cudaMemcpy(&n_ovf, cnt.p, 8, cudaMemcpyDeviceToHost));
    std::vector<unsigned long long> h(dense);
    SCB_CUDA(cudaMemcpy(h.data(), hist.p, (uint64_t)dense * 8, cudaMemcpyDeviceToHost));
    std::vector<std::pair<uint64_t, uint64_t>> rows;
    if (n_ovf <= ovf_cap) {
        std::vector<unsigned long long> o(n_ovf);
        if (n_ovf) SCB_CUDA(cudaMemcpy(o.data(), ovf.p, n_ovf * 8, cudaMemcpyDeviceToHost));
        rows_from_hist(h, std::move(o), rows);
    } else {
        // more large counters than the overflow list holds: histogram the table on the host
        std::vector<uint32_t> t(slots);
        SCB_CUDA(cudaMemcpy(t.data(), ctx->table, slots * 4, cudaMemcpyDeviceToHost));
        std::sort(t.begin(), t.end());
        for (size_t i = 0; i < t.size();) {
            size_t j = i;
            while (j < t.size() && t[j] == t[i]) j++;
            rows.emplace_back(t[i], j - i);
            i = j;
        }
    }
    return emit_rows(rows, values, counts, capacity, n_rows);
}

scb_status scb_batch_stats(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                           scb_stats* stats) {
    if (!ctx || !stats) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    CtxLock lk(ctx);
    std::memset(stats, 0, sizeof(*stats));
    return for_each_chunk(ctx, seqs, offsets, n, [&](Lane& L, TileArgs& a, const Chunk&) -> scb_status {
        SCB_TRY(run_tiles(ctx, L, kModeStats, a, L.stream));
        unsigned long long c[kCntSlots];
        SCB_TRY(read_counters(ctx, L, L.stream, c));
        stats->windows += c[kCntWindows];
        stats->super_kmers += c[kCntSuperKmers];
        stats->smers += c[kCntSmers];
        stats->sectors += c[kCntSectors];
        return SCB_OK;
    });
}

scb_status scb_debug_window_minimizers(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                                       uint32_t* out) {
    if (!ctx || !out) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    CtxLock lk(ctx);
    DevBuf dbg;
    return for_each_chunk(ctx, seqs, offsets, n, [&](Lane& L, TileArgs& a, const Chunk& ch) -> scb_status {
        const uint64_t nb = ch.byte1 - ch.byte0;
        SCB_TRY(dbg.ensure(std::max<uint64_t>(nb, 1) * 4));
        launch_fill_u32(dbg.as<uint32_t>(), 0xFFFFFFFFu, nb, L.stream);
        a.dbg = dbg.as<uint32_t>();
        SCB_TRY(run_tiles(ctx, L, kModeDebugMin, a, L.stream));
        unsigned long long c[kCntSlots];
        SCB_TRY(read_counters(ctx, L, L.stream, c));
        std::vector<uint32_t> h(nb);
        if (nb) SCB_CUDA(cudaMemcpy(h.data(), dbg.p, nb * 4, cudaMemcpyDeviceToHost));
        for (uint64_t i = 0; i < nb; i++) {
            out[ch.byte0 - offsets[0] + i] = h[i] == 0xFFFFFFFFu ? h[i] : (uint32_t)(h[i] + ch.byte0 - offsets[0]);
        }
        return SCB_OK;
    });
}

scb_status scb_set_timing(scb_ctx* ctx, int enable) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    CtxLock lk(ctx);
    if (enable) {
        for (auto& e : ctx->lane.ev) {
            if (!e) SCB_CUDA(cudaEventCreate(&e));
        }
    }
    ctx->timing = enable != 0;
    ctx->times = scb_timings{};
    ctx->lane.spans = 0;
    return SCB_OK;
}

scb_status scb_set_graphs(scb_ctx* ctx, int enable) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    CtxLock lk(ctx);
    ctx->graphs = enable != 0;
    return SCB_OK;
}

scb_status scb_set_fused_build(scb_ctx* ctx, int enable) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    CtxLock lk(ctx);
    ctx->fused_build = enable != 0;
    return SCB_OK;
}

scb_status scb_set_piece_bytes(scb_ctx* ctx, uint64_t piece_bytes) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    CtxLock lk(ctx);
    ctx->piece_bytes = piece_bytes;
    return SCB_OK;
}

scb_status scb_set_host_pack(scb_ctx* ctx, int enable) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    CtxLock lk(ctx);
    ctx->host_pack = enable != 0;
    return SCB_OK;
}

scb_status scb_h2d_bytes(scb_ctx* ctx, uint64_t* bytes) {
    if (!ctx || !bytes) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    CtxLock lk(ctx);
    *bytes = ctx->h2d_bytes;
    return SCB_OK;
}

scb_status scb_graph_stats(const scb_ctx* ctx, uint64_t* captures, uint64_t* replays, uint64_t* fallbacks) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    if (captures) *captures = ctx->lane.captures;
    if (replays) *replays = ctx->lane.replays;
    if (fallbacks) *fallbacks = ctx->lane.graph_fallbacks;
    return SCB_OK;
}

scb_status scb_get_timings(const scb_ctx* ctx, scb_timings* out) {
    if (!ctx || !out) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    *out = ctx->times;
    return SCB_OK;
}

scb_status scb_reset(scb_ctx* ctx) {
    if (!ctx) return fail_kind(SCB_ERR_INTERNAL_STATE, "null context");
    CtxLock lk(ctx);
    SCB_TRY(sync_ctx_streams(ctx));
    SCB_TRY(ensure_lane_work(ctx, ctx->lane, 0));  // the lane's stream
    cudaStream_t st = ctx->lane.stream;
    SCB_CUDA(cudaMemsetAsync(ctx->table, 0, ctx->table_bytes, st));
    SCB_CUDA(cudaMemsetAsync(ctx->status, 0, 64, st));
    SCB_CUDA(cudaStreamSynchronize(st));
    ctx->inserted_kmers = 0;
    ctx->inserted_smers = 0;
    ctx->frozen = false;
    return SCB_OK;
}

uint64_t scb_table_bytes(const scb_ctx* ctx) { return ctx ? ctx->table_bytes : 0; }

scb_status scb_table_download(const scb_ctx* cctx, void* host, uint64_t bytes) {
    if (!cctx || !host) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    scb_ctx* ctx = const_cast<scb_ctx*>(cctx);
    CtxLock lk(ctx);
    if (bytes != ctx->table_bytes) return fail_kind(SCB_ERR_INTERNAL_STATE, "table size mismatch");
    SCB_CUDA(cudaMemcpy(host, ctx->table, bytes, cudaMemcpyDeviceToHost));
    return SCB_OK;
}

scb_status scb_table_download_range(const scb_ctx* cctx, uint64_t offset, void* host, uint64_t bytes) {
    if (!cctx || (!host && bytes)) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    scb_ctx* ctx = const_cast<scb_ctx*>(cctx);
    CtxLock lk(ctx);
    if (offset > ctx->table_bytes || bytes > ctx->table_bytes - offset) {
        return fail_kind(SCB_ERR_INTERNAL_STATE, "range [" + std::to_string(offset) + ", +" + std::to_string(bytes) +
                                                     ") is outside the " + std::to_string(ctx->table_bytes) +
                                                     "-byte table");
    }
    if (bytes) SCB_CUDA(cudaMemcpy(host, static_cast<const uint8_t*>(ctx->table) + offset, bytes,
                                   cudaMemcpyDeviceToHost));
    return SCB_OK;
}

scb_status scb_table_upload(scb_ctx* ctx, const void* host, uint64_t bytes, uint64_t inserted_kmers) {
    if (!ctx || !host) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    CtxLock lk(ctx);
    if (bytes != ctx->table_bytes) return fail_kind(SCB_ERR_INTERNAL_STATE, "table size mismatch");
    SCB_CUDA(cudaMemcpy(ctx->table, host, bytes, cudaMemcpyHostToDevice));
    ctx->inserted_kmers = inserted_kmers;
    ctx->frozen = true;
    return SCB_OK;
}

// ---------------------------------------------------------------------------------------
// .scb (api.rs:28-29, 388-608)
// ---------------------------------------------------------------------------------------
static void put64(std::vector<uint8_t>& b, uint64_t v) {
    for (int i = 0; i < 8; i++) b.push_back((uint8_t)(v >> (8 * i)));
}
static void put32(std::vector<uint8_t>& b, uint32_t v) {
    for (int i = 0; i < 4; i++) b.push_back((uint8_t)(v >> (8 * i)));
}

static const uint8_t kMagic[8] = {'S', 'C', 'B', 'I', 'D', 'X', 0, 0};
static const uint32_t kFormatVersion = 2;

scb_status scb_save(const scb_ctx* cctx, const char* path) {
    if (!cctx || !path) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    scb_ctx* ctx = const_cast<scb_ctx*>(cctx);
    CtxLock lk(ctx);
    std::vector<uint8_t> head;
    head.insert(head.end(), kMagic, kMagic + 8);
    put32(head, kFormatVersion);
    const scb_config& c = ctx->cfg;
    put64(head, c.k);
    put64(head, c.m);
    put64(head, c.s);
    put64(head, c.n_hashes);
    head.push_back(c.counter_bits);
    head.push_back(c.counter_slots_exponent);
    head.push_back(c.block_slots_exponent);
    put64(head, c.threads);
    put64(head, c.queue);
    put64(head, ctx->inserted_kmers);
    put64(head, ctx->shard_count);
    put64(head, ctx->subblocks);
    put64(head, ctx->block_slots);
    put64(head, ctx->shard_mask);
    put32(head, ctx->shard_shift);
    put64(head, ctx->block_slots_mask);
    put64(head, ctx->nb_blocks);
    put64(head, ctx->block_mask);
    put64(head, c.n_hashes);
    FILE* fp = std::fopen(path, "wb");
    if (!fp) return fail(SCB_ERR_IO, std::string("I/O error for '") + path + "': cannot create file");
    bool ok = std::fwrite(head.data(), 1, head.size(), fp) == head.size();
    // the table is already in file order: stream it through a pinned buffer
    const uint64_t chunk = 64ull << 20;
    void* pinned = nullptr;
    if (cudaMallocHost(&pinned, chunk) != cudaSuccess) {
        std::fclose(fp);
        return fail_kind(SCB_ERR_INTERNAL_STATE, "pinned host allocation failed");
    }
    for (uint64_t off = 0; ok && off < ctx->table_bytes; off += chunk) {
        const uint64_t nb = std::min(chunk, ctx->table_bytes - off);
        if (cudaMemcpy(pinned, (const uint8_t*)ctx->table + off, nb, cudaMemcpyDeviceToHost) != cudaSuccess) {
            ok = false;
            break;
        }
        ok = std::fwrite(pinned, 1, nb, fp) == nb;
    }
    cudaFreeHost(pinned);
    ok = (std::fclose(fp) == 0) && ok;
    if (!ok) return fail(SCB_ERR_IO, std::string("I/O error for '") + path + "': write failed");
    return SCB_OK;
}

static bool get_exact(FILE* fp, void* dst, size_t n) { return std::fread(dst, 1, n, fp) == n; }
static bool get64(FILE* fp, uint64_t& v) {
    uint8_t b[8];
    if (!get_exact(fp, b, 8)) return false;
    v = 0;
    for (int i = 0; i < 8; i++) v |= (uint64_t)b[i] << (8 * i);
    return true;
}
static bool get32(FILE* fp, uint32_t& v) {
    uint8_t b[4];
    if (!get_exact(fp, b, 4)) return false;
    v = 0;
    for (int i = 0; i < 4; i++) v |= (uint32_t)b[i] << (8 * i);
    return true;
}

scb_status scb_load(const char* path, scb_ctx** out) {
    if (!path || !out) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    *out = nullptr;
    FILE* fp = std::fopen(path, "rb");
    if (!fp) return fail(SCB_ERR_IO, std::string("I/O error for '") + path + "': cannot open file");
    struct Closer {
        FILE* f;
        ~Closer() { std::fclose(f); }
    } closer{fp};
    const std::string io_short = std::string("I/O error for '") + path + "': failed to fill whole buffer";
    uint8_t magic[8];
    if (!get_exact(fp, magic, 8)) return fail(SCB_ERR_IO, io_short);
    if (std::memcmp(magic, kMagic, 8) != 0)
        return fail_kind(SCB_ERR_INVALID_INDEX_FORMAT, "bad SuperCountingBloom index magic");
    uint32_t version = 0;
    if (!get32(fp, version)) return fail(SCB_ERR_IO, io_short);
    if (version != kFormatVersion)
        return fail_kind(SCB_ERR_INVALID_INDEX_FORMAT, "unsupported index format version " + std::to_string(version));
    scb_config c{};
    if (!get64(fp, c.k) || !get64(fp, c.m) || !get64(fp, c.s) || !get64(fp, c.n_hashes) ||
        !get_exact(fp, &c.counter_bits, 1))
        return fail(SCB_ERR_IO, io_short);
    if (c.counter_bits != 8 && c.counter_bits != 16 && c.counter_bits != 32)
        return fail_kind(SCB_ERR_INVALID_INDEX_FORMAT, "unsupported counter width " + std::to_string(c.counter_bits));
    uint64_t inserted = 0;
    if (!get_exact(fp, &c.counter_slots_exponent, 1) || !get_exact(fp, &c.block_slots_exponent, 1) ||
        !get64(fp, c.threads) || !get64(fp, c.queue) || !get64(fp, inserted))
        return fail(SCB_ERR_IO, io_short);
    SCB_TRY(validate_config(&c));
    uint64_t sc, sb, bs, sm, bsm, nb, bm, nh;
    uint32_t ss;
    if (!get64(fp, sc) || !get64(fp, sb) || !get64(fp, bs) || !get64(fp, sm) || !get32(fp, ss) || !get64(fp, bsm) ||
        !get64(fp, nb) || !get64(fp, bm) || !get64(fp, nh))
        return fail(SCB_ERR_IO, io_short);
    scb_ctx probe;
    probe.cfg = c;
    fill_geometry(&probe);
    if (sc != probe.shard_count || sb != probe.subblocks || bs != probe.block_slots || sm != probe.shard_mask ||
        ss != probe.shard_shift || bsm != probe.block_slots_mask || nb != probe.nb_blocks || bm != probe.block_mask ||
        nh != c.n_hashes)
        return fail_kind(SCB_ERR_INVALID_INDEX_FORMAT, "stored filter layout does not match config");
    scb_ctx* ctx = nullptr;
    SCB_TRY(alloc_ctx(&c, &ctx));
    const uint64_t chunk = 64ull << 20;
    void* pinned = nullptr;
    if (cudaMallocHost(&pinned, chunk) != cudaSuccess) {
        delete ctx;
        return fail_kind(SCB_ERR_INTERNAL_STATE, "pinned host allocation failed");
    }
    for (uint64_t off = 0; off < ctx->table_bytes; off += chunk) {
        const uint64_t nbytes = std::min(chunk, ctx->table_bytes - off);
        if (!get_exact(fp, pinned, nbytes)) {
            cudaFreeHost(pinned);
            delete ctx;
            return fail(SCB_ERR_IO, io_short);
        }
        if (cudaMemcpy((uint8_t*)ctx->table + off, pinned, nbytes, cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaFreeHost(pinned);
            delete ctx;
            return fail_kind(SCB_ERR_INTERNAL_STATE, "table upload failed");
        }
    }
    cudaFreeHost(pinned);
    uint8_t extra;
    if (std::fread(&extra, 1, 1, fp) == 1) {
        delete ctx;
        return fail_kind(SCB_ERR_INVALID_INDEX_FORMAT, "trailing bytes after serialized index");
    }
    ctx->inserted_kmers = inserted;
    ctx->frozen = true;
    *out = ctx;
    return SCB_OK;
}


static void tuning_to_public(const Tuning& t, scb_tuning* out) {
    out->small_batch_bytes = t.small_bytes;
    out->insert_small = t.insert_small;
    out->insert_large = t.insert_large;
    out->query_small = t.query_small;
    out->query_large = t.query_large;
    out->bucket_records = t.bucket_records;
    out->apply_threads = t.apply_threads;
    out->host_batch_bytes = t.host_batch_bytes;
}

scb_status scb_get_tuning(const scb_ctx* ctx, scb_tuning* out) {
    if (!ctx || !out) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    std::memset(out, 0, sizeof(*out));
    tuning_to_public(ctx->tuning, out);
    return SCB_OK;
}

scb_status scb_autotune(scb_ctx* ctx, const uint8_t* seqs, const uint64_t* offsets, uint64_t n, scb_tuning* out) {
    if (!ctx || !seqs || !offsets) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    SCB_TRY(check_offsets(offsets, n));
    const uint64_t base = n ? offsets[0] : 0;
    const uint64_t total = n ? offsets[n] - base : 0;
    if (total == 0 || total > kMaxBatchBytes - 64)
        return fail_kind(SCB_ERR_INTERNAL_STATE, "the autotuning sample must hold 1 byte to 2 GiB of sequences");
    cudaSetDevice(ctx->device);
    scb_ctx* scratch_raw = nullptr;
    SCB_TRY(alloc_ctx(&ctx->cfg, &scratch_raw));
    std::unique_ptr<scb_ctx> scratch(scratch_raw);
    // the sample on the device, offsets rebased to its first byte
    DevBuf d_seq, d_off;
    SCB_TRY(d_seq.ensure(total + 64));
    SCB_TRY(d_off.ensure((n + 1) * 8));
    std::vector<uint64_t> off(offsets, offsets + n + 1);
    for (auto& v : off) v -= base;
    SCB_CUDA(cudaMemcpy(d_seq.p, seqs + base, total, cudaMemcpyHostToDevice));
    SCB_CUDA(cudaMemcpy(d_off.p, off.data(), (n + 1) * 8, cudaMemcpyHostToDevice));
    // small class: a prefix of about 1/32 of the sample (at least 64 KiB)
    uint64_t n_small = 0;
    const uint64_t small_target = std::max<uint64_t>(total / 32, 64 << 10);
    while (n_small < n && off[n_small + 1] <= small_target) n_small++;
    if (n_small == 0) n_small = 1;
    const uint64_t small_bytes = off[n_small];

    struct Cand {
        scb_strategy s;
        uint32_t bucket, threads;
    };
    uint32_t measured = 0;
    // build + stream-query of the first nseq sequences with one candidate; second run timed
    auto measure = [&](const Cand& c, uint64_t nseq, uint64_t nbytes, double& ins, double& q) -> scb_status {
        scratch->insert_strategy = scratch->query_strategy = c.s;
        scratch->tuning = Tuning();
        scratch->tuning.bucket_records = c.bucket;
        scratch->tuning.apply_threads = c.threads;
        for (int rep = 0; rep < 2; rep++) {
            SCB_TRY(scb_reset(scratch.get()));
            SCB_TRY(scb_set_timing(scratch.get(), 1));
            uint64_t km = 0, sm = 0;
            scb_report r;
            SCB_TRY(scb_build_and_stream_query_device(scratch.get(), d_seq.as<uint8_t>(), d_off.as<uint64_t>(), nseq,
                                                      nbytes, nullptr, &km, &sm, &r));
            scb_timings t;
            SCB_TRY(scb_get_timings(scratch.get(), &t));
            ins = t.pack_ms + t.insert_ms;
            q = t.query_ms;
        }
        SCB_TRY(scb_set_timing(scratch.get(), 0));
        measured++;
        return SCB_OK;
    };

    std::vector<Cand> cands = {{SCB_STRATEGY_PLAIN, 512, 256}, {SCB_STRATEGY_FUSED, 512, 256}};
    if (grouped_supported(ctx)) {
        // records-per-bucket targets that give the sample distinct bucket sizes; where the
        // 4096-counter cap makes several alike, only the default (512) or the one nearest to it
        // is measured, so a tie in noise never moves the setting
        std::vector<std::pair<uint32_t, uint32_t>> shifts;  // (shift, target)
        for (uint32_t b : {512u, 256u, 1024u, 2048u}) {
            const uint32_t sh = bucket_shift_for(ctx, records_estimate(ctx, total), b);
            bool seen = false;
            for (auto& x : shifts) seen = seen || x.first == sh;
            if (!seen) shifts.push_back({sh, b});
        }
        for (auto& x : shifts) {
            for (uint32_t t : {256u, 512u}) cands.push_back({SCB_STRATEGY_GROUPED, x.second, t});
        }
    }
    Tuning best;
    double best_ins = 1e30, best_q = 1e30, best_group = 1e30;
    Cand best_ins_c = cands[1], best_q_c = cands[1], best_g_c = cands[1];
    for (const Cand& c : cands) {
        double ins = 0, q = 0;
        SCB_TRY(measure(c, n, total, ins, q));
        if (ins < best_ins) {
            best_ins = ins;
            best_ins_c = c;
        }
        if (q < best_q) {
            best_q = q;
            best_q_c = c;
        }
        if (c.s == SCB_STRATEGY_GROUPED && ins + q < best_group) {
            best_group = ins + q;
            best_g_c = c;
        }
    }
    best.insert_large = best_ins_c.s;
    best.query_large = best_q_c.s;
    if (best_group < 1e30) {
        best.bucket_records = best_g_c.bucket;
        best.apply_threads = best_g_c.threads;
    }
    // small batches: the three strategies, grouped with the parameters chosen above
    double s_ins = 1e30, s_q = 1e30;
    for (scb_strategy st : {SCB_STRATEGY_PLAIN, SCB_STRATEGY_FUSED, SCB_STRATEGY_GROUPED}) {
        if (st == SCB_STRATEGY_GROUPED && !grouped_supported(ctx)) continue;
        double ins = 0, q = 0;
        SCB_TRY(measure({st, best.bucket_records, best.apply_threads}, n_small, small_bytes, ins, q));
        if (ins < s_ins) {
            s_ins = ins;
            best.insert_small = st;
        }
        if (q < s_q) {
            s_q = q;
            best.query_small = st;
        }
    }
    const bool split = best.insert_small != best.insert_large || best.query_small != best.query_large;
    // switch at the geometric midpoint of the two measured batch sizes
    best.small_bytes = split ? (uint64_t)std::sqrt((double)small_bytes * (double)total) : 0;
    // reads per batch of host calls: insert the whole sample through the host path in batches
    // of a quarter, a half and all of it
    best.valid = true;
    double best_host = 1e30;
    uint64_t best_chunk = best.host_batch_bytes;
    for (uint64_t div : {4ull, 2ull, 1ull}) {
        const uint64_t chunk = std::max<uint64_t>(total / div, 1 << 20);
        scratch->tuning = best;
        scratch->tuning.host_batch_bytes = chunk;
        scratch->insert_strategy = scratch->query_strategy = SCB_STRATEGY_AUTO;
        double ms = 0;
        for (int rep = 0; rep < 2; rep++) {  // the first run captures the batches' graphs
            SCB_TRY(scb_reset(scratch.get()));
            const auto t0 = std::chrono::steady_clock::now();
            uint64_t km = 0, sm = 0;
            SCB_TRY(scb_insert_batch(scratch.get(), seqs, offsets, n, &km, &sm));
            ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        }
        measured++;
        if (ms < best_host) {
            best_host = ms;
            best_chunk = div == 1 ? kMaxBatchBytes - 64 : chunk;
        }
        if (chunk >= total) break;
    }
    best.host_batch_bytes = best_chunk;
    ctx->tuning = best;
    {
        std::lock_guard<std::mutex> lk(g_tune_mu);
        g_tune_cache[tune_key(ctx->cfg)] = best;
    }
    if (out) {
        std::memset(out, 0, sizeof(*out));
        tuning_to_public(best, out);
        out->insert_ms = best_ins;
        out->query_ms = best_q;
        out->candidates = measured;
    }
    return SCB_OK;
}

}  // extern "C"

// ---------------------------------------------------------------------------------------
// Allocation-free query report.
//
// For callers that must not call cudaMalloc while they run: real-time serving threads that keep
// the allocator's latency (and the device-wide synchronisation cudaMalloc / cudaFree can imply)
// out of the request path, and hosts that hand this library a fixed device-memory budget at
// start-up.  The per-call scratch of the fused report query (2-bit codes, ACGT and
// sequence-start bitmaps, counters, the tile work counter) lives in one file-scope device array
// instead of buffers allocated per call.
//
// Limits: batches of at most kNoallocMaxBytes sequence bytes.  The array takes
// kNoallocScratchBytes on every GPU that loads this library, until the process exits.  Its
// device address is looked up once per device (with that device current) and kept, so the
// entry point must not be used after a cudaDeviceReset of that device.  All calls share the
// array: the call clears what must start at zero, and two calls whose work overlaps on the GPU
// (different streams or threads) race on it, so such callers serialise their calls.
// ---------------------------------------------------------------------------------------
namespace {

constexpr uint64_t kNoallocMaxBytes = 32ull << 20;  // 32 MiB of sequence bytes per call
constexpr uint64_t kNoallocGroups = kNoallocMaxBytes / 32;
constexpr uint64_t kNoallocCodesBytes = (2 * kNoallocGroups + kPadWords) * 4;
constexpr uint64_t kNoallocBitsBytes = (kNoallocGroups + kPadWords) * 4;
constexpr uint64_t kNoallocCodesOff = 256;  // counters (16 x u64) and the tile counter come first
constexpr uint64_t kNoallocValidOff = kNoallocCodesOff + ((kNoallocCodesBytes + 255) / 256) * 256;
constexpr uint64_t kNoallocStartOff = kNoallocValidOff + ((kNoallocBitsBytes + 255) / 256) * 256;
constexpr uint64_t kNoallocScratchBytes = kNoallocStartOff + ((kNoallocBitsBytes + 255) / 256) * 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

// Device address of g_noalloc_scratch, looked up once per device with that device current.
std::mutex g_noalloc_mu;
void* g_noalloc_addr[64] = {nullptr};

scb_status noalloc_scratch(int device, unsigned char** out) {
    if (device < 0 || device >= 64) return fail_kind(SCB_ERR_INTERNAL_STATE, "device index out of range");
    std::lock_guard<std::mutex> lk(g_noalloc_mu);
    if (!g_noalloc_addr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            return fail_kind(SCB_ERR_INTERNAL_STATE,
                             std::string("cudaGetSymbolAddress of the static scratch failed: ") + cudaGetErrorString(e));
        }
        g_noalloc_addr[device] = p;
    }
    *out = static_cast<unsigned char*>(g_noalloc_addr[device]);
    return SCB_OK;
}

}  // namespace

extern "C" scb_status scb_query_report_device_noalloc(scb_ctx* ctx, const uint8_t* d_seqs, const uint64_t* d_offsets,
                                                      uint64_t n_seqs, uint64_t n_bytes, void* stream,
                                                      scb_report* report) {
    SCB_TRY(need_frozen(ctx));
    if (!report) return fail_kind(SCB_ERR_INTERNAL_STATE, "null report");
    if (n_bytes > kNoallocMaxBytes) {
        return fail_kind(SCB_ERR_INTERNAL_STATE, "scb_query_report_device_noalloc takes at most " +
                                                     std::to_string(kNoallocMaxBytes) + " sequence bytes per call, got " +
                                                     std::to_string(n_bytes));
    }
    CtxLock lk(ctx);
    unsigned char* base = nullptr;
    SCB_TRY(noalloc_scratch(ctx->device, &base));
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    const uint64_t groups = (n_bytes + 31) / 32;
    unsigned long long* cnt = reinterpret_cast<unsigned long long*>(base);
    unsigned int* tiles = reinterpret_cast<unsigned int*>(base + kCntSlots * 8);
    uint32_t* codes = reinterpret_cast<uint32_t*>(base + kNoallocCodesOff);
    uint32_t* valid = reinterpret_cast<uint32_t*>(base + kNoallocValidOff);
    uint32_t* seqstart = reinterpret_cast<uint32_t*>(base + kNoallocStartOff);
    // the array keeps the previous call's contents: clear everything this call reads
    SCB_CUDA(cudaMemsetAsync(base, 0, kNoallocCodesOff, st));
    SCB_CUDA(cudaMemsetAsync(codes, 0, (2 * groups + kPadWords) * 4, st));
    SCB_CUDA(cudaMemsetAsync(valid, 0, (groups + kPadWords) * 4, st));
    SCB_CUDA(cudaMemsetAsync(seqstart, 0, (groups + kPadWords) * 4, st));
    if (n_bytes) launch_pack(d_seqs, n_bytes, codes, valid, st);
    launch_seqstart(d_offsets, n_seqs, n_bytes, seqstart, st);
    launch_seq_windows(d_offsets, n_seqs, ctx->g.k, cnt, nullptr, st);
    TileArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = ctx->g;
    a.codes = codes;
    a.valid = valid;
    a.seqstart = seqstart;
    a.n_bytes = n_bytes;
    a.n_code_words = 2 * groups;
    a.n_bit_words = groups;
    a.n_tiles = (uint32_t)((n_bytes + kTileWindows - 1) / kTileWindows);
    a.table = ctx->table;
    a.status = ctx->status;
    a.cnt = cnt;
    a.tile_counter = tiles;
    a.offsets = d_offsets;
    a.n_seqs = n_seqs;
    if (a.n_tiles) launch_tiles(kModeReport, a, tile_grid(kModeReport, ctx->g.bits, ctx->sm_count, a.n_tiles), st);
    SCB_CUDA(cudaGetLastError());
    unsigned long long c[kCntSlots];
    uint32_t status = 0;
    SCB_CUDA(cudaMemcpyAsync(c, cnt, kCntSlots * 8, cudaMemcpyDeviceToHost, st));
    SCB_CUDA(cudaMemcpyAsync(&status, ctx->status, 4, cudaMemcpyDeviceToHost, st));
    SCB_CUDA(cudaStreamSynchronize(st));
    if (status) return fail_kind(SCB_ERR_INTERNAL_STATE, "device status word 0x" + std::to_string(status));
    report->records_processed = c[kCntRecords];
    report->total_windows = c[kCntTotalWindows];
    report->valid_kmers = c[kCntValid];
    report->positive_estimates = c[kCntPositive];
    report->estimate_checksum = c[kCntChecksum];
    return SCB_OK;
}
