// Serving loop over a frozen, device-resident index: continuous batching of query requests.
//
// Requests (host buffers of sequences, per-window outputs) are split into pieces of whole
// sequences that fit one batch.  A scheduler thread keeps a FIFO of pending pieces and a fixed
// set of slots; each slot owns device buffers and pinned staging for one batch, sized so that
// all slots together fit the configured device-memory budget (admission control).  Whenever a
// slot is free and pieces are pending, the scheduler packs the oldest pieces into a batch and
// launches it on the slot's stream: H2D copy, 2-bit packing, the fused per-window abundance
// kernel (which, with the whole-stream spectrum on, also feeds the stream's distinct-k-mer set
// from the same estimates), narrowing of the estimates to the counters' width, D2H copy.  The
// device work of a batch (clears, packing, sequence starts, abundance kernel, narrowing) is one
// replay of a CUDA graph captured once per slot: the batch's sizes reach the
// kernels through a parameter block that a one-thread kernel writes before the replay, and the
// kernels' grids do not depend on the batch, so the same graph serves every batch shape.
// Batches of different slots overlap on the GPU; requests that arrive while
// others run are admitted as soon as a slot frees.  A host callback at the end of each batch
// wakes the scheduler, which scatters the results into the requests' output buffers and
// completes the requests whose pieces are all done.  Each slot has its own completion thread,
// which copies its batch's results out of pinned memory into the requests' buffers outside the
// server lock (a large batch with helper threads), so the copies of different slots run in
// parallel and never hold up the scheduler.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <thread>
#include <unordered_map>
#include <vector>

#include "scb_internal.h"

using namespace scb;

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Request {
    uint64_t id = 0;
    const uint8_t* seqs = nullptr;
    const uint64_t* offsets = nullptr;
    uint64_t n = 0;
    uint64_t* out = nullptr;
    uint8_t* valid = nullptr;
    uint64_t windows = 0;
    uint32_t pieces_left = 0;
    bool admitted = false;
    bool done = false;
    Clock::time_point submit, admit, finish;
};

struct Piece {
    Request* req = nullptr;
    uint64_t seq0 = 0, seq1 = 0;   // sequences of the request
    uint64_t win0 = 0, windows = 0;  // first output window (in the request) and count
    uint64_t bytes = 0;
};

struct Slot {
    cudaStream_t stream = nullptr;
    DevBuf ascii, offsets, woff, codes, valid, seqstart, out, outv, cnt, tiles, params;
    DevBuf outn;  // the estimates narrowed to the counters' width for the copy to the host
    cudaGraphExec_t graph = nullptr;  // the slot's batch, captured when the server starts
    uint64_t graph_launches = 0;
    uint8_t* h_ascii = nullptr;
    uint64_t* h_offsets = nullptr;
    uint64_t* h_woff = nullptr;
    uint8_t* h_outn = nullptr;  // narrowed estimates (2 or 4 bytes per window)
    uint8_t* h_outv = nullptr;
    std::vector<Piece> pieces;
    std::vector<uint64_t> piece_win;  // first window of each piece inside the batch output
    bool busy = false;
    std::atomic<bool> complete{false};
    // completion thread: woken by the batch's host callback
    std::thread finisher;
    std::mutex fmu;
    std::condition_variable fcv;
    ~Slot() {
        if (graph) cudaGraphExecDestroy(graph);
        if (h_ascii) cudaFreeHost(h_ascii);
        if (h_offsets) cudaFreeHost(h_offsets);
        if (h_woff) cudaFreeHost(h_woff);
        if (h_outn) cudaFreeHost(h_outn);
        if (h_outv) cudaFreeHost(h_outv);
        if (stream) cudaStreamDestroy(stream);
    }
};

uint64_t windows_of_seq(uint64_t len, uint64_t k) { return len >= k ? len + 1 - k : 0; }

}  // namespace

struct scb_server {
    scb_ctx* ctx = nullptr;
    scb_server_config cfg{};
    std::vector<std::unique_ptr<Slot>> slots;
    std::mutex mu;
    std::condition_variable wake;     // scheduler
    std::condition_variable settled;  // waiters
    std::deque<Piece> pending;
    std::unordered_map<uint64_t, std::unique_ptr<Request>> reqs;
    std::thread worker;
    bool stop = false;
    uint64_t next_id = 1;
    std::string error;  // first asynchronous failure, reported by waits
    // statistics since the last reset
    std::vector<double> latencies;
    uint64_t stat_windows = 0, stat_batches = 0;
    bool use_graphs = true;
    uint64_t captures = 0, replays = 0;
    // bytes per window of the estimates copied to the host: 2 for 8- and 16-bit counters, 4 for
    // 32-bit ones (an estimate never exceeds the counters' maximum); widened to u64 on the host
    uint32_t out_width = 2;
    // whole-stream spectrum: distinct canonical k-mers of every batch (set of 2^k keys, ~0 empty),
    // the dense histogram of their estimates, values past it (32-bit counters), and the counters
    // the distinct kernel adds to (windows, distinct keys, overflow entries)
    bool spectrum = false;
    DevBuf spec_set, spec_hist, spec_ovf, spec_cnt;
    uint64_t spec_mask = 0, spec_ovf_cap = 0;
    uint32_t spec_dense = 0;
    Clock::time_point first_submit{}, last_finish{};
    bool have_first = false;

    void run();
    void finish(Slot& s);
    void copy_out(Slot& s);
    uint64_t host_share = 1;  // threads a slot's copy-out may use: the host's threads / slots
    std::atomic<bool> stop_finishers{false};
    void add_spectrum(TileArgs& d, unsigned int* tile_counter) const;
    scb_status clear_spectrum(cudaStream_t st);
    scb_status launch(Slot& s);
    scb_status record(Slot& s, cudaStream_t st);
    scb_status capture(Slot& s);
    void complete(Slot& s);
};

namespace {

// Host callback at the end of a batch: set the slot's flag and wake the scheduler.  It takes no
// lock (a host function must not block); a wake-up lost between the scheduler's check and its
// sleep costs at most the scheduler's 100 us poll interval.
void CUDART_CB on_batch_done(void* p) {
    auto* pair = static_cast<std::pair<scb_server*, Slot*>*>(p);
    pair->second->complete.store(true, std::memory_order_release);
    pair->second->fcv.notify_one();
    delete pair;
}

}  // namespace

// Tile arguments of the abundance kernel over a slot's buffers (sizes of the batch, or of the
// shape class when the kernel reads the batch's own sizes from the parameter block).
static TileArgs tile_args(const scb_server& srv, const Slot& s, uint64_t bytes, uint64_t seqs) {
    const scb_ctx* c = srv.ctx;
    const uint64_t groups = (bytes + 31) / 32;
    TileArgs a;
    std::memset(&a, 0, sizeof(a));
    a.g = c->g;
    a.codes = s.codes.as<uint32_t>();
    a.valid = s.valid.as<uint32_t>();
    a.seqstart = s.seqstart.as<uint32_t>();
    a.n_bytes = bytes;
    a.n_code_words = 2 * groups;
    a.n_bit_words = groups;
    a.n_tiles = (uint32_t)((bytes + kTileWindows - 1) / kTileWindows);
    a.table = c->table;
    a.status = c->status;
    a.cnt = s.cnt.as<unsigned long long>();
    a.tile_counter = s.tiles.as<unsigned int>();
    a.offsets = s.offsets.as<uint64_t>();
    a.n_seqs = seqs;
    a.woff = s.woff.as<uint64_t>();
    a.out = s.out.as<unsigned long long>();
    a.out_valid = s.outv.as<uint8_t>();
    return a;
}

// Points a batch's tile arguments at the server's stream-wide distinct-k-mer set (kernel (f)): the
// abundance kernel in its kModeAbundDistinct form also inserts each window's canonical k-mer and
// counts the estimate of every new one.
void scb_server::add_spectrum(TileArgs& d, unsigned int* tile_counter) const {
    d.cnt = spec_cnt.as<unsigned long long>();
    d.tile_counter = tile_counter;
    d.set_keys = spec_set.as<unsigned long long>();
    d.set_mask = spec_mask;
    d.hist = spec_hist.as<unsigned long long>();
    d.hist_dense = spec_dense;
    d.ovf = spec_ovf.as<unsigned long long>();
    d.ovf_cap = spec_ovf_cap;
}

scb_status scb_server::clear_spectrum(cudaStream_t st) {
    SCB_CUDA(cudaMemsetAsync(spec_set.p, 0xFF, (spec_mask + 1) * 8, st));
    SCB_CUDA(cudaMemsetAsync(spec_hist.p, 0, (uint64_t)spec_dense * 8, st));
    SCB_CUDA(cudaMemsetAsync(spec_cnt.p, 0, kCntSlots * 8, st));
    SCB_CUDA(cudaStreamSynchronize(st));
    return SCB_OK;
}

// The graph body of one slot batch: sizes from the slot's parameter block, fixed grids.
scb_status scb_server::record(Slot& s, cudaStream_t st) {
    const BatchParams* bp = s.params.as<BatchParams>();
    const int sms = ctx->sm_count;
    SCB_CUDA(cudaMemsetAsync(s.cnt.p, 0, kCntSlots * 8, st));
    SCB_CUDA(cudaMemsetAsync(s.tiles.p, 0, 64, st));
    launch_clear_dyn(bp, s.seqstart.as<uint32_t>(), s.out.as<unsigned long long>(), s.outv.as<uint8_t>(), sms, st);
    launch_pack_dyn(bp, s.codes.as<uint32_t>(), s.valid.as<uint32_t>(), sms, st);
    launch_seqstart_dyn(bp, s.seqstart.as<uint32_t>(), sms, st);
    // capacities of the slot; the tile kernel reads the batch's sizes from bp
    TileArgs a = tile_args(*this, s, cfg.max_batch_bytes, cfg.max_batch_seqs);
    a.dyn = bp;
    if (spectrum) {  // one estimate per window serves the abundances and the stream's key set
        add_spectrum(a, s.tiles.as<unsigned int>());
        launch_tiles(kModeAbundDistinct, a, tile_grid(kModeAbundDistinct, ctx->g.bits, sms, a.n_tiles), st);
    } else {
        launch_tiles(kModeAbund, a, tile_grid(kModeAbund, ctx->g.bits, sms, a.n_tiles), st);
    }
    launch_narrow_out(bp, 0, s.out.as<unsigned long long>(), s.outn.p, out_width, sms, st);
    SCB_CUDA(cudaGetLastError());
    return SCB_OK;
}

scb_status scb_server::capture(Slot& s) {
    SCB_CUDA(cudaStreamBeginCapture(s.stream, cudaStreamCaptureModeRelaxed));
    record_launches_into(&s.graph_launches);
    const scb_status rs = record(s, s.stream);
    record_launches_into(nullptr);
    cudaGraph_t graph = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s.stream, &graph);
    if (rs != SCB_OK || e != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        if (rs != SCB_OK) return rs;
        return fail_kind(SCB_ERR_INTERNAL_STATE, std::string("graph capture: ") + cudaGetErrorString(e));
    }
    const cudaError_t ei = cudaGraphInstantiate(&s.graph, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) {
        s.graph = nullptr;
        return fail_kind(SCB_ERR_INTERNAL_STATE, std::string("graph instantiate: ") + cudaGetErrorString(ei));
    }
    captures++;
    return SCB_OK;
}

scb_status scb_server::launch(Slot& s) {
    scb_ctx* c = ctx;
    cudaStream_t st = s.stream;
    // stage the pieces contiguously in pinned memory, with batch-local offsets and window offsets
    uint64_t bytes = 0, seqs = 0, wins = 0;
    s.piece_win.clear();
    for (const Piece& p : s.pieces) {
        const Request& r = *p.req;
        s.piece_win.push_back(wins);
        for (uint64_t j = p.seq0; j < p.seq1; j++) {
            const uint64_t len = r.offsets[j + 1] - r.offsets[j];
            std::memcpy(s.h_ascii + bytes, r.seqs + r.offsets[j], len);
            s.h_offsets[seqs] = bytes;
            s.h_woff[seqs] = wins;
            bytes += len;
            wins += windows_of_seq(len, c->cfg.k);
            seqs++;
        }
    }
    s.h_offsets[seqs] = bytes;
    const uint64_t groups = (bytes + 31) / 32;
    if (bytes) SCB_CUDA(cudaMemcpyAsync(s.ascii.p, s.h_ascii, bytes, cudaMemcpyHostToDevice, st));
    SCB_CUDA(cudaMemcpyAsync(s.offsets.p, s.h_offsets, (seqs + 1) * 8, cudaMemcpyHostToDevice, st));
    if (seqs) SCB_CUDA(cudaMemcpyAsync(s.woff.p, s.h_woff, seqs * 8, cudaMemcpyHostToDevice, st));
    if (bytes && use_graphs) {
        if (!s.graph) SCB_TRY(capture(s));
        launch_set_params(s.params.as<BatchParams>(),
                          BatchParams{bytes, seqs, s.ascii.as<uint8_t>(), s.offsets.as<uint64_t>()}, st);
        SCB_CUDA(cudaGraphLaunch(s.graph, st));
        note_launches(s.graph_launches);
        replays++;
    } else {
        SCB_CUDA(cudaMemsetAsync(s.codes.p, 0, (2 * groups + kPadWords) * 4, st));
        SCB_CUDA(cudaMemsetAsync(s.valid.p, 0, (groups + kPadWords) * 4, st));
        SCB_CUDA(cudaMemsetAsync(s.seqstart.p, 0, (groups + kPadWords) * 4, st));
        SCB_CUDA(cudaMemsetAsync(s.cnt.p, 0, kCntSlots * 8, st));
        SCB_CUDA(cudaMemsetAsync(s.tiles.p, 0, 64, st));
        if (wins) {
            SCB_CUDA(cudaMemsetAsync(s.out.p, 0, wins * 8, st));
            SCB_CUDA(cudaMemsetAsync(s.outv.p, 0, wins, st));
        }
        if (bytes) {
            launch_pack(s.ascii.as<uint8_t>(), bytes, s.codes.as<uint32_t>(), s.valid.as<uint32_t>(), st);
            launch_seqstart(s.offsets.as<uint64_t>(), seqs, bytes, s.seqstart.as<uint32_t>(), st);
            TileArgs a = tile_args(*this, s, bytes, seqs);
            if (spectrum) {
                add_spectrum(a, s.tiles.as<unsigned int>());
                launch_tiles(kModeAbundDistinct, a, tile_grid(kModeAbundDistinct, c->g.bits, c->sm_count, a.n_tiles),
                             st);
            } else {
                launch_tiles(kModeAbund, a, tile_grid(kModeAbund, c->g.bits, c->sm_count, a.n_tiles), st);
            }
            if (wins) {
                launch_narrow_out(nullptr, wins, s.out.as<unsigned long long>(), s.outn.p, out_width, c->sm_count,
                                  st);
            }
            SCB_CUDA(cudaGetLastError());
        }
    }
    if (wins) {
        SCB_CUDA(cudaMemcpyAsync(s.h_outn, s.outn.p, wins * out_width, cudaMemcpyDeviceToHost, st));
        SCB_CUDA(cudaMemcpyAsync(s.h_outv, s.outv.p, wins, cudaMemcpyDeviceToHost, st));
    }
    s.complete.store(false, std::memory_order_relaxed);
    s.busy = true;
    auto* ud = new std::pair<scb_server*, Slot*>(this, &s);
    const cudaError_t e = cudaLaunchHostFunc(st, on_batch_done, ud);
    if (e != cudaSuccess) {
        delete ud;
        s.busy = false;
        return fail_kind(SCB_ERR_INTERNAL_STATE, std::string("cudaLaunchHostFunc: ") + cudaGetErrorString(e));
    }
    stat_batches++;
    return SCB_OK;
}

// Copies a finished batch's per-window results from the slot's pinned buffers into the requests'
// buffers, widening the estimates to u64 (the validity bytes are copied as they are).  A large
// batch (a full 16 MiB batch writes about 150 MB into the requests) is split into parts of 512 Ki
// windows that host_share threads work through together (the host's threads divided among the
// slots), so the copy-out keeps up with the GPU instead of holding the slot.
void scb_server::copy_out(Slot& s) {
    struct Part {
        uint64_t* est;           // the request's estimates
        uint8_t* valid;          // and validity bytes
        const uint8_t* src;      // the slot's narrowed estimates of the first window
        const uint8_t* src_valid;
        uint64_t n;              // windows
    };
    constexpr uint64_t kPart = 512ull << 10;
    const uint32_t w = out_width;
    std::vector<Part> parts;
    uint64_t total = 0;
    for (size_t i = 0; i < s.pieces.size(); i++) {
        const Piece& p = s.pieces[i];
        for (uint64_t off = 0; off < p.windows; off += kPart) {
            const uint64_t b = s.piece_win[i] + off;
            parts.push_back(Part{p.req->out + p.win0 + off, p.req->valid + p.win0 + off, s.h_outn + b * w,
                                 s.h_outv + b, std::min(kPart, p.windows - off)});
        }
        total += p.windows;
    }
    auto run = [w](const Part& q) {
        if (w == 2) {
            const uint16_t* src = reinterpret_cast<const uint16_t*>(q.src);
            for (uint64_t j = 0; j < q.n; j++) q.est[j] = src[j];
        } else {
            const uint32_t* src = reinterpret_cast<const uint32_t*>(q.src);
            for (uint64_t j = 0; j < q.n; j++) q.est[j] = src[j];
        }
        std::memcpy(q.valid, q.src_valid, q.n);
    };
    const unsigned helpers = (unsigned)std::min<uint64_t>(host_share, parts.size()) - 1u;
    if (helpers == 0 || total < 2 * kPart) {
        for (const Part& q : parts) run(q);
        return;
    }
    std::atomic<size_t> next{0};
    auto work = [&] {
        for (size_t i = next.fetch_add(1); i < parts.size(); i = next.fetch_add(1)) run(parts[i]);
    };
    std::vector<std::thread> th;
    th.reserve(helpers);
    for (unsigned t = 0; t < helpers; t++) th.emplace_back(work);
    work();
    for (auto& x : th) x.join();
}

// The slot's completion thread: waits for its batch's host callback (polling every 100 us, so a
// notification that arrives before the wait is never lost for long), copies the results into the
// requests' buffers without the server lock (a request's buffers stay valid until its wait returns,
// which needs this batch), then completes the pieces under the lock.
void scb_server::finish(Slot& s) {
    cudaSetDevice(ctx->device);
    while (true) {
        {
            std::unique_lock<std::mutex> lk(s.fmu);
            s.fcv.wait_for(lk, std::chrono::microseconds(100),
                           [&] { return s.complete.load(std::memory_order_acquire) || stop_finishers.load(); });
        }
        if (!s.complete.load(std::memory_order_acquire)) {
            if (stop_finishers.load()) break;
            continue;
        }
        copy_out(s);
        std::lock_guard<std::mutex> lk(mu);
        s.complete.store(false, std::memory_order_relaxed);
        complete(s);
        wake.notify_one();
    }
}

void scb_server::complete(Slot& s) {
    const auto now = Clock::now();
    for (size_t i = 0; i < s.pieces.size(); i++) {
        const Piece& p = s.pieces[i];
        Request& r = *p.req;
        if (--r.pieces_left == 0) {
            r.done = true;
            r.finish = now;
            latencies.push_back(ms_between(r.submit, r.finish));
            stat_windows += r.windows;
            last_finish = now;
        }
    }
    s.pieces.clear();
    s.busy = false;
    settled.notify_all();
}

void scb_server::run() {
    cudaSetDevice(ctx->device);
    std::unique_lock<std::mutex> lk(mu);
    while (true) {
        if (stop && pending.empty()) {
            bool idle = true;
            for (auto& sp : slots) idle = idle && !sp->busy;
            if (idle) break;
        }
        // admit pending pieces into free slots, oldest first
        for (auto& sp : slots) {
            if (pending.empty()) break;
            if (sp->busy) continue;
            uint64_t bytes = 0, seqs = 0;
            while (!pending.empty()) {
                const Piece& p = pending.front();
                const uint64_t ps = p.seq1 - p.seq0;
                if (!sp->pieces.empty() && (bytes + p.bytes > cfg.max_batch_bytes || seqs + ps > cfg.max_batch_seqs)) break;
                bytes += p.bytes;
                seqs += ps;
                if (!p.req->admitted) {
                    p.req->admitted = true;
                    p.req->admit = Clock::now();
                }
                sp->pieces.push_back(p);
                pending.pop_front();
            }
            if (launch(*sp) != SCB_OK) {
                if (error.empty()) error = last_error_slot();
                // fail the batch's requests rather than leave their waiters blocked
                for (const Piece& p : sp->pieces) {
                    if (--p.req->pieces_left == 0) {
                        p.req->done = true;
                        p.req->finish = Clock::now();
                    }
                }
                sp->pieces.clear();
                sp->busy = false;
                settled.notify_all();
            }
        }
        wake.wait_for(lk, std::chrono::microseconds(100), [&] {
            bool free_slot = false;
            for (auto& sp : slots) free_slot = free_slot || !sp->busy;
            return (free_slot && !pending.empty()) || (stop && pending.empty());
        });
    }
}

extern "C" {

scb_status scb_server_create(scb_ctx* ctx, const scb_server_config* cfg_in, scb_server** out) {
    if (!ctx || !out) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    *out = nullptr;
    if (!ctx->frozen) return fail_kind(SCB_ERR_INTERNAL_STATE, "serving needs a frozen index (into_index)");
    scb_server_config cfg = cfg_in ? *cfg_in : scb_server_config{};
    if (cfg.max_batch_bytes == 0) cfg.max_batch_bytes = 64ull << 20;
    if (cfg.max_batch_seqs == 0) cfg.max_batch_seqs = std::max<uint64_t>(1024, cfg.max_batch_bytes / 64);
    if (cfg.max_inflight == 0) cfg.max_inflight = 4;
    if (cfg.max_batch_bytes > kMaxBatchBytes / 2)
        return fail_kind(SCB_ERR_INVALID_CONFIG, "max_batch_bytes above 1 GiB");
    // device bytes of one slot: reads, 2-bit codes, two bitmaps, offsets, window offsets,
    // u64 + u8 outputs and the narrowed u16/u32 copy per window (at most one window per byte)
    const uint64_t B = cfg.max_batch_bytes, R = cfg.max_batch_seqs;
    const uint64_t groups = (B + 31) / 32;
    const uint64_t slot_bytes = (groups * 32 + 64) + (2 * groups + kPadWords) * 4 + 2 * (groups + kPadWords) * 4 +
                                (R + 1) * 8 * 2 + B * 13 + kCntSlots * 8 + 64;
    uint64_t n_slots = cfg.memory_budget_bytes ? cfg.memory_budget_bytes / slot_bytes : cfg.max_inflight;
    n_slots = std::min<uint64_t>(n_slots, cfg.max_inflight);
    if (n_slots == 0)
        return fail_kind(SCB_ERR_INVALID_CONFIG, "memory budget below one batch slot (" + std::to_string(slot_bytes) +
                                                     " bytes); lower max_batch_bytes or raise the budget");
    cudaSetDevice(ctx->device);
    auto srv = std::make_unique<scb_server>();
    srv->ctx = ctx;
    srv->cfg = cfg;
    srv->cfg.max_inflight = (uint32_t)n_slots;
    srv->host_share = std::max<uint64_t>(1, std::thread::hardware_concurrency() / n_slots);
    srv->use_graphs = ctx->graphs;
    srv->out_width = ctx->g.bits <= 16 ? 2u : 4u;
    for (uint64_t i = 0; i < n_slots; i++) {
        auto s = std::make_unique<Slot>();
        SCB_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
        SCB_TRY(s->ascii.ensure(groups * 32 + 64));
        SCB_TRY(s->offsets.ensure((R + 1) * 8));
        SCB_TRY(s->woff.ensure((R + 1) * 8));
        SCB_TRY(s->codes.ensure((2 * groups + kPadWords) * 4));
        SCB_TRY(s->valid.ensure((groups + kPadWords) * 4));
        SCB_TRY(s->seqstart.ensure((groups + kPadWords) * 4));
        SCB_TRY(s->out.ensure(std::max<uint64_t>(B, 1) * 8));
        SCB_TRY(s->outn.ensure(std::max<uint64_t>(B, 1) * 4));
        SCB_TRY(s->outv.ensure(B + 16));  // cleared in 16-byte stores
        SCB_TRY(s->cnt.ensure(kCntSlots * 8));
        SCB_TRY(s->tiles.ensure(64));
        SCB_TRY(s->params.ensure(sizeof(BatchParams)));
        SCB_CUDA(cudaMallocHost((void**)&s->h_ascii, B + 64));
        SCB_CUDA(cudaMallocHost((void**)&s->h_offsets, (R + 1) * 8));
        SCB_CUDA(cudaMallocHost((void**)&s->h_woff, (R + 1) * 8));
        SCB_CUDA(cudaMallocHost((void**)&s->h_outn, std::max<uint64_t>(B, 1) * srv->out_width));
        SCB_CUDA(cudaMallocHost((void**)&s->h_outv, std::max<uint64_t>(B, 1)));
        srv->slots.push_back(std::move(s));
    }
    if (cfg.spectrum_keys) {
        uint64_t cap = 1024;
        while (cap < 2 * cfg.spectrum_keys) cap <<= 1;
        srv->spectrum = true;
        srv->spec_mask = cap - 1;
        srv->spec_dense = ctx->g.bits == 8 ? 256u : 65536u;
        srv->spec_ovf_cap = ctx->g.bits == 32 ? cfg.spectrum_keys : 1;
        SCB_TRY(srv->spec_set.ensure(cap * 8));
        SCB_TRY(srv->spec_hist.ensure((uint64_t)srv->spec_dense * 8));
        SCB_TRY(srv->spec_ovf.ensure(srv->spec_ovf_cap * 8));
        SCB_TRY(srv->spec_cnt.ensure(kCntSlots * 8));
        SCB_TRY(srv->clear_spectrum(srv->slots[0]->stream));
    }
    // every slot's graph is captured here, before the first request: a slot that first runs while
    // others are busy (the first burst of arrivals) would otherwise hold its batch behind a capture
    if (srv->use_graphs) {
        for (auto& sp : srv->slots) SCB_TRY(srv->capture(*sp));
    }
    scb_server* raw = srv.release();
    for (auto& sp : raw->slots) {
        Slot* s = sp.get();
        s->finisher = std::thread([raw, s] { raw->finish(*s); });
    }
    raw->worker = std::thread([raw] { raw->run(); });
    *out = raw;
    return SCB_OK;
}

scb_status scb_server_submit(scb_server* s, const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                             uint64_t* abundances, uint8_t* valid, uint64_t* ticket) {
    if (!s || !offsets || !ticket) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    const uint64_t k = s->ctx->cfg.k;
    auto r = std::make_unique<Request>();
    r->seqs = seqs;
    r->offsets = offsets;
    r->n = n;
    r->out = abundances;
    r->valid = valid;
    // split into pieces of whole sequences that fit one batch
    std::vector<Piece> pieces;
    uint64_t win = 0;
    Piece cur;
    cur.req = r.get();
    for (uint64_t j = 0; j < n; j++) {
        if (offsets[j + 1] < offsets[j]) return fail_kind(SCB_ERR_INTERNAL_STATE, "offsets must be non-decreasing");
        const uint64_t len = offsets[j + 1] - offsets[j];
        if (len > s->cfg.max_batch_bytes)
            return fail_kind(SCB_ERR_INTERNAL_STATE, "a sequence longer than the server's max_batch_bytes");
        const uint64_t w = windows_of_seq(len, k);
        if (cur.seq1 > cur.seq0 &&
            (cur.bytes + len > s->cfg.max_batch_bytes || cur.seq1 - cur.seq0 + 1 > s->cfg.max_batch_seqs)) {
            pieces.push_back(cur);
            cur = Piece();
            cur.req = r.get();
            cur.seq0 = cur.seq1 = j;
            cur.win0 = win;
        }
        cur.seq1 = j + 1;
        cur.bytes += len;
        cur.windows += w;
        win += w;
    }
    if (cur.seq1 > cur.seq0) pieces.push_back(cur);
    if (win && (!abundances || !valid)) return fail_kind(SCB_ERR_INTERNAL_STATE, "null output buffers");
    r->windows = win;
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return fail_kind(SCB_ERR_CHANNEL_CLOSED, "worker channel closed: the server is shutting down");
    r->id = s->next_id++;
    r->submit = Clock::now();
    if (!s->have_first) {
        s->first_submit = r->submit;
        s->have_first = true;
    }
    r->pieces_left = (uint32_t)pieces.size();
    if (pieces.empty()) {
        r->done = true;
        r->admit = r->finish = r->submit;
        s->latencies.push_back(0.0);
    }
    for (auto& p : pieces) s->pending.push_back(p);
    *ticket = r->id;
    s->reqs.emplace(r->id, std::move(r));
    s->wake.notify_one();
    return SCB_OK;
}

scb_status scb_server_wait(scb_server* s, uint64_t ticket, scb_request_stats* stats) {
    if (!s) return fail_kind(SCB_ERR_INTERNAL_STATE, "null server");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(ticket);
    if (it == s->reqs.end()) return fail_kind(SCB_ERR_INTERNAL_STATE, "unknown ticket");
    Request* r = it->second.get();
    s->settled.wait(lk, [&] { return r->done; });
    if (stats) {
        stats->queue_ms = ms_between(r->submit, r->admit);
        stats->service_ms = ms_between(r->admit, r->finish);
        stats->total_ms = ms_between(r->submit, r->finish);
        stats->windows = r->windows;
    }
    s->reqs.erase(it);
    if (!s->error.empty()) return fail(SCB_ERR_INTERNAL_STATE, s->error);
    return SCB_OK;
}

scb_status scb_server_get_summary(scb_server* s, scb_server_summary* out) {
    if (!s || !out) return fail_kind(SCB_ERR_INTERNAL_STATE, "null argument");
    std::lock_guard<std::mutex> lk(s->mu);
    std::memset(out, 0, sizeof(*out));
    std::vector<double> v = s->latencies;
    std::sort(v.begin(), v.end());
    out->requests = v.size();
    out->windows = s->stat_windows;
    out->batches = s->stat_batches;
    out->slots = (uint32_t)s->slots.size();
    if (!v.empty()) {
        auto pct = [&](double q) {
            const double pos = q * (double)(v.size() - 1);
            const size_t lo = (size_t)pos;
            const size_t hi = std::min(lo + 1, v.size() - 1);
            return v[lo] + (v[hi] - v[lo]) * (pos - (double)lo);
        };
        out->p50_ms = pct(0.50);
        out->p99_ms = pct(0.99);
        out->max_ms = v.back();
        double sum = 0;
        for (double x : v) sum += x;
        out->mean_ms = sum / (double)v.size();
    }
    if (s->have_first) out->span_s = std::chrono::duration<double>(s->last_finish - s->first_submit).count();
    return SCB_OK;
}

scb_status scb_server_graph_stats(scb_server* s, uint64_t* captures, uint64_t* replays) {
    if (!s) return fail_kind(SCB_ERR_INTERNAL_STATE, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    if (captures) *captures = s->captures;
    if (replays) *replays = s->replays;
    return SCB_OK;
}

scb_status scb_server_reset_stats(scb_server* s) {
    if (!s) return fail_kind(SCB_ERR_INTERNAL_STATE, "null server");
    std::lock_guard<std::mutex> lk(s->mu);
    s->latencies.clear();
    s->stat_windows = 0;
    s->stat_batches = 0;
    s->have_first = false;
    if (s->spectrum) {
        cudaSetDevice(s->ctx->device);
        for (auto& sp : s->slots) SCB_CUDA(cudaStreamSynchronize(sp->stream));
        SCB_TRY(s->clear_spectrum(s->slots[0]->stream));
    }
    return SCB_OK;
}

scb_status scb_server_spectrum(scb_server* s, uint64_t* values, uint64_t* counts, uint64_t capacity,
                               uint64_t* n_rows, uint64_t* distinct_keys, uint64_t* queried_kmers) {
    if (!s) return fail_kind(SCB_ERR_INTERNAL_STATE, "null server");
    if (!s->spectrum) return fail_kind(SCB_ERR_INTERNAL_STATE, "the server was created without spectrum_keys");
    std::unique_lock<std::mutex> lk(s->mu);
    // every submitted piece answered: nothing pending, no slot busy
    s->settled.wait(lk, [&] {
        if (!s->pending.empty()) return false;
        for (auto& sp : s->slots) {
            if (sp->busy) return false;
        }
        return true;
    });
    cudaSetDevice(s->ctx->device);
    for (auto& sp : s->slots) SCB_CUDA(cudaStreamSynchronize(sp->stream));
    cudaStream_t st = s->slots[0]->stream;
    unsigned long long c[kCntSlots];
    uint32_t status = 0;
    std::vector<unsigned long long> dense(s->spec_dense);
    SCB_CUDA(cudaMemcpyAsync(c, s->spec_cnt.p, kCntSlots * 8, cudaMemcpyDeviceToHost, st));
    SCB_CUDA(cudaMemcpyAsync(&status, s->ctx->status, 4, cudaMemcpyDeviceToHost, st));
    SCB_CUDA(cudaMemcpyAsync(dense.data(), s->spec_hist.p, (uint64_t)s->spec_dense * 8, cudaMemcpyDeviceToHost, st));
    SCB_CUDA(cudaStreamSynchronize(st));
    if (status) {
        return fail_kind(SCB_ERR_INTERNAL_STATE, "device status word 0x" + std::to_string(status) +
                                                     " (2 = the stream has more distinct k-mers than spectrum_keys)");
    }
    const uint64_t n_ovf = std::min<uint64_t>(c[kCntOverflow], s->spec_ovf_cap);
    std::vector<unsigned long long> ovf(n_ovf);
    if (n_ovf) SCB_CUDA(cudaMemcpy(ovf.data(), s->spec_ovf.p, n_ovf * 8, cudaMemcpyDeviceToHost));
    std::vector<std::pair<uint64_t, uint64_t>> rows;
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
    if (distinct_keys) *distinct_keys = c[kCntDistinct];
    if (queried_kmers) *queried_kmers = c[kCntValid];
    if (n_rows) *n_rows = rows.size();
    if (!values || !counts) return SCB_OK;
    if (capacity < rows.size()) return fail_kind(SCB_ERR_INTERNAL_STATE, "row capacity too small");
    for (size_t i = 0; i < rows.size(); i++) {
        values[i] = rows[i].first;
        counts[i] = rows[i].second;
    }
    return SCB_OK;
}

void scb_server_destroy(scb_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->wake.notify_all();
    if (s->worker.joinable()) s->worker.join();  // returns once every slot is idle
    cudaSetDevice(s->ctx->device);
    for (auto& sp : s->slots) cudaStreamSynchronize(sp->stream);
    s->stop_finishers.store(true);
    for (auto& sp : s->slots) {
        sp->fcv.notify_all();
        if (sp->finisher.joinable()) sp->finisher.join();
    }
    delete s;
}

}  // extern "C"
