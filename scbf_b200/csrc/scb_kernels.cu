// SuperCountingBloom kernels for sm_100a.
//
//  (a) k_pack          ASCII -> 2-bit codes + ACGT bitmap, 32 bytes per thread, vector loads
//  (b)-(f) k_tiles     one persistent kernel over a device work queue of 1024-window tiles of
//                      the flat base stream.  A tile stages its codes and bitmaps in shared
//                      memory, computes the canonical m-mer hash keys once, picks each window's
//                      minimizer (kernel b), hashes s-mers (c) and then inserts (d), queries
//                      (e) or feeds the distinct-k-mer spectrum (f).  Reads of any length share
//                      the same tiles, so 150 bp and 100 kbp reads balance without per-read work.
//  plain pipeline      k_tiles<Materialize> writes per-window block ids and super-k-mer end
//                      flags to HBM, then k_plain_insert / k_plain_query run one thread per
//                      window from global memory: the one-launch-per-stage baseline.
//
// Insert semantics (filter.rs:199-237) in per-window form: super-k-mer j with windows
// [a_j, e_j] inserts s-mers a_j .. e_j + k - s into its block.  Window g therefore inserts its
// own s-mer g, and the last window of each super-k-mer also inserts s-mers g+1 .. g+k-s.
// Saturating increments commute, so any order gives the reference's counters.
// Query semantics (filter.rs:462-508): window g's estimate is the min over s-mers g .. g+k-s of
// their n_hashes-probe minimum inside window g's block, which is what the reference's deque
// computes per super-k-mer.
#include <atomic>
#include <cstdio>
#include <type_traits>

#include "scb_kernels.cuh"

namespace scb {

namespace {
std::atomic<uint64_t> g_launches{0};
}

// While a thread records a graph, its launches are counted into the graph (run at each replay).
thread_local uint64_t* t_recording = nullptr;
void note_launch() {
    if (t_recording) {
        ++*t_recording;
    } else {
        g_launches.fetch_add(1, std::memory_order_relaxed);
    }
}
void note_launches(uint64_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void record_launches_into(uint64_t* counter) { t_recording = counter; }
uint64_t kernel_launch_count() { return g_launches.load(std::memory_order_relaxed); }

// ---------------------------------------------------------------------------------------
// (a) packing
// ---------------------------------------------------------------------------------------
__device__ __forceinline__ void pack_word(uint32_t w, uint32_t& code8, uint32_t& valid4) {
    const uint32_t u = w & 0xDFDFDFDFu;  // upper-case letters
    const uint32_t m = __vcmpeq4(u, 0x41414141u) | __vcmpeq4(u, 0x43434343u) | __vcmpeq4(u, 0x47474747u) |
                       __vcmpeq4(u, 0x54545454u);
    uint32_t c = (w >> 1) & 0x03030303u;
    code8 = (c | (c >> 6) | (c >> 12) | (c >> 18)) & 0xFFu;
    uint32_t v = m & 0x01010101u;
    valid4 = (v | (v >> 7) | (v >> 14) | (v >> 21)) & 0xFu;
}

__global__ void k_pack(const uint8_t* __restrict__ ascii, uint64_t n, uint32_t* __restrict__ codes,
                       uint32_t* __restrict__ valid, uint64_t n_groups, int aligned) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t gi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; gi < n_groups; gi += stride) {
        const uint64_t base = gi * 32;
        uint32_t w[8];
        if (aligned && base + 32 <= n) {
            const uint4 x = __ldcs(reinterpret_cast<const uint4*>(ascii + base));
            const uint4 y = __ldcs(reinterpret_cast<const uint4*>(ascii + base + 16));
            w[0] = x.x; w[1] = x.y; w[2] = x.z; w[3] = x.w;
            w[4] = y.x; w[5] = y.y; w[6] = y.z; w[7] = y.w;
        } else {
#pragma unroll
            for (int j = 0; j < 8; j++) {
                uint32_t v = 0;
                for (int b = 0; b < 4; b++) {
                    const uint64_t idx = base + 4 * j + b;
                    if (idx < n) v |= (uint32_t)ascii[idx] << (8 * b);
                }
                w[j] = v;
            }
        }
        uint32_t c0 = 0, c1 = 0, vm = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            uint32_t c8, v4;
            pack_word(w[j], c8, v4);
            if (j < 4) {
                c0 |= c8 << (8 * j);
            } else {
                c1 |= c8 << (8 * (j - 4));
            }
            vm |= v4 << (4 * j);
        }
        codes[2 * gi] = c0;
        codes[2 * gi + 1] = c1;
        valid[gi] = vm;
    }
}

// Graph-replayable kernels.  The batch's sizes and inputs come from the device parameter block
// and every launch has a fixed grid (grid-stride loops), so a captured graph serves batches of any
// size that fit its buffers.

// Packing: groups [0, groups(n)) from the reads, then kPadWords zero words after the batch in
// both arrays (the padding the tile kernels may read).
__global__ void k_pack_dyn(const BatchParams* __restrict__ bp, uint32_t* __restrict__ codes,
                           uint32_t* __restrict__ valid) {
    const uint64_t n = bp->n_bytes;
    const uint64_t n_groups = (n + 31) / 32;
    const uint8_t* __restrict__ ascii = bp->ascii;
    const bool aligned = (reinterpret_cast<uintptr_t>(ascii) & 15u) == 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t gi = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; gi < n_groups + kPadWords; gi += stride) {
        if (gi >= n_groups) {
            const uint64_t t = gi - n_groups;
            valid[n_groups + t] = 0;
            codes[2 * n_groups + t] = 0;
            continue;
        }
        const uint64_t base = gi * 32;
        uint32_t w[8];
        if (aligned && base + 32 <= n) {
            const uint4 x = __ldcs(reinterpret_cast<const uint4*>(ascii + base));
            const uint4 y = __ldcs(reinterpret_cast<const uint4*>(ascii + base + 16));
            w[0] = x.x; w[1] = x.y; w[2] = x.z; w[3] = x.w;
            w[4] = y.x; w[5] = y.y; w[6] = y.z; w[7] = y.w;
        } else {
#pragma unroll
            for (int j = 0; j < 8; j++) {
                uint32_t v = 0;
                for (int b = 0; b < 4; b++) {
                    const uint64_t idx = base + 4 * j + b;
                    if (idx < n) v |= (uint32_t)ascii[idx] << (8 * b);
                }
                w[j] = v;
            }
        }
        uint32_t c0 = 0, c1 = 0, vm = 0;
#pragma unroll
        for (int j = 0; j < 8; j++) {
            uint32_t c8, v4;
            pack_word(w[j], c8, v4);
            if (j < 4) {
                c0 |= c8 << (8 * j);
            } else {
                c1 |= c8 << (8 * (j - 4));
            }
            vm |= v4 << (4 * j);
        }
        codes[2 * gi] = c0;
        codes[2 * gi + 1] = c1;
        valid[gi] = vm;
    }
}

// Clears the sequence-start bitmap of the batch and, when given, its per-window outputs (at most
// one window per byte).
__global__ void k_clear_dyn(const BatchParams* __restrict__ bp, uint32_t* __restrict__ seqstart,
                            unsigned long long* __restrict__ out, uint8_t* __restrict__ out_valid) {
    const uint64_t n = bp->n_bytes;
    const uint64_t n_words = (n + 31) / 32 + kPadWords;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t t0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    for (uint64_t i = t0; i < n_words; i += stride) seqstart[i] = 0;
    if (out) {
        for (uint64_t i = t0; i < n; i += stride) out[i] = 0;
        for (uint64_t i = t0; i < (n + 15) / 16; i += stride) reinterpret_cast<uint4*>(out_valid)[i] = make_uint4(0, 0, 0, 0);
    }
}

// Sequence starts (after k_clear_dyn).
__global__ void k_seqstart_dyn(const BatchParams* __restrict__ bp, uint32_t* __restrict__ seqstart) {
    const uint64_t n_bytes = bp->n_bytes, n_seqs = bp->n_seqs;
    const uint64_t* __restrict__ offsets = bp->offsets;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_seqs; j += stride) {
        const uint64_t a = offsets[j], b = offsets[j + 1];
        if (b > a && a < n_bytes) atomicOr(&seqstart[a >> 5], 1u << (a & 31));
    }
}

// Window and record counts (the QueryFastaReport totals).
__global__ void k_seq_windows_dyn(const BatchParams* __restrict__ bp, uint32_t k, unsigned long long* cnt) {
    const uint64_t n_seqs = bp->n_seqs;
    const uint64_t* __restrict__ offsets = bp->offsets;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    unsigned long long total = 0, recs = 0;
    const uint64_t n_iter = (n_seqs + stride - 1) / stride;
    for (uint64_t it = 0; it < n_iter; it++) {
        const uint64_t j = it * stride + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (j < n_seqs) {
            const uint64_t len = offsets[j + 1] - offsets[j];
            total += len >= k ? len + 1 - k : 0;
            recs += 1;
        }
    }
    warp_add_u64(&cnt[kCntTotalWindows], total);
    warp_add_u64(&cnt[kCntRecords], recs);
}

// Writes a batch's parameter block from kernel arguments (ahead of a graph replay), so the
// replay never waits on a copy engine that a large upload keeps busy.
__global__ void k_set_params(BatchParams* bp, BatchParams v) { *bp = v; }

void launch_set_params(BatchParams* bp, const BatchParams& v, cudaStream_t st) {
    k_set_params<<<1, 1, 0, st>>>(bp, v);
    note_launch();
}

void launch_pack_dyn(const BatchParams* bp, uint32_t* codes, uint32_t* valid, int sm_count, cudaStream_t st) {
    k_pack_dyn<<<(unsigned)(sm_count * 8), 256, 0, st>>>(bp, codes, valid);
    note_launch();
}

void launch_clear_dyn(const BatchParams* bp, uint32_t* seqstart, unsigned long long* out, uint8_t* out_valid,
                      int sm_count, cudaStream_t st) {
    k_clear_dyn<<<(unsigned)(sm_count * 4), 256, 0, st>>>(bp, seqstart, out, out_valid);
    note_launch();
}

void launch_seqstart_dyn(const BatchParams* bp, uint32_t* seqstart, int sm_count, cudaStream_t st) {
    k_seqstart_dyn<<<(unsigned)(sm_count * 2), 256, 0, st>>>(bp, seqstart);
    note_launch();
}

void launch_seq_windows_dyn(const BatchParams* bp, uint32_t k, unsigned long long* cnt, int sm_count,
                            cudaStream_t st) {
    k_seq_windows_dyn<<<(unsigned)(sm_count * 2), 256, 0, st>>>(bp, k, cnt);
    note_launch();
}

__global__ void k_seqstart(const uint64_t* __restrict__ offsets, uint64_t n_seqs, uint64_t n_bytes,
                           uint32_t* __restrict__ seqstart) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; j < n_seqs; j += stride) {
        const uint64_t a = offsets[j], b = offsets[j + 1];
        if (b > a && a < n_bytes) atomicOr(&seqstart[a >> 5], 1u << (a & 31));
    }
}

// Per-sequence window counts: woff[j] = max(0, len_j + 1 - k) (scanned afterwards), plus the
// records / total-windows fields of the report (api.rs:284-285).
__global__ void k_seq_windows(const uint64_t* __restrict__ offsets, uint64_t n_seqs, uint32_t k,
                              unsigned long long* cnt, uint64_t* woff) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    unsigned long long total = 0, recs = 0;
    const uint64_t n_iter = (n_seqs + stride - 1) / stride;
    for (uint64_t it = 0; it < n_iter; it++) {
        const uint64_t j = it * stride + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (j < n_seqs) {
            const uint64_t len = offsets[j + 1] - offsets[j];
            const uint64_t nw = len >= k ? len + 1 - k : 0;
            if (woff) woff[j] = nw;
            total += nw;
            recs += 1;
        }
    }
    warp_add_u64(&cnt[kCntTotalWindows], total);
    warp_add_u64(&cnt[kCntRecords], recs);
}

// Exclusive scan of u64 (three phases, recursive over block sums).
constexpr int kScanThreads = 1024;

__global__ void k_scan_blocks(uint64_t* data, uint64_t n, uint64_t* block_sums) {
    __shared__ uint64_t warp_tot[32];
    const uint64_t i = (uint64_t)blockIdx.x * kScanThreads + threadIdx.x;
    const uint64_t v = i < n ? data[i] : 0;
    uint64_t x = v;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int off = 1; off < 32; off <<= 1) {
        const uint64_t y = __shfl_up_sync(0xFFFFFFFFu, x, off);
        if (lane >= off) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
        uint64_t t = warp_tot[lane];
        for (int off = 1; off < 32; off <<= 1) {
            const uint64_t y = __shfl_up_sync(0xFFFFFFFFu, t, off);
            if (lane >= off) t += y;
        }
        warp_tot[lane] = t;
    }
    __syncthreads();
    const uint64_t incl = x + (wid > 0 ? warp_tot[wid - 1] : 0);
    if (i < n) data[i] = incl - v;
    if (threadIdx.x == kScanThreads - 1) block_sums[blockIdx.x] = incl;
}

__global__ void k_scan_add(uint64_t* data, uint64_t n, const uint64_t* block_prefix) {
    const uint64_t i = (uint64_t)blockIdx.x * kScanThreads + threadIdx.x;
    if (i < n) data[i] += block_prefix[blockIdx.x];
}

void launch_scan_inplace(uint64_t* data, uint64_t n, uint64_t* scratch, cudaStream_t st) {
    if (n == 0) return;
    const uint64_t nb = (n + kScanThreads - 1) / kScanThreads;
    k_scan_blocks<<<(unsigned)nb, kScanThreads, 0, st>>>(data, n, scratch);
    note_launch();
    if (nb > 1) {
        launch_scan_inplace(scratch, nb, scratch + nb, st);
        k_scan_add<<<(unsigned)nb, kScanThreads, 0, st>>>(data, n, scratch);
        note_launch();
    }
}

// ---------------------------------------------------------------------------------------
// Tile kernel
// ---------------------------------------------------------------------------------------
constexpr int kBack = 32;  // windows evaluated before a tile in stats mode (>= w)
constexpr int kFwd = 1;    // windows evaluated after a tile (super-k-mer end detection)
constexpr int kEvalMax = kTileWindows + kBack + kFwd;
// The cut's tiles: kBack windows before and kFwd after fill kTileWindows evaluated windows exactly,
// so every window's minimum comes from the four-window strips.
constexpr int kCutWindows = kTileWindows - kBack - kFwd;
constexpr int kKeysMax = kEvalMax + 32;
constexpr int kCodeWordsMax = (kEvalMax + 96 + 16) / 16 + 8;
constexpr int kBitWordsMax = (kEvalMax + 128 + 32) / 32 + 8;
constexpr uint16_t kNoWindow = 0xFFFFu;

constexpr int kNtChunks = 11;  // ceil(32 / 3) 3-base chunks of an m-mer

struct TileSmem {
    uint32_t codes[kCodeWordsMax];
    uint32_t valid[kBitWordsMax];
    uint32_t start[kBitWordsMax];
    uint32_t pk[kKeysMax];  // packed m-mer key: (hash >> 16) << 16 | position relative to e0
    alignas(8) uint16_t poff[kEvalMax];
    uint32_t block[kEvalMax];
    uint16_t ends[kTileWindows];
    // canonical ntHash tables: 3-base chunk contributions (fw, rc) and one-base roll terms
    uint32_t nt3f[kNtChunks * 64];
    uint32_t nt3r[kNtChunks * 64];
    uint32_t rollf[16];
    uint32_t rollr[16];
    uint32_t n_ends;
    uint32_t tile;
    uint64_t seq_lo, seq_hi;
    uint32_t warp_cnt[kTileThreads / 32];
    uint32_t warp_run[kTileThreads / 32];
};


// Fills the per-CTA ntHash tables for m-mers of length m:
//   nt3f[c][x] = XOR over bases t of chunk c of rotl(seed(base), 7 * (m - 1 - (3c + t)))
//   nt3r[c][x] = XOR over bases t of chunk c of rotl(seed(base ^ 2), 7 * (3c + t))
//   rollf[o | i << 2] = rotl(seed(o), 7m) ^ seed(i)
//   rollr[o | i << 2] = rotr(seed(o ^ 2), 7) ^ rotl(seed(i ^ 2), 7(m - 1))
// so that fw / rc of an m-mer are XORs of ceil(m/3) lookups and one base rolls in two.
__device__ void fill_nt_tables(TileSmem& sm, uint32_t m) {
    for (uint32_t e = threadIdx.x; e < kNtChunks * 64; e += blockDim.x) {
        const uint32_t c = e >> 6, x = e & 63;
        uint32_t f = 0, r = 0;
        for (uint32_t t = 0; t < 3; t++) {
            const uint32_t u = 3 * c + t;
            if (u >= m) break;
            const uint32_t b = (x >> (2 * t)) & 3u;
            f ^= rotl32(nt_seed(b), kNtRot * (m - 1 - u));
            r ^= rotl32(nt_seed(b ^ 2u), kNtRot * u);
        }
        sm.nt3f[e] = f;
        sm.nt3r[e] = r;
    }
    if (threadIdx.x < 16) {
        const uint32_t o = threadIdx.x & 3u, i = threadIdx.x >> 2;
        sm.rollf[threadIdx.x] = rotl32(nt_seed(o), kNtRot * m) ^ nt_seed(i);
        sm.rollr[threadIdx.x] = rotr32(nt_seed(o ^ 2u), kNtRot) ^ rotl32(nt_seed(i ^ 2u), kNtRot * (m - 1));
    }
}

// Canonical ntHash key of the m-mer whose 2-bit codes are in v (masked to m bases).
__device__ __forceinline__ void nt_direct_tab(const TileSmem& sm, uint64_t v, uint32_t m, uint32_t& fw,
                                              uint32_t& rc) {
    fw = 0;
    rc = 0;
    const uint32_t nch = (m + 2) / 3;
    for (uint32_t c = 0; c < nch; c++) {
        const uint32_t x = (uint32_t)(v >> (6 * c)) & 63u;
        fw ^= sm.nt3f[c * 64 + x];
        rc ^= sm.nt3r[c * 64 + x];
    }
}

// Block id of the super-k-mer whose minimizer m-mer starts at relative base b.
__device__ __forceinline__ uint32_t minimizer_block(const uint32_t* codes_s, uint32_t b, uint32_t m, uint64_t block_mask) {
    const uint64_t mm = codes64(codes_s, b) & len_mask(m);
    return (uint32_t)(xorshift64(canonical(mm, m)) & block_mask);
}

__device__ __forceinline__ uint32_t code_at(const uint32_t* words, uint32_t b) {
    return (words[b >> 4] >> (2 * (b & 15))) & 3u;
}

// Window minimum of four consecutive windows i0..i0+3 (needs w >= 4): window i0+j covers the
// packed keys [i0+j, i0+j+w-1] = suffix [i0+j, i0+3] of the first four keys, the middle
// [i0+4, i0+w-1] shared by all four, and the first j keys of the tail [i0+w, i0+w+2].  Lout[j]
// gets the minimum of the packed keys (leftmost minimum), Rout[j] of the keys with inverted
// position bits (rightmost minimum).
__device__ __forceinline__ void strip_minima(const uint32_t* pk, uint32_t i0, uint32_t w, uint32_t* Lout,
                                             uint32_t* Rout) {
    uint32_t a[4];
#pragma unroll
    for (int j = 0; j < 4; j++) a[j] = pk[i0 + j];
    uint32_t sl[4], sr[4];
    sl[3] = a[3];
    sr[3] = a[3] ^ 0xFFFFu;
#pragma unroll
    for (int j = 2; j >= 0; j--) {
        sl[j] = min(a[j], sl[j + 1]);
        sr[j] = min(a[j] ^ 0xFFFFu, sr[j + 1]);
    }
    uint32_t ml = 0xFFFFFFFFu, mr = 0xFFFFFFFFu;
    for (uint32_t o = 4; o < w; o++) {
        const uint32_t p = pk[i0 + o];
        ml = min(ml, p);
        mr = min(mr, p ^ 0xFFFFu);
    }
    uint32_t pl = 0xFFFFFFFFu, pr = 0xFFFFFFFFu;
#pragma unroll
    for (int j = 0; j < 4; j++) {
        if (j > 0) {
            const uint32_t t = pk[i0 + w + j - 1];
            pl = min(pl, t);
            pr = min(pr, t ^ 0xFFFFu);
        }
        Lout[j] = min(min(sl[j], ml), pl);
        Rout[j] = min(min(sr[j], mr), pr);
    }
}

// Largest j in [lo, hi] with offsets[j] <= pos.
__device__ __forceinline__ uint64_t seq_of(const uint64_t* offsets, uint64_t lo, uint64_t hi, uint64_t pos) {
    while (lo < hi) {
        const uint64_t mid = (lo + hi + 1) >> 1;
        if (__ldg(offsets + mid) <= pos) {
            lo = mid;
        } else {
            hi = mid - 1;
        }
    }
    return lo;
}

__device__ __forceinline__ bool set_insert(unsigned long long* keys, uint64_t mask, uint64_t key, uint32_t* status) {
    uint64_t i = xorshift64(key ^ 0x5851F42D4C957F2Dull) & mask;
    for (uint64_t probe = 0; probe <= mask; probe++) {
        const unsigned long long cur = __ldcg(keys + i);
        if (cur == key) return false;
        if (cur == ~0ull) {
            const unsigned long long prev = atomicCAS(keys + i, ~0ull, (unsigned long long)key);
            if (prev == ~0ull) return true;
            if (prev == key) return false;
        }
        i = (i + 1) & mask;
    }
    atomicOr(status, kStatusHashFull);
    return false;
}

template <int BITS>
__device__ __forceinline__ uint32_t window_estimate(const TileArgs& a, const DevGeom& g, const uint32_t* codes_s,
                                                    uint64_t rel, uint64_t base) {
    uint32_t r = CounterTraits<BITS>::kMax;
    const uint64_t sm = len_mask(g.s);
    for (uint32_t t = 0; t + g.s <= g.k; t++) {
        const uint64_t smer = canonical(codes64(codes_s, rel + t) & sm, g.s);
        const uint32_t e = estimate_smer<BITS>(a.table, g, base, smer);
        r = e < r ? e : r;
    }
    return r;
}

// KMC: 0 for any k and m, or (k << 8) | m compiled in (the cut of the default geometry, k = 31,
// m = 21, w = 11: the window-minimum strips unroll and the k- and m-masks are constants).
template <int MODE, int BITS, int KMC = 0>
__global__ void __launch_bounds__(kTileThreads, 8) k_tiles(TileArgs a) {
    __shared__ TileSmem sm;
    const DevGeom g = a.g;
    const uint32_t kv = KMC ? (uint32_t)(KMC >> 8) : g.k;
    const uint32_t mv = KMC ? (uint32_t)(KMC & 255) : g.m;
    const uint32_t wv = kv - mv + 1;
    const uint32_t tid = threadIdx.x;
    uint32_t* table32 = reinterpret_cast<uint32_t*>(a.table);
    unsigned long long c_win = 0, c_smer = 0, c_valid = 0, c_pos = 0, c_sum = 0, c_sk = 0, c_sec = 0, c_dist = 0;
    const uint64_t s_mask = len_mask(g.s);
    const uint32_t ks = kv - g.s;
    // modes that read a block id for every valid window (the cut computes it at ends only)
    constexpr bool kBlockPerWindow = MODE == kModeInsert || MODE == kModeReport || MODE == kModeAbund ||
                                     MODE == kModeDistinct || MODE == kModeAbundDistinct ||
                                     MODE == kModeMaterialize;
    constexpr bool kAbund = MODE == kModeAbund || MODE == kModeAbundDistinct;
    constexpr bool kDistinct = MODE == kModeDistinct || MODE == kModeAbundDistinct;
    // batch sizes: from the parameter block on graph replays, else from the arguments
    uint64_t n_bytes = a.n_bytes, n_seqs = a.n_seqs, n_code_words = a.n_code_words, n_bit_words = a.n_bit_words;
    uint32_t n_tiles = a.n_tiles;
    const uint64_t* offsets = a.offsets;
    if (a.dyn) {
        n_bytes = a.dyn->n_bytes;
        n_seqs = a.dyn->n_seqs;
        offsets = a.dyn->offsets;
        n_bit_words = (n_bytes + 31) / 32;
        n_code_words = 2 * n_bit_words;
        n_tiles = (uint32_t)((n_bytes + kTileWindows - 1) / kTileWindows);
    }
    constexpr uint32_t kWin = MODE == kModeCut ? (uint32_t)kCutWindows : (uint32_t)kTileWindows;  // tile windows
    if constexpr (MODE == kModeCut) n_tiles = (uint32_t)((n_bytes + kWin - 1) / kWin);
    fill_nt_tables(sm, mv);

    while (true) {
        if (tid == 0) sm.tile = atomicAdd(a.tile_counter, 1u);
        __syncthreads();
        const uint32_t tile = sm.tile;
        if (tile >= n_tiles) break;
        const uint64_t t0 = (uint64_t)tile * kWin;
        const uint32_t back = (MODE == kModeStats || MODE == kModeCut)
                                  ? (uint32_t)(t0 < (uint64_t)kBack ? t0 : (uint64_t)kBack)
                                  : 0u;
        const uint64_t e0 = t0 - back;
        const uint32_t n_eval = MODE == kModeCut ? (uint32_t)kTileWindows : back + kTileWindows + kFwd;
        const uint32_t n_keys = n_eval + wv - 1;

        // stage codes and bitmaps of the tile
        const uint64_t cb = e0 & ~15ull;
        const uint64_t cw0 = cb >> 4;
        const uint32_t n_cw = (uint32_t)((e0 + n_eval + 96 - cb) >> 4) + 3;
        for (uint32_t i = tid; i < n_cw; i += blockDim.x) {
            sm.codes[i] = (cw0 + i < n_code_words) ? __ldg(a.codes + cw0 + i) : 0u;
        }
        const uint64_t bb = e0 & ~31ull;
        const uint64_t bw0 = bb >> 5;
        const uint32_t n_bw = (uint32_t)((e0 + n_eval + 128 - bb) >> 5) + 3;
        for (uint32_t i = tid; i < n_bw; i += blockDim.x) {
            const bool in = bw0 + i < n_bit_words;
            sm.valid[i] = in ? __ldg(a.valid + bw0 + i) : 0u;
            sm.start[i] = in ? __ldg(a.seqstart + bw0 + i) : 0u;
        }
        if (kAbund && tid == 0) {
            sm.seq_lo = seq_of(offsets, 0, n_seqs, t0);
            const uint64_t last = t0 + kTileWindows;
            sm.seq_hi = seq_of(offsets, sm.seq_lo, n_seqs, last);
        }
        if (tid == 0) sm.n_ends = 0;
        __syncthreads();

        // canonical m-mer hash keys for m-mer positions e0 .. e0 + n_keys - 1, packed as
        // (hash >> 16) << 16 | position so that one integer min picks the leftmost minimum
        {
            const uint32_t per = (n_keys + blockDim.x - 1) / blockDim.x;  // <= 5 with 1024-window tiles
            const uint32_t q0 = tid * per;
            const uint32_t q1 = min(q0 + per, n_keys);
            if (q0 < q1) {
                const uint64_t b0 = e0 + q0 - cb;
                uint32_t fw, rc;
                uint64_t outs = codes64(sm.codes, b0);  // bases leaving: b0, b0+1, ...
                nt_direct_tab(sm, outs & len_mask(mv), mv, fw, rc);
                sm.pk[q0] = ((fw + rc) & 0xFFFF0000u) | q0;
                uint64_t ins = codes64(sm.codes, b0 + mv);  // bases entering: b0+m, b0+m+1, ...
                for (uint32_t q = q0 + 1; q < q1; q++) {
                    const uint32_t idx = ((uint32_t)outs & 3u) | (((uint32_t)ins & 3u) << 2);
                    outs >>= 2;
                    ins >>= 2;
                    fw = rotl32(fw, kNtRot) ^ sm.rollf[idx];
                    rc = rotr32(rc, kNtRot) ^ sm.rollr[idx];
                    sm.pk[q] = ((fw + rc) & 0xFFFF0000u) | q;
                }
            }
        }
        __syncthreads();

        // (b) minimizer of each evaluated window: leftmost minimum = min(pk), rightmost minimum =
        // min(pk ^ 0xFFFF) (the position bits inverted); strand from the count of T/G bases.
        // Windows 0..1023 go in strips of four per thread; the rest (and w < 4) one at a time.
        const uint32_t strip_end = wv >= 4 ? (uint32_t)kTileWindows : 0u;
        if (strip_end) {
            const uint32_t i0 = 4 * tid;
            const uint64_t pos0 = e0 + i0;
            const uint64_t vb = bits64(sm.valid, pos0 - bb), sb = bits64(sm.start, pos0 - bb);
            uint32_t lm[4], rm[4];
            strip_minima(sm.pk, i0, wv, lm, rm);
            // the T/G count of each window (bit 1 of a base's code), rolled one base at a time; with
            // k compiled in, the bases that leave and enter come from two 64-bit reads of the codes
            const uint64_t c_lo = codes64(sm.codes, pos0 - cb);  // bases pos0 .. pos0 + 31
            const uint64_t c_hi = KMC ? codes64(sm.codes, pos0 - cb + 32) : 0ull;
            uint32_t tg = __popcll(c_lo & len_mask(kv) & 0xAAAAAAAAAAAAAAAAull);
#pragma unroll
            for (uint32_t j = 0; j < 4; j++) {
                if (j > 0) {  // roll the T/G count by one base
                    if constexpr (KMC != 0) {
                        const uint32_t in = j - 1 + kv;  // base entering, relative to pos0
                        const uint32_t bit_in = in < 32 ? (uint32_t)(c_lo >> (2 * in + 1)) & 1u
                                                        : (uint32_t)(c_hi >> (2 * (in - 32) + 1)) & 1u;
                        tg += bit_in - ((uint32_t)(c_lo >> (2 * (j - 1) + 1)) & 1u);
                    } else {
                        const uint64_t out_b = pos0 + j - 1 - cb;
                        tg += (code_at(sm.codes, out_b + kv) >> 1) - (code_at(sm.codes, out_b) >> 1);
                    }
                }
                uint16_t po = kNoWindow;
                if (window_ok(vb >> j, sb >> j, kv)) {
                    po = (uint16_t)((2 * tg > kv) ? (lm[j] & 0xFFFFu) : ((rm[j] & 0xFFFFu) ^ 0xFFFFu));
                    if constexpr (kBlockPerWindow) sm.block[i0 + j] = minimizer_block(sm.codes, e0 + po - cb, mv, g.block_mask);
                }
                sm.poff[i0 + j] = po;
            }
        }
        for (uint32_t i = strip_end + tid; i < n_eval; i += blockDim.x) {
            const uint64_t pos = e0 + i;
            uint16_t po = kNoWindow;
            if (window_ok(bits64(sm.valid, pos - bb), bits64(sm.start, pos - bb), kv)) {
                uint32_t lmin = 0xFFFFFFFFu, rmin = 0xFFFFFFFFu;
                for (uint32_t o = 0; o < wv; o++) {
                    const uint32_t p = sm.pk[i + o];
                    lmin = min(lmin, p);
                    rmin = min(rmin, p ^ 0xFFFFu);
                }
                const uint64_t kval = codes64(sm.codes, pos - cb) & len_mask(kv);
                const uint32_t tg = __popcll(kval & 0xAAAAAAAAAAAAAAAAull);
                po = (uint16_t)((2 * tg > kv) ? (lmin & 0xFFFFu) : ((rmin & 0xFFFFu) ^ 0xFFFFu));
                if constexpr (kBlockPerWindow) sm.block[i] = minimizer_block(sm.codes, e0 + po - cb, mv, g.block_mask);
            }
            sm.poff[i] = po;
        }
        __syncthreads();

        if constexpr (MODE == kModeInsert) {
            for (uint32_t i = tid; i < kTileWindows; i += blockDim.x) {
                const uint16_t po = sm.poff[i];
                if (po == kNoWindow) continue;
                const uint64_t pos = t0 + i;
                const uint64_t base = block_base(g, sm.block[i]);
                const uint64_t smer = canonical(codes64(sm.codes, pos - cb) & s_mask, g.s);
                insert_smer<BITS>(table32, g, base, smer, a.status);
                c_win++;
                c_smer++;
                if (sm.poff[i + 1] != po) {
                    c_sk++;
                    if (ks > 0) sm.ends[atomicAdd(&sm.n_ends, 1u)] = (uint16_t)i;
                }
            }
            __syncthreads();
            const uint32_t n_tasks = sm.n_ends * ks;
            for (uint32_t f = tid; f < n_tasks; f += blockDim.x) {
                const uint32_t e = sm.ends[f / ks];
                const uint32_t u = 1 + f % ks;
                const uint64_t smer = canonical(codes64(sm.codes, t0 + e + u - cb) & s_mask, g.s);
                insert_smer<BITS>(table32, g, block_base(g, sm.block[e]), smer, a.status);
                c_smer++;
            }
        } else if constexpr (MODE == kModeReport || kAbund || kDistinct) {
            for (uint32_t i = tid; i < kTileWindows; i += blockDim.x) {
                if (sm.poff[i] == kNoWindow) continue;
                const uint64_t pos = t0 + i;
                const uint32_t r = window_estimate<BITS>(a, g, sm.codes, pos - cb, block_base(g, sm.block[i]));
                if constexpr (MODE == kModeReport) {
                    c_valid++;
                    c_pos += r > 0;
                    c_sum += r;
                }
                if constexpr (kAbund) {
                    const uint64_t j = seq_of(offsets, sm.seq_lo, sm.seq_hi, pos);
                    const uint64_t o = a.woff[j] + (pos - __ldg(offsets + j));
                    a.out[o] = r;
                    a.out_valid[o] = 1;
                }
                if constexpr (kDistinct) {
                    c_valid++;
                    const uint64_t key = canonical(codes64(sm.codes, pos - cb) & len_mask(kv), kv);
                    if (set_insert(a.set_keys, a.set_mask, key, a.status)) {
                        c_dist++;
                        if (r < a.hist_dense) {
                            atomicAdd(a.hist + r, 1ull);
                        } else {
                            const unsigned long long o = atomicAdd(&a.cnt[kCntOverflow], 1ull);
                            if (o < a.ovf_cap) {
                                a.ovf[o] = r;
                            } else {
                                atomicOr(a.status, kStatusOverflowFull);
                            }
                        }
                    }
                }
            }
        } else if constexpr (MODE == kModeStats) {
            const uint32_t bytes_per = BITS / 8;
            const uint64_t block_sectors = ((1ull << g.block_log2) * bytes_per + 31) / 32;
            for (uint32_t i = back + tid; i < back + kTileWindows; i += blockDim.x) {
                const uint16_t po = sm.poff[i];
                if (po == kNoWindow) continue;
                c_win++;
                if (sm.poff[i + 1] == po) continue;
                c_sk++;
                uint32_t st = i;
                while (st > 0 && sm.poff[st - 1] == po) st--;
                const uint32_t n_sm = (i - st + 1) + ks;
                c_smer += n_sm;
                if (block_sectors <= 256) {
                    uint32_t seen[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                    const uint64_t base_rel = 0;
                    (void)base_rel;
                    for (uint32_t q = 0; q < n_sm; q++) {
                        const uint64_t smer = canonical(codes64(sm.codes, e0 + st + q - cb) & s_mask, g.s);
                        uint64_t hash = xorshift64(smer);
                        for (uint32_t h = 1;; h++) {
                            const uint32_t sec = (uint32_t)(((hash & g.bs_mask) * bytes_per) >> 5);
                            seen[sec >> 5] |= 1u << (sec & 31);
                            if (h >= g.h) break;
                            hash = xorshift64(hash);
                        }
                    }
                    uint32_t d = 0;
                    for (int x = 0; x < 8; x++) d += __popc(seen[x]);
                    c_sec += d;
                } else {
                    c_sec += (unsigned long long)n_sm * g.h;
                }
            }
        } else if constexpr (MODE == kModeCut) {
            // one record per super-k-mer, emitted at its last window: (block, first window, windows).
            // Thread t looks at evaluated windows 4t .. 4t+3 (its strip); the tile's own windows
            // are [back, back + kCutWindows).  A window starts a super-k-mer when its minimizer
            // position differs from the window before, and ends one when it differs from the
            // window after.  A block-wide running maximum of start positions gives each end its
            // first window (a super-k-mer spans at most w <= 32 = kBack windows, so every one
            // that ends in the tile starts inside the evaluated range).
            const uint32_t lane = tid & 31, wid = tid >> 5;
            const uint32_t i0 = 4 * tid;
            const uint2 raw = *reinterpret_cast<const uint2*>(sm.poff + i0);
            const uint32_t p[4] = {raw.x & 0xFFFFu, raw.x >> 16, raw.y & 0xFFFFu, raw.y >> 16};
            const uint32_t pv = tid ? (uint32_t)sm.poff[i0 - 1] : (uint32_t)kNoWindow;
            const uint32_t pn = sm.poff[i0 + 4];  // index kTileWindows: never a tile window's successor
            const uint32_t lo = back, hi = back + (uint32_t)kCutWindows;
            uint32_t mine = 0, run = 0, endmask = 0;
            uint32_t rs[4];  // 1 + the latest start in this strip up to each window (0: none yet)
#pragma unroll
            for (uint32_t j = 0; j < 4; j++) {
                const uint32_t i = i0 + j;
                const uint32_t before = j ? p[j - 1] : pv, after = j < 3 ? p[j + 1] : pn;
                const bool ok = p[j] != kNoWindow;
                if (ok && before != p[j]) run = i + 1;
                rs[j] = run;
                const bool in = i >= lo && i < hi;
                c_win += (ok && in) ? 1u : 0u;
                if (ok && in && after != p[j]) {
                    endmask |= 1u << j;
                    mine++;
                }
            }
            uint32_t incl = mine, rmax = run;
            for (int off = 1; off < 32; off <<= 1) {
                const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, incl, off);
                const uint32_t z = __shfl_up_sync(0xFFFFFFFFu, rmax, off);
                if ((int)lane >= off) {
                    incl += y;
                    rmax = max(rmax, z);
                }
            }
            uint32_t rprev = __shfl_up_sync(0xFFFFFFFFu, rmax, 1);
            if (lane == 0) rprev = 0;
            if (lane == 31) {
                sm.warp_cnt[wid] = incl;
                sm.warp_run[wid] = rmax;
            }
            __syncthreads();
            // the warps' totals: an 8-lane scan of their counts (sum) and run starts (maximum)
            constexpr uint32_t kWarps = kTileThreads / 32;
            uint32_t wc = lane < kWarps ? sm.warp_cnt[lane] : 0u;
            uint32_t wr = lane < kWarps ? sm.warp_run[lane] : 0u;
#pragma unroll
            for (uint32_t off = 1; off < kWarps; off <<= 1) {
                const uint32_t yc = __shfl_up_sync(0xFFFFFFFFu, wc, off);
                const uint32_t yr = __shfl_up_sync(0xFFFFFFFFu, wr, off);
                if (lane >= off) {
                    wc += yc;
                    wr = max(wr, yr);
                }
            }
            const uint32_t tile_total = __shfl_sync(0xFFFFFFFFu, wc, kWarps - 1);
            const uint32_t prev_c = __shfl_sync(0xFFFFFFFFu, wc, wid ? wid - 1 : 0);
            const uint32_t prev_r = __shfl_sync(0xFFFFFFFFu, wr, wid ? wid - 1 : 0);
            uint32_t before = incl - mine + (wid ? prev_c : 0u);
            if (wid) rprev = max(rprev, prev_r);
            // compact the tile's ends (window | first window << 16, in window order, in the block
            // array the cut does not otherwise use) so the per-record work below runs on full warps
#pragma unroll
            for (uint32_t j = 0; j < 4; j++) {
                if ((endmask >> j) & 1u) sm.block[before++] = (i0 + j) | ((max(rprev, rs[j]) - 1u) << 16);
            }
            __syncthreads();
            // each record takes the next slot of its bucket's region; past the region it goes to
            // the overflow list (sorted into place by the bucketing step)
            const uint32_t local_mask = (1u << a.bucket_shift) - 1u;
            for (uint32_t e = tid; e < tile_total; e += blockDim.x) {
                const uint32_t v = sm.block[e];
                const uint32_t i = v & 0xFFFFu, st = v >> 16;
                const uint16_t po = sm.poff[i];
                const uint32_t nwin = i - st + 1;
                c_sk++;
                c_smer += nwin + ks;
                const uint32_t block = minimizer_block(sm.codes, e0 + po - cb, mv, g.block_mask);
                const unsigned long long val =
                    (unsigned long long)(e0 + st) | ((unsigned long long)nwin << kRecWindowsShift);
                // the super-k-mer's bases (64 from its first one) travel with the record, so the
                // apply reads them in slot order instead of gathering them from the batch's codes
                const uint32_t b0 = (uint32_t)(e0 + st - cb);
                const uint64_t lo = codes64(sm.codes, b0), hi = codes64(sm.codes, b0 + 32u);
                const uint4 bases4 = make_uint4((uint32_t)lo, (uint32_t)(lo >> 32), (uint32_t)hi, (uint32_t)(hi >> 32));
                const uint32_t bucket = block >> a.bucket_shift;
                const unsigned long long slot = atomicAdd(a.bucket_hist + bucket, 1ull);
                if (slot < a.bucket_cap) {
                    const uint64_t at = (uint64_t)bucket * a.bucket_cap + slot;
                    a.sorted[at] = val | ((unsigned long long)(block & local_mask) << kRecLocalShift);
                    __stcs(a.sbases + at, bases4);  // read once, by the apply
                } else {
                    const unsigned long long o = atomicAdd(a.rec_count, 1ull);
                    if (o < a.rec_cap) {
                        a.rec_key[o] = block;
                        a.rec_val[o] = val;
                        a.rec_bases[o] = bases4;
                    }
                }
            }
        } else if constexpr (MODE == kModeDebugMin) {
            for (uint32_t i = tid; i < kTileWindows; i += blockDim.x) {
                const uint64_t pos = t0 + i;
                if (sm.poff[i] != kNoWindow && pos < n_bytes) a.dbg[pos] = (uint32_t)(e0 + sm.poff[i]);
            }
        } else if constexpr (MODE == kModeMaterialize) {
            for (uint32_t i = tid; i < kTileWindows; i += blockDim.x) {
                const uint64_t pos = t0 + i;
                if (pos >= n_bytes) continue;
                const uint16_t po = sm.poff[i];
                a.wblock[pos] = po == kNoWindow ? 0xFFFFFFFFu : sm.block[i];
                a.wend[pos] = (po != kNoWindow && sm.poff[i + 1] != po) ? 1 : 0;
            }
        }
        __syncthreads();
    }
    warp_add_u64(&a.cnt[kCntWindows], c_win);
    warp_add_u64(&a.cnt[kCntSmers], c_smer);
    warp_add_u64(&a.cnt[kCntValid], c_valid);
    warp_add_u64(&a.cnt[kCntPositive], c_pos);
    warp_add_u64(&a.cnt[kCntChecksum], c_sum);
    warp_add_u64(&a.cnt[kCntSuperKmers], c_sk);
    warp_add_u64(&a.cnt[kCntSectors], c_sec);
    warp_add_u64(&a.cnt[kCntDistinct], c_dist);
}

template <int MODE>
static void launch_tiles_bits(const TileArgs& a, int grid, cudaStream_t st) {
    constexpr int kDefaultKM = (31 << 8) | 21;
    if (MODE == kModeCut && (((int)a.g.k << 8) | (int)a.g.m) == kDefaultKM) {
        switch (a.g.bits) {
            case 8: k_tiles<MODE, 8, kDefaultKM><<<grid, kTileThreads, 0, st>>>(a); break;
            case 16: k_tiles<MODE, 16, kDefaultKM><<<grid, kTileThreads, 0, st>>>(a); break;
            default: k_tiles<MODE, 32, kDefaultKM><<<grid, kTileThreads, 0, st>>>(a); break;
        }
    } else {
        switch (a.g.bits) {
            case 8: k_tiles<MODE, 8><<<grid, kTileThreads, 0, st>>>(a); break;
            case 16: k_tiles<MODE, 16><<<grid, kTileThreads, 0, st>>>(a); break;
            default: k_tiles<MODE, 32><<<grid, kTileThreads, 0, st>>>(a); break;
        }
    }
    note_launch();
}

void launch_tiles(int mode, const TileArgs& a, int grid, cudaStream_t st) {
    if (grid <= 0) return;
    switch (mode) {
        case kModeInsert: launch_tiles_bits<kModeInsert>(a, grid, st); break;
        case kModeReport: launch_tiles_bits<kModeReport>(a, grid, st); break;
        case kModeAbund: launch_tiles_bits<kModeAbund>(a, grid, st); break;
        case kModeDistinct: launch_tiles_bits<kModeDistinct>(a, grid, st); break;
        case kModeAbundDistinct: launch_tiles_bits<kModeAbundDistinct>(a, grid, st); break;
        case kModeStats: launch_tiles_bits<kModeStats>(a, grid, st); break;
        case kModeDebugMin: launch_tiles_bits<kModeDebugMin>(a, grid, st); break;
        case kModeMaterialize: launch_tiles_bits<kModeMaterialize>(a, grid, st); break;
        case kModeCut: launch_tiles_bits<kModeCut>(a, grid, st); break;
        default: break;
    }
}

int tile_grid(int mode, int bits, int sm_count, uint32_t n_tiles) {
    int per_sm = 0;
    const void* fn = nullptr;
#define SCB_PICK(MODEV)                                                              \
    fn = bits == 8 ? (const void*)k_tiles<MODEV, 8>                                  \
                   : (bits == 16 ? (const void*)k_tiles<MODEV, 16> : (const void*)k_tiles<MODEV, 32>)
    switch (mode) {
        case kModeInsert: SCB_PICK(kModeInsert); break;
        case kModeReport: SCB_PICK(kModeReport); break;
        case kModeAbund: SCB_PICK(kModeAbund); break;
        case kModeDistinct: SCB_PICK(kModeDistinct); break;
        case kModeAbundDistinct: SCB_PICK(kModeAbundDistinct); break;
        case kModeStats: SCB_PICK(kModeStats); break;
        case kModeDebugMin: SCB_PICK(kModeDebugMin); break;
        case kModeCut: SCB_PICK(kModeCut); break;
        default: SCB_PICK(kModeMaterialize); break;
    }
#undef SCB_PICK
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kTileThreads, 0) != cudaSuccess || per_sm < 1) {
        per_sm = 1;
    }
    const uint64_t want = (uint64_t)per_sm * (uint64_t)sm_count;
    return (int)(n_tiles < want ? n_tiles : want);
}

// ---------------------------------------------------------------------------------------
// Plain pipeline: one thread per window, everything from global memory.
// ---------------------------------------------------------------------------------------
template <int BITS>
__global__ void k_plain_insert(TileArgs a) {
    const DevGeom g = a.g;
    uint32_t* table32 = reinterpret_cast<uint32_t*>(a.table);
    const uint64_t s_mask = len_mask(g.s);
    const uint32_t ks = g.k - g.s;
    unsigned long long c_win = 0, c_smer = 0, c_sk = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t n_iter = (a.n_bytes + stride - 1) / stride;
    for (uint64_t it = 0; it < n_iter; it++) {
        const uint64_t pos = it * stride + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (pos >= a.n_bytes) continue;
        const uint32_t blk = a.wblock[pos];
        if (blk == 0xFFFFFFFFu) continue;
        const uint64_t base = block_base(g, blk);
        insert_smer<BITS>(table32, g, base, canonical(codes64(a.codes, pos) & s_mask, g.s), a.status);
        c_win++;
        c_smer++;
        if (a.wend[pos]) {
            c_sk++;
            for (uint32_t u = 1; u <= ks; u++) {
                insert_smer<BITS>(table32, g, base, canonical(codes64(a.codes, pos + u) & s_mask, g.s), a.status);
                c_smer++;
            }
        }
    }
    warp_add_u64(&a.cnt[kCntWindows], c_win);
    warp_add_u64(&a.cnt[kCntSmers], c_smer);
    warp_add_u64(&a.cnt[kCntSuperKmers], c_sk);
}

template <int MODE, int BITS>
__global__ void k_plain_query(TileArgs a) {
    const DevGeom g = a.g;
    unsigned long long c_valid = 0, c_pos = 0, c_sum = 0;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t n_iter = (a.n_bytes + stride - 1) / stride;
    for (uint64_t it = 0; it < n_iter; it++) {
        const uint64_t pos = it * stride + (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
        if (pos >= a.n_bytes) continue;
        const uint32_t blk = a.wblock[pos];
        if (blk == 0xFFFFFFFFu) continue;
        const uint32_t r = window_estimate<BITS>(a, g, a.codes, pos, block_base(g, blk));
        if constexpr (MODE == kModeReport) {
            c_valid++;
            c_pos += r > 0;
            c_sum += r;
        } else {
            const uint64_t j = seq_of(a.offsets, 0, a.n_seqs, pos);
            const uint64_t o = a.woff[j] + (pos - __ldg(a.offsets + j));
            a.out[o] = r;
            a.out_valid[o] = 1;
        }
    }
    warp_add_u64(&a.cnt[kCntValid], c_valid);
    warp_add_u64(&a.cnt[kCntPositive], c_pos);
    warp_add_u64(&a.cnt[kCntChecksum], c_sum);
}

static int plain_grid(uint64_t n) {
    const uint64_t blocks = (n + 255) / 256;
    return (int)(blocks < (1u << 20) ? (blocks ? blocks : 1) : (1u << 20));
}

void launch_plain_insert(const TileArgs& a, cudaStream_t st) {
    const int grid = plain_grid(a.n_bytes);
    switch (a.g.bits) {
        case 8: k_plain_insert<8><<<grid, 256, 0, st>>>(a); break;
        case 16: k_plain_insert<16><<<grid, 256, 0, st>>>(a); break;
        default: k_plain_insert<32><<<grid, 256, 0, st>>>(a); break;
    }
    note_launch();
}

void launch_plain_query(int mode, const TileArgs& a, cudaStream_t st) {
    const int grid = plain_grid(a.n_bytes);
    if (mode == kModeReport) {
        switch (a.g.bits) {
            case 8: k_plain_query<kModeReport, 8><<<grid, 256, 0, st>>>(a); break;
            case 16: k_plain_query<kModeReport, 16><<<grid, 256, 0, st>>>(a); break;
            default: k_plain_query<kModeReport, 32><<<grid, 256, 0, st>>>(a); break;
        }
    } else {
        switch (a.g.bits) {
            case 8: k_plain_query<kModeAbund, 8><<<grid, 256, 0, st>>>(a); break;
            case 16: k_plain_query<kModeAbund, 16><<<grid, 256, 0, st>>>(a); break;
            default: k_plain_query<kModeAbund, 32><<<grid, 256, 0, st>>>(a); break;
        }
    }
    note_launch();
}

// ---------------------------------------------------------------------------------------
// Counter histogram (filter.rs:50-54, 267-275): value -> number of counters.
// ---------------------------------------------------------------------------------------
constexpr uint32_t kHistSmem = 8192;

template <int BITS>
__global__ void k_counter_hist(const void* __restrict__ table, uint64_t slots, unsigned long long* hist,
                               uint32_t dense, unsigned long long* ovf, uint64_t ovf_cap,
                               unsigned long long* ovf_count) {
    __shared__ unsigned int sh[kHistSmem];
    for (uint32_t i = threadIdx.x; i < kHistSmem; i += blockDim.x) sh[i] = 0;
    __syncthreads();
    const uint32_t lane = threadIdx.x & 31;
    const uint64_t warps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint64_t wid = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    unsigned long long zeros = 0;
    for (uint64_t base = wid * 32; base < slots; base += warps * 32) {
        const uint64_t idx = base + lane;
        const bool in = idx < slots;
        const uint32_t v = in ? load_counter<BITS>(table, idx) : 0xFFFFFFFFu;
        const bool is_zero = in && v == 0;
        zeros += is_zero;
        const bool other = in && v != 0;
        const unsigned mask = __ballot_sync(0xFFFFFFFFu, other);
        if (other) {
            const unsigned peers = __match_any_sync(mask, v);
            if (lane == (uint32_t)(__ffs(peers) - 1)) {
                const unsigned c = __popc(peers);
                if (v < kHistSmem) {
                    atomicAdd(&sh[v], c);
                } else if (v < dense) {
                    atomicAdd(hist + v, (unsigned long long)c);
                } else {
                    const unsigned long long o = atomicAdd(ovf_count, (unsigned long long)c);
                    for (unsigned q = 0; q < c; q++) {
                        if (o + q < ovf_cap) ovf[o + q] = v;
                    }
                }
            }
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < kHistSmem; i += blockDim.x) {
        if (sh[i]) atomicAdd(hist + i, (unsigned long long)sh[i]);
    }
    warp_add_u64(hist, zeros);
}

void launch_counter_hist(const void* table, uint64_t slots, int bits, unsigned long long* hist, uint32_t dense,
                         unsigned long long* ovf, uint64_t ovf_cap, unsigned long long* ovf_count, cudaStream_t st) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const uint64_t want = (slots + 255) / 256;
    const int grid = (int)(want < (uint64_t)sms * 4 ? (want ? want : 1) : (uint64_t)sms * 4);
    switch (bits) {
        case 8: k_counter_hist<8><<<grid, 256, 0, st>>>(table, slots, hist, dense, ovf, ovf_cap, ovf_count); break;
        case 16: k_counter_hist<16><<<grid, 256, 0, st>>>(table, slots, hist, dense, ovf, ovf_cap, ovf_count); break;
        default: k_counter_hist<32><<<grid, 256, 0, st>>>(table, slots, hist, dense, ovf, ovf_cap, ovf_count); break;
    }
    note_launch();
}

// ---------------------------------------------------------------------------------------
// Grouped pipeline: records bucketed by block; each work item's blocks live in shared memory.
// ---------------------------------------------------------------------------------------
// Overflow records (those past their bucket's region) into bucket order after the regions:
// position = base + the bucket's overflow offset + its running count.
__global__ void k_scatter(const uint32_t* __restrict__ key, const unsigned long long* __restrict__ val,
                          const uint4* __restrict__ vbases, const unsigned long long* __restrict__ count,
                          uint64_t cap, uint32_t shift, unsigned long long* __restrict__ cursor, uint64_t base,
                          unsigned long long* __restrict__ sorted, uint4* __restrict__ sbases) {
    const uint64_t n = *count;
    if (n > cap) return;  // the overflow list ran out of room: the host redoes the batch
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint32_t local_mask = (1u << shift) - 1u;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const unsigned long long v = val[i];
        const uint32_t block = key[i];
        const unsigned long long pos = base + atomicAdd(cursor + (block >> shift), 1ull);
        sorted[pos] = v | ((unsigned long long)(block & local_mask) << kRecLocalShift);
        sbases[pos] = vbases[i];
    }
}

// Work items per bucket: its region's records (at most bucket_cap) and its overflow records, in
// items of at most kItemRecords; also each bucket's overflow count (for the overflow offsets).
__global__ void k_item_counts(const unsigned long long* __restrict__ counts, uint64_t n_buckets, uint64_t bucket_cap,
                              uint64_t* __restrict__ item_count, uint64_t* __restrict__ ovf_count,
                              const unsigned long long* __restrict__ rec_count, uint64_t rec_cap) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const bool overflow = *rec_count > rec_cap;  // no work items: nothing is applied
    for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b <= n_buckets; b += stride) {
        if (b == n_buckets || overflow) {
            item_count[b] = 0;
            ovf_count[b] = 0;
        } else {
            const uint64_t c = counts[b];
            const uint64_t m = c < bucket_cap ? c : bucket_cap, o = c - m;
            item_count[b] = (m + kItemRecords - 1) / kItemRecords + (o + kItemRecords - 1) / kItemRecords;
            ovf_count[b] = o;
        }
    }
}

__global__ void k_item_write(const unsigned long long* __restrict__ counts, uint64_t bucket_cap,
                             const uint64_t* __restrict__ item_off, const uint64_t* __restrict__ ovf_off,
                             uint64_t ovf_base, uint64_t n_buckets, uint4* __restrict__ items) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t b = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; b < n_buckets; b += stride) {
        const uint64_t c = counts[b];
        const uint64_t m = c < bucket_cap ? c : bucket_cap, o = c - m;
        const uint64_t i0 = item_off[b];
        const uint32_t excl = item_off[b + 1] - i0 == 1 ? 1u : 0u;  // the bucket's only item
        uint64_t t = 0;
        for (uint64_t r = 0; r < m; r += kItemRecords, t++) {
            const uint64_t cnt = min((uint64_t)kItemRecords, m - r);
            items[i0 + t] = make_uint4((uint32_t)b, (uint32_t)(b * bucket_cap + r), (uint32_t)cnt, excl);
        }
        for (uint64_t r = 0; r < o; r += kItemRecords, t++) {
            const uint64_t cnt = min((uint64_t)kItemRecords, o - r);
            items[i0 + t] = make_uint4((uint32_t)b, (uint32_t)(ovf_base + ovf_off[b] + r), (uint32_t)cnt, excl);
        }
    }
}

// Windows of the work items whose keys go to the global set of the spectrum apply: those that are
// not their bucket's only one, and those with more than kSpecSet / 2 windows (too many for the
// shared-memory set).  One thread per item, summed into *out.
__global__ void k_shared_item_windows(const uint4* __restrict__ items, const unsigned long long* __restrict__ n_items,
                                      const unsigned long long* __restrict__ recs, unsigned long long* out) {
    const uint64_t n = *n_items;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    unsigned long long sum = 0;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint4 it = items[i];
        unsigned long long wins = 0;
        for (uint32_t r = 0; r < it.z; r++) wins += (recs[it.y + r] >> kRecWindowsShift) & 63u;
        if (!it.w || 2 * wins > kSpecSet) sum += wins;
    }
    warp_add_u64(out, sum);
}

void launch_shared_item_windows(const uint4* items, const unsigned long long* n_items, const unsigned long long* recs,
                                unsigned long long* out, cudaStream_t st) {
    k_shared_item_windows<<<592, 256, 0, st>>>(items, n_items, recs, out);
    note_launch();
}

// Largest r in [0, n) with pre[r] <= v (pre[0] = 0, pre non-decreasing).
__device__ __forceinline__ uint32_t find_rec(const uint32_t* pre, uint32_t n, uint32_t v) {
    uint32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        const uint32_t mid = (lo + hi + 1) >> 1;
        if (pre[mid] <= v) {
            lo = mid;
        } else {
            hi = mid - 1;
        }
    }
    return lo;
}

__device__ __forceinline__ uint64_t codes64_ldg(const uint32_t* words, uint64_t b) {
    const uint64_t w = b >> 4;
    const uint32_t sh = (uint32_t)(b & 15) * 2u;
    const uint32_t w0 = __ldg(words + w), w1 = __ldg(words + w + 1), w2 = __ldg(words + w + 2);
    return ((uint64_t)__funnelshift_r(w1, w2, sh) << 32) | __funnelshift_r(w0, w1, sh);
}

// Block-wide exclusive prefix of (n_r + ks) and n_r over the chunk's records into spre / wpre.
__device__ __forceinline__ void chunk_prefix(const unsigned long long* rv, uint32_t nrec, uint32_t ks, uint32_t* spre,
                                             uint32_t* wpre, uint32_t* warp_tot) {
    const uint32_t tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    uint32_t w = 0;
    if (tid < nrec) w = (uint32_t)((rv[tid] >> kRecWindowsShift) & 63u);
    const uint32_t s = tid < nrec ? w + ks : 0u;
    uint32_t pack_s = s, pack_w = w;
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t ys = __shfl_up_sync(0xFFFFFFFFu, pack_s, off);
        const uint32_t yw = __shfl_up_sync(0xFFFFFFFFu, pack_w, off);
        if ((int)lane >= off) {
            pack_s += ys;
            pack_w += yw;
        }
    }
    if (lane == 31) {
        warp_tot[2 * wid] = pack_s;
        warp_tot[2 * wid + 1] = pack_w;
    }
    __syncthreads();
    uint32_t add_s = 0, add_w = 0;
    for (uint32_t x = 0; x < wid; x++) {
        add_s += warp_tot[2 * x];
        add_w += warp_tot[2 * x + 1];
    }
    if (tid < nrec) {
        spre[tid + 1] = pack_s + add_s;
        wpre[tid + 1] = pack_w + add_w;
    }
    if (tid == 0) {
        spre[0] = 0;
        wpre[0] = 0;
    }
    __syncthreads();
}

template <int BITS>
struct CounterType {
    using type = uint32_t;
};
template <>
struct CounterType<8> {
    using type = uint8_t;
};
template <>
struct CounterType<16> {
    using type = uint16_t;
};

// Shared-memory layout of k_apply (offsets in bytes, all 16-byte aligned):
//   cells   bucket counters: u32 deltas (insert) or the counters at native width (query)
//   rv      the chunk's records
//   spre    exclusive prefix of s-mers per record, wpre the same for windows
//   bases   the 2-bit code words of each record of the chunk
//   rbases  the same words reverse-complemented (word j = revcomp of word 7 - j), plus spare
//           words that the last record's reads may touch
//   smap    record of each s-mer of the chunk, wmap record of each window (query)
//   touched one flag per block of the bucket
//   est     s-mer minima of the chunk (query; 16-bit for 8/16-bit counters)
//   skeys   the work item's distinct canonical k-mers (spectrum), shist the CTA's histogram
struct ApplyLayout {
    uint32_t cells, rv, spre, wpre, bases, rbases, smap, wmap, touched, est, kept, skeys, shist, total;
};

// s-mers (and windows) of one staged chunk of records; a record has at most 31 + 31
constexpr uint32_t kSmerBudget = 4096;
// 2-bit code words staged per record: its record bases, whose first base is the first window's,
// hold its <= w + k - 1 <= 63 bases.  codes64 may read up to two words further (into the next
// record's words or the spare words); those bits lie past the s-mer and are masked off.
constexpr uint32_t kRecBaseWords = 4;
// probe-slot loads a query thread keeps in flight
constexpr uint32_t kProbeBatch = 4;

__host__ __device__ inline uint32_t align16(uint32_t x) { return (x + 15u) & ~15u; }

// lean: a query over kept probe slots stages no bases (items without slots read the codes from
// global memory), which leaves room for more CTAs per SM.
__host__ __device__ inline ApplyLayout apply_layout(int mode, int bits, uint32_t bucket_slots, uint32_t bucket_blocks,
                                                    bool lean = false) {
    ApplyLayout l;
    const bool deltas = mode == kModeInsert || mode == kModeBuild;  // u32 deltas in the cells
    const bool queries = mode != kModeInsert;                        // window map and s-mer minima
    const uint32_t cell_bytes = deltas ? 4u : (uint32_t)bits / 8u;
    const uint32_t max_smers = kSmerBudget, max_windows = kSmerBudget;
    l.cells = 0;
    l.rv = align16(bucket_slots * cell_bytes);
    l.spre = l.rv + align16(kApplyChunk * 8u);
    l.wpre = l.spre + align16((kApplyChunk + 1u) * 4u);
    l.bases = l.wpre + align16((kApplyChunk + 1u) * 4u);
    l.rbases = l.bases + (lean ? 0u : align16(kApplyChunk * kRecBaseWords * 4u));
    l.smap = l.rbases + (lean ? 0u : align16(kApplyChunk * kRecBaseWords * 4u + 16u));  // + the last record's over-read
    const uint32_t est_bytes = align16(max_smers * (bits <= 16 ? 2u : 4u));
    if (mode == kModeBuild) {
        // the build's query phase needs neither the s-mer map nor the staged bases: its window
        // map takes the s-mer map's bytes, its s-mer minima the bases' when they fit
        l.wmap = l.smap;
        l.touched = l.smap + align16(max_smers);
        const bool est_in_bases = est_bytes <= l.smap - l.bases;
        l.est = est_in_bases ? l.bases : l.touched + align16(bucket_blocks);
        l.kept = l.touched + align16(bucket_blocks) + (est_in_bases ? 0u : est_bytes);
    } else {
        l.wmap = l.smap + align16(max_smers);
        l.touched = l.wmap + (queries ? align16(max_windows) : 0u);
        l.est = l.touched + align16(bucket_blocks);
        l.kept = l.est + (queries ? est_bytes : 0u);
    }
    l.skeys = l.kept;
    l.shist = l.skeys + (mode == kModeSpectrum ? kSpecSet * 8u : 0u);
    l.total = l.shist + (mode == kModeSpectrum ? kSpecBins * 4u : 0u);
    return l;
}

// Inserts a canonical k-mer into a shared-memory open-addressing set (~0 marks an empty slot; no
// canonical k-mer has that value).  True when the key is new.  The set holds at least twice as
// many slots as the keys offered to it, so a free slot is always found.
__device__ __forceinline__ bool smem_set_insert(unsigned long long* keys, uint32_t mask, uint64_t key) {
    uint32_t i = (uint32_t)(((key ^ (key >> 31)) * 0x9E3779B97F4A7C15ull) >> 40) & mask;
    for (uint32_t probe = 0; probe <= mask; probe++) {
        const unsigned long long cur = *reinterpret_cast<volatile unsigned long long*>(keys + i);
        if (cur == key) return false;
        if (cur == ~0ull) {
            const unsigned long long prev = atomicCAS(keys + i, ~0ull, (unsigned long long)key);
            if (prev == ~0ull) return true;
            if (prev == key) return false;
        }
        i = (i + 1) & mask;
    }
    return false;
}

// Commits a work item's u32 deltas (cells, bucket_blocks blocks of 2^bs_log2 counters) to the
// table: min(old + delta, MAX) per counter (counter.rs saturation), 16 bytes per thread when the
// item is its bucket's only one, 32-bit words when blocks are word-aligned, saturating CAS per
// counter otherwise (items of a split bucket commit concurrently).  keep_finals (an exclusive item
// only) leaves each touched counter's committed value in its cell.
template <int BITS>
__device__ __forceinline__ void commit_item(uint32_t* cells, const uint8_t* touched, const GroupArgs& a,
                                            uint64_t bucket, uint32_t bs_log2, uint32_t bucket_blocks,
                                            bool exclusive, bool keep_finals) {
    using T = CounterTraits<BITS>;
    using Cnt = typename CounterType<BITS>::type;
    constexpr uint32_t kVecLog2 = BITS == 8 ? 4u : (BITS == 16 ? 3u : 2u);
    constexpr uint32_t lanes = T::kLanes;
    const DevGeom& g = a.g;
    const uint32_t tid = threadIdx.x;
    const uint32_t bs = 1u << bs_log2;
    const uint32_t bucket_slots = bs * bucket_blocks;
    uint32_t* table32 = reinterpret_cast<uint32_t*>(a.table);
    const bool word_ok = exclusive && (bs % lanes) == 0;
    if (exclusive && bs_log2 >= kVecLog2) {
        // 16 bytes of the table per thread: kVec counters, their u32 deltas in shared memory
        constexpr uint32_t kVec = 1u << kVecLog2;
        const uint32_t vlog = bs_log2 - kVecLog2;
        const uint32_t n_vec = bucket_blocks << vlog;
        const uint4* d4 = reinterpret_cast<const uint4*>(cells);
        for (uint32_t x = tid; x < n_vec; x += blockDim.x) {
            const uint32_t lb = x >> vlog;
            if (!touched[lb]) continue;
            const uint64_t base = block_base(g, (bucket << a.bucket_shift) | lb);
            uint4* wp = reinterpret_cast<uint4*>(reinterpret_cast<Cnt*>(a.table) + base) + (x & ((1u << vlog) - 1u));
            const uint4 o4 = __ldcg(wp);
            uint32_t d[kVec];
#pragma unroll
            for (uint32_t q = 0; q < kVec / 4; q++) {
                const uint4 v = d4[x * (kVec / 4) + q];
                d[4 * q] = v.x;
                d[4 * q + 1] = v.y;
                d[4 * q + 2] = v.z;
                d[4 * q + 3] = v.w;
            }
            const uint32_t ow[4] = {o4.x, o4.y, o4.z, o4.w};
            uint32_t nw[4];
#pragma unroll
            for (uint32_t w = 0; w < 4; w++) {
                uint32_t acc = 0;
#pragma unroll
                for (uint32_t l = 0; l < lanes; l++) {
                    const uint64_t cur = (ow[w] >> (l * BITS)) & T::kMax;
                    const uint64_t sum = cur + d[w * lanes + l];
                    acc |= (uint32_t)(sum < T::kMax ? sum : T::kMax) << (l * BITS);
                }
                nw[w] = acc;
            }
            __stcg(wp, make_uint4(nw[0], nw[1], nw[2], nw[3]));
            if (keep_finals) {
                uint4* c4w = reinterpret_cast<uint4*>(cells);
#pragma unroll
                for (uint32_t q = 0; q < kVec / 4; q++) {
                    uint32_t fv[4];
#pragma unroll
                    for (uint32_t j = 0; j < 4; j++) {
                        const uint32_t c = 4 * q + j;  // counter c of the vector: word c / lanes
                        fv[j] = (nw[c / lanes] >> ((c % lanes) * BITS)) & T::kMax;
                    }
                    c4w[x * (kVec / 4) + q] = make_uint4(fv[0], fv[1], fv[2], fv[3]);
                }
            }
        }
    } else if (word_ok) {
        const uint32_t block_words = bs / lanes;
        for (uint32_t x = tid; x < bucket_blocks * block_words; x += blockDim.x) {
            const uint32_t lb = x / block_words, wi = x % block_words;
            if (!touched[lb]) continue;
            const uint64_t base = block_base(g, (bucket << a.bucket_shift) | lb);
            uint32_t* wp = table32 + base / lanes + wi;
            const uint32_t old = __ldcg(wp);
            uint32_t nw = 0;
            const uint32_t cb = (lb << bs_log2) + wi * lanes;
#pragma unroll
            for (uint32_t l = 0; l < lanes; l++) {
                const uint64_t cur = (old >> (l * BITS)) & T::kMax;
                const uint64_t sum = cur + cells[cb + l];
                const uint32_t nv = (uint32_t)(sum < T::kMax ? sum : T::kMax);
                nw |= nv << (l * BITS);
                if (keep_finals) cells[cb + l] = nv;
            }
            __stcg(wp, nw);
        }
    } else {
        for (uint32_t x = tid; x < bucket_slots; x += blockDim.x) {
            const uint32_t lb = x >> bs_log2;
            const uint32_t d = cells[x];
            if (!touched[lb] || d == 0) continue;
            const uint64_t base = block_base(g, (bucket << a.bucket_shift) | lb);
            sat_add<BITS>(table32, base + (x & (bs - 1)), d, a.status);
        }
    }
}

// NH = 4: four hashes per s-mer (the default geometry), unrolled; NH = 0: any n_hashes.  Kept
// probe slots are 16-bit lanes (n_hashes <= 4), each the counter's index within the bucket's
// shared-memory cells, so the query needs neither the s-mer nor its record.
// KSC: 0 for any k and s, or (k << 8) | s of the default geometry (k = 31, s = 25) compiled in, so
// that the s-mer and window loops and masks are constants (measured 4-5 % faster).
constexpr int kDefaultKS = (31 << 8) | 25;

template <int MODE, int BITS, int NH, bool LEAN, int KSC = 0>
__device__ __forceinline__ void apply_body(const GroupArgs& a, uint32_t bs_log2, uint32_t bucket_blocks) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    using T = CounterTraits<BITS>;
    using Cnt = typename CounterType<BITS>::type;
    constexpr bool kDeltas = MODE == kModeInsert || MODE == kModeBuild;  // cells hold u32 deltas
    constexpr bool kBuild = MODE == kModeBuild;
    constexpr bool kSpec = MODE == kModeSpectrum;
    constexpr bool kStaged = MODE == kModeReport || kSpec;  // cells hold the table's counters
    using Cell = typename std::conditional<kDeltas, uint32_t, Cnt>::type;
    using Est = typename std::conditional<(BITS <= 16), uint16_t, uint32_t>::type;
    constexpr uint32_t kVecLog2 = BITS == 8 ? 4u : (BITS == 16 ? 3u : 2u);  // log2 counters per 16 bytes
    const DevGeom g = a.g;
    const uint32_t bs = 1u << bs_log2;
    const uint32_t bucket_slots = bs * bucket_blocks;
    const ApplyLayout lay = apply_layout(MODE, BITS, bucket_slots, bucket_blocks, LEAN);
    Cell* cells = reinterpret_cast<Cell*>(smem_raw + lay.cells);
    unsigned long long* rv = reinterpret_cast<unsigned long long*>(smem_raw + lay.rv);
    uint32_t* spre = reinterpret_cast<uint32_t*>(smem_raw + lay.spre);
    uint32_t* wpre = reinterpret_cast<uint32_t*>(smem_raw + lay.wpre);
    uint32_t* bases = reinterpret_cast<uint32_t*>(smem_raw + lay.bases);
    uint32_t* rbases = reinterpret_cast<uint32_t*>(smem_raw + lay.rbases);
    uint8_t* smap = smem_raw + lay.smap;
    uint8_t* wmap = smem_raw + lay.wmap;
    uint8_t* touched = smem_raw + lay.touched;
    Est* est = reinterpret_cast<Est*>(smem_raw + lay.est);
    // build: this CTA's region of the kept probe words (written by the insert, read back by the
    // query of the same item moments later, so it stays in L2)
    unsigned long long* kept = (kBuild && blockIdx.x < a.kept_ctas) ? a.kept + (uint64_t)blockIdx.x * kKeptSmers
                                                                     : nullptr;
    unsigned long long* skeys = reinterpret_cast<unsigned long long*>(smem_raw + lay.skeys);
    uint32_t* shist = reinterpret_cast<uint32_t*>(smem_raw + lay.shist);
    __shared__ uint4 item;
    __shared__ uint32_t item_fused;
    __shared__ unsigned item_idx;
    __shared__ uint32_t item_smers;
    __shared__ unsigned long long item_probes;
    __shared__ uint32_t warp_tot[2 * (kApplyMaxThreads / 32)];

    const uint32_t tid = threadIdx.x;
    const uint32_t kv = KSC ? (uint32_t)(KSC >> 8) : g.k;
    const uint32_t sv = KSC ? (uint32_t)(KSC & 255) : g.s;
    const uint32_t ks = kv - sv;
    const uint64_t s_mask = len_mask(sv);
    const uint64_t n_items = *a.n_items;
    if (a.rec_count && *a.rec_count > a.rec_cap) return;  // records outgrew their slots: host redoes it
    unsigned long long c_valid = 0, c_pos = 0, c_sum = 0, c_dist = 0;
    const uint32_t spec_bins = kSpec ? min(kSpecBins, a.hist_dense) : 0u;
    if constexpr (kSpec) {
        for (uint32_t x = tid; x < spec_bins; x += blockDim.x) shist[x] = 0;
    }

    while (true) {
        if (tid == 0) {
            const unsigned idx = atomicAdd(a.work_counter, 1u);
            item = idx < n_items ? a.items[idx] : make_uint4(0xFFFFFFFFu, 0, 0, 0);
            item_idx = idx;
            item_smers = 0;
        }
        __syncthreads();
        const uint4 it = item;
        if (it.x == 0xFFFFFFFFu) break;
        const uint64_t bucket = it.x;
        const uint64_t first = it.y;
        const uint32_t count = it.z;
        const bool exclusive = it.w != 0;

        // probe slots of the item: the insert reserves room for all its s-mers, the query finds
        // where the insert put them
        unsigned long long pbase = kNoProbes;
        // build: the item answers its own query when its counters are final once it commits (the
        // bucket's only item) and its probe slots fit the kept array; otherwise it stores them and
        // goes to the list the query kernel works through
        bool fused = false;
        if (a.probes) {
            if constexpr (kDeltas) {
                uint32_t n = 0;
                for (uint32_t r = tid; r < count; r += blockDim.x) {
                    n += (uint32_t)((a.recs[first + r] >> kRecWindowsShift) & 63u) + ks;
                }
                n = __reduce_add_sync(0xFFFFFFFFu, n);
                if ((tid & 31) == 0 && n) atomicAdd(&item_smers, n);
                __syncthreads();
                if (tid == 0) {
                    bool f = false;
                    if constexpr (kBuild) {
                        f = kept != nullptr && exclusive && item_smers <= kKeptSmers && (bs % T::kLanes) == 0;
                    }
                    unsigned long long b = kNoProbes;
                    if (!f) {
                        b = atomicAdd(a.probe_count, (unsigned long long)item_smers);
                        if (b + item_smers > a.probe_cap) b = kNoProbes;
                    }
                    if constexpr (kBuild) {
                        if (!f) {
                            const unsigned long long d = atomicAdd(a.dcount, 1ull);
                            a.ditems[d] = it;
                            a.ditem_base[d] = b;
                        }
                    } else {
                        a.item_base[item_idx] = b;
                    }
                    item_probes = b;
                    item_fused = f ? 1u : 0u;
                }
            } else {
                if (tid == 0) item_probes = a.item_base[item_idx];
            }
            __syncthreads();
            pbase = item_probes;
            if constexpr (kBuild) fused = item_fused != 0;
        }
        const bool have_probes = MODE == kModeReport && pbase != kNoProbes;
        // spectrum: the item's windows deduplicate in a shared-memory set of at least twice as
        // many slots when the item is its bucket's only one (every occurrence of a canonical
        // k-mer has the same minimizer, so the same block and bucket); otherwise in the global set
        uint32_t set_cap = 0;
        if constexpr (kSpec) {
            uint32_t n = 0;
            for (uint32_t r = tid; r < count; r += blockDim.x) {
                n += (uint32_t)((a.recs[first + r] >> kRecWindowsShift) & 63u);
            }
            n = __reduce_add_sync(0xFFFFFFFFu, n);
            if ((tid & 31) == 0 && n) atomicAdd(&item_smers, n);
            __syncthreads();
            const uint32_t wins = item_smers;
            if (exclusive && 2 * wins <= kSpecSet) {
                set_cap = 256;
                while (set_cap < 2 * wins) set_cap <<= 1;
                for (uint32_t x = tid; x < set_cap; x += blockDim.x) skeys[x] = ~0ull;
            }
        }
        uint64_t poff = 0;  // s-mers of the item's earlier chunks

        for (uint32_t x = tid; x < bucket_blocks; x += blockDim.x) touched[x] = 0;
        if constexpr (kDeltas) {
            if ((bucket_slots & 3u) == 0) {
                uint4* c4 = reinterpret_cast<uint4*>(cells);
                for (uint32_t x = tid; x < bucket_slots / 4; x += blockDim.x) c4[x] = make_uint4(0u, 0u, 0u, 0u);
            } else {
                for (uint32_t x = tid; x < bucket_slots; x += blockDim.x) cells[x] = 0;
            }
        }
        __syncthreads();
        if constexpr (kStaged) {
            // stage the counters of the blocks this item reads, 16 bytes per load when a block
            // holds at least that much
            for (uint32_t r = tid; r < count; r += blockDim.x) touched[a.recs[first + r] >> kRecLocalShift] = 1;
            __syncthreads();
            if (bs_log2 >= kVecLog2) {
                const uint32_t vlog = bs_log2 - kVecLog2;
                const uint32_t n_vec = bucket_blocks << vlog;
                uint4* c4 = reinterpret_cast<uint4*>(cells);
                for (uint32_t x = tid; x < n_vec; x += blockDim.x) {
                    const uint32_t lb = x >> vlog;
                    if (!touched[lb]) continue;
                    const uint64_t base = block_base(g, (bucket << a.bucket_shift) | lb);
                    const uint4* src = reinterpret_cast<const uint4*>(reinterpret_cast<const Cnt*>(a.table) + base);
                    c4[x] = __ldg(src + (x & ((1u << vlog) - 1u)));
                }
            } else {
                for (uint32_t x = tid; x < bucket_slots; x += blockDim.x) {
                    const uint32_t lb = x >> bs_log2;
                    if (!touched[lb]) continue;
                    const uint64_t base = block_base(g, (bucket << a.bucket_shift) | lb);
                    cells[x] = (Cell)load_counter<BITS>(a.table, base + (x & (bs - 1)));
                }
            }
            __syncthreads();
        }

        for (uint32_t c0 = 0; c0 < count;) {
            const uint32_t nrec = min(kApplyChunk, count - c0);
            if (tid < nrec) rv[tid] = a.recs[first + c0 + tid];
            __syncthreads();
            chunk_prefix(rv, nrec, ks, spre, wpre, warp_tot);
            // the leading records whose s-mers fit the chunk's budget (at least one)
            const uint32_t nuse = (uint32_t)__syncthreads_count(tid < nrec && spre[tid + 1] <= kSmerBudget);
            // stage the records' bases (one 16-byte entry per record, read in slot order) and
            // their reverse complements (a query with the insert's probe slots needs no bases)
            for (uint32_t r = tid; r < (have_probes || LEAN ? 0u : nuse); r += blockDim.x) {
                const uint4 b = __ldcs(a.sbases + first + c0 + r);
                reinterpret_cast<uint4*>(bases)[r] = b;
                reinterpret_cast<uint4*>(rbases)[r] = make_uint4(revcomp16(b.w), revcomp16(b.z), revcomp16(b.y),
                                                                 revcomp16(b.x));
            }
            if (tid < nuse) {  // record index of its s-mers (not needed with kept slots) / windows
                const uint32_t s0 = spre[tid], s1 = have_probes ? s0 : spre[tid + 1];
                for (uint32_t f = s0; f < s1; f++) smap[f] = (uint8_t)tid;
                if constexpr (kDeltas) touched[(uint32_t)(rv[tid] >> kRecLocalShift)] = 1;
                if constexpr (kStaged) {
                    const uint32_t w0i = wpre[tid], w1i = wpre[tid + 1];
                    for (uint32_t vv = w0i; vv < w1i; vv++) wmap[vv] = (uint8_t)tid;
                }
            }
            __syncthreads();
            const uint32_t nrec_used = nuse;
            const uint32_t S = spre[nrec_used];
            if constexpr (MODE == kModeReport) {
                if (have_probes) {
                    // the insert's slots of the chunk's s-mers: kProbeBatch loads in flight per
                    // thread, then the counter minima from shared memory
                    const unsigned long long* src = a.probes + pbase + poff;
                    for (uint32_t f0 = tid; f0 < S; f0 += kProbeBatch * blockDim.x) {
                        unsigned long long pk[kProbeBatch];
#pragma unroll
                        for (uint32_t j = 0; j < kProbeBatch; j++) {
                            const uint32_t f = f0 + j * blockDim.x;
                            pk[j] = f < S ? __ldcs(src + f) : 0ull;
                        }
#pragma unroll
                        for (uint32_t j = 0; j < kProbeBatch; j++) {
                            const uint32_t f = f0 + j * blockDim.x;
                            if (f >= S) break;
                            uint32_t e;
                            if constexpr (NH == 4) {
                                const uint32_t lo = (uint32_t)pk[j], hi = (uint32_t)(pk[j] >> 32);
                                const uint32_t c0 = cells[lo & 0xFFFFu], c1 = cells[lo >> 16];
                                const uint32_t c2 = cells[hi & 0xFFFFu], c3 = cells[hi >> 16];
                                e = min(min(c0, c1), min(c2, c3));
                            } else {
                                e = T::kMax;
                                for (uint32_t h = 0; h < g.h; h++) {
                                    const uint32_t c = cells[(uint32_t)(pk[j] >> (16 * h)) & 0xFFFFu];
                                    e = c < e ? c : e;
                                }
                            }
                            est[f] = (Est)e;
                        }
                    }
                }
            }
            // hash the s-mers (insert; query without stored slots)
            for (uint32_t f = have_probes ? S : tid; f < S; f += blockDim.x) {
                const uint32_t r = smap[f];
                const unsigned long long v = rv[r];
                const uint32_t lb = (uint32_t)(v >> kRecLocalShift);
                const uint32_t start = (uint32_t)v;
                const uint32_t rel = f - spre[r];  // base offset in the staged words
                // forward s-mer from the staged words; its reverse complement from the mirrored
                // words: base t of it is the complement of forward base rel + s - 1 - t, which
                // sits at position 16 * kRecBaseWords - rel - s + t of the mirrored stream (bits
                // read past the record's words land above 2s and are masked off)
                uint64_t smer;
                if constexpr (LEAN) {  // no staged bases: the codes from global memory
                    smer = canonical(codes64(a.codes, start + (f - spre[r])) & s_mask, sv);
                } else {
                    const uint64_t fw = codes64(bases + r * kRecBaseWords, rel) & s_mask;
                    const uint64_t rc = codes64(rbases + r * kRecBaseWords, 16u * kRecBaseWords - rel - sv) & s_mask;
                    smer = fw < rc ? fw : rc;
                }
                uint64_t hash = xorshift64(smer);
                Cell* blk = cells + (lb << bs_log2);
                if constexpr (kDeltas) {
                    unsigned long long pk = 0;
                    if constexpr (NH == 4) {
                        uint32_t sl[4];
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            sl[j] = (uint32_t)(hash & g.bs_mask);
                            if (j < 3) hash = xorshift64(hash);  // no mix after the last probe
                        }
#pragma unroll
                        for (int j = 0; j < 4; j++) atomicAdd(blk + sl[j], 1u);
                        const uint32_t cb = lb << bs_log2;  // the block's first cell in the bucket
                        pk = (unsigned long long)((cb + sl[0]) | ((cb + sl[1]) << 16)) |
                             ((unsigned long long)((cb + sl[2]) | ((cb + sl[3]) << 16)) << 32);
                    } else {
                        for (uint32_t h = 1;; h++) {  // n_hashes >= 1; no mix after the last probe
                            const uint32_t slot = (uint32_t)(hash & g.bs_mask);
                            atomicAdd(blk + slot, 1u);
                            pk |= (unsigned long long)((lb << bs_log2) + slot) << (((h - 1) & 3) * 16);
                            if (h >= g.h) break;
                            hash = xorshift64(hash);
                        }
                    }
                    if (kBuild && fused) {
                        __stcg(kept + poff + f, pk);
                    } else if (pbase != kNoProbes) {
                        __stcs(a.probes + pbase + poff + f, pk);
                    }
                } else {
                    uint32_t e = T::kMax;
                    if constexpr (NH == 4) {
#pragma unroll
                        for (int j = 0; j < 4; j++) {
                            const uint32_t c = blk[hash & g.bs_mask];
                            e = c < e ? c : e;
                            if (j < 3) hash = xorshift64(hash);
                        }
                    } else {
                        for (uint32_t h = 1;; h++) {
                            const uint32_t c = blk[hash & g.bs_mask];
                            e = c < e ? c : e;
                            if (h >= g.h) break;
                            hash = xorshift64(hash);
                        }
                    }
                    est[f] = (Est)e;
                }
            }
            __syncthreads();
            if constexpr (MODE == kModeReport) {
                const uint32_t W = wpre[nrec_used];
                for (uint32_t v = tid; v < W; v += blockDim.x) {
                    const uint32_t r = wmap[v];
                    const Est* e = est + spre[r] + (v - wpre[r]);
                    uint32_t m = e[0];
                    for (uint32_t t = 1; t <= ks; t++) m = min(m, (uint32_t)e[t]);
                    c_valid++;
                    c_pos += m > 0;
                    c_sum += m;
                }
                __syncthreads();
            }
            if constexpr (kSpec) {
                // fastx.rs:255-308, 392-410: each window's canonical k-mer (from the staged bases
                // and their mirror) counts its estimate once, the first time the key is seen
                const uint32_t W = wpre[nrec_used];
                const uint64_t kmask = len_mask(kv);
                for (uint32_t v = tid; v < W; v += blockDim.x) {
                    const uint32_t r = wmap[v];
                    const uint32_t off = v - wpre[r];
                    const Est* e = est + spre[r] + off;
                    uint32_t m = e[0];
                    for (uint32_t t = 1; t <= ks; t++) m = min(m, (uint32_t)e[t]);
                    const uint64_t fw = codes64(bases + r * kRecBaseWords, off) & kmask;
                    const uint64_t rc = codes64(rbases + r * kRecBaseWords, 16u * kRecBaseWords - off - kv) & kmask;
                    const uint64_t key = fw < rc ? fw : rc;
                    c_valid++;
                    const bool fresh = set_cap ? smem_set_insert(skeys, set_cap - 1, key)
                                               : set_insert(a.set_keys, a.set_mask, key, a.status);
                    if (fresh) {
                        c_dist++;
                        if (m < spec_bins) {
                            atomicAdd(shist + m, 1u);
                        } else if (m < a.hist_dense) {
                            atomicAdd(a.hist + m, 1ull);
                        } else {
                            const unsigned long long o = atomicAdd(&a.cnt[kCntOverflow], 1ull);
                            if (o < a.ovf_cap) {
                                a.ovf[o] = m;
                            } else {
                                atomicOr(a.status, kStatusOverflowFull);
                            }
                        }
                    }
                }
                __syncthreads();
            }
            c0 += nrec_used;
            poff += S;
        }

        if constexpr (kDeltas) {
            commit_item<BITS>(cells, touched, a, bucket, bs_log2, bucket_blocks, exclusive, kBuild && fused);
        }
        if constexpr (kBuild) {
            if (fused) {
                // the item's query (src/filter.rs:462-508): every record's blocks are final, in the
                // cells; each s-mer's estimate from its kept probe slots, then window minima, chunk
                // by chunk as the insert went (same chunks, so the same kept offsets)
                __syncthreads();
                uint64_t qoff = 0;
                for (uint32_t c0 = 0; c0 < count;) {
                    const uint32_t nrec = min(kApplyChunk, count - c0);
                    if (tid < nrec) rv[tid] = a.recs[first + c0 + tid];
                    __syncthreads();
                    chunk_prefix(rv, nrec, ks, spre, wpre, warp_tot);
                    const uint32_t nuse = (uint32_t)__syncthreads_count(tid < nrec && spre[tid + 1] <= kSmerBudget);
                    if (tid < nuse) {
                        const uint32_t w0i = wpre[tid], w1i = wpre[tid + 1];
                        for (uint32_t vv = w0i; vv < w1i; vv++) wmap[vv] = (uint8_t)tid;
                    }
                    const uint32_t S = spre[nuse];
                    // kProbeBatch kept probe words in flight per thread (L2 hits: the insert above
                    // wrote them), then the counter minima from the committed cells
                    for (uint32_t f0 = tid; f0 < S; f0 += kProbeBatch * blockDim.x) {
                        unsigned long long pk[kProbeBatch];
#pragma unroll
                        for (uint32_t j = 0; j < kProbeBatch; j++) {
                            const uint32_t f = f0 + j * blockDim.x;
                            pk[j] = f < S ? __ldcg(kept + qoff + f) : 0ull;
                        }
#pragma unroll
                        for (uint32_t j = 0; j < kProbeBatch; j++) {
                            const uint32_t f = f0 + j * blockDim.x;
                            if (f >= S) break;
                            uint32_t e;
                            if constexpr (NH == 4) {
                                const uint32_t lo = (uint32_t)pk[j], hi = (uint32_t)(pk[j] >> 32);
                                e = min(min(cells[lo & 0xFFFFu], cells[lo >> 16]),
                                        min(cells[hi & 0xFFFFu], cells[hi >> 16]));
                            } else {
                                e = T::kMax;
                                for (uint32_t h = 0; h < g.h; h++) {
                                    e = min(e, (uint32_t)cells[(uint32_t)(pk[j] >> (16 * h)) & 0xFFFFu]);
                                }
                            }
                            est[f] = (Est)e;
                        }
                    }
                    __syncthreads();
                    const uint32_t W = wpre[nuse];
                    for (uint32_t v = tid; v < W; v += blockDim.x) {
                        const uint32_t r = wmap[v];
                        const Est* e = est + spre[r] + (v - wpre[r]);
                        uint32_t m = e[0];
                        for (uint32_t t = 1; t <= ks; t++) m = min(m, (uint32_t)e[t]);
                        c_valid++;
                        c_pos += m > 0;
                        c_sum += m;
                    }
                    __syncthreads();
                    c0 += nuse;
                    qoff += S;
                }
            }
        }
        __syncthreads();
    }
    unsigned long long* rc = a.cnt;
    if constexpr (kBuild) rc = a.qcnt;
    warp_add_u64(&rc[kCntValid], c_valid);
    warp_add_u64(&rc[kCntPositive], c_pos);
    warp_add_u64(&rc[kCntChecksum], c_sum);
    if constexpr (kSpec) {
        warp_add_u64(&rc[kCntDistinct], c_dist);
        __syncthreads();
        for (uint32_t x = tid; x < spec_bins; x += blockDim.x) {
            if (shist[x]) atomicAdd(a.hist + x, (unsigned long long)shist[x]);
        }
    }
}

template <int MODE, int BITS, int NH, int KSC>
__global__ void __launch_bounds__(kApplyMaxThreads) k_apply_insert(GroupArgs a, uint32_t bs_log2,
                                                                    uint32_t bucket_blocks) {
    apply_body<MODE, BITS, NH, false, KSC>(a, bs_log2, bucket_blocks);
}

// The query is held to 2048 threads per SM at every CTA width (at most 32 registers), which
// measured faster than the compiler's own choice; the insert measured faster without it.
template <int MODE, int BITS, int NH, bool LEAN, int KSC>
__global__ void __launch_bounds__(kApplyMaxThreads, 2048 / kApplyMaxThreads) k_apply_query(GroupArgs a,
                                                                                           uint32_t bs_log2,
                                                                                           uint32_t bucket_blocks) {
    apply_body<MODE, BITS, NH, LEAN, KSC>(a, bs_log2, bucket_blocks);
}

template <int MODE, int BITS, int NH, int KSC>
__global__ void __launch_bounds__(kApplyMaxThreads) k_apply_spectrum(GroupArgs a, uint32_t bs_log2,
                                                                      uint32_t bucket_blocks) {
    apply_body<MODE, BITS, NH, false, KSC>(a, bs_log2, bucket_blocks);
}

static size_t apply_smem(int mode, int bits, uint32_t bucket_slots, uint32_t bucket_blocks, bool lean) {
    return apply_layout(mode, bits, bucket_slots, bucket_blocks, lean).total;
}

template <int MODE, int BITS>
static void launch_apply_t(const GroupArgs& a, int bs_log2, uint32_t bucket_blocks, int sm_count, uint64_t max_items,
                           cudaStream_t st) {
    const bool lean = MODE == kModeReport && a.probes != nullptr;
    const size_t smem = apply_smem(MODE, BITS, (1u << bs_log2) * bucket_blocks, bucket_blocks, lean);
    void (*fn)(GroupArgs, uint32_t, uint32_t);
    const bool dflt = a.g.h == 4 && (((int)a.g.k << 8) | (int)a.g.s) == kDefaultKS;
    if constexpr (MODE == kModeInsert || MODE == kModeBuild) {
        fn = dflt ? k_apply_insert<MODE, BITS, 4, kDefaultKS>
                  : (a.g.h == 4 ? k_apply_insert<MODE, BITS, 4, 0> : k_apply_insert<MODE, BITS, 0, 0>);
    } else if constexpr (MODE == kModeSpectrum) {
        fn = dflt ? k_apply_spectrum<MODE, BITS, 4, kDefaultKS>
                  : (a.g.h == 4 ? k_apply_spectrum<MODE, BITS, 4, 0> : k_apply_spectrum<MODE, BITS, 0, 0>);
    } else {
        if (lean) {
            fn = dflt ? k_apply_query<MODE, BITS, 4, true, kDefaultKS>
                      : (a.g.h == 4 ? k_apply_query<MODE, BITS, 4, true, 0> : k_apply_query<MODE, BITS, 0, true, 0>);
        } else {
            fn = dflt ? k_apply_query<MODE, BITS, 4, false, kDefaultKS>
                      : (a.g.h == 4 ? k_apply_query<MODE, BITS, 4, false, 0> : k_apply_query<MODE, BITS, 0, false, 0>);
        }
    }
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    // one thread per staged record at least (256 or 512 threads)
    const int threads = a.apply_threads == 512 ? 512 : (int)kApplyChunk;
    int per_sm = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess || per_sm < 1) {
        per_sm = 1;
    }
    uint64_t grid = (uint64_t)per_sm * sm_count;
    if (grid > max_items) grid = max_items;
    if (grid == 0) grid = 1;
    fn<<<(unsigned)grid, threads, smem, st>>>(a, (uint32_t)bs_log2, bucket_blocks);
    note_launch();
}



void launch_apply(int mode, const GroupArgs& a, int bs_log2, uint32_t bucket_blocks, int sm_count, uint64_t max_items,
                  cudaStream_t st) {
    if (mode == kModeInsert) {
        switch (a.g.bits) {
            case 8: launch_apply_t<kModeInsert, 8>(a, bs_log2, bucket_blocks, sm_count, max_items, st); break;
            case 16: launch_apply_t<kModeInsert, 16>(a, bs_log2, bucket_blocks, sm_count, max_items, st); break;
            default: launch_apply_t<kModeInsert, 32>(a, bs_log2, bucket_blocks, sm_count, max_items, st); break;
        }
    } else if (mode == kModeSpectrum) {
        switch (a.g.bits) {
            case 8: launch_apply_t<kModeSpectrum, 8>(a, bs_log2, bucket_blocks, sm_count, max_items, st); break;
            case 16: launch_apply_t<kModeSpectrum, 16>(a, bs_log2, bucket_blocks, sm_count, max_items, st); break;
            default: launch_apply_t<kModeSpectrum, 32>(a, bs_log2, bucket_blocks, sm_count, max_items, st); break;
        }
    } else if (mode == kModeBuild) {
        switch (a.g.bits) {
            case 8: launch_apply_t<kModeBuild, 8>(a, bs_log2, bucket_blocks, sm_count, max_items, st); break;
            case 16: launch_apply_t<kModeBuild, 16>(a, bs_log2, bucket_blocks, sm_count, max_items, st); break;
            default: launch_apply_t<kModeBuild, 32>(a, bs_log2, bucket_blocks, sm_count, max_items, st); break;
        }
    } else {
        switch (a.g.bits) {
            case 8: launch_apply_t<kModeReport, 8>(a, bs_log2, bucket_blocks, sm_count, max_items, st); break;
            case 16: launch_apply_t<kModeReport, 16>(a, bs_log2, bucket_blocks, sm_count, max_items, st); break;
            default: launch_apply_t<kModeReport, 32>(a, bs_log2, bucket_blocks, sm_count, max_items, st); break;
        }
    }
}

void launch_scatter(const uint32_t* rec_key, const unsigned long long* rec_val, const uint4* rec_bases,
                    const unsigned long long* rec_count, uint64_t rec_cap, uint32_t bucket_shift,
                    unsigned long long* cursor, uint64_t base, unsigned long long* sorted, uint4* sbases,
                    cudaStream_t st) {
    const uint64_t blocks = (rec_cap + 255) / 256;
    k_scatter<<<(unsigned)(blocks < 4096 ? (blocks ? blocks : 1) : 4096), 256, 0, st>>>(
        rec_key, rec_val, rec_bases, rec_count, rec_cap, bucket_shift, cursor, base, sorted, sbases);
    note_launch();
}

void launch_item_counts(const unsigned long long* counts, uint64_t n_buckets, uint64_t bucket_cap, uint64_t* item_count,
                        uint64_t* ovf_count, const unsigned long long* rec_count, uint64_t rec_cap, cudaStream_t st) {
    const uint64_t blocks = (n_buckets + 1 + 255) / 256;
    k_item_counts<<<(unsigned)(blocks < 16384 ? blocks : 16384), 256, 0, st>>>(counts, n_buckets, bucket_cap,
                                                                              item_count, ovf_count, rec_count,
                                                                              rec_cap);
    note_launch();
}

void launch_item_write(const unsigned long long* counts, uint64_t bucket_cap, const uint64_t* item_off,
                       const uint64_t* ovf_off, uint64_t ovf_base, uint64_t n_buckets, uint4* items,
                       cudaStream_t st) {
    const uint64_t blocks = (n_buckets + 255) / 256;
    k_item_write<<<(unsigned)(blocks < 16384 ? (blocks ? blocks : 1) : 16384), 256, 0, st>>>(
        counts, bucket_cap, item_off, ovf_off, ovf_base, n_buckets, items);
    note_launch();
}

// ---------------------------------------------------------------------------------------
// Small launches
// ---------------------------------------------------------------------------------------
__global__ void k_fill_u32(uint32_t* p, uint32_t v, uint64_t n) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) p[i] = v;
}

void launch_fill_u32(uint32_t* p, uint32_t v, uint64_t n, cudaStream_t st) {
    if (n == 0) return;
    const uint64_t blocks = (n + 255) / 256;
    k_fill_u32<<<(unsigned)(blocks < 65536 ? blocks : 65536), 256, 0, st>>>(p, v, n);
    note_launch();
}

void launch_pack(const uint8_t* ascii, uint64_t n_bytes, uint32_t* codes, uint32_t* valid, cudaStream_t st) {
    const uint64_t n_groups = (n_bytes + 31) / 32;
    if (n_groups == 0) return;
    const int aligned = ((reinterpret_cast<uintptr_t>(ascii) & 15) == 0) ? 1 : 0;
    const uint64_t blocks = (n_groups + 255) / 256;
    k_pack<<<(unsigned)(blocks < (1u << 20) ? blocks : (1u << 20)), 256, 0, st>>>(ascii, n_bytes, codes, valid,
                                                                                  n_groups, aligned);
    note_launch();
}

void launch_seqstart(const uint64_t* offsets, uint64_t n_seqs, uint64_t n_bytes, uint32_t* seqstart,
                     cudaStream_t st) {
    if (n_seqs == 0) return;
    const uint64_t blocks = (n_seqs + 255) / 256;
    k_seqstart<<<(unsigned)(blocks < 65536 ? blocks : 65536), 256, 0, st>>>(offsets, n_seqs, n_bytes, seqstart);
    note_launch();
}

void launch_seq_windows(const uint64_t* offsets, uint64_t n_seqs, uint32_t k, unsigned long long* cnt,
                        uint64_t* woff, cudaStream_t st) {
    if (n_seqs == 0) return;
    const uint64_t blocks = (n_seqs + 255) / 256;
    k_seq_windows<<<(unsigned)(blocks < 4096 ? blocks : 4096), 256, 0, st>>>(offsets, n_seqs, k, cnt, woff);
    note_launch();
}

}  // namespace scb
