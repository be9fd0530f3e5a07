// Device helpers for the SuperCountingBloom kernels (sm_100a).
//
// Data layout in HBM for one batch of concatenated sequences (N bytes):
//   codes    : 2-bit base codes, 16 bases per 32-bit word; base g at bits 2*(g%16) of word g/16
//              (code = (ascii >> 1) & 3: A=0, C=1, T=2, G=3; complement = code ^ 2)
//   valid    : 1 bit per base (is A/C/G/T in either case), base g at bit g%32 of word g/32
//   seqstart : 1 bit per base, set where a non-empty sequence starts
// A k-mer window at g is valid when bases g..g+k-1 are valid and no sequence starts inside
// g+1..g+k-1, i.e. the window lies inside one maximal ACGT run of one sequence.
// The counter table is kept in .scb file order (shard-major), so save/load is one copy.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace scb {

// Status bits written to the context's device status word.
constexpr uint32_t kStatusCasLimit = 1u << 0;   // a saturating CAS loop gave up
constexpr uint32_t kStatusHashFull = 1u << 1;   // the distinct-k-mer set ran out of probes
constexpr uint32_t kStatusOverflowFull = 1u << 2;  // histogram overflow list full
constexpr int kMaxCasTries = 1 << 20;

// Geometry of one filter, precomputed on the host (filter.rs:90-116 layout).
struct DevGeom {
    uint32_t k, m, s, h, w;   // w = k - m + 1 m-mers per window
    uint32_t bits;            // counter width
    uint32_t block_log2;      // block_slots_exponent
    uint32_t shard_shift;     // log2(shard_count)
    uint32_t sub_log2;        // log2(subblocks)
    uint32_t pad_;
    uint64_t block_mask;      // nb_blocks - 1
    uint64_t shard_mask;      // shard_count - 1
    uint64_t bs_mask;         // block_slots - 1
};

// filter.rs:629-635 (SplitMix64 finaliser, golden-ratio increment).
__device__ __forceinline__ uint64_t xorshift64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

// filter.rs:217-219 + CounterShard::index: file-order index of the block's first counter.
// (shard * subblocks + subblock) * block_slots, with subblocks a power of two.
__device__ __forceinline__ uint64_t block_base(const DevGeom& g, uint64_t block) {
    return (((block & g.shard_mask) << g.sub_log2) | (block >> g.shard_shift)) << g.block_log2;
}

__device__ __forceinline__ uint64_t len_mask(uint32_t len) {
    return len >= 32 ? ~0ull : ((1ull << (2 * len)) - 1ull);
}

// Reverse complement of a len-base value (base t at bits 2t..2t+1), same bit order.
__device__ __forceinline__ uint64_t revcomp(uint64_t v, uint32_t len) {
    uint64_t r = __brevll(v);
    r = ((r >> 1) & 0x5555555555555555ull) | ((r & 0x5555555555555555ull) << 1);
    const uint32_t sh = 64u - 2u * len;
    r = sh >= 64 ? 0 : (r >> sh);
    return r ^ (0xAAAAAAAAAAAAAAAAull >> sh);
}

// Reverse complement of the 16 bases of one code word (base t moves to 15 - t).
__device__ __forceinline__ uint32_t revcomp16(uint32_t w) {
    uint32_t r = __brev(w);
    r = ((r >> 1) & 0x55555555u) | ((r & 0x55555555u) << 1);
    return r ^ 0xAAAAAAAAu;
}

__device__ __forceinline__ uint64_t canonical(uint64_t fwd, uint32_t len) {
    const uint64_t rc = revcomp(fwd, len);
    return fwd < rc ? fwd : rc;
}

// 64 bits of a 2-bit code stream starting at base b (words of 16 bases).  Reads words
// b/16 .. b/16+2, which the caller keeps in bounds.  Positions are below 2^31 (a batch's bases
// or a tile's shared-memory stream), so the index arithmetic stays 32-bit.
__device__ __forceinline__ uint64_t codes64(const uint32_t* words, uint32_t b) {
    const uint32_t w = b >> 4;
    const uint32_t sh = (b & 15u) * 2u;
    const uint32_t w0 = words[w], w1 = words[w + 1], w2 = words[w + 2];
    const uint32_t lo = __funnelshift_r(w0, w1, sh);
    const uint32_t hi = __funnelshift_r(w1, w2, sh);
    return ((uint64_t)hi << 32) | lo;
}

// 64 bits of a bitmap starting at bit b (words of 32 bits); reads words b/32 .. b/32+2.
__device__ __forceinline__ uint64_t bits64(const uint32_t* words, uint32_t b) {
    const uint32_t w = b >> 5;
    const uint32_t sh = b & 31u;
    const uint32_t w0 = words[w], w1 = words[w + 1], w2 = words[w + 2];
    const uint32_t lo = __funnelshift_r(w0, w1, sh);
    const uint32_t hi = __funnelshift_r(w1, w2, sh);
    return ((uint64_t)hi << 32) | lo;
}

// Window validity from the valid / seqstart bitmaps (bits starting at the window's base).
__device__ __forceinline__ bool window_ok(uint64_t valid_bits, uint64_t start_bits, uint32_t k) {
    const uint64_t km = k >= 64 ? ~0ull : ((1ull << k) - 1ull);
    return ((valid_bits & km) == km) && (((start_bits >> 1) & (km >> 1)) == 0);
}

// ---------------------------------------------------------------------------------------
// Canonical ntHash of m-mers (restatement of the seq-hash / simd-minimizers hash): 32-bit,
// rotation 7 per character, original ntHash seeds (low 32 bits) per letter; hash = fw + rc.
// ---------------------------------------------------------------------------------------
constexpr uint32_t kNtRot = 7u;

__device__ __forceinline__ uint32_t nt_seed(uint32_t c) {
    const uint32_t lo = (c & 1u) ? 0x62a02b4cu : 0x95c60474u;  // C : A
    const uint32_t hi = (c & 1u) ? 0x82572324u : 0x4be24456u;  // G : T
    return (c & 2u) ? hi : lo;
}
__device__ __forceinline__ uint32_t rotl32(uint32_t x, uint32_t r) { return __funnelshift_l(x, x, r); }
__device__ __forceinline__ uint32_t rotr32(uint32_t x, uint32_t r) { return __funnelshift_r(x, x, r); }

// Forward / reverse ntHash of the m-mer whose codes are in v (base t at bits 2t).
__device__ __forceinline__ void nt_direct(uint64_t v, uint32_t m, uint32_t& fw, uint32_t& rc) {
    fw = 0;
    rc = 0;
    for (uint32_t t = 0; t < m; t++) {
        const uint32_t c = (uint32_t)(v >> (2 * t)) & 3u;
        fw ^= rotl32(nt_seed(c), kNtRot * (m - 1 - t));
        rc ^= rotl32(nt_seed(c ^ 2u), kNtRot * t);
    }
}

// Roll both hashes one base forward: c_out leaves at the left, c_in enters at the right.
__device__ __forceinline__ void nt_roll(uint32_t& fw, uint32_t& rc, uint32_t c_out, uint32_t c_in, uint32_t m) {
    fw = rotl32(fw, kNtRot) ^ rotl32(nt_seed(c_out), kNtRot * m) ^ nt_seed(c_in);
    rc = rotr32(rc, kNtRot) ^ rotr32(nt_seed(c_out ^ 2u), kNtRot) ^ rotl32(nt_seed(c_in ^ 2u), kNtRot * (m - 1));
}

// ---------------------------------------------------------------------------------------
// Counters
// ---------------------------------------------------------------------------------------
template <int BITS>
struct CounterTraits {
    static constexpr uint32_t kLanes = 32 / BITS;
    static constexpr uint32_t kMax = BITS == 32 ? 0xFFFFFFFFu : ((1u << BITS) - 1u);
};

// counter.rs saturating_increment on a counter packed in a 32-bit word, through atomicCAS.
// Saturated counters need no write.  The loop is lock-free (each failure means another
// thread's CAS succeeded); it is bounded all the same and reports through *status.
template <int BITS>
__device__ __forceinline__ void sat_inc(uint32_t* table32, uint64_t idx, uint32_t* status) {
    using T = CounterTraits<BITS>;
    uint32_t* p = table32 + (idx / T::kLanes);
    const uint32_t sh = (uint32_t)(idx % T::kLanes) * BITS;
    uint32_t old = __ldcg(p);
    for (int it = 0; it < kMaxCasTries; ++it) {
        if (((old >> sh) & T::kMax) == T::kMax) return;
        const uint32_t prev = atomicCAS(p, old, old + (1u << sh));
        if (prev == old) return;
        old = prev;
    }
    atomicOr(status, kStatusCasLimit);
}

// Saturating add of `delta` (>= 1) to one counter, same protocol.
template <int BITS>
__device__ __forceinline__ void sat_add(uint32_t* table32, uint64_t idx, uint32_t delta, uint32_t* status) {
    using T = CounterTraits<BITS>;
    uint32_t* p = table32 + (idx / T::kLanes);
    const uint32_t sh = (uint32_t)(idx % T::kLanes) * BITS;
    uint32_t old = __ldcg(p);
    for (int it = 0; it < kMaxCasTries; ++it) {
        const uint32_t cur = (old >> sh) & T::kMax;
        if (cur == T::kMax) return;
        const uint32_t room = T::kMax - cur;
        const uint32_t add = delta < room ? delta : room;
        const uint32_t prev = atomicCAS(p, old, old + (add << sh));
        if (prev == old) return;
        old = prev;
    }
    atomicOr(status, kStatusCasLimit);
}

template <int BITS>
__device__ __forceinline__ uint32_t load_counter(const void* table, uint64_t idx) {
    if constexpr (BITS == 8) {
        return __ldg(reinterpret_cast<const unsigned char*>(table) + idx);
    } else if constexpr (BITS == 16) {
        return __ldg(reinterpret_cast<const unsigned short*>(table) + idx);
    } else {
        return __ldg(reinterpret_cast<const unsigned int*>(table) + idx);
    }
}

// filter.rs:562-571: min over the n_hashes probes of an s-mer inside one block.
template <int BITS>
__device__ __forceinline__ uint32_t estimate_smer(const void* table, const DevGeom& g, uint64_t base, uint64_t smer) {
    uint64_t hash = xorshift64(smer);
    uint32_t est = CounterTraits<BITS>::kMax;
    for (uint32_t i = 1;; i++) {  // n_hashes >= 1; the chain's value after the last probe is unused
        const uint32_t v = load_counter<BITS>(table, base + (hash & g.bs_mask));
        est = v < est ? v : est;
        if (i >= g.h) break;
        hash = xorshift64(hash);
    }
    return est;
}

// filter.rs:224-233: the n_hashes saturating increments of one s-mer inside one block.
template <int BITS>
__device__ __forceinline__ void insert_smer(uint32_t* table32, const DevGeom& g, uint64_t base, uint64_t smer,
                                            uint32_t* status) {
    uint64_t hash = xorshift64(smer);
    for (uint32_t i = 1;; i++) {
        sat_inc<BITS>(table32, base + (hash & g.bs_mask), status);
        if (i >= g.h) break;
        hash = xorshift64(hash);
    }
}

// Warp-aggregated add of a 64-bit value to a global counter.
__device__ __forceinline__ void warp_add_u64(unsigned long long* dst, unsigned long long v) {
    for (int off = 16; off > 0; off >>= 1) v += __shfl_down_sync(0xFFFFFFFFu, v, off);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(dst, v);
}

}  // namespace scb
