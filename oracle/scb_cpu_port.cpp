// Multi-threaded CPU port of the reference's build + stream-query pipeline (TEST / BASELINE
// INFRASTRUCTURE: timed as the CPU baseline, never part of the product library).
//
// Structure follows the reference:
//   - one producer splits each record at non-ACGT bytes, keeps chunks of length >= k and sends
//     an owned copy of each chunk through a bounded queue of `queue` entries
//     (fastx.rs:206-253 build_filter, fastx.rs:310-369 stream_query_kmers);
//   - `threads` workers pack each chunk and insert / query it;
//   - the counter table is split into min(nb_blocks, 1024) shards, each behind its own mutex,
//     locked once per super-k-mer (filter.rs:57-65, 130-134, 217-222).
// The per-chunk arithmetic is the oracle's (scb_oracle.c) made incremental: rolling ntHash,
// rolling TG count and rolling canonical s-mers, as the crate's scalar code path computes them.
// Its results are checked against the oracle in tests/test_oracle.py.

#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdint>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "scb_oracle.h"

namespace {

constexpr uint32_t kSeed[4] = {0x95c60474u, 0x62a02b4cu, 0x4be24456u, 0x82572324u};
constexpr uint32_t kRot = 7u;

inline uint32_t rotl(uint32_t x, uint32_t r) {
    r &= 31u;
    return r ? (x << r) | (x >> (32u - r)) : x;
}
inline uint32_t rotr(uint32_t x, uint32_t r) {
    r &= 31u;
    return r ? (x >> r) | (x << (32u - r)) : x;
}

// Bounded multi-producer / multi-consumer queue (the crossbeam bounded channel).
class BoundedQueue {
  public:
    explicit BoundedQueue(size_t cap) : cap_(cap ? cap : 1) {}
    void push(std::vector<uint8_t>&& v) {
        std::unique_lock<std::mutex> lk(mu_);
        not_full_.wait(lk, [&] { return q_.size() < cap_; });
        q_.push_back(std::move(v));
        not_empty_.notify_one();
    }
    bool pop(std::vector<uint8_t>& out) {
        std::unique_lock<std::mutex> lk(mu_);
        not_empty_.wait(lk, [&] { return !q_.empty() || closed_; });
        if (q_.empty()) return false;
        out = std::move(q_.front());
        q_.pop_front();
        not_full_.notify_one();
        return true;
    }
    void close() {
        std::lock_guard<std::mutex> lk(mu_);
        closed_ = true;
        not_empty_.notify_all();
    }

  private:
    size_t cap_;
    std::deque<std::vector<uint8_t>> q_;
    bool closed_ = false;
    std::mutex mu_;
    std::condition_variable not_full_, not_empty_;
};

struct Geometry {
    uint64_t k, m, s, h;
    int bits;
    ora_layout L;
};

// Super-k-mer cut of one chunk of codes: starts and block base indices.
struct SuperKmers {
    std::vector<uint32_t> starts;
    std::vector<uint64_t> bases;
    std::vector<uint64_t> shards;
};

void cut_super_kmers(const Geometry& g, const uint8_t* codes, size_t len, SuperKmers& out,
                     std::vector<uint32_t>& keys) {
    out.starts.clear();
    out.bases.clear();
    out.shards.clear();
    const size_t k = g.k, m = g.m, w = k - m + 1;
    const size_t n_mmers = len - m + 1;
    keys.resize(n_mmers);
    // rolling canonical ntHash
    uint32_t fw = 0, rc = 0;
    for (size_t t = 0; t < m; t++) {
        fw ^= rotl(kSeed[codes[t]], uint32_t(kRot * (m - 1 - t)));
        rc ^= rotl(kSeed[codes[t] ^ 2], uint32_t(kRot * t));
    }
    keys[0] = (fw + rc) >> 16;
    for (size_t j = 1; j < n_mmers; j++) {
        uint8_t out_c = codes[j - 1], in_c = codes[j + m - 1];
        fw = rotl(fw, kRot) ^ rotl(kSeed[out_c], uint32_t(kRot * m)) ^ kSeed[in_c];
        rc = rotr(rc, kRot) ^ rotr(kSeed[out_c ^ 2], kRot) ^ rotl(kSeed[in_c ^ 2], uint32_t(kRot * (m - 1)));
        keys[j] = (fw + rc) >> 16;
    }
    size_t tg = 0;
    for (size_t t = 0; t < k; t++) tg += codes[t] >> 1;
    size_t prev = SIZE_MAX;
    const uint64_t mmask = m == 32 ? ~0ULL : ((1ULL << (2 * m)) - 1);
    for (size_t i = 0; i + k <= len; i++) {
        if (i > 0) tg += (codes[i + k - 1] >> 1) - (codes[i - 1] >> 1);
        uint32_t best = 0xFFFFFFFFu;
        size_t left = 0, right = 0;
        for (size_t o = 0; o < w; o++) {
            uint32_t key = keys[i + o];
            if (key < best) {
                best = key;
                left = right = o;
            } else if (key == best) {
                right = o;
            }
        }
        size_t p = i + ((2 * tg > k) ? left : right);
        if (i == 0 || p != prev) {
            uint64_t f = 0, r = 0;
            for (size_t t = 0; t < m; t++) {
                f |= uint64_t(codes[p + t]) << (2 * t);
                r |= uint64_t(codes[p + m - 1 - t] ^ 2) << (2 * t);
            }
            (void)mmask;
            uint64_t minv = std::min(f, r);
            uint64_t block = ora_xorshift_u64(minv) & g.L.block_mask;
            uint64_t shard = block & g.L.shard_mask;
            uint64_t sub = block >> g.L.shard_shift;
            out.starts.push_back(uint32_t(i));
            out.bases.push_back((shard * g.L.subblocks + sub) * g.L.block_slots);
            out.shards.push_back(shard);
        }
        prev = p;
    }
}

// Canonical s-mers of positions [0, n) of a chunk, rolling.
void canonical_smers(const uint8_t* codes, size_t n, size_t s, std::vector<uint64_t>& out) {
    out.resize(n);
    const uint64_t mask = s == 32 ? ~0ULL : ((1ULL << (2 * s)) - 1);
    uint64_t f = 0, r = 0;
    for (size_t t = 0; t + 1 < s; t++) {
        f |= uint64_t(codes[t]) << (2 * t);
        r = ((r << 2) | uint64_t(codes[t] ^ 2)) & mask;
    }
    for (size_t pos = 0; pos < n; pos++) {
        uint8_t c = codes[pos + s - 1];
        f = (f | (uint64_t(c) << (2 * (s - 1)))) & mask;
        r = ((r << 2) | uint64_t(c ^ 2)) & mask;
        out[pos] = std::min(f, r);
        f >>= 2;
    }
}

template <typename C>
struct Port {
    Geometry g;
    C* table;
    std::vector<std::mutex>* locks;

    uint64_t insert_chunk(const uint8_t* codes, size_t len, SuperKmers& sk, std::vector<uint32_t>& keys,
                          std::vector<uint64_t>& smers) {
        cut_super_kmers(g, codes, len, sk, keys);
        const size_t nw = len - g.k + 1;
        canonical_smers(codes, nw + g.k - g.s, g.s, smers);
        uint64_t inserted = 0;
        const C maxv = C(~C(0));
        for (size_t i = 0; i < sk.starts.size(); i++) {
            size_t st = sk.starts[i];
            size_t en = i + 1 < sk.starts.size() ? sk.starts[i + 1] : nw;
            size_t end_smer = en + (g.k - g.s);
            C* blk = table + sk.bases[i];
            std::lock_guard<std::mutex> lk((*locks)[sk.shards[i]]);
            for (size_t pos = st; pos < end_smer; pos++) {
                uint64_t hash = ora_xorshift_u64(smers[pos]);
                for (uint64_t h = 0; h < g.h; h++) {
                    C& c = blk[hash & g.L.block_slots_mask];
                    if (c != maxv) c++;
                    hash = ora_xorshift_u64(hash);
                }
                inserted++;
            }
        }
        return inserted;
    }

    void query_chunk(const uint8_t* codes, size_t len, SuperKmers& sk, std::vector<uint32_t>& keys,
                     std::vector<uint64_t>& smers, std::vector<uint64_t>& est, std::vector<size_t>& dq,
                     ora_report& rep) {
        cut_super_kmers(g, codes, len, sk, keys);
        const size_t nw = len - g.k + 1;
        canonical_smers(codes, nw + g.k - g.s, g.s, smers);
        const size_t window = g.k - g.s + 1;
        for (size_t i = 0; i < sk.starts.size(); i++) {
            size_t st = sk.starts[i];
            size_t en = i + 1 < sk.starts.size() ? sk.starts[i + 1] : nw;
            size_t smer_count = en - st + window - 1;
            const C* blk = table + sk.bases[i];
            est.resize(smer_count);
            for (size_t o = 0; o < smer_count; o++) {
                uint64_t hash = ora_xorshift_u64(smers[st + o]);
                C e = C(~C(0));
                for (uint64_t h = 0; h < g.h; h++) {
                    e = std::min(e, blk[hash & g.L.block_slots_mask]);
                    hash = ora_xorshift_u64(hash);
                }
                est[o] = e;
            }
            dq.resize(smer_count);
            size_t head = 0, tail = 0;
            for (size_t o = 0; o < smer_count; o++) {
                while (tail > head && est[dq[tail - 1]] >= est[o]) tail--;
                dq[tail++] = o;
                while (tail > head && dq[head] + window <= o) head++;
                if (o + 1 >= window) {
                    uint64_t v = est[dq[head]];
                    rep.valid_kmers++;
                    if (v > 0) rep.positive_estimates++;
                    rep.estimate_checksum += v;
                }
            }
        }
    }
};

void produce_chunks(const uint8_t* seqs, const uint64_t* offsets, uint64_t n, uint64_t k, BoundedQueue& q,
                    uint64_t* chunks, uint64_t* kmers) {
    for (uint64_t r = 0; r < n; r++) {
        const uint8_t* s = seqs + offsets[r];
        size_t len = offsets[r + 1] - offsets[r];
        size_t i = 0;
        while (i < len) {
            while (i < len && !ora_is_acgt(s[i])) i++;
            size_t a = i;
            while (i < len && ora_is_acgt(s[i])) i++;
            if (i - a >= k) {
                if (chunks) (*chunks)++;
                if (kmers) *kmers += i - a + 1 - k;
                q.push(std::vector<uint8_t>(s + a, s + i));
            }
        }
    }
    q.close();
}

template <typename C>
int run_port(ora_filter* f, const uint8_t* seqs, const uint64_t* offsets, uint64_t n, uint64_t threads,
             uint64_t queue, uint64_t* ikmers, uint64_t* ismers, ora_report* rep, double* build_s,
             double* query_s) {
    const ora_config* cfg = ora_filter_config(f);
    Port<C> port;
    port.g.k = cfg->k;
    port.g.m = cfg->m;
    port.g.s = cfg->s;
    port.g.h = cfg->n_hashes;
    port.g.bits = cfg->counter_bits;
    ora_layout_from_config(cfg, &port.g.L);
    port.table = static_cast<C*>(ora_filter_table(f));
    std::vector<std::mutex> locks(port.g.L.shard_count);
    port.locks = &locks;
    if (threads == 0) threads = 1;

    auto t0 = std::chrono::steady_clock::now();
    uint64_t chunks = 0, kmers = 0;
    std::vector<uint64_t> smers_per(threads, 0);
    {
        BoundedQueue q(queue);
        std::vector<std::thread> workers;
        for (uint64_t t = 0; t < threads; t++) {
            workers.emplace_back([&, t] {
                std::vector<uint8_t> chunk;
                SuperKmers sk;
                std::vector<uint32_t> keys;
                std::vector<uint64_t> sm;
                uint64_t local = 0;
                while (q.pop(chunk)) {
                    for (auto& b : chunk) b = ora_base_code(b);
                    local += port.insert_chunk(chunk.data(), chunk.size(), sk, keys, sm);
                }
                smers_per[t] = local;
            });
        }
        produce_chunks(seqs, offsets, n, cfg->k, q, &chunks, &kmers);
        for (auto& w : workers) w.join();
    }
    auto t1 = std::chrono::steady_clock::now();
    uint64_t smers = 0;
    for (auto v : smers_per) smers += v;

    std::vector<ora_report> reps(threads);
    {
        BoundedQueue q(queue);
        std::vector<std::thread> workers;
        for (uint64_t t = 0; t < threads; t++) {
            workers.emplace_back([&, t] {
                std::vector<uint8_t> chunk;
                SuperKmers sk;
                std::vector<uint32_t> keys;
                std::vector<uint64_t> sm, est;
                std::vector<size_t> dq;
                ora_report local;
                std::memset(&local, 0, sizeof(local));
                while (q.pop(chunk)) {
                    for (auto& b : chunk) b = ora_base_code(b);
                    local.records_processed++;
                    local.total_windows += chunk.size() + 1 - port.g.k;
                    port.query_chunk(chunk.data(), chunk.size(), sk, keys, sm, est, dq, local);
                }
                reps[t] = local;
            });
        }
        produce_chunks(seqs, offsets, n, cfg->k, q, nullptr, nullptr);
        for (auto& w : workers) w.join();
    }
    auto t2 = std::chrono::steady_clock::now();
    std::memset(rep, 0, sizeof(*rep));
    for (auto& r : reps) {
        rep->records_processed += r.records_processed;
        rep->total_windows += r.total_windows;
        rep->valid_kmers += r.valid_kmers;
        rep->positive_estimates += r.positive_estimates;
        rep->estimate_checksum += r.estimate_checksum;
    }
    ora_filter_set_inserted_kmers(f, ora_filter_inserted_kmers(f) + kmers);
    *ikmers = kmers;
    *ismers = smers;
    *build_s = std::chrono::duration<double>(t1 - t0).count();
    *query_s = std::chrono::duration<double>(t2 - t1).count();
    return 0;
}

}  // namespace

extern "C" int ora_port_build_and_stream_query(ora_filter* f, const uint8_t* seqs, const uint64_t* offsets,
                                               uint64_t n, uint64_t threads, uint64_t queue,
                                               uint64_t* inserted_kmers, uint64_t* inserted_smers,
                                               ora_report* rep, double* build_s, double* query_s) {
    switch (ora_filter_config(f)->counter_bits) {
        case 8:
            return run_port<uint8_t>(f, seqs, offsets, n, threads, queue, inserted_kmers, inserted_smers, rep,
                                     build_s, query_s);
        case 16:
            return run_port<uint16_t>(f, seqs, offsets, n, threads, queue, inserted_kmers, inserted_smers,
                                      rep, build_s, query_s);
        default:
            return run_port<uint32_t>(f, seqs, offsets, n, threads, queue, inserted_kmers, inserted_smers,
                                      rep, build_s, query_s);
    }
}
