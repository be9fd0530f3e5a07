/*
 * CPU oracle (test infrastructure) -- plain-C restatement of the reference crate
 * super-counting-bloom 0.1.0.  See scb_oracle.h for the parity status of each part.
 * Every function cites the reference file:line it follows.  Simplicity over speed:
 * m-mer hashes and window minima are computed directly, one position at a time.
 */
#include "scb_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------- */
/* Config and layout                                                          */
/* ------------------------------------------------------------------------- */

static int fail(char* msg, size_t cap, const char* text) {
    if (msg && cap) {
        snprintf(msg, cap, "%s", text);
    }
    return 1;
}

/* config.rs:50-92, config.rs:103-107 (checked_pow2), filter.rs:96-100 */
int ora_validate(const ora_config* c, char* msg, size_t cap) {
    if (c->k == 0 || c->k > 32) return fail(msg, cap, "k must be in 1..=32");
    if (c->m == 0 || c->m > c->k) return fail(msg, cap, "m must be in 1..=k");
    if (c->s == 0 || c->s > c->k || c->s > 32) return fail(msg, cap, "s must be in 1..=k and <= 32");
    if (c->k % 2 == 0) return fail(msg, cap, "canonical SIMD minimizers require odd k");
    if (c->n_hashes == 0) return fail(msg, cap, "n_hashes must be positive");
    if (c->block_slots_exponent >= c->counter_slots_exponent)
        return fail(msg, cap, "block_slots_exponent must be smaller than counter_slots_exponent");
    if (c->threads == 0) return fail(msg, cap, "threads must be positive");
    if (c->queue == 0) return fail(msg, cap, "queue must be positive");
    if (c->counter_bits != 8 && c->counter_bits != 16 && c->counter_bits != 32)
        return fail(msg, cap, "unsupported counter width");
    if (c->counter_slots_exponent >= 64) return fail(msg, cap, "counter_slots_exponent is too large");
    return 0;
}

/* filter.rs:90-116 */
int ora_layout_from_config(const ora_config* c, ora_layout* L) {
    if (ora_validate(c, NULL, 0)) return 1;
    uint64_t counter_slots = 1ULL << c->counter_slots_exponent;
    uint64_t block_slots = 1ULL << c->block_slots_exponent;
    uint64_t nb_blocks = counter_slots / block_slots; /* always a power of two here */
    uint64_t shard_count = nb_blocks < 1024 ? nb_blocks : 1024;
    uint32_t shift = 0;
    while ((1ULL << shift) < shard_count) shift++;
    L->shard_count = shard_count;
    L->subblocks = nb_blocks / shard_count;
    L->block_slots = block_slots;
    L->shard_mask = shard_count - 1;
    L->shard_shift = shift;
    L->block_slots_mask = block_slots - 1;
    L->nb_blocks = nb_blocks;
    L->block_mask = nb_blocks - 1;
    L->n_hashes = c->n_hashes;
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Hashing and packed-sequence primitives                                     */
/* ------------------------------------------------------------------------- */

/* filter.rs:629-635: SplitMix64 finaliser with the golden-ratio increment. */
uint64_t ora_xorshift_u64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ULL;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ULL;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBULL;
    return x ^ (x >> 31);
}

/* packed-seq 4.4.2 (restated): a base's code is bits 1..2 of its ASCII byte, which gives
 * A=0, C=1, T=2, G=3 for both cases; the complement of a code is code ^ 2. */
uint8_t ora_base_code(uint8_t b) { return (uint8_t)((b >> 1) & 3); }

/* api.rs:929-931 */
int ora_is_acgt(uint8_t b) {
    if (b >= 'a' && b <= 'z') b = (uint8_t)(b - 32);
    return b == 'A' || b == 'C' || b == 'G' || b == 'T';
}

/* packed-seq read_kmer (restated): base pos+t sits in bits 2t..2t+1. */
uint64_t ora_read_kmer(const uint8_t* codes, size_t len, size_t pos) {
    uint64_t v = 0;
    for (size_t t = 0; t < len; t++) v |= (uint64_t)codes[pos + t] << (2 * t);
    return v;
}

/* packed-seq read_revcomp_kmer (restated): the reverse complement, same bit order. */
uint64_t ora_read_revcomp_kmer(const uint8_t* codes, size_t len, size_t pos) {
    uint64_t v = 0;
    for (size_t t = 0; t < len; t++) v |= (uint64_t)(codes[pos + len - 1 - t] ^ 2) << (2 * t);
    return v;
}

/* filter.rs:622-627 */
uint64_t ora_canonical_kmer(const uint8_t* codes, size_t len, size_t pos) {
    uint64_t a = ora_read_kmer(codes, len, pos);
    uint64_t b = ora_read_revcomp_kmer(codes, len, pos);
    return a < b ? a : b;
}

/* seq-hash / simd-minimizers canonical ntHash (restated from the ntHash and SimdMinimizers
 * papers): 32-bit ntHash with per-character rotation 7 and the original ntHash seeds (low 32
 * bits, per letter).  The canonical hash is fw + rc (wrapping), so an m-mer and its reverse
 * complement hash equally. */
static const uint32_t NT_SEED[4] = {
    0x95c60474u, /* A (code 0) */
    0x62a02b4cu, /* C (code 1) */
    0x4be24456u, /* T (code 2) */
    0x82572324u, /* G (code 3) */
};
#define NT_ROT 7u

static uint32_t rotl32(uint32_t x, uint32_t r) {
    r &= 31u;
    return r ? (x << r) | (x >> (32u - r)) : x;
}

uint32_t ora_mmer_hash(const uint8_t* codes, size_t pos, size_t m) {
    uint32_t fw = 0, rc = 0;
    for (size_t t = 0; t < m; t++) {
        uint8_t c = codes[pos + t];
        fw ^= rotl32(NT_SEED[c], (uint32_t)(NT_ROT * (m - 1 - t)));
        rc ^= rotl32(NT_SEED[c ^ 2], (uint32_t)(NT_ROT * t));
    }
    return fw + rc;
}

/* simd-minimizers canonical window minimum (restated from the SimdMinimizers paper): the order
 * key of an m-mer is the upper 16 bits of its hash (the lower 16 bits carry the position in the
 * crate's sliding-window minimum).  A window of w = k-m+1 m-mers is read on the forward strand
 * when more than half of its k bases are T or G (code bit 1 set); the forward strand takes the
 * leftmost minimal key, the reverse strand the rightmost.  k is odd, so the rule is
 * strand-symmetric.  Returns the chosen m-mer's position. */
size_t ora_window_minimizer(const uint8_t* codes, const uint32_t* hashes, size_t i, size_t k, size_t m) {
    size_t w = k - m + 1;
    uint32_t best = 0xFFFFFFFFu;
    size_t left = 0, right = 0;
    for (size_t o = 0; o < w; o++) {
        uint32_t key = hashes[i + o] >> 16;
        if (key < best) {
            best = key;
            left = right = o;
        } else if (key == best) {
            right = o;
        }
    }
    size_t tg = 0;
    for (size_t t = 0; t < k; t++) tg += codes[i + t] >> 1;
    return i + ((2 * tg > k) ? left : right);
}

/* filter.rs:608-620: super-k-mer starts (first k-mer index of each run of windows sharing a
 * minimizer position) and the canonical m-mer value of each super-k-mer's minimizer. */
size_t ora_super_kmers(const uint8_t* codes, size_t len, size_t k, size_t m, uint32_t* starts,
                       uint64_t* minimizers) {
    if (len < k) return 0;
    size_t n_mmers = len - m + 1;
    uint32_t* hashes = (uint32_t*)malloc(n_mmers * sizeof(uint32_t));
    for (size_t j = 0; j < n_mmers; j++) hashes[j] = ora_mmer_hash(codes, j, m);
    size_t n = 0, prev = (size_t)-1;
    for (size_t i = 0; i + k <= len; i++) {
        size_t p = ora_window_minimizer(codes, hashes, i, k, m);
        if (i == 0 || p != prev) {
            starts[n] = (uint32_t)i;
            minimizers[n] = ora_canonical_kmer(codes, m, p);
            n++;
        }
        prev = p;
    }
    free(hashes);
    return n;
}

/* ------------------------------------------------------------------------- */
/* Filter                                                                     */
/* ------------------------------------------------------------------------- */

struct ora_filter {
    ora_config cfg;
    ora_layout L;
    uint8_t* table; /* file order: shard-major, then subblock, then slot */
    uint64_t slots;
    uint64_t inserted_kmers, inserted_smers;
};

ora_filter* ora_filter_new(const ora_config* cfg) {
    ora_layout L;
    if (ora_layout_from_config(cfg, &L)) return NULL;
    ora_filter* f = (ora_filter*)calloc(1, sizeof(ora_filter));
    f->cfg = *cfg;
    f->L = L;
    f->slots = 1ULL << cfg->counter_slots_exponent;
    f->table = (uint8_t*)calloc(f->slots, cfg->counter_bits / 8);
    if (!f->table) {
        free(f);
        return NULL;
    }
    return f;
}

void ora_filter_free(ora_filter* f) {
    if (!f) return;
    free(f->table);
    free(f);
}

/* A fresh filter on the existing allocation (SuperCountingBloom::new of the same config): every
 * counter back to zero and the insert totals cleared.  The pages stay mapped, so a caller that
 * times work on a cleared filter times no first-touch page faults. */
void ora_filter_clear(ora_filter* f) {
    memset(f->table, 0, (size_t)ora_filter_table_bytes(f));
    f->inserted_kmers = 0;
    f->inserted_smers = 0;
}

void* ora_filter_table(ora_filter* f) { return f->table; }
uint64_t ora_filter_table_bytes(const ora_filter* f) { return f->slots * (f->cfg.counter_bits / 8); }
uint64_t ora_filter_inserted_kmers(const ora_filter* f) { return f->inserted_kmers; }
uint64_t ora_filter_inserted_smers(const ora_filter* f) { return f->inserted_smers; }
void ora_filter_set_inserted_kmers(ora_filter* f, uint64_t v) { f->inserted_kmers = v; }
const ora_config* ora_filter_config(const ora_filter* f) { return &f->cfg; }

/* filter.rs:217-219 + CounterShard::index (filter.rs:33-37): file-order index of a block's
 * first counter.  Shards are written one after the other (filter.rs:575-580). */
static uint64_t block_base(const ora_layout* L, uint64_t minimizer) {
    uint64_t block = ora_xorshift_u64(minimizer) & L->block_mask;
    uint64_t shard = block & L->shard_mask;
    uint64_t subblock = block >> L->shard_shift;
    return (shard * L->subblocks + subblock) * L->block_slots;
}

static uint64_t counter_get(const ora_filter* f, uint64_t idx) {
    switch (f->cfg.counter_bits) {
        case 8: return f->table[idx];
        case 16: return ((const uint16_t*)f->table)[idx];
        default: return ((const uint32_t*)f->table)[idx];
    }
}

/* counter.rs:21-23, 50-52, 97-99: saturating +1. */
static void counter_increment(ora_filter* f, uint64_t idx) {
    switch (f->cfg.counter_bits) {
        case 8:
            if (f->table[idx] != 0xFFu) f->table[idx]++;
            break;
        case 16: {
            uint16_t* t = (uint16_t*)f->table;
            if (t[idx] != 0xFFFFu) t[idx]++;
            break;
        }
        default: {
            uint32_t* t = (uint32_t*)f->table;
            if (t[idx] != 0xFFFFFFFFu) t[idx]++;
            break;
        }
    }
}

static uint64_t counter_max(const ora_filter* f) {
    return f->cfg.counter_bits == 8 ? 0xFFu : f->cfg.counter_bits == 16 ? 0xFFFFu : 0xFFFFFFFFu;
}

/* filter.rs:199-237 */
uint64_t ora_insert_packed(ora_filter* f, const uint8_t* codes, size_t len) {
    const ora_config* c = &f->cfg;
    if (len < c->k) return 0;
    size_t nw = len - c->k + 1;
    uint32_t* starts = (uint32_t*)malloc(nw * sizeof(uint32_t));
    uint64_t* mins = (uint64_t*)malloc(nw * sizeof(uint64_t));
    size_t n = ora_super_kmers(codes, len, c->k, c->m, starts, mins);
    uint64_t inserted = 0;
    for (size_t i = 0; i < n; i++) {
        size_t start_kmer = starts[i];
        size_t end_kmer = i + 1 < n ? starts[i + 1] : len + 1 - c->k;
        uint64_t base = block_base(&f->L, mins[i]);
        size_t end_smer = end_kmer + (c->k - c->s);
        for (size_t pos = start_kmer; pos < end_smer; pos++) {
            uint64_t smer = ora_canonical_kmer(codes, c->s, pos);
            uint64_t hash = ora_xorshift_u64(smer);
            for (uint64_t h = 0; h < f->L.n_hashes; h++) {
                counter_increment(f, base + (hash & f->L.block_slots_mask));
                hash = ora_xorshift_u64(hash);
            }
            inserted++;
        }
    }
    free(starts);
    free(mins);
    return inserted;
}

/* filter.rs:562-571 */
static uint64_t estimate_smer(const ora_filter* f, uint64_t base, uint64_t smer) {
    uint64_t hash = ora_xorshift_u64(smer);
    uint64_t est = counter_max(f);
    for (uint64_t h = 0; h < f->L.n_hashes; h++) {
        uint64_t v = counter_get(f, base + (hash & f->L.block_slots_mask));
        if (v < est) est = v;
        hash = ora_xorshift_u64(hash);
    }
    return est;
}

/* filter.rs:462-508: s-mer estimates of one super-k-mer, then the sliding minimum over
 * windows of k-s+1 s-mers kept with a monotonic deque of offsets. */
static size_t estimate_super_kmer(const ora_filter* f, uint64_t base, const uint8_t* codes,
                                  size_t start_kmer, size_t end_kmer, uint64_t* out) {
    const ora_config* c = &f->cfg;
    size_t window = c->k - c->s + 1;
    size_t kmer_count = end_kmer - start_kmer;
    size_t smer_count = kmer_count + window - 1;
    uint64_t* est = (uint64_t*)malloc(smer_count * sizeof(uint64_t));
    size_t* dq = (size_t*)malloc(smer_count * sizeof(size_t));
    for (size_t o = 0; o < smer_count; o++) {
        est[o] = estimate_smer(f, base, ora_canonical_kmer(codes, c->s, start_kmer + o));
    }
    size_t head = 0, tail = 0, written = 0; /* deque is dq[head..tail) */
    for (size_t o = 0; o < smer_count; o++) {
        while (tail > head && est[dq[tail - 1]] >= est[o]) tail--;
        dq[tail++] = o;
        while (tail > head && dq[head] + window <= o) head++;
        if (o + 1 >= window) out[written++] = est[dq[head]];
    }
    free(est);
    free(dq);
    return written;
}

/* filter.rs:337-369 */
void ora_estimate_packed(const ora_filter* f, const uint8_t* codes, size_t len, uint64_t* out) {
    const ora_config* c = &f->cfg;
    if (len < c->k) return;
    size_t nw = len - c->k + 1;
    uint32_t* starts = (uint32_t*)malloc(nw * sizeof(uint32_t));
    uint64_t* mins = (uint64_t*)malloc(nw * sizeof(uint64_t));
    size_t n = ora_super_kmers(codes, len, c->k, c->m, starts, mins);
    size_t written = 0;
    for (size_t i = 0; i < n; i++) {
        size_t start_kmer = starts[i];
        size_t end_kmer = i + 1 < n ? starts[i + 1] : len + 1 - c->k;
        written += estimate_super_kmer(f, block_base(&f->L, mins[i]), codes, start_kmer, end_kmer,
                                       out + written);
    }
    free(starts);
    free(mins);
}

/* ------------------------------------------------------------------------- */
/* ASCII sequences: N-splitting and batches (api.rs)                         */
/* ------------------------------------------------------------------------- */

/* Calls fn(start, end) for each maximal ACGT run of seq[0..len) (api.rs:687-704, 812-829). */
typedef void (*run_fn)(void* ctx, const uint8_t* seq, size_t start, size_t end);

static void for_each_run(const uint8_t* seq, size_t len, run_fn fn, void* ctx) {
    size_t run_start = (size_t)-1;
    for (size_t i = 0; i < len; i++) {
        if (ora_is_acgt(seq[i])) {
            if (run_start == (size_t)-1) run_start = i;
        } else if (run_start != (size_t)-1) {
            fn(ctx, seq, run_start, i);
            run_start = (size_t)-1;
        }
    }
    if (run_start != (size_t)-1) fn(ctx, seq, run_start, len);
}

static uint8_t* encode_run(const uint8_t* seq, size_t start, size_t end) {
    uint8_t* codes = (uint8_t*)malloc(end - start + 1);
    for (size_t i = start; i < end; i++) codes[i - start] = ora_base_code(seq[i]);
    return codes;
}

typedef struct {
    ora_filter* f;
    uint64_t kmers, smers;
} insert_ctx;

/* api.rs:708-726 */
static void insert_run(void* vctx, const uint8_t* seq, size_t start, size_t end) {
    insert_ctx* ic = (insert_ctx*)vctx;
    if (end - start < ic->f->cfg.k) return;
    uint8_t* codes = encode_run(seq, start, end);
    ic->kmers += end - start + 1 - ic->f->cfg.k;
    ic->smers += ora_insert_packed(ic->f, codes, end - start);
    free(codes);
}

/* api.rs:123-138 + 676-706 for each sequence of the batch. */
void ora_insert_batch(ora_filter* f, const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                      uint64_t* inserted_kmers, uint64_t* inserted_smers) {
    insert_ctx ic = {f, 0, 0};
    for (uint64_t r = 0; r < n; r++) {
        size_t len = offsets[r + 1] - offsets[r];
        if (len < f->cfg.k) continue;
        for_each_run(seqs + offsets[r], len, insert_run, &ic);
    }
    f->inserted_kmers += ic.kmers;
    f->inserted_smers += ic.smers;
    if (inserted_kmers) *inserted_kmers = ic.kmers;
    if (inserted_smers) *inserted_smers = ic.smers;
}

typedef struct {
    const ora_filter* f;
    uint64_t* out;
    uint8_t* valid;
} query_ctx;

/* api.rs:833-853 */
static void query_run(void* vctx, const uint8_t* seq, size_t start, size_t end) {
    query_ctx* qc = (query_ctx*)vctx;
    if (end - start < qc->f->cfg.k) return;
    uint8_t* codes = encode_run(seq, start, end);
    size_t nw = end - start + 1 - qc->f->cfg.k;
    ora_estimate_packed(qc->f, codes, end - start, qc->out + start);
    memset(qc->valid + start, 1, nw);
    free(codes);
}

static uint64_t n_windows(uint64_t len, uint64_t k) { return len >= k ? len + 1 - k : 0; }

/* api.rs:799-831 for each sequence; outputs concatenated per sequence. */
void ora_query_batch(const ora_filter* f, const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                     uint64_t* out, uint8_t* valid) {
    uint64_t w = 0;
    for (uint64_t r = 0; r < n; r++) {
        size_t len = offsets[r + 1] - offsets[r];
        uint64_t nw = n_windows(len, f->cfg.k);
        if (nw == 0) continue;
        memset(out + w, 0, nw * sizeof(uint64_t));
        memset(valid + w, 0, nw);
        query_ctx qc = {f, out + w, valid + w};
        for_each_run(seqs + offsets[r], len, query_run, &qc);
        w += nw;
    }
}

/* api.rs:273-327 (the per-worker loop at api.rs:283-296, merged). */
void ora_query_report(const ora_filter* f, const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                      ora_report* rep) {
    memset(rep, 0, sizeof(*rep));
    for (uint64_t r = 0; r < n; r++) {
        size_t len = offsets[r + 1] - offsets[r];
        uint64_t nw = n_windows(len, f->cfg.k);
        rep->records_processed++;
        if (nw == 0) continue;
        uint64_t* out = (uint64_t*)calloc(nw, sizeof(uint64_t));
        uint8_t* valid = (uint8_t*)calloc(nw, 1);
        query_ctx qc = {f, out, valid};
        for_each_run(seqs + offsets[r], len, query_run, &qc);
        rep->total_windows += nw;
        for (uint64_t i = 0; i < nw; i++) {
            if (!valid[i]) continue;
            rep->valid_kmers++;
            if (out[i] > 0) rep->positive_estimates++;
            rep->estimate_checksum += out[i];
        }
        free(out);
        free(valid);
    }
}

/* ------------------------------------------------------------------------- */
/* Distinct-k-mer spectrum and counter histogram                              */
/* ------------------------------------------------------------------------- */

/* Open-addressing map u64 -> u64 (keys never equal EMPTY: a canonical k-mer of k <= 32 is
 * never all-ones, because its reverse complement would be smaller). */
#define EMPTY_KEY 0xFFFFFFFFFFFFFFFFULL
typedef struct {
    uint64_t* keys;
    uint64_t* vals;
    uint64_t cap, size;
} u64map;

static void map_init(u64map* m, uint64_t cap) {
    m->cap = 16;
    while (m->cap < cap * 2) m->cap <<= 1;
    m->keys = (uint64_t*)malloc(m->cap * sizeof(uint64_t));
    m->vals = (uint64_t*)malloc(m->cap * sizeof(uint64_t));
    memset(m->keys, 0xFF, m->cap * sizeof(uint64_t));
    m->size = 0;
}

static void map_free(u64map* m) {
    free(m->keys);
    free(m->vals);
}

static void map_grow(u64map* m);

/* Returns pointer to the value; *inserted says whether the key was new. */
static uint64_t* map_entry(u64map* m, uint64_t key, int* inserted) {
    if ((m->size + 1) * 2 > m->cap) map_grow(m);
    uint64_t i = ora_xorshift_u64(key) & (m->cap - 1);
    while (m->keys[i] != EMPTY_KEY) {
        if (m->keys[i] == key) {
            *inserted = 0;
            return &m->vals[i];
        }
        i = (i + 1) & (m->cap - 1);
    }
    m->keys[i] = key;
    m->vals[i] = 0;
    m->size++;
    *inserted = 1;
    return &m->vals[i];
}

static void map_grow(u64map* m) {
    u64map bigger;
    map_init(&bigger, m->cap);
    for (uint64_t i = 0; i < m->cap; i++) {
        if (m->keys[i] == EMPTY_KEY) continue;
        int ins;
        *map_entry(&bigger, m->keys[i], &ins) = m->vals[i];
    }
    map_free(m);
    *m = bigger;
}

typedef struct {
    const ora_filter* f;
    u64map* map;
    uint64_t queried, mismatches;
} spectrum_ctx;

/* filter.rs:302-335 + 407-460 on one run: key = canonical k-mer, value = estimate, first
 * insertion wins (filter.rs:454). */
static void spectrum_run(void* vctx, const uint8_t* seq, size_t start, size_t end) {
    spectrum_ctx* sc = (spectrum_ctx*)vctx;
    const ora_config* c = &sc->f->cfg;
    if (end - start < c->k) return;
    uint8_t* codes = encode_run(seq, start, end);
    size_t nw = end - start + 1 - c->k;
    uint64_t* est = (uint64_t*)malloc(nw * sizeof(uint64_t));
    ora_estimate_packed(sc->f, codes, end - start, est);
    for (size_t i = 0; i < nw; i++) {
        int inserted;
        uint64_t* v = map_entry(sc->map, ora_canonical_kmer(codes, c->k, i), &inserted);
        if (inserted) {
            *v = est[i];
        } else if (*v != est[i]) {
            sc->mismatches++;
        }
    }
    sc->queried += nw;
    free(est);
    free(codes);
}

static int cmp_u64pair(const void* a, const void* b) {
    const uint64_t* x = (const uint64_t*)a;
    const uint64_t* y = (const uint64_t*)b;
    return x[0] < y[0] ? -1 : x[0] > y[0] ? 1 : 0;
}

/* Turns a value->count map into rows sorted by value (fastx.rs:402-410, filter.rs:190-192). */
static uint64_t emit_rows(u64map* hist, uint64_t* values, uint64_t* counts, uint64_t cap) {
    uint64_t rows = hist->size;
    uint64_t* pairs = (uint64_t*)malloc((rows ? rows : 1) * 2 * sizeof(uint64_t));
    uint64_t r = 0;
    for (uint64_t i = 0; i < hist->cap; i++) {
        if (hist->keys[i] == EMPTY_KEY) continue;
        pairs[2 * r] = hist->keys[i];
        pairs[2 * r + 1] = hist->vals[i];
        r++;
    }
    qsort(pairs, rows, 2 * sizeof(uint64_t), cmp_u64pair);
    if (values && counts && cap >= rows) {
        for (uint64_t i = 0; i < rows; i++) {
            values[i] = pairs[2 * i];
            counts[i] = pairs[2 * i + 1];
        }
    }
    free(pairs);
    return rows;
}

/* The spectrum path splits records at non-ACGT bytes and keeps chunks of length >= k
 * (fastx.rs:14-19, 231-243); with the API's is_acgt rule this is the same run set. */
uint64_t ora_spectrum_distinct(const ora_filter* f, const uint8_t* seqs, const uint64_t* offsets,
                               uint64_t n, uint64_t* values, uint64_t* counts, uint64_t cap,
                               uint64_t* distinct_keys, uint64_t* queried_kmers, uint64_t* mismatches) {
    u64map map;
    map_init(&map, 1024);
    spectrum_ctx sc = {f, &map, 0, 0};
    for (uint64_t r = 0; r < n; r++) {
        size_t len = offsets[r + 1] - offsets[r];
        for_each_run(seqs + offsets[r], len, spectrum_run, &sc);
    }
    u64map hist;
    map_init(&hist, 1024);
    for (uint64_t i = 0; i < map.cap; i++) {
        if (map.keys[i] == EMPTY_KEY) continue;
        int ins;
        (*map_entry(&hist, map.vals[i], &ins))++;
    }
    uint64_t rows = emit_rows(&hist, values, counts, cap);
    if (distinct_keys) *distinct_keys = map.size;
    if (queried_kmers) *queried_kmers = sc.queried;
    if (mismatches) *mismatches = sc.mismatches;
    map_free(&hist);
    map_free(&map);
    return rows;
}

/* filter.rs:50-54 + 267-275 */
uint64_t ora_counter_histogram(const ora_filter* f, uint64_t* values, uint64_t* counts, uint64_t cap) {
    u64map hist;
    map_init(&hist, 1024);
    for (uint64_t i = 0; i < f->slots; i++) {
        int ins;
        (*map_entry(&hist, counter_get(f, i), &ins))++;
    }
    uint64_t rows = emit_rows(&hist, values, counts, cap);
    map_free(&hist);
    return rows;
}

/* ------------------------------------------------------------------------- */
/* .scb serialization (api.rs:28-29, 388-608; counter.rs LE slices)          */
/* ------------------------------------------------------------------------- */

static const uint8_t INDEX_MAGIC[8] = {'S', 'C', 'B', 'I', 'D', 'X', 0, 0};
#define INDEX_FORMAT_VERSION 2u

static void put_u64(FILE* fp, uint64_t v) {
    uint8_t b[8];
    for (int i = 0; i < 8; i++) b[i] = (uint8_t)(v >> (8 * i));
    fwrite(b, 1, 8, fp);
}
static void put_u32(FILE* fp, uint32_t v) {
    uint8_t b[4];
    for (int i = 0; i < 4; i++) b[i] = (uint8_t)(v >> (8 * i));
    fwrite(b, 1, 4, fp);
}
static void put_u8(FILE* fp, uint8_t v) { fwrite(&v, 1, 1, fp); }

/* api.rs:388-414 with write_config (466-480) and write_layout (515-529). */
int ora_save(const ora_filter* f, const char* path) {
    FILE* fp = fopen(path, "wb");
    if (!fp) return 1;
    fwrite(INDEX_MAGIC, 1, 8, fp);
    put_u32(fp, INDEX_FORMAT_VERSION);
    put_u64(fp, f->cfg.k);
    put_u64(fp, f->cfg.m);
    put_u64(fp, f->cfg.s);
    put_u64(fp, f->cfg.n_hashes);
    put_u8(fp, f->cfg.counter_bits);
    put_u8(fp, f->cfg.counter_slots_exponent);
    put_u8(fp, f->cfg.block_slots_exponent);
    put_u64(fp, f->cfg.threads);
    put_u64(fp, f->cfg.queue);
    put_u64(fp, f->inserted_kmers);
    put_u64(fp, f->L.shard_count);
    put_u64(fp, f->L.subblocks);
    put_u64(fp, f->L.block_slots);
    put_u64(fp, f->L.shard_mask);
    put_u32(fp, f->L.shard_shift);
    put_u64(fp, f->L.block_slots_mask);
    put_u64(fp, f->L.nb_blocks);
    put_u64(fp, f->L.block_mask);
    put_u64(fp, f->L.n_hashes);
    /* filter.rs:575-580: shards in order; the table is already in that order, LE. */
    size_t bytes = (size_t)ora_filter_table_bytes(f);
    int bad = fwrite(f->table, 1, bytes, fp) != bytes;
    bad |= fclose(fp) != 0;
    return bad;
}

static int get_bytes(FILE* fp, void* dst, size_t n) { return fread(dst, 1, n, fp) == n ? 0 : 1; }
static int get_u64(FILE* fp, uint64_t* v) {
    uint8_t b[8];
    if (get_bytes(fp, b, 8)) return 1;
    *v = 0;
    for (int i = 0; i < 8; i++) *v |= (uint64_t)b[i] << (8 * i);
    return 0;
}
static int get_u32(FILE* fp, uint32_t* v) {
    uint8_t b[4];
    if (get_bytes(fp, b, 4)) return 1;
    *v = 0;
    for (int i = 0; i < 4; i++) *v |= (uint32_t)b[i] << (8 * i);
    return 0;
}

/* api.rs:416-464 + 599-608 */
ora_filter* ora_load(const char* path, char* msg, size_t cap) {
    FILE* fp = fopen(path, "rb");
    if (!fp) {
        fail(msg, cap, "io: cannot open");
        return NULL;
    }
    uint8_t magic[8];
    uint32_t version = 0;
    ora_config c;
    memset(&c, 0, sizeof(c));
    uint64_t inserted = 0;
    ora_layout stored;
    memset(&stored, 0, sizeof(stored));
    ora_filter* f = NULL;
    if (get_bytes(fp, magic, 8)) {
        fail(msg, cap, "io: short read");
        goto done;
    }
    if (memcmp(magic, INDEX_MAGIC, 8) != 0) {
        fail(msg, cap, "invalid index format: bad SuperCountingBloom index magic");
        goto done;
    }
    if (get_u32(fp, &version)) {
        fail(msg, cap, "io: short read");
        goto done;
    }
    if (version != INDEX_FORMAT_VERSION) {
        fail(msg, cap, "invalid index format: unsupported index format version");
        goto done;
    }
    if (get_u64(fp, &c.k) || get_u64(fp, &c.m) || get_u64(fp, &c.s) || get_u64(fp, &c.n_hashes) ||
        get_bytes(fp, &c.counter_bits, 1)) {
        fail(msg, cap, "io: short read");
        goto done;
    }
    if (c.counter_bits != 8 && c.counter_bits != 16 && c.counter_bits != 32) {
        fail(msg, cap, "invalid index format: unsupported counter width");
        goto done;
    }
    if (get_bytes(fp, &c.counter_slots_exponent, 1) || get_bytes(fp, &c.block_slots_exponent, 1) ||
        get_u64(fp, &c.threads) || get_u64(fp, &c.queue) || get_u64(fp, &inserted)) {
        fail(msg, cap, "io: short read");
        goto done;
    }
    if (ora_validate(&c, msg, cap)) goto done;
    if (get_u64(fp, &stored.shard_count) || get_u64(fp, &stored.subblocks) ||
        get_u64(fp, &stored.block_slots) || get_u64(fp, &stored.shard_mask) ||
        get_u32(fp, &stored.shard_shift) || get_u64(fp, &stored.block_slots_mask) ||
        get_u64(fp, &stored.nb_blocks) || get_u64(fp, &stored.block_mask) ||
        get_u64(fp, &stored.n_hashes)) {
        fail(msg, cap, "io: short read");
        goto done;
    }
    {
        ora_layout expected;
        ora_layout_from_config(&c, &expected);
        if (stored.shard_count != expected.shard_count || stored.subblocks != expected.subblocks ||
            stored.block_slots != expected.block_slots || stored.shard_mask != expected.shard_mask ||
            stored.shard_shift != expected.shard_shift ||
            stored.block_slots_mask != expected.block_slots_mask ||
            stored.nb_blocks != expected.nb_blocks || stored.block_mask != expected.block_mask ||
            stored.n_hashes != expected.n_hashes) {
            fail(msg, cap, "invalid index format: stored filter layout does not match config");
            goto done;
        }
    }
    f = ora_filter_new(&c);
    if (!f) {
        fail(msg, cap, "internal state: allocation failed");
        goto done;
    }
    if (get_bytes(fp, f->table, (size_t)ora_filter_table_bytes(f))) {
        fail(msg, cap, "io: short read");
        ora_filter_free(f);
        f = NULL;
        goto done;
    }
    {
        uint8_t extra;
        if (fread(&extra, 1, 1, fp) == 1) {
            fail(msg, cap, "invalid index format: trailing bytes after serialized index");
            ora_filter_free(f);
            f = NULL;
            goto done;
        }
    }
    f->inserted_kmers = inserted;
done:
    fclose(fp);
    return f;
}

/* ------------------------------------------------------------------------- */
/* Batch-level instrumentation                                                */
/* ------------------------------------------------------------------------- */

typedef struct {
    uint64_t k, m;
    uint64_t base_offset;
    uint32_t* out;
} wm_ctx;

static void window_minimizer_run(void* vctx, const uint8_t* seq, size_t start, size_t end) {
    wm_ctx* wc = (wm_ctx*)vctx;
    size_t len = end - start;
    if (len < wc->k) return;
    uint8_t* codes = encode_run(seq, start, end);
    size_t n_mmers = len - wc->m + 1;
    uint32_t* hashes = (uint32_t*)malloc(n_mmers * sizeof(uint32_t));
    for (size_t j = 0; j < n_mmers; j++) hashes[j] = ora_mmer_hash(codes, j, wc->m);
    for (size_t i = 0; i + wc->k <= len; i++) {
        size_t p = ora_window_minimizer(codes, hashes, i, wc->k, wc->m);
        wc->out[wc->base_offset + start + i] = (uint32_t)(wc->base_offset + start + p);
    }
    free(hashes);
    free(codes);
}

void ora_batch_window_minimizers(const uint8_t* seqs, const uint64_t* offsets, uint64_t n,
                                 uint64_t k, uint64_t m, uint32_t* out) {
    uint64_t total = offsets[n];
    for (uint64_t i = 0; i < total; i++) out[i] = 0xFFFFFFFFu;
    for (uint64_t r = 0; r < n; r++) {
        wm_ctx wc = {k, m, offsets[r], out};
        for_each_run(seqs + offsets[r], offsets[r + 1] - offsets[r], window_minimizer_run, &wc);
    }
}

typedef struct {
    const ora_config* cfg;
    const ora_layout* L;
    uint64_t sk, smers, sectors;
} sector_ctx;

static void sector_run(void* vctx, const uint8_t* seq, size_t start, size_t end) {
    sector_ctx* sc = (sector_ctx*)vctx;
    const ora_config* c = sc->cfg;
    size_t len = end - start;
    if (len < c->k) return;
    uint8_t* codes = encode_run(seq, start, end);
    size_t nw = len - c->k + 1;
    uint32_t* starts = (uint32_t*)malloc(nw * sizeof(uint32_t));
    uint64_t* mins = (uint64_t*)malloc(nw * sizeof(uint64_t));
    size_t n = ora_super_kmers(codes, len, c->k, c->m, starts, mins);
    uint64_t bytes_per_counter = c->counter_bits / 8;
    uint64_t block_bytes = sc->L->block_slots * bytes_per_counter;
    uint64_t n_sectors = (block_bytes + 31) / 32;
    uint8_t* seen = (uint8_t*)calloc(n_sectors, 1);
    for (size_t i = 0; i < n; i++) {
        size_t s0 = starts[i];
        size_t e0 = i + 1 < n ? starts[i + 1] : len + 1 - c->k;
        memset(seen, 0, n_sectors);
        uint64_t distinct = 0;
        for (size_t pos = s0; pos < e0 + (c->k - c->s); pos++) {
            uint64_t hash = ora_xorshift_u64(ora_canonical_kmer(codes, c->s, pos));
            for (uint64_t h = 0; h < c->n_hashes; h++) {
                uint64_t sec = ((hash & sc->L->block_slots_mask) * bytes_per_counter) / 32;
                if (!seen[sec]) {
                    seen[sec] = 1;
                    distinct++;
                }
                hash = ora_xorshift_u64(hash);
            }
            sc->smers++;
        }
        sc->sectors += distinct;
    }
    sc->sk += n;
    free(seen);
    free(starts);
    free(mins);
    free(codes);
}

void ora_batch_sector_stats(const ora_config* cfg, const uint8_t* seqs, const uint64_t* offsets,
                            uint64_t n, uint64_t* super_kmers, uint64_t* smers, uint64_t* sectors) {
    ora_layout L;
    ora_layout_from_config(cfg, &L);
    sector_ctx sc = {cfg, &L, 0, 0, 0};
    for (uint64_t r = 0; r < n; r++) {
        size_t len = offsets[r + 1] - offsets[r];
        if (len < cfg->k) continue;
        for_each_run(seqs + offsets[r], len, sector_run, &sc);
    }
    *super_kmers = sc.sk;
    *smers = sc.smers;
    *sectors = sc.sectors;
}
