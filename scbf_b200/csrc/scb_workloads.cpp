// Seeded synthetic sequencing workloads (host, multi-threaded).  Every read draws from its own
// random stream derived from (seed, read index), so the output does not depend on the thread
// count.  Bases are written as ASCII A/C/G/T/N; offsets are n+1 uint64.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace {

struct Rng {  // xoshiro256** seeded through splitmix64
    uint64_t s[4];
    static uint64_t splitmix(uint64_t& x) {
        uint64_t z = (x += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    Rng(uint64_t seed, uint64_t stream) {
        uint64_t x = seed * 0xD1B54A32D192ED03ull + stream * 0x9E3779B97F4A7C15ull + 0x632BE59BD9B4E019ull;
        for (auto& v : s) v = splitmix(x);
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {
        const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    double uniform() { return (next() >> 11) * 0x1.0p-53; }
    uint64_t below(uint64_t n) { return n ? (uint64_t)(((unsigned __int128)next() * n) >> 64) : 0; }
    // number of failures before the next success of a Bernoulli(p) sequence
    uint64_t geometric(double p) {
        if (p <= 0) return UINT64_MAX;
        if (p >= 1) return 0;
        const double u = 1.0 - uniform();
        return (uint64_t)std::floor(std::log(u) / std::log1p(-p));
    }
    double normal() {
        const double u1 = 1.0 - uniform(), u2 = uniform();
        return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
    }
};

const char kLetters[4] = {'A', 'C', 'G', 'T'};  // letter index; complement = 3 - index

template <typename F>
void parallel_for(uint64_t n, F&& fn) {
    unsigned t = std::max(1u, std::thread::hardware_concurrency());
    t = (unsigned)std::min<uint64_t>(t, std::max<uint64_t>(1, n / 1024));
    std::vector<std::thread> th;
    for (unsigned i = 0; i < t; i++) {
        th.emplace_back([&, i] {
            for (uint64_t j = n * i / t; j < n * (i + 1) / t; j++) fn(j);
        });
    }
    for (auto& x : th) x.join();
}

// In-place substitutions (each base w.p. rate -> one of the 3 other letters) and N runs
// (runs start w.p. n_rate / mean_run per base, length U{1..max_run}, clipped at the read end).
void mutate(Rng& r, uint8_t* idx, uint64_t len, double sub_rate) {
    for (uint64_t p = r.geometric(sub_rate); p < len; p += 1 + r.geometric(sub_rate)) {
        idx[p] = (uint8_t)((idx[p] + 1 + r.below(3)) & 3);
    }
}

void n_runs(Rng& r, char* out, uint64_t len, double n_rate, int max_run) {
    if (n_rate <= 0) return;
    const double start_p = n_rate / ((1.0 + max_run) / 2.0);
    for (uint64_t p = r.geometric(start_p); p < len; p += 1 + r.geometric(start_p)) {
        const uint64_t L = 1 + r.below((uint64_t)max_run);
        for (uint64_t q = p; q < std::min(len, p + L); q++) out[q] = 'N';
    }
}

}  // namespace

extern "C" {

// Uniform random genome as letter indices 0..3.
void scbw_random_genome(uint8_t* g, uint64_t len, uint64_t seed) {
    const uint64_t blocks = (len + 65535) / 65536;
    parallel_for(blocks, [&](uint64_t b) {
        Rng r(seed, 0xA11CE + b);
        const uint64_t a = b * 65536, e = std::min(len, a + 65536);
        for (uint64_t i = a; i < e; i += 32) {
            uint64_t x = r.next();
            for (uint64_t j = i; j < std::min(e, i + 32); j++, x >>= 2) g[j] = (uint8_t)(x & 3);
        }
    });
}

// Fixed-length reads, uniform start, 50/50 strand, substitutions, N runs.
void scbw_short_reads(const uint8_t* g, uint64_t glen, uint64_t n_reads, uint64_t read_len, uint64_t seed,
                      double sub_rate, double n_rate, int n_max_run, uint8_t* out, uint64_t* offsets) {
    parallel_for(n_reads, [&](uint64_t i) {
        Rng r(seed, i);
        uint8_t buf[4096];
        std::vector<uint8_t> big;
        uint8_t* idx = buf;
        if (read_len > sizeof(buf)) {
            big.resize(read_len);
            idx = big.data();
        }
        const uint64_t st = r.below(glen - read_len + 1);
        const bool rev = r.next() & 1;
        for (uint64_t j = 0; j < read_len; j++) idx[j] = rev ? (uint8_t)(3 - g[st + read_len - 1 - j]) : g[st + j];
        mutate(r, idx, read_len, sub_rate);
        char* o = reinterpret_cast<char*>(out + i * read_len);
        for (uint64_t j = 0; j < read_len; j++) o[j] = kLetters[idx[j]];
        n_runs(r, o, read_len, n_rate, n_max_run);
        offsets[i + 1] = (i + 1) * read_len;
    });
    offsets[0] = 0;
}

// Log-normal read lengths (median, sigma) clipped to [lo, hi]; fills lens[n].
void scbw_lognormal_lengths(uint64_t n, double median, double sigma, uint64_t lo, uint64_t hi, uint64_t seed,
                            uint64_t* lens) {
    Rng r(seed, 0x10C);
    for (uint64_t i = 0; i < n; i++) {
        const double v = std::exp(std::log(median) + sigma * r.normal());
        lens[i] = (uint64_t)std::min<double>((double)hi, std::max<double>((double)lo, v));
    }
}

// Reads of given template lengths with substitution / insertion / deletion rates; read i is
// written at out[offsets[i]] (offsets precomputed by the caller from out_lens, which this
// function fills in a first pass when offsets == nullptr).
void scbw_noisy_reads(const uint8_t* g, uint64_t glen, uint64_t n, const uint64_t* tlens, uint64_t seed,
                      double sub, double ins, double del, uint64_t* out_lens, const uint64_t* offsets, uint8_t* out) {
    parallel_for(n, [&](uint64_t i) {
        Rng r(seed, (1ull << 40) + i);
        const uint64_t L = std::min(tlens[i], glen);
        const uint64_t st = r.below(glen - L + 1);
        const bool rev = r.next() & 1;
        char* o = out && offsets ? reinterpret_cast<char*>(out + offsets[i]) : nullptr;
        uint64_t w = 0;
        for (uint64_t j = 0; j < L; j++) {
            const uint8_t b = rev ? (uint8_t)(3 - g[st + L - 1 - j]) : g[st + j];
            const double u = r.uniform();
            if (u < del) continue;
            if (u < del + ins) {
                const uint64_t extra = r.below(4);  // drawn in both passes
                if (o) {
                    o[w] = kLetters[b];
                    o[w + 1] = kLetters[extra];
                }
                w += 2;
                continue;
            }
            uint8_t c = b;
            if (u < del + ins + sub) c = (uint8_t)((b + 1 + r.below(3)) & 3);
            if (o) o[w] = kLetters[c];
            w++;
        }
        if (out_lens) out_lens[i] = w;
    });
}

// Overwrites copies of repeat families into the genome (sequentially, deterministic).
void scbw_plant_repeats(uint8_t* g, uint64_t glen, uint64_t n_families, uint64_t fam_min, uint64_t fam_max,
                        double copy_lo, double copy_hi, double repeat_frac, double divergence, uint64_t seed) {
    Rng r(seed, 0xBEEF);
    std::vector<uint64_t> flen(n_families);
    std::vector<double> copies(n_families);
    double total = 0;
    for (uint64_t f = 0; f < n_families; f++) {
        flen[f] = fam_min + r.below(fam_max - fam_min + 1);
        copies[f] = std::exp(std::log(copy_lo) + r.uniform() * (std::log(copy_hi) - std::log(copy_lo)));
        total += flen[f] * copies[f];
    }
    const double scale = repeat_frac * (double)glen / total;
    std::vector<uint8_t> fam, cp;
    for (uint64_t f = 0; f < n_families; f++) {
        fam.resize(flen[f]);
        for (auto& b : fam) b = (uint8_t)r.below(4);
        const uint64_t nc = std::max<uint64_t>(1, (uint64_t)std::llround(copies[f] * scale));
        for (uint64_t c = 0; c < nc && glen > fam.size(); c++) {
            const uint64_t pos = r.below(glen - fam.size());
            cp = fam;
            mutate(r, cp.data(), cp.size(), divergence);
            std::memcpy(g + pos, cp.data(), cp.size());
        }
    }
}

// dst read i = src read order[i]; dst_offsets must already hold the prefix sums of the
// permuted lengths.
void scbw_gather_reads(const uint8_t* src, const uint64_t* src_offsets, const uint64_t* order, uint64_t n,
                       uint8_t* dst, const uint64_t* dst_offsets) {
    parallel_for(n, [&](uint64_t i) {
        const uint64_t j = order[i];
        std::memcpy(dst + dst_offsets[i], src + src_offsets[j], src_offsets[j + 1] - src_offsets[j]);
    });
}

// Letter indices -> ASCII.
void scbw_to_ascii(const uint8_t* idx, uint64_t n, uint8_t* out) {
    parallel_for((n + 65535) / 65536, [&](uint64_t b) {
        for (uint64_t i = b * 65536; i < std::min(n, (b + 1) * 65536); i++) out[i] = (uint8_t)kLetters[idx[i]];
    });
}

}  // extern "C"
