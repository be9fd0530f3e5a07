// Host-side 2-bit packing of reads (kernel (a)'s layout, computed on the CPU) so that a host
// entry point copies 3 bits per base to the device instead of the 8-bit letters.
//
// Layout (the same as the device packing kernel's):
//   codes: 16 bases per 32-bit word, base g at bits 2 * (g % 16) of word g / 16, code = (byte >> 1) & 3
//   valid: 32 bases per 32-bit word, base g at bit g % 32 of word g / 32, set for A/C/G/T in either case
// followed by kPadWords zero words in both arrays.  Bytes past n inside the last 32-byte group
// count as zero bytes (code 0, not valid), as on the device.
//
// Each 32-byte group is independent, so threads take contiguous ranges of groups.  With AVX2 a
// group is 10 vector operations: the validity bits come out of one movemask, the codes out of two
// multiply-add steps that merge 2-bit fields (bytes -> 4-bit -> 8-bit) and a byte gather.

#include <immintrin.h>

#include <algorithm>
#include <cstdint>
#include <cstring>
#include <thread>
#include <vector>

namespace scb {

constexpr uint64_t kHostPadWords = 16;  // = kPadWords of the kernels

namespace {

// Scalar form of one group of up to 32 bytes.
void pack_group_scalar(const uint8_t* p, uint64_t len, uint32_t* c0, uint32_t* c1, uint32_t* vm) {
    uint64_t codes = 0;
    uint32_t valid = 0;
    for (uint64_t j = 0; j < len; j++) {
        const uint8_t b = p[j];
        const uint8_t u = b & 0xDF;
        codes |= (uint64_t)((b >> 1) & 3u) << (2 * j);
        valid |= (uint32_t)(u == 'A' || u == 'C' || u == 'G' || u == 'T') << j;
    }
    *c0 = (uint32_t)codes;
    *c1 = (uint32_t)(codes >> 32);
    *vm = valid;
}

__attribute__((target("avx2"))) void pack_range_avx2(const uint8_t* ascii, uint64_t n, uint64_t g0, uint64_t g1,
                                                      uint32_t* codes, uint32_t* valid) {
    const __m256i upper = _mm256_set1_epi8((char)0xDF);
    const __m256i A = _mm256_set1_epi8('A'), Cc = _mm256_set1_epi8('C'), G = _mm256_set1_epi8('G'),
                  T = _mm256_set1_epi8('T');
    const __m256i three = _mm256_set1_epi8(3);
    const __m256i pair = _mm256_set1_epi16(0x0401);      // byte0 * 1 + byte1 * 4
    const __m256i quad = _mm256_set1_epi32(0x00100001);  // half0 * 1 + half1 * 16
    // low byte of each 32-bit lane to the lane's first four bytes, per 128-bit half
    const __m256i gather = _mm256_setr_epi8(0, 4, 8, 12, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, 0, 4, 8, 12,
                                            -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1, -1);
    const uint64_t full = n / 32;  // groups with all 32 bytes
    for (uint64_t gi = g0; gi < g1; gi++) {
        if (gi >= full) {
            const uint64_t len = gi * 32 < n ? n - gi * 32 : 0;
            pack_group_scalar(ascii + gi * 32, len, codes + 2 * gi, codes + 2 * gi + 1, valid + gi);
            continue;
        }
        const __m256i x = _mm256_loadu_si256(reinterpret_cast<const __m256i*>(ascii + gi * 32));
        const __m256i u = _mm256_and_si256(x, upper);
        const __m256i ok = _mm256_or_si256(_mm256_or_si256(_mm256_cmpeq_epi8(u, A), _mm256_cmpeq_epi8(u, Cc)),
                                           _mm256_or_si256(_mm256_cmpeq_epi8(u, G), _mm256_cmpeq_epi8(u, T)));
        valid[gi] = (uint32_t)_mm256_movemask_epi8(ok);
        const __m256i c = _mm256_and_si256(_mm256_srli_epi16(x, 1), three);  // (byte >> 1) & 3 per byte
        const __m256i c4 = _mm256_maddubs_epi16(c, pair);                     // 2 bases per 16-bit lane
        const __m256i c8 = _mm256_madd_epi16(c4, quad);                       // 4 bases per 32-bit lane
        const __m256i b = _mm256_shuffle_epi8(c8, gather);                    // 4 bytes per half
        const uint32_t lo = (uint32_t)_mm256_extract_epi32(b, 0), hi = (uint32_t)_mm256_extract_epi32(b, 4);
        codes[2 * gi] = lo;
        codes[2 * gi + 1] = hi;
    }
}

void pack_range_scalar(const uint8_t* ascii, uint64_t n, uint64_t g0, uint64_t g1, uint32_t* codes, uint32_t* valid) {
    for (uint64_t gi = g0; gi < g1; gi++) {
        const uint64_t len = gi * 32 < n ? std::min<uint64_t>(32, n - gi * 32) : 0;
        pack_group_scalar(ascii + gi * 32, len, codes + 2 * gi, codes + 2 * gi + 1, valid + gi);
    }
}

bool have_avx2() {
    static const bool yes = __builtin_cpu_supports("avx2");
    return yes;
}

}  // namespace

// Packs n bytes into codes (2 * groups + kHostPadWords words) and valid (groups + kHostPadWords
// words), groups = ceil(n / 32), on up to `threads` host threads.
void host_pack(const uint8_t* ascii, uint64_t n, uint32_t* codes, uint32_t* valid, unsigned threads) {
    const uint64_t groups = (n + 31) / 32;
    auto range = [&](uint64_t g0, uint64_t g1) {
        if (have_avx2()) {
            pack_range_avx2(ascii, n, g0, g1, codes, valid);
        } else {
            pack_range_scalar(ascii, n, g0, g1, codes, valid);
        }
    };
    const uint64_t parts = std::max<uint64_t>(1, std::min<uint64_t>(threads, groups / (1 << 14)));
    if (parts <= 1) {
        range(0, groups);
    } else {
        std::vector<std::thread> th;
        for (uint64_t t = 0; t < parts; t++) th.emplace_back(range, groups * t / parts, groups * (t + 1) / parts);
        for (auto& x : th) x.join();
    }
    std::memset(codes + 2 * groups, 0, kHostPadWords * 4);
    std::memset(valid + groups, 0, kHostPadWords * 4);
}

}  // namespace scb

// Test hook (not in include/scb.h): the packing of n bytes, for the layout tests.
extern "C" void scb_internal_host_pack(const uint8_t* ascii, uint64_t n, uint32_t* codes, uint32_t* valid,
                                       unsigned threads) {
    scb::host_pack(ascii, n, codes, valid, threads);
}
