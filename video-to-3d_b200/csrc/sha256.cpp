// SHA-256 (FIPS 180-4) on the host: the digest of ContentHash::of_bytes
// (crates/video-to-3d-core/src/scene_project.rs:463-465), which identifies a
// stage artifact by the SHA-256 of its JSON document.  A single message
// hashes block after block, so this runs on the host while the document
// streams back from the device.  Processors with the SHA extensions run the
// compression through sha256rnds2 / sha256msg1 / sha256msg2; others (or
// V3D_SHA256_PORTABLE=1) through the portable rounds.
#include <cpuid.h>
#include <immintrin.h>

#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "../../include/v3d_dense.h"
#include "host.hpp"

namespace v3d {
namespace {

// Round constants and initial hash value from their definitions: the first
// 32 bits of the fractional parts of the cube roots of the first 64 primes,
// and of the square roots of the first 8, by exact integer roots of
// p * 2^96 and p * 2^64.
struct Constants {
    uint32_t k[64];
    uint32_t h0[8];
};

using u128 = unsigned __int128;

uint64_t iroot(u128 x, int degree) {
    uint64_t lo = 0, hi = uint64_t(1) << 40;  // roots here stay below 2^36
    while (hi - lo > 1) {
        const uint64_t mid = lo + (hi - lo) / 2;
        u128 p = mid;
        for (int i = 1; i < degree; ++i) p *= mid;
        if (p <= x) lo = mid;
        else hi = mid;
    }
    return lo;
}

Constants make_constants() {
    Constants c{};
    uint32_t primes[64];
    int n = 0;
    for (uint32_t v = 2; n < 64; ++v) {
        bool prime = true;
        for (int i = 0; i < n && primes[i] * primes[i] <= v; ++i)
            if (v % primes[i] == 0) prime = false;
        if (prime) primes[n++] = v;
    }
    for (int i = 0; i < 64; ++i) c.k[i] = (uint32_t)iroot((u128)primes[i] << 96, 3);
    for (int i = 0; i < 8; ++i) c.h0[i] = (uint32_t)iroot((u128)primes[i] << 64, 2);
    return c;
}

const Constants& constants() {
    static const Constants c = make_constants();
    return c;
}

inline uint32_t rotr(uint32_t x, int n) { return (x >> n) | (x << (32 - n)); }

void compress_portable(uint32_t h[8], const uint8_t* p, size_t blocks) {
    const uint32_t* K = constants().k;
    for (; blocks; --blocks, p += 64) {
        uint32_t w[64];
        for (int t = 0; t < 16; ++t)
            w[t] = (uint32_t)p[4 * t] << 24 | (uint32_t)p[4 * t + 1] << 16 | (uint32_t)p[4 * t + 2] << 8 |
                   p[4 * t + 3];
        for (int t = 16; t < 64; ++t) {
            const uint32_t s0 = rotr(w[t - 15], 7) ^ rotr(w[t - 15], 18) ^ (w[t - 15] >> 3);
            const uint32_t s1 = rotr(w[t - 2], 17) ^ rotr(w[t - 2], 19) ^ (w[t - 2] >> 10);
            w[t] = w[t - 16] + s0 + w[t - 7] + s1;
        }
        uint32_t a = h[0], b = h[1], c = h[2], d = h[3], e = h[4], f = h[5], g = h[6], hh = h[7];
        for (int t = 0; t < 64; ++t) {
            const uint32_t t1 = hh + (rotr(e, 6) ^ rotr(e, 11) ^ rotr(e, 25)) + ((e & f) ^ (~e & g)) + K[t] + w[t];
            const uint32_t t2 = (rotr(a, 2) ^ rotr(a, 13) ^ rotr(a, 22)) + ((a & b) ^ (a & c) ^ (b & c));
            hh = g;
            g = f;
            f = e;
            e = d + t1;
            d = c;
            c = b;
            b = a;
            a = t1 + t2;
        }
        h[0] += a;
        h[1] += b;
        h[2] += c;
        h[3] += d;
        h[4] += e;
        h[5] += f;
        h[6] += g;
        h[7] += hh;
    }
}

// The SHA extensions keep the state as two vectors, {A,B,E,F} and {C,D,G,H}
// (highest lane first).  sha256rnds2(cdgh, abef, wk) runs two rounds with the
// two lowest lanes of wk and returns the new {A,B,E,F}; the old {A,B,E,F} is
// then the new {C,D,G,H}.  The schedule words W[t..t+3] sit in one vector,
// lowest lane first: W[t+16..t+19] = sha256msg2(sha256msg1(W[t..], W[t+4..])
// + W[t+9..t+12], W[t+12..]).
__attribute__((target("sha,sse4.1,ssse3"))) void compress_sha_ext(uint32_t h[8], const uint8_t* p,
                                                                   size_t blocks) {
    const uint32_t* K = constants().k;
    const __m128i big_endian = _mm_set_epi8(12, 13, 14, 15, 8, 9, 10, 11, 4, 5, 6, 7, 0, 1, 2, 3);
    __m128i abef = _mm_set_epi32((int)h[0], (int)h[1], (int)h[4], (int)h[5]);
    __m128i cdgh = _mm_set_epi32((int)h[2], (int)h[3], (int)h[6], (int)h[7]);
    for (; blocks; --blocks, p += 64) {
        const __m128i abef0 = abef, cdgh0 = cdgh;
        __m128i w[4];
        for (int j = 0; j < 4; ++j)
            w[j] = _mm_shuffle_epi8(_mm_loadu_si128(reinterpret_cast<const __m128i*>(p + 16 * j)), big_endian);
        for (int g = 0; g < 16; ++g) {
            __m128i wk = _mm_add_epi32(w[g & 3], _mm_loadu_si128(reinterpret_cast<const __m128i*>(K + 4 * g)));
            __m128i next = _mm_sha256rnds2_epu32(cdgh, abef, wk);
            cdgh = abef;
            abef = next;
            wk = _mm_shuffle_epi32(wk, 0x0E);
            next = _mm_sha256rnds2_epu32(cdgh, abef, wk);
            cdgh = abef;
            abef = next;
            if (g < 12) {
                __m128i x = _mm_sha256msg1_epu32(w[g & 3], w[(g + 1) & 3]);
                x = _mm_add_epi32(x, _mm_alignr_epi8(w[(g + 3) & 3], w[(g + 2) & 3], 4));
                w[g & 3] = _mm_sha256msg2_epu32(x, w[(g + 3) & 3]);
            }
        }
        abef = _mm_add_epi32(abef, abef0);
        cdgh = _mm_add_epi32(cdgh, cdgh0);
    }
    alignas(16) uint32_t s[4], t[4];
    _mm_store_si128(reinterpret_cast<__m128i*>(s), abef);
    _mm_store_si128(reinterpret_cast<__m128i*>(t), cdgh);
    h[0] = s[3];
    h[1] = s[2];
    h[4] = s[1];
    h[5] = s[0];
    h[2] = t[3];
    h[3] = t[2];
    h[6] = t[1];
    h[7] = t[0];
}

bool use_sha_ext() {
    static const bool yes = [] {
        const char* env = std::getenv("V3D_SHA256_PORTABLE");
        if (env && env[0] == '1') return false;
        unsigned a = 0, b = 0, c = 0, d = 0;
        if (!__get_cpuid(1, &a, &b, &c, &d)) return false;
        const bool ssse3_sse41 = (c & (1u << 9)) && (c & (1u << 19));
        if (!__get_cpuid_count(7, 0, &a, &b, &c, &d)) return false;
        return ssse3_sse41 && (b & (1u << 29));
    }();
    return yes;
}

void compress(uint32_t h[8], const uint8_t* p, size_t blocks) {
    if (use_sha_ext()) compress_sha_ext(h, p, blocks);
    else compress_portable(h, p, blocks);
}

}  // namespace

Sha256::Sha256() { std::memcpy(h, constants().h0, sizeof(h)); }

void Sha256::update(const void* data, size_t n) {
    const uint8_t* p = static_cast<const uint8_t*>(data);
    length += n;
    if (fill) {
        const size_t take = n < 64 - fill ? n : 64 - fill;
        std::memcpy(buf + fill, p, take);
        fill += take;
        p += take;
        n -= take;
        if (fill < 64) return;
        compress(h, buf, 1);
        fill = 0;
    }
    if (n >= 64) {
        compress(h, p, n / 64);
        p += n / 64 * 64;
        n %= 64;
    }
    std::memcpy(buf, p, n);
    fill = n;
}

void Sha256::finish(uint8_t digest[32]) {
    const uint64_t bits = length * 8;
    uint8_t pad[72] = {0x80};
    const size_t zeros = (fill < 56 ? 56 - fill : 120 - fill);
    for (int i = 0; i < 8; ++i) pad[zeros + i] = (uint8_t)(bits >> (56 - 8 * i));
    update(pad, zeros + 8);
    for (int i = 0; i < 8; ++i)
        for (int j = 0; j < 4; ++j) digest[4 * i + j] = (uint8_t)(h[i] >> (24 - 8 * j));
}

}  // namespace v3d

extern "C" void v3d_sha256(const void* bytes, uint64_t n, uint8_t* digest) {
    v3d::Sha256 s;
    if (n) s.update(bytes, n);
    s.finish(digest);
}
