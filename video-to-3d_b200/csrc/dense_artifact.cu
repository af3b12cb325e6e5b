// The dense artifact's bulk as serde_json text, formatted on the device
// (v3d_encode_dense_evidence).  DenseStageArtifact::to_json and content_hash
// (reconstruction_stages.rs:287-380) write DenseEvidence
// (reconstruction_stages.rs:250-256); its points, grid sites and point
// attributes are nearly all of the document.
//
// One thread owns one array element (or one of the four pieces of glue
// between the arrays: "[", "],"grid_sites":[", "],"point_attributes":[",
// "]").  k_measure finds the shortest round-trip decimal of each f32 and the
// element's text length, and scans the lengths within its block; k_block_bases
// scans the block totals; k_emit lets each warp format its 32 elements into
// shared memory and store the contiguous text with 16-byte stores.  The
// host copies the text back in chunks while a host thread hashes it
// (SHA-256, sha256.cpp), so the digest is ready when the last byte lands.
//
// Shortest digits, exactly: with v = m * 2^e2 and its rounding interval
// [mm, mp] * 2^(e2-2) (bounds included when m is even, as round-to-nearest-
// even parsing reads them), the value and both bounds are divided by 10^k9,
// k9 = floor(log10 v) - 8, with exact floors (a double estimate corrected by
// exact comparisons of d * 10^k against X * 2^c on 160-bit integers).  The
// shortest decimal is then the largest power 10^s with a multiple inside the
// integer interval, and the digit string is the value rounded to that
// position (half to even) and clamped into the interval: the closest of the
// shortest, as serde_json's formatter (zmij, after ryu) prints.
#include <cub/block/block_scan.cuh>

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <mutex>
#include <thread>

#include "../../include/v3d_dense.h"
#include "host.hpp"
#include "v3d_device.cuh"

namespace v3d {
namespace {

// ---- exact arithmetic for the digit search --------------------------------

// 5^j for j <= 60, five 32-bit limbs each (least significant first).
struct Pow5Table {
    uint32_t w[61][5];
};

constexpr Pow5Table make_pow5_table() {
    Pow5Table t{};
    t.w[0][0] = 1;
    for (int j = 1; j <= 60; ++j) {
        uint64_t carry = 0;
        for (int i = 0; i < 5; ++i) {
            const uint64_t p = (uint64_t)t.w[j - 1][i] * 5u + carry;
            t.w[j][i] = (uint32_t)p;
            carry = p >> 32;
        }
    }
    return t;
}

__device__ const Pow5Table g_pow5 = make_pow5_table();

struct U160 {
    uint32_t w[5];
};

// m * 5^j; the callers keep the product below 2^160.
__device__ __forceinline__ U160 mul_pow5(int j, uint32_t m) {
    U160 r;
    uint64_t carry = 0;
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        const uint64_t p = (uint64_t)__ldg(&g_pow5.w[j][i]) * m + carry;
        r.w[i] = (uint32_t)p;
        carry = p >> 32;
    }
    return r;
}

__device__ __forceinline__ U160 small(uint32_t x) { return U160{{x, 0u, 0u, 0u, 0u}}; }

__device__ __forceinline__ int bitlen(const U160& a) {
#pragma unroll
    for (int i = 4; i >= 0; --i)
        if (a.w[i]) return 32 * i + 32 - __clz(a.w[i]);
    return 0;
}

// a << s for 0 <= s < 160 with the result below 2^160.
__device__ __forceinline__ U160 shl(U160 a, int s) {
    const int q = s >> 5, b = s & 31;
#pragma unroll
    for (int t = 0; t < 4; ++t)
        if (t < q) {
            a.w[4] = a.w[3];
            a.w[3] = a.w[2];
            a.w[2] = a.w[1];
            a.w[1] = a.w[0];
            a.w[0] = 0u;
        }
    U160 r;
    r.w[0] = a.w[0] << b;
#pragma unroll
    for (int i = 1; i < 5; ++i) r.w[i] = __funnelshift_l(a.w[i - 1], a.w[i], b);
    return r;
}

__device__ __forceinline__ int cmp(const U160& a, const U160& b) {
#pragma unroll
    for (int i = 4; i >= 0; --i)
        if (a.w[i] != b.w[i]) return a.w[i] < b.w[i] ? -1 : 1;
    return 0;
}

// Sign of d * 10^k - X * 2^c, exactly, for 0 < d < 2^32, 0 < X < 2^27,
// -54 <= k <= 40 (both sides stay below 2^153 after alignment).
__device__ int cmp_dec_bin(uint32_t d, int k, uint32_t X, int c) {
    U160 A, B;
    int ea, eb = c;
    if (k >= 0) {
        A = mul_pow5(k, d);  // d * 5^k * 2^k
        ea = k;
        B = small(X);
    } else {
        A = small(d);  // d * 2^k against X * 5^-k * 2^c
        ea = k;
        B = mul_pow5(-k, X);
    }
    const int la = bitlen(A) + ea, lb = bitlen(B) + eb;
    if (la != lb) return la < lb ? -1 : 1;
    if (ea > eb) A = shl(A, ea - eb);
    else if (eb > ea) B = shl(B, eb - ea);
    return cmp(A, B);
}

// floor(X * 2^c / 10^k) (< 2^31 for the scales used here), whether the
// quotient is exact, and, when not, where the fraction lies against one half
// (1 below, 2 exactly, 3 above).  The double estimate is off by less than
// 4e-7 here (ldexp is exact, exp10 within an ulp, the product within half an
// ulp, quotients below 1.1e9), so a fraction at least kMargin from 0, 1/2 and
// 1 decides all three; only the rare quotients near those use the exact
// comparisons.
constexpr double kMargin = 1.0 / 65536.0;

__device__ uint32_t floor_scaled(uint32_t X, int c, int k, double scale, bool* exact, int* half) {
    const double approx = (double)X * scale;  // scale = 2^c 10^-k
    if (approx >= 4.0e9) {  // a scale one decade too fine: saturate, the caller moves k
        *exact = false;
        *half = 1;
        return 0xFFFFFFFFu;
    }
    const double whole = floor(approx), frac = approx - whole;
    if (frac > kMargin && frac < 1.0 - kMargin && fabs(frac - 0.5) > kMargin) {
        *exact = false;
        *half = frac < 0.5 ? 1 : 3;
        return (uint32_t)whole;
    }
    uint32_t q = (uint32_t)approx;  // within one of the floor
    int t = cmp_dec_bin(q, k, X, c);
    for (int i = 0; i < 4 && t > 0; ++i) t = cmp_dec_bin(--q, k, X, c);
    for (int i = 0; i < 4; ++i) {
        const int t1 = cmp_dec_bin(q + 1u, k, X, c);
        if (t1 > 0) break;
        ++q;
        t = t1;
    }
    *exact = t == 0;
    *half = 0;
    if (!*exact) {
        const int th = cmp_dec_bin(2u * q + 1u, k, X, c + 1);  // (2q + 1) 10^k against 2 X 2^c
        *half = th > 0 ? 1 : (th == 0 ? 2 : 3);
    }
    return q;
}

// One f32 as serde_json writes it: shortest digits and the exponent of the
// last digit, or a flag for zero / non-finite.  8 bytes.
struct Dec {
    uint32_t digits;
    int16_t exp10;
    uint8_t len;
    uint8_t flags;
};
constexpr uint8_t kNeg = 1, kZero = 2, kNonFinite = 4;

__device__ __forceinline__ int ndigits(uint32_t d) {
    int n = 1;
    while (d >= 10u) {
        d /= 10u;
        ++n;
    }
    return n;
}

__device__ Dec decimal_of(float f) {
    Dec r{0u, 0, 0, 0};
    const uint32_t bits = __float_as_uint(f);
    if ((bits & 0x7F800000u) == 0x7F800000u) {
        r.flags = kNonFinite;
        return r;
    }
    if (bits >> 31) r.flags |= kNeg;
    const uint32_t mag = bits & 0x7FFFFFFFu;
    if (mag == 0u) {
        r.flags |= kZero;
        return r;
    }
    const uint32_t ieee_m = mag & 0x7FFFFFu, ieee_e = mag >> 23;
    const uint32_t m = ieee_e ? (ieee_m | 0x800000u) : ieee_m;
    const int e2 = ieee_e ? (int)ieee_e - 150 : -149;
    const bool even = (m & 1u) == 0u;
    // the value and its rounding interval in units of 2^(e2-2); the gap below
    // halves at the bottom of a binade (not below the smallest normal)
    const uint32_t mv = 4u * m, mp = mv + 2u, mm = mv - ((ieee_m != 0u || ieee_e <= 1u) ? 2u : 1u);
    const int c = e2 - 2;
    // k9 such that 10^8 <= v / 10^k9 < 10^9: floor(E log10 2) for v in
    // [2^E, 2^(E+1)) is off by at most one, which the exact quotient's range
    // corrects
    const int E = e2 + 31 - __clz(m);
    int k9 = (int)floor((double)E * 0.30102999566398120) - 8;
    bool ev, el, eu;
    int frac, unused;
    double scale = ldexp(exp10((double)-k9), c);  // one scale for the value and both bounds
    uint32_t qv = floor_scaled(mv, c, k9, scale, &ev, &frac);
    for (int i = 0; i < 2 && (qv < 100000000u || qv >= 1000000000u); ++i) {
        k9 += qv < 100000000u ? -1 : 1;
        scale = ldexp(exp10((double)-k9), c);
        qv = floor_scaled(mv, c, k9, scale, &ev, &frac);
    }
    const uint32_t ql = floor_scaled(mm, c, k9, scale, &el, &unused);
    const uint32_t qu = floor_scaled(mp, c, k9, scale, &eu, &unused);
    const uint32_t lo = (el && even) ? ql : ql + 1u;
    const uint32_t hi = (eu && !even) ? qu - 1u : qu;
    // v / 10^k9 - qv: 0 exact, 1 below one half, 2 one half, 3 above
    if (ev) frac = 0;
    uint32_t p = 1u;
    int s = 0;
    while (s < 9) {
        const uint32_t p10 = p * 10u;
        if (hi / p10 < (lo + p10 - 1u) / p10) break;
        p = p10;
        ++s;
    }
    uint32_t d = qv / p;
    const uint32_t rem = qv - d * p;
    bool up;
    if (s == 0) {
        up = frac == 3 || (frac == 2 && (d & 1u));
    } else {
        const uint32_t half = p / 2u;
        up = rem > half || (rem == half && (frac != 0 || (d & 1u)));
    }
    d += up ? 1u : 0u;
    d = min(max(d, (lo + p - 1u) / p), hi / p);
    int k = k9 + s;
    while (d % 10u == 0u) {
        d /= 10u;
        ++k;
    }
    r.digits = d;
    r.exp10 = (int16_t)k;
    r.len = (uint8_t)ndigits(d);
    return r;
}

// ---- text ------------------------------------------------------------------

__device__ __forceinline__ int exp_len(int x) { return (x < 0 ? 1 : 0) + ((x >= 10 || x <= -10) ? 2 : 1); }

// serde_json's f32 notation (the ryu crate's, kept by zmij).
__device__ int text_len(const Dec& dc) {
    if (dc.flags & kNonFinite) return 4;  // null
    const int sign = (dc.flags & kNeg) ? 1 : 0;
    if (dc.flags & kZero) return sign + 3;
    const int n = dc.len, k = dc.exp10, kk = n + k;
    if (k >= 0 && kk <= 13) return sign + kk + 2;
    if (kk > 0 && kk <= 13) return sign + n + 1;
    if (kk > -6 && kk <= 0) return sign + 2 - kk + n;
    return sign + n + (n > 1 ? 1 : 0) + 1 + exp_len(kk - 1);
}

__device__ char* write_f32(char* p, const Dec& dc) {
    if (dc.flags & kNonFinite) {
        p[0] = 'n';
        p[1] = 'u';
        p[2] = 'l';
        p[3] = 'l';
        return p + 4;
    }
    if (dc.flags & kNeg) *p++ = '-';
    if (dc.flags & kZero) {
        p[0] = '0';
        p[1] = '.';
        p[2] = '0';
        return p + 3;
    }
    const int n = dc.len, k = dc.exp10, kk = n + k;
    uint32_t d = dc.digits;
    if (k >= 0 && kk <= 13) {  // 1234e7 -> 12340000000.0
        for (int i = n - 1; i >= 0; --i, d /= 10u) p[i] = (char)('0' + d % 10u);
        for (int i = n; i < kk; ++i) p[i] = '0';
        p[kk] = '.';
        p[kk + 1] = '0';
        return p + kk + 2;
    }
    if (kk > 0 && kk <= 13) {  // 1234e-2 -> 12.34
        for (int i = n - 1; i >= 0; --i, d /= 10u) p[i + (i >= kk ? 1 : 0)] = (char)('0' + d % 10u);
        p[kk] = '.';
        return p + n + 1;
    }
    if (kk > -6 && kk <= 0) {  // 1234e-6 -> 0.001234
        p[0] = '0';
        p[1] = '.';
        const int o = 2 - kk;
        for (int i = 2; i < o; ++i) p[i] = '0';
        for (int i = n - 1; i >= 0; --i, d /= 10u) p[o + i] = (char)('0' + d % 10u);
        return p + o + n;
    }
    // 1e30, 1.234e-33
    for (int i = n - 1; i >= 1; --i, d /= 10u) p[i + 1] = (char)('0' + d % 10u);
    p[0] = (char)('0' + d);
    int q = 1;
    if (n > 1) {
        p[1] = '.';
        q = n + 1;
    }
    p[q++] = 'e';
    int x = kk - 1;
    if (x < 0) {
        p[q++] = '-';
        x = -x;
    }
    if (x >= 10) p[q++] = (char)('0' + x / 10);
    p[q++] = (char)('0' + x % 10);
    return p + q;
}

__device__ __forceinline__ char* write_u32(char* p, uint32_t v) {
    const int n = ndigits(v);
    for (int i = n - 1; i >= 0; --i, v /= 10u) p[i] = (char)('0' + v % 10u);
    return p + n;
}

template <int N>
__device__ __forceinline__ char* put(char* p, const char (&s)[N]) {
#pragma unroll
    for (int i = 0; i < N - 1; ++i) p[i] = s[i];
    return p + N - 1;
}

// ---- element index space ---------------------------------------------------
// [glue 0][points][glue 1][sites][glue 2][attributes][glue 3]
struct Layout {
    uint64_t np, ns, na, E;
};

enum Kind { kGlue0, kPoint, kGlue1, kSite, kGlue2, kAttr, kGlue3 };

__device__ __forceinline__ int kind_of(uint64_t e, const Layout& L, uint64_t* i) {
    if (e == 0) return kGlue0;
    if (e <= L.np) {
        *i = e - 1;
        return kPoint;
    }
    if (e == L.np + 1) return kGlue1;
    if (e <= L.np + 1 + L.ns) {
        *i = e - L.np - 2;
        return kSite;
    }
    if (e == L.np + L.ns + 2) return kGlue2;
    if (e <= L.np + L.ns + 2 + L.na) {
        *i = e - L.np - L.ns - 3;
        return kAttr;
    }
    return kGlue3;
}

constexpr int kThreads = 256;
constexpr int kMaxElement = 124;  // 1 comma + 122 for the longest point, rounded up

struct Summary {
    unsigned long long glue[4];  // body offsets of the four glue pieces
    unsigned long long total;    // body bytes
    unsigned long long non_finite;
};

struct Arrays {
    const v3d_point* pts;
    const v3d_grid_site* sites;
    const v3d_point_attributes* attrs;
    Layout L;
};

__global__ void __launch_bounds__(kThreads) k_measure(Arrays in, Dec* __restrict__ dec,
                                                      uint32_t* __restrict__ local_end,
                                                      unsigned long long* __restrict__ block_total,
                                                      Summary* __restrict__ summary) {
    using Scan = cub::BlockScan<uint32_t, kThreads>;
    __shared__ typename Scan::TempStorage scan;
    const uint64_t e = (uint64_t)blockIdx.x * kThreads + threadIdx.x;
    uint32_t len = 0, nonfinite = 0;
    if (e < in.L.E) {
        uint64_t i = 0;
        switch (kind_of(e, in.L, &i)) {
            case kGlue0:
            case kGlue3: len = 1; break;
            case kGlue1: len = 16; break;  // ],"grid_sites":[
            case kGlue2: len = 22; break;  // ],"point_attributes":[
            case kPoint: {
                const v3d_point pt = in.pts[i];
                const Dec a = decimal_of(pt.x), b = decimal_of(pt.y), c = decimal_of(pt.z),
                          d = decimal_of(pt.confidence);
                dec[4 * i] = a;
                dec[4 * i + 1] = b;
                dec[4 * i + 2] = c;
                dec[4 * i + 3] = d;
                len = (i ? 1 : 0) + 45 + text_len(a) + text_len(b) + text_len(c) + text_len(d) +
                      ndigits(pt.r) + ndigits(pt.g) + ndigits(pt.b);
                nonfinite = (a.flags & kNonFinite ? 1 : 0) + (b.flags & kNonFinite ? 1 : 0) +
                            (c.flags & kNonFinite ? 1 : 0) + (d.flags & kNonFinite ? 1 : 0);
                break;
            }
            case kSite: {
                const v3d_grid_site s = in.sites[i];
                len = (i ? 1 : 0) + 11 + ndigits(s.x) + ndigits(s.y);
                break;
            }
            case kAttr: {
                const v3d_point_attributes at = in.attrs[i];
                const Dec a = decimal_of(at.reciprocal_consistency), b = decimal_of(at.depth_margin);
                dec[4 * in.L.np + 2 * i] = a;
                dec[4 * in.L.np + 2 * i + 1] = b;
                len = (i ? 1 : 0) + 43 + text_len(a) + text_len(b);
                nonfinite = (a.flags & kNonFinite ? 1 : 0) + (b.flags & kNonFinite ? 1 : 0);
                break;
            }
        }
    }
    uint32_t end, total;
    Scan(scan).InclusiveSum(len, end, total);
    if (e < in.L.E) local_end[e] = end;
    if (threadIdx.x == 0) block_total[blockIdx.x] = total;
    if (nonfinite) atomicAdd(&summary->non_finite, (unsigned long long)nonfinite);
}

// Exclusive scan of the block totals by one block, 8 consecutive totals a
// thread; base[b] is block b's first body byte.
__global__ void __launch_bounds__(512) k_block_bases(const unsigned long long* __restrict__ totals,
                                                     uint64_t n, unsigned long long* __restrict__ base,
                                                     Summary* __restrict__ summary) {
    constexpr int kItems = 8, kTile = 512 * kItems;
    using Scan = cub::BlockScan<unsigned long long, 512>;
    __shared__ typename Scan::TempStorage scan;
    __shared__ unsigned long long carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint64_t b0 = 0; b0 < n; b0 += kTile) {
        const uint64_t first = b0 + (uint64_t)threadIdx.x * kItems;
        unsigned long long v[kItems], ex[kItems], sum;
#pragma unroll
        for (int k = 0; k < kItems; ++k) v[k] = first + k < n ? totals[first + k] : 0ull;
        Scan(scan).ExclusiveSum(v, ex, sum);
        const unsigned long long c = carry;
#pragma unroll
        for (int k = 0; k < kItems; ++k)
            if (first + k < n) base[first + k] = c + ex[k];
        __syncthreads();
        if (threadIdx.x == 0) carry = c + sum;
        __syncthreads();
    }
    if (threadIdx.x == 0) summary->total = carry;
}

__device__ char* write_element(char* p, uint64_t e, const Arrays& in, const Dec* __restrict__ dec) {
    uint64_t i = 0;
    switch (kind_of(e, in.L, &i)) {
        case kGlue0: return put(p, "[");
        case kGlue1: return put(p, "],\"grid_sites\":[");
        case kGlue2: return put(p, "],\"point_attributes\":[");
        case kGlue3: return put(p, "]");
        case kPoint: {
            const v3d_point pt = in.pts[i];
            if (i) *p++ = ',';
            p = write_f32(put(p, "{\"x\":"), dec[4 * i]);
            p = write_f32(put(p, ",\"y\":"), dec[4 * i + 1]);
            p = write_f32(put(p, ",\"z\":"), dec[4 * i + 2]);
            p = write_f32(put(p, ",\"confidence\":"), dec[4 * i + 3]);
            p = write_u32(put(p, ",\"r\":"), pt.r);
            p = write_u32(put(p, ",\"g\":"), pt.g);
            p = write_u32(put(p, ",\"b\":"), pt.b);
            return put(p, "}");
        }
        case kSite: {
            const v3d_grid_site s = in.sites[i];
            if (i) *p++ = ',';
            p = write_u32(put(p, "{\"x\":"), s.x);
            p = write_u32(put(p, ",\"y\":"), s.y);
            return put(p, "}");
        }
        default: {  // kAttr
            if (i) *p++ = ',';
            p = write_f32(put(p, "{\"reciprocal_consistency\":"), dec[4 * in.L.np + 2 * i]);
            p = write_f32(put(p, ",\"depth_margin\":"), dec[4 * in.L.np + 2 * i + 1]);
            return put(p, "}");
        }
    }
}

// Each warp formats 32 consecutive elements into its shared-memory stage,
// placed so that the stage and the body agree modulo 16, then stores the
// text: 16-byte stores for the aligned interior, bytes at the two ragged ends
// (the neighbouring warps own the rest of those 16-byte words).
__global__ void __launch_bounds__(kThreads) k_emit(Arrays in, const Dec* __restrict__ dec,
                                                   const uint32_t* __restrict__ local_end,
                                                   const unsigned long long* __restrict__ base,
                                                   char* __restrict__ body, Summary* __restrict__ summary) {
    __shared__ __align__(16) char stage[kThreads / 32][32 * kMaxElement + 16];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    char* sm = stage[warp];
    const uint64_t e0 = (uint64_t)blockIdx.x * kThreads + (uint64_t)warp * 32;
    if (e0 >= in.L.E) return;  // the whole warp leaves together
    const uint64_t e = e0 + lane;
    const bool valid = e < in.L.E;
    const unsigned long long b = base[blockIdx.x];
    unsigned long long my_start = 0, my_end = 0;
    if (valid) {
        my_end = b + local_end[e];
        my_start = (e % kThreads) ? b + local_end[e - 1] : b;
    }
    const int last = in.L.E - e0 > 32 ? 31 : (int)(in.L.E - 1 - e0);
    const unsigned long long start = __shfl_sync(0xFFFFFFFFu, my_start, 0);
    const unsigned long long end = __shfl_sync(0xFFFFFFFFu, my_end, last);
    const int sb = (int)(start & 15ull);
    if (valid) {
        char* p = sm + sb + (my_start - start);
        write_element(p, e, in, dec);
        uint64_t i;
        const int kind = kind_of(e, in.L, &i);
        if (kind == kGlue1) summary->glue[1] = my_start;
        else if (kind == kGlue2) summary->glue[2] = my_start;
        else if (kind == kGlue3) summary->glue[3] = my_start;
    }
    __syncwarp();
    const unsigned long long a0 = (start + 15ull) & ~15ull, a1 = end & ~15ull;
    if (a0 <= a1) {
        if (start + lane < a0) body[start + lane] = sm[sb + lane];
        if (a1 + lane < end) body[a1 + lane] = sm[sb + (a1 - start) + lane];
        for (unsigned long long v = a0 + 16ull * lane; v < a1; v += 512ull)
            *reinterpret_cast<uint4*>(body + v) = *reinterpret_cast<const uint4*>(sm + sb + (v - start));
    } else {
        for (unsigned long long q = start + lane; q < end; q += 32ull) body[q] = sm[sb + (q - start)];
    }
}

constexpr uint64_t kGlueBytes = 1 + 16 + 22 + 1;
constexpr uint64_t kMaxPoint = 123, kMaxSite = 32, kMaxAttr = 78;  // comma included

}  // namespace
}  // namespace v3d

using namespace v3d;

extern "C" uint64_t v3d_dense_document_bound(uint64_t n_points, uint64_t n_grid_sites,
                                             uint64_t n_point_attributes, uint64_t prefix_bytes,
                                             uint64_t suffix_bytes) {
    return prefix_bytes + suffix_bytes + kGlueBytes + kMaxPoint * n_points + kMaxSite * n_grid_sites +
           kMaxAttr * n_point_attributes;
}

extern "C" void v3d_pack_dense_points(const v3d_point* points, uint64_t n, uint8_t* values_f32_le,
                                      uint8_t* rgb) {
    static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "f32::to_le_bytes is the in-memory layout");
    static_assert(offsetof(v3d_point, x) == 0 && offsetof(v3d_point, confidence) == 12,
                  "x, y, z, confidence lead v3d_point");
    for (uint64_t i = 0; i < n; ++i) {
        std::memcpy(values_f32_le + 16 * i, &points[i], 16);
        rgb[3 * i] = points[i].r;
        rgb[3 * i + 1] = points[i].g;
        rgb[3 * i + 2] = points[i].b;
    }
}

extern "C" int32_t v3d_pack_mesh_triangles(const v3d_mesh_triangle* triangles, uint64_t nt,
                                           const v3d_triangle_source* sources, uint64_t ns,
                                           const v3d_derived_vertex_source* derived, uint64_t nd,
                                           uint64_t point_count, uint8_t* indices_u32_le,
                                           uint8_t* confidence_f32_le, uint8_t* sources_u32_le,
                                           uint8_t* derived_u32_le, uint8_t* derived_barycentric_f64_le,
                                           const char** error) {
    static_assert(__BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__, "to_le_bytes is the in-memory layout");
    const char* const source_range =
        "failed to serialize reconstruction: triangle source exceeds browser transport range";
    auto fail = [&](const char* why) {
        if (error) *error = why;
        return (int32_t)V3D_ERR_INVALID_ARGUMENT;
    };
    if (error) *error = nullptr;
    if ((nt && (!triangles || !indices_u32_le || !confidence_f32_le)) || (ns && (!sources || !sources_u32_le)) ||
        (nd && (!derived || !derived_u32_le || !derived_barycentric_f64_le)))
        return V3D_ERR_INVALID_ARGUMENT;
    auto put_u32 = [](uint8_t* at, uint64_t v) {
        const uint32_t w = (uint32_t)v;
        std::memcpy(at, &w, 4);
    };
    for (uint64_t i = 0; i < ns; ++i) {
        const uint64_t v[4] = {sources[i].triangle, sources[i].corners[0], sources[i].corners[1],
                               sources[i].corners[2]};
        for (int k = 0; k < 4; ++k) {
            if (v[k] > 0xFFFFFFFFull) return fail(source_range);
            put_u32(sources_u32_le + 16 * i + 4 * k, v[k]);
        }
    }
    for (uint64_t i = 0; i < nd; ++i) {
        const v3d_derived_vertex_source& d = derived[i];
        const uint64_t v[5] = {d.point_index, d.source_triangle, d.source_corners[0], d.source_corners[1],
                               d.source_corners[2]};
        for (int k = 0; k < 5; ++k) {
            if (v[k] > 0xFFFFFFFFull) return fail(source_range);
            put_u32(derived_u32_le + 20 * i + 4 * k, v[k]);
        }
        std::memcpy(derived_barycentric_f64_le + 24 * i, d.barycentric, 24);
    }
    for (uint64_t t = 0; t < nt; ++t) {
        const uint64_t v[3] = {triangles[t].a, triangles[t].b, triangles[t].c};
        for (int k = 0; k < 3; ++k) {
            if (v[k] >= point_count)
                return fail("failed to serialize reconstruction: mesh triangle references a missing dense point");
            if (v[k] > 0xFFFFFFFFull)
                return fail("failed to serialize reconstruction: dense point index exceeds browser transport range");
            put_u32(indices_u32_le + 12 * t + 4 * k, v[k]);
        }
        std::memcpy(confidence_f32_le + 4 * t, &triangles[t].confidence, 4);
    }
    return V3D_OK;
}

extern "C" int32_t v3d_encode_dense_evidence(
    v3d_context* ctx, const v3d_point* points, uint64_t np, const v3d_grid_site* sites, uint64_t ns,
    const v3d_point_attributes* attrs, uint64_t na, const char* prefix, uint64_t prefix_bytes,
    const char* suffix, uint64_t suffix_bytes, char* document, uint64_t capacity, v3d_dense_document* out) {
    if (!ctx || !out || (np && !points) || (ns && !sites) || (na && !attrs) || (prefix_bytes && !prefix) ||
        (suffix_bytes && !suffix))
        return V3D_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    if (np >= (1ull << 32) || ns >= (1ull << 32) || na >= (1ull << 32)) {
        ctx->last_error = "the dense document takes fewer than 2^32 points, grid sites and attributes";
        return V3D_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(ctx->stream);
    Layout L{np, ns, na, np + ns + na + 4};
    const uint64_t blocks = (L.E + kThreads - 1) / kThreads;
    const uint64_t body_cap = v3d_dense_document_bound(np, ns, na, 0, 0);
    Carve cv;
    const size_t o_pts = cv.take<v3d_point>(np), o_sites = cv.take<v3d_grid_site>(ns),
                 o_attrs = cv.take<v3d_point_attributes>(na), o_dec = cv.take<Dec>(4 * np + 2 * na),
                 o_end = cv.take<uint32_t>(L.E), o_tot = cv.take<unsigned long long>(blocks),
                 o_base = cv.take<unsigned long long>(blocks), o_sum = cv.take<Summary>(1),
                 o_body = cv.take<char>(body_cap);
    if (!ensure_arena(ctx, cv.off + 256)) {
        ctx->last_error = "device arena allocation failed";
        return V3D_ERR_OUT_OF_MEMORY;
    }
    char* base = static_cast<char*>(ctx->arena);
    Arrays in{reinterpret_cast<const v3d_point*>(base + o_pts),
              reinterpret_cast<const v3d_grid_site*>(base + o_sites),
              reinterpret_cast<const v3d_point_attributes*>(base + o_attrs), L};
    auto* d_dec = reinterpret_cast<Dec*>(base + o_dec);
    auto* d_end = reinterpret_cast<uint32_t*>(base + o_end);
    auto* d_tot = reinterpret_cast<unsigned long long*>(base + o_tot);
    auto* d_base = reinterpret_cast<unsigned long long*>(base + o_base);
    auto* d_sum = reinterpret_cast<Summary*>(base + o_sum);
    char* d_body = base + o_body;
    if (np) V3D_CTX_CK(cudaMemcpyAsync(base + o_pts, points, sizeof(v3d_point) * np, cudaMemcpyHostToDevice, st));
    if (ns)
        V3D_CTX_CK(cudaMemcpyAsync(base + o_sites, sites, sizeof(v3d_grid_site) * ns, cudaMemcpyHostToDevice, st));
    if (na)
        V3D_CTX_CK(cudaMemcpyAsync(base + o_attrs, attrs, sizeof(v3d_point_attributes) * na,
                                   cudaMemcpyHostToDevice, st));
    V3D_CTX_CK(cudaMemsetAsync(d_sum, 0, sizeof(Summary), st));

    const uint64_t launches0 = g_kernel_launches;
    cudaEvent_t ev0, ev1;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    struct Events {
        cudaEvent_t a, b;
        ~Events() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } events{ev0, ev1};
    cudaEventRecord(ev0, st);
    V3D_COUNTED k_measure<<<(unsigned)blocks, kThreads, 0, st>>>(in, d_dec, d_end, d_tot, d_sum);
    V3D_CTX_CK(cudaGetLastError());
    V3D_COUNTED k_block_bases<<<1, 512, 0, st>>>(d_tot, blocks, d_base, d_sum);
    V3D_CTX_CK(cudaGetLastError());
    V3D_COUNTED k_emit<<<(unsigned)blocks, kThreads, 0, st>>>(in, d_dec, d_end, d_base, d_body, d_sum);
    V3D_CTX_CK(cudaGetLastError());
    cudaEventRecord(ev1, st);
    Summary sum{};
    V3D_CTX_CK(cudaMemcpyAsync(&sum, d_sum, sizeof(Summary), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaStreamSynchronize(st));
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess) ctx->last_ms = ms;
    ctx->last_launches = g_kernel_launches - launches0;

    const uint64_t body = sum.total;
    out->points_bytes = sum.glue[1] + 1;
    out->grid_sites_bytes = sum.glue[2] - (sum.glue[1] + 15) + 1;
    out->point_attributes_bytes = sum.glue[3] - (sum.glue[2] + 21) + 1;
    out->non_finite = sum.non_finite;
    out->document_bytes = prefix_bytes + body + suffix_bytes;
    if (body > body_cap || sum.glue[3] + 1 != body) {
        ctx->last_error = "dense document layout check failed";
        return V3D_ERR_INTERNAL;
    }
    if (!document || capacity < out->document_bytes) {
        ctx->last_error = "the document buffer is smaller than the document";
        return V3D_ERR_INVALID_ARGUMENT;
    }

    // Stream the body back in chunks; a host thread hashes each part as soon
    // as it is in place.
    const uint64_t total = out->document_bytes;
    std::mutex m;
    std::condition_variable cv_ready;
    uint64_t ready = 0;
    bool failed = false;
    auto publish = [&](uint64_t n, bool failure) {
        {
            std::lock_guard<std::mutex> g(m);
            ready = n;
            failed = failed || failure;
        }
        cv_ready.notify_one();
    };
    std::thread hasher;
    auto hash_document = [&] {
        Sha256 h;
        uint64_t done = 0;
        while (done < total) {
            uint64_t r;
            {
                std::unique_lock<std::mutex> g(m);
                cv_ready.wait(g, [&] { return ready > done || failed; });
                if (failed) return;
                r = ready;
            }
            h.update(document + done, r - done);
            done = r;
        }
        h.finish(out->sha256);
    };
    try {
        hasher = std::thread(hash_document);
    } catch (const std::exception&) {
        ctx->last_error = "could not start the hashing thread";
        return V3D_ERR_INTERNAL;
    }
    if (prefix_bytes) std::memcpy(document, prefix, prefix_bytes);
    publish(prefix_bytes, false);
    constexpr uint64_t kChunk = 8ull << 20;
    cudaError_t err = cudaSuccess;
    for (uint64_t o = 0; o < body && err == cudaSuccess; o += kChunk) {
        const uint64_t n = std::min(kChunk, body - o);
        err = cudaMemcpyAsync(document + prefix_bytes + o, d_body + o, n, cudaMemcpyDeviceToHost, st);
        if (err == cudaSuccess) err = cudaStreamSynchronize(st);
        if (err == cudaSuccess) publish(prefix_bytes + o + n, false);
    }
    if (err == cudaSuccess) {
        if (suffix_bytes) std::memcpy(document + prefix_bytes + body, suffix, suffix_bytes);
        publish(total, false);
    } else {
        publish(0, true);
    }
    hasher.join();
    if (err != cudaSuccess) {
        std::memset(out->sha256, 0, sizeof(out->sha256));
        ctx->last_error = std::string("reading the document back: ") + cudaGetErrorString(err);
        return V3D_ERR_CUDA;
    }
    return V3D_OK;
}
