// TEST INFRASTRUCTURE — CPU oracle of the dense artifact wire format.
//
// DenseStageArtifact::to_json (crates/video-to-3d-core/src/
// reconstruction_stages.rs:287-380) writes the dense evidence with serde_json
// 1.0.154 (Cargo.lock; float_roundtrip feature, Cargo.toml:13), which formats
// every f32 through the zmij 1.0.23 crate.  Neither crate is vendored in the
// reference, so this file restates their published behaviour:
//   * digits: the shortest decimal that reads back to the same f32 under
//     round-to-nearest-even parsing, the closest of those to the f32, ties to
//     an even last digit (the contract of Ryu, Ulf Adams, PLDI 2018, and of
//     its successors);
//   * notation: serde_json's f32 notation (the ryu crate's, which zmij keeps):
//     with n digits d and decimal exponent k of the last digit, kk = n + k,
//       0 <= k and kk <= 13   digits, kk - n zeros, ".0"   (1234e7 -> 12340000000.0)
//       0 < kk <= 13          digits with the point after kk (1234e-2 -> 12.34)
//       -6 < kk <= 0          "0." then -kk zeros then digits (1234e-6 -> 0.001234)
//       n == 1                d "e" (kk - 1)                 (1e30, 1e-7)
//       otherwise             d "." rest "e" (kk - 1)        (1.234e33)
//     a leading '-' for negative values (-0.0 included), "0.0" for zero and
//     null for NaN and the infinities (serde_json's serialize_f32).
// The digit search here does not follow Ryu: for p = 1..9 it takes glibc's
// exactly rounded p-digit decimal (printf %.*e, round half to even), and that
// decimal's neighbour on the far side of the value, and keeps the first that
// strtof (exactly rounded) reads back to the same f32.  Those two candidates
// are the only p-digit decimals that can lie in the value's rounding interval
// on the far and near side, so the first hit is the shortest, and the
// nearest-first order makes it the closest.  The digits are pinned against
// numpy's shortest float32 repr (Dragon4 in unique mode) in
// tests/test_artifact_cpu.py; the notation is unpinned: no golden document
// exists in the reference and the crates cannot be built here.
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>

#include "oracle.hpp"

namespace v3do {
namespace {

bool reads_back(uint64_t d, int k, float f) {
    char buf[64];
    std::snprintf(buf, sizeof(buf), "%llue%d", (unsigned long long)d, k);
    const float g = std::strtof(buf, nullptr);
    uint32_t a, b;
    std::memcpy(&a, &g, 4);
    std::memcpy(&b, &f, 4);
    return a == b;
}

}  // namespace

// Shortest round-trip digits of a finite nonzero |f|: f == digits * 10^exp10,
// digits without trailing zeros.
void shortest_f32(float f, uint32_t* digits, int* exp10) {
    const float a = std::fabs(f);
    for (int p = 1; p <= 9; ++p) {
        char buf[64];
        std::snprintf(buf, sizeof(buf), "%.*e", p - 1, (double)a);
        // d.ddde[+-]xx -> integer digits and the exponent of the last digit
        uint64_t d = 0;
        const char* s = buf;
        for (; *s && *s != 'e'; ++s)
            if (*s >= '0' && *s <= '9') d = d * 10 + (uint64_t)(*s - '0');
        const int e = std::atoi(s + 1);
        const int k = e - (p - 1);
        uint64_t hit = 0;
        int hk = k;
        if (reads_back(d, k, a)) {
            hit = d;
        } else {
            // the neighbour on the far side of the value
            char vb[64];
            std::snprintf(vb, sizeof(vb), "%llue%d", (unsigned long long)d, k);
            const double dv = std::strtod(vb, nullptr);  // the decimal, to the nearest double
            // the decimal and the f32 differ by far more than a double's ulp
            const uint64_t other = dv > (double)a ? d - 1 : d + 1;
            if (other > 0 && reads_back(other, k, a)) hit = other;
        }
        if (hit) {
            while (hit % 10 == 0) {
                hit /= 10;
                ++hk;
            }
            *digits = (uint32_t)hit;
            *exp10 = hk;
            return;
        }
    }
    // unreachable: 9 significant digits always identify an f32
    *digits = 0;
    *exp10 = 0;
}

size_t format_f32(float f, char* out) {
    if (!std::isfinite(f)) {
        std::memcpy(out, "null", 4);
        return 4;
    }
    size_t n = 0;
    if (std::signbit(f)) out[n++] = '-';
    if (f == 0.0f) {
        std::memcpy(out + n, "0.0", 3);
        return n + 3;
    }
    uint32_t d;
    int k;
    shortest_f32(f, &d, &k);
    char dig[16];
    const int len = std::snprintf(dig, sizeof(dig), "%u", d);
    const int kk = len + k;
    if (k >= 0 && kk <= 13) {
        std::memcpy(out + n, dig, len);
        n += len;
        for (int i = len; i < kk; ++i) out[n++] = '0';
        out[n++] = '.';
        out[n++] = '0';
    } else if (kk > 0 && kk <= 13) {
        std::memcpy(out + n, dig, kk);
        n += kk;
        out[n++] = '.';
        std::memcpy(out + n, dig + kk, len - kk);
        n += len - kk;
    } else if (kk > -6 && kk <= 0) {
        out[n++] = '0';
        out[n++] = '.';
        for (int i = 0; i < -kk; ++i) out[n++] = '0';
        std::memcpy(out + n, dig, len);
        n += len;
    } else {
        out[n++] = dig[0];
        if (len > 1) {
            out[n++] = '.';
            std::memcpy(out + n, dig + 1, len - 1);
            n += len - 1;
        }
        n += std::snprintf(out + n, 8, "e%d", kk - 1);
    }
    return n;
}

namespace {

struct Writer {
    std::string s;
    uint64_t non_finite = 0;
    void raw(const char* t) { s += t; }
    void f32(float v) {
        char b[32];
        if (!std::isfinite(v)) ++non_finite;
        s.append(b, format_f32(v, b));
    }
    void u(uint64_t v) { s += std::to_string(v); }
};

}  // namespace
}  // namespace v3do

using namespace v3do;

extern "C" {

// Shortest digits and exponent (returns 1 for finite nonzero input, else 0).
int32_t v3do_shortest_f32(float f, uint32_t* digits, int32_t* exp10) {
    if (!std::isfinite(f) || f == 0.0f) return 0;
    int k;
    shortest_f32(f, digits, &k);
    *exp10 = k;
    return 1;
}

uint64_t v3do_format_f32(float f, char* out) { return format_f32(f, out); }

// The three arrays of DenseEvidence (reconstruction_stages.rs:250-256) in
// serde_json's compact form, framed like v3d_encode_dense_evidence; the digest
// is left zero (tests hash the document with hashlib).
int32_t v3do_encode_dense_evidence(const v3d_point* points, uint64_t n_points,
                                   const v3d_grid_site* sites, uint64_t n_sites,
                                   const v3d_point_attributes* attrs, uint64_t n_attrs,
                                   const char* prefix, uint64_t prefix_bytes, const char* suffix,
                                   uint64_t suffix_bytes, char* document, uint64_t capacity,
                                   v3d_dense_document* out) {
    if (!out || (n_points && !points) || (n_sites && !sites) || (n_attrs && !attrs))
        return V3D_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    Writer w;
    w.s.assign(prefix ? prefix : "", prefix ? prefix_bytes : 0);
    size_t mark = w.s.size();
    w.raw("[");
    for (uint64_t i = 0; i < n_points; ++i) {
        const v3d_point& p = points[i];
        w.raw(i ? ",{\"x\":" : "{\"x\":");
        w.f32(p.x);
        w.raw(",\"y\":");
        w.f32(p.y);
        w.raw(",\"z\":");
        w.f32(p.z);
        w.raw(",\"confidence\":");
        w.f32(p.confidence);
        w.raw(",\"r\":");
        w.u(p.r);
        w.raw(",\"g\":");
        w.u(p.g);
        w.raw(",\"b\":");
        w.u(p.b);
        w.raw("}");
    }
    w.raw("]");
    out->points_bytes = w.s.size() - mark;
    w.raw(",\"grid_sites\":");
    mark = w.s.size();
    w.raw("[");
    for (uint64_t i = 0; i < n_sites; ++i) {
        w.raw(i ? ",{\"x\":" : "{\"x\":");
        w.u(sites[i].x);
        w.raw(",\"y\":");
        w.u(sites[i].y);
        w.raw("}");
    }
    w.raw("]");
    out->grid_sites_bytes = w.s.size() - mark;
    w.raw(",\"point_attributes\":");
    mark = w.s.size();
    w.raw("[");
    for (uint64_t i = 0; i < n_attrs; ++i) {
        w.raw(i ? ",{\"reciprocal_consistency\":" : "{\"reciprocal_consistency\":");
        w.f32(attrs[i].reciprocal_consistency);
        w.raw(",\"depth_margin\":");
        w.f32(attrs[i].depth_margin);
        w.raw("}");
    }
    w.raw("]");
    out->point_attributes_bytes = w.s.size() - mark;
    if (suffix) w.s.append(suffix, suffix_bytes);
    out->document_bytes = w.s.size();
    out->non_finite = w.non_finite;
    if (w.s.size() > capacity || !document) return V3D_ERR_INVALID_ARGUMENT;
    std::memcpy(document, w.s.data(), w.s.size());
    return V3D_OK;
}

// pack_dense_points (crates/video-to-3d-wasm/src/lib.rs:227-240).
void v3do_pack_dense_points(const v3d_point* points, uint64_t n, uint8_t* values_f32_le,
                            uint8_t* rgb) {
    for (uint64_t i = 0; i < n; ++i) {
        const float v[4] = {points[i].x, points[i].y, points[i].z, points[i].confidence};
        for (int j = 0; j < 4; ++j) {
            uint32_t b;
            std::memcpy(&b, &v[j], 4);
            for (int q = 0; q < 4; ++q) values_f32_le[16 * i + 4 * j + q] = (uint8_t)(b >> (8 * q));
        }
        rgb[3 * i] = points[i].r;
        rgb[3 * i + 1] = points[i].g;
        rgb[3 * i + 2] = points[i].b;
    }
}

// pack_mesh_triangles (crates/video-to-3d-wasm/src/lib.rs:269-326), byte by
// byte; returns 0, or 1 + the index of the failing message (0 source range,
// 1 missing point, 2 point index range).
int32_t v3do_pack_mesh_triangles(const v3d_mesh_triangle* triangles, uint64_t nt,
                                 const v3d_triangle_source* sources, uint64_t ns,
                                 const v3d_derived_vertex_source* derived, uint64_t nd, uint64_t point_count,
                                 uint8_t* indices, uint8_t* confidence, uint8_t* src, uint8_t* der,
                                 uint8_t* bary) {
    auto le32 = [](uint8_t* at, uint64_t v) {
        for (int q = 0; q < 4; ++q) at[q] = (uint8_t)(v >> (8 * q));
    };
    auto le64 = [](uint8_t* at, uint64_t v) {
        for (int q = 0; q < 8; ++q) at[q] = (uint8_t)(v >> (8 * q));
    };
    size_t o = 0;
    for (uint64_t i = 0; i < ns; ++i) {
        const uint64_t v[4] = {sources[i].triangle, sources[i].corners[0], sources[i].corners[1],
                               sources[i].corners[2]};
        for (uint64_t x : v) {
            if (x > 0xFFFFFFFFull) return 1;
            le32(src + o, x);
            o += 4;
        }
    }
    o = 0;
    size_t ob = 0;
    for (uint64_t i = 0; i < nd; ++i) {
        const uint64_t v[5] = {derived[i].point_index, derived[i].source_triangle, derived[i].source_corners[0],
                               derived[i].source_corners[1], derived[i].source_corners[2]};
        for (uint64_t x : v) {
            if (x > 0xFFFFFFFFull) return 1;
            le32(der + o, x);
            o += 4;
        }
        for (double w : derived[i].barycentric) {
            uint64_t b;
            std::memcpy(&b, &w, 8);
            le64(bary + ob, b);
            ob += 8;
        }
    }
    o = 0;
    for (uint64_t t = 0; t < nt; ++t) {
        for (uint64_t x : {triangles[t].a, triangles[t].b, triangles[t].c}) {
            if (x >= point_count) return 2;
            if (x > 0xFFFFFFFFull) return 3;
            le32(indices + o, x);
            o += 4;
        }
        uint32_t c;
        std::memcpy(&c, &triangles[t].confidence, 4);
        le32(confidence + 4 * t, c);
    }
    return 0;
}

}  // extern "C"
