// Geometry of the connected-surface merge (surface_merge.rs,
// surface_merge_clip.rs, surface_merge_stitch.rs), shared by its device
// kernels and its host stages so both evaluate every f64 expression in the
// same order: nalgebra's (3-vector dot (x*x + y*y) + z*z, 3x3 products column
// by column), every multiply and add rounded separately (the device side
// through explicitly rounded intrinsics, the host side compiled with
// -ffp-contract=off).
#pragma once

#include <cmath>
#include <cstdint>
#include <cstring>

#ifdef __CUDACC__
#define MG_HD __host__ __device__ __forceinline__
#else
#define MG_HD inline
#endif

namespace v3d {
namespace mg {

#ifdef __CUDA_ARCH__
MG_HD double mul(double a, double b) { return __dmul_rn(a, b); }
MG_HD double add(double a, double b) { return __dadd_rn(a, b); }
MG_HD double sub(double a, double b) { return __dsub_rn(a, b); }
MG_HD double dvd(double a, double b) { return __ddiv_rn(a, b); }
MG_HD double sqr(double a) { return __dsqrt_rn(a); }
#else
MG_HD double mul(double a, double b) { return a * b; }
MG_HD double add(double a, double b) { return a + b; }
MG_HD double sub(double a, double b) { return a - b; }
MG_HD double dvd(double a, double b) { return a / b; }
MG_HD double sqr(double a) { return std::sqrt(a); }
#endif

constexpr double kGeomEps = 1.0e-9;  // GEOMETRIC_EPSILON, surface_merge.rs:57
constexpr double kF64Eps = 2.220446049250313e-16;
constexpr double kF64MinPositive = 2.2250738585072014e-308;

struct V2 {
    double x, y;
};
struct V3 {
    double x, y, z;
};

MG_HD V2 v2(double x, double y) { return V2{x, y}; }
MG_HD V2 operator+(V2 a, V2 b) { return V2{add(a.x, b.x), add(a.y, b.y)}; }
MG_HD V2 operator-(V2 a, V2 b) { return V2{sub(a.x, b.x), sub(a.y, b.y)}; }
MG_HD V2 operator*(V2 a, double s) { return V2{mul(a.x, s), mul(a.y, s)}; }
MG_HD V2 operator/(V2 a, double s) { return V2{dvd(a.x, s), dvd(a.y, s)}; }
MG_HD double cross2(V2 a, V2 b) { return sub(mul(a.x, b.y), mul(a.y, b.x)); }
MG_HD double dot2(V2 a, V2 b) { return add(mul(a.x, b.x), mul(a.y, b.y)); }
MG_HD double norm2(V2 a) { return sqr(add(mul(a.x, a.x), mul(a.y, a.y))); }

MG_HD V3 operator+(V3 a, V3 b) { return V3{add(a.x, b.x), add(a.y, b.y), add(a.z, b.z)}; }
MG_HD V3 operator-(V3 a, V3 b) { return V3{sub(a.x, b.x), sub(a.y, b.y), sub(a.z, b.z)}; }
MG_HD V3 operator*(V3 a, double s) { return V3{mul(a.x, s), mul(a.y, s), mul(a.z, s)}; }
MG_HD double dot3(V3 a, V3 b) { return add(add(mul(a.x, b.x), mul(a.y, b.y)), mul(a.z, b.z)); }
MG_HD double norm3(V3 a) { return sqr(dot3(a, a)); }
MG_HD V3 cross3(V3 a, V3 b) {
    return V3{sub(mul(a.y, b.z), mul(a.z, b.y)), sub(mul(a.z, b.x), mul(a.x, b.z)),
              sub(mul(a.x, b.y), mul(a.y, b.x))};
}

// f64::signum (+0.0 -> 1.0, -0.0 -> -1.0)
MG_HD double signum(double v) {
    if (v != v) return v;
#ifdef __CUDA_ARCH__
    return signbit(v) ? -1.0 : 1.0;
#else
    return std::signbit(v) ? -1.0 : 1.0;
#endif
}
MG_HD double fmin_(double a, double b) { return fmin(a, b); }
MG_HD double fmax_(double a, double b) { return fmax(a, b); }

// ReferenceCamera::project (surface_merge.rs:109-118): x_cam = R x + t.
struct Cam {
    double R[9];
    double t[3];
};
MG_HD V3 to_camera(const Cam& c, V3 p) {
    V3 r;
    r.x = add(add(mul(c.R[0], p.x), mul(c.R[1], p.y)), mul(c.R[2], p.z));
    r.y = add(add(mul(c.R[3], p.x), mul(c.R[4], p.y)), mul(c.R[5], p.z));
    r.z = add(add(mul(c.R[6], p.x), mul(c.R[7], p.y)), mul(c.R[8], p.z));
    return V3{add(r.x, c.t[0]), add(r.y, c.t[1]), add(r.z, c.t[2])};
}
// image (x, y) and depth; false behind the camera or not finite
MG_HD bool project(const Cam& c, V3 p, double& ix, double& iy, double& depth) {
    V3 q = to_camera(c, p);
    if (!(q.z > kGeomEps) || !isfinite(q.x) || !isfinite(q.y) || !isfinite(q.z)) return false;
    ix = dvd(q.x, q.z);
    iy = dvd(q.y, q.z);
    depth = q.z;
    return true;
}

// A projected triangle: corners (x, y) in normalized image coordinates, depth.
struct PT {
    double x[3], y[3], z[3];
    MG_HD V2 p(int i) const { return V2{x[i], y[i]}; }
};
MG_HD bool project_triangle(const Cam& c, const V3 corners[3], PT& out) {
    for (int i = 0; i < 3; ++i)
        if (!project(c, corners[i], out.x[i], out.y[i], out.z[i])) return false;
    return true;
}
MG_HD double image_area(const PT& t) {
    return fabs(cross2(t.p(1) - t.p(0), t.p(2) - t.p(0))) * 0.5;
}
MG_HD double signed_image_area(const PT& t) { return mul(cross2(t.p(1) - t.p(0), t.p(2) - t.p(0)), 0.5); }
// inverse_depth (surface_merge.rs:1653-1663); false for None
MG_HD bool inverse_depth(const PT& t, V2 point, double& out) {
    V2 a = t.p(0), b = t.p(1), c = t.p(2);
    double det = cross2(b - a, c - a);
    if (fabs(det) <= mul(kGeomEps, kGeomEps)) return false;
    double wb = dvd(cross2(point - a, c - a), det);
    double wc = dvd(cross2(b - a, point - a), det);
    double inv = add(add(dvd(sub(sub(1.0, wb), wc), t.z[0]), dvd(wb, t.z[1])), dvd(wc, t.z[2]));
    if (!(isfinite(inv) && inv > 0.0)) return false;
    out = inv;
    return true;
}
// the plane through the corners in camera coordinates (ReferenceCamera::plane)
MG_HD bool camera_plane(const Cam& c, const V3 corners[3], V3& normal, double& offset) {
    V3 a = to_camera(c, corners[0]), b = to_camera(c, corners[1]), d = to_camera(c, corners[2]);
    normal = cross3(b - a, d - a);
    if (!(norm3(normal) > kGeomEps)) return false;
    offset = dot3(normal, a);
    return true;
}

// ---- polygons in fixed storage (device and host) ---------------------------------
// A triangle clipped by three half-planes keeps at most 6 corners.
template <int CAP>
struct Poly {
    V2 v[CAP];
    int n = 0;
};

// polygon_area (surface_merge.rs:1875-1884)
template <int CAP>
MG_HD double poly_area(const Poly<CAP>& p) {
    if (p.n < 3) return 0.0;
    double s = -0.0;
    for (int i = 0; i < p.n; ++i) s = add(s, cross2(p.v[i], p.v[(i + 1) % p.n]));
    return fabs(s) * 0.5;
}

// split_polygon's included part (surface_merge.rs:1886-1913)
template <int CAP>
MG_HD void split_in(const Poly<CAP>& in, V2 a, V2 b, double orientation, Poly<CAP>& out) {
    out.n = 0;
    if (in.n == 0) return;
    const V2 ba = b - a;
    for (int i = 0; i < in.n; ++i) {
        V2 prev = in.v[(i + in.n - 1) % in.n], cur = in.v[i];
        double before = mul(orientation, cross2(ba, prev - a));
        double after = mul(orientation, cross2(ba, cur - a));
        if ((before < 0.0 && after > 0.0) || (before > 0.0 && after < 0.0)) {
            if (out.n < CAP) out.v[out.n] = prev + (cur - prev) * dvd(before, sub(before, after));
            ++out.n;
        }
        if (after >= 0.0) {
            if (out.n < CAP) out.v[out.n] = cur;
            ++out.n;
        }
    }
    if (out.n > CAP) out.n = CAP + 1;  // overflow marker: never reached for triangle clips
}

// The candidate triangle clipped to a kept triangle (Footprint::visit_overlaps,
// surface_merge.rs:1432-1452); false when the storage would overflow.
MG_HD bool clip_to_triangle(const PT& candidate, const PT& kept, Poly<8>& out) {
    Poly<8> a, b;
    a.n = 3;
    for (int i = 0; i < 3; ++i) a.v[i] = candidate.p(i);
    const double winding = cross2(kept.p(1) - kept.p(0), kept.p(2) - kept.p(0));
    const double o = signum(winding);
    Poly<8>* src = &a;
    Poly<8>* dst = &b;
    for (int e = 0; e < 3; ++e) {
        split_in(*src, kept.p(e), kept.p((e + 1) % 3), o, *dst);
        if (dst->n > 8) return false;
        Poly<8>* t = src;
        src = dst;
        dst = t;
        if (src->n == 0) break;
    }
    out = *src;
    return true;
}

// back_projected_area (surface_merge.rs:1628-1645)
template <int CAP>
MG_HD double back_projected_area(const Poly<CAP>& poly, V3 normal, double offset) {
    V3 lifted[CAP];
    for (int i = 0; i < poly.n; ++i) {
        V3 ray{poly.v[i].x, poly.v[i].y, 1.0};
        double along = dot3(normal, ray);
        if (!(fabs(along) > kGeomEps)) return 0.0;
        lifted[i] = ray * dvd(offset, along);
    }
    V3 sum{0.0, 0.0, 0.0};
    for (int i = 0; i < poly.n; ++i) sum = sum + cross3(lifted[i], lifted[(i + 1) % poly.n]);
    return norm3(sum) * 0.5;
}

// ---- LevelGrid cell arithmetic (surface_merge.rs:1704-1734) -----------------------------
constexpr int kMaxGridLevels = 48;
constexpr int64_t kMaxAnchorCellSpan = 3;

// Rust `f64 as i64`: saturating, NaN to 0
MG_HD int64_t sat_i64(double v) {
    if (v != v) return 0;
    if (v >= 9223372036854775807.0) return INT64_MAX;
    if (v <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)v;
}
MG_HD int64_t sat_sub(int64_t a, int64_t b) {
    if (b > 0 && a < INT64_MIN + b) return INT64_MIN;
    if (b < 0 && a > INT64_MAX + b) return INT64_MAX;
    return a - b;
}
// the cell range of [low, high] on one axis at `level`; false for None
MG_HD bool axis_range(double cell, int level, double low, double high, int64_t& first,
                      int64_t& last) {
    const double size = mul(cell, ldexp(1.0, level));
    double f = floor(dvd(low, size)), l = floor(dvd(high, size));
    if (!isfinite(f) || !isfinite(l) || f > l) return false;
    first = sat_i64(f);
    last = sat_i64(l);
    return true;
}

// A frozen 2-D grid (one footprint): buckets sorted by (level, x, y).
struct GridBucket {
    int64_t x, y;
    int32_t level;
    uint32_t start;  // into the footprint's item list; the bucket ends at the next start
};

MG_HD bool bucket_less(const GridBucket& b, int32_t level, int64_t x, int64_t y) {
    if (b.level != level) return b.level < level;
    if (b.x != x) return b.x < x;
    return b.y < y;
}

}  // namespace mg
}  // namespace v3d
