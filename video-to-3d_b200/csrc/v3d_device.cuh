// Device-side types and arithmetic of the dense plane-sweep pass.
//
// Two arithmetic policies evaluate a window cost:
//  * exact: every tap in f64 through the reference's own formulas
//    (dense_legacy.rs:996-1029 unproject/project, 1113-1127 bilinear,
//    1032-1095 patch_error), written with __dadd_rn/__dmul_rn/__ddiv_rn so no
//    multiply-add is ever fused — the results are bit-identical to the
//    reference's IEEE f64 evaluation;
//  * fast: per-plane homographies composed in f64 on the host and applied in
//    f32 per tap, f32 bilinear samples and f32 window sums.
// Per-candidate geometry (hypothesis depths, unproject/project of the chosen
// point, fusion) always runs in exact f64.
#pragma once

#include <cuda_bf16.h>
#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

namespace v3d {

// Kernel launches enqueued by this host thread: every launch site counts
// itself with V3D_COUNTED, and a call reports the difference across it.
extern thread_local uint64_t g_kernel_launches;
#define V3D_COUNTED ++::v3d::g_kernel_launches;

constexpr int kMaxRadius = 4;
constexpr int kMaxTaps = (2 * kMaxRadius + 1) * (2 * kMaxRadius + 1);
constexpr int kMaxSources = 16;
constexpr int kMaxPlanes = 256;

// Reference constants that no profile changes (dense_legacy.rs:8-19).
constexpr double kMaxReciprocalRelativeDepthError = 0.08;
constexpr double kMaxFusionRelativePositionError = 0.08;
constexpr int kMinFusionObservations = 2;
constexpr int kMinSurfaceNeighbors = 3;
constexpr double kMaxSurfaceNeighborSpread = 0.06;
constexpr double kSurfaceCompletionConfidenceScale = 0.85;

enum StorageFormat : int32_t { kU8 = 0, kF32 = 1, kF16 = 2, kBF16 = 3 };

struct DevCamera {
    double R[9];  // world->camera rotation, row-major
    double t[3];
};

struct DevImage {
    const void* data;  // device pointer, tightly packed rows
    uint32_t width, height;
};

struct DevSource {
    DevCamera cam;
    DevImage img;
    double search_min, search_max;  // the source's own depth envelope
    // fast policy: ref pixel (x,y,1) -> source homogeneous pixel = A p + (1/d) b
    float fwd_A[9], fwd_b[3];
    // fast policy: source pixel -> reference homogeneous pixel = A p + (1/d) b
    float bwd_A[9], bwd_b[3];
};

struct DevReference {
    DevCamera cam;
    DevImage img;
    const uint8_t* rgba;  // reference RGBA8 frame, or nullptr for gray storage
    double focal;
    double search_min, search_max;
    uint32_t border, stride, nx, ny;
    int32_t n_src;
    int32_t planes;    // depth hypotheses of this reference (and of its sources' sweeps)
    uint64_t inv_off;  // first entry of its [kMaxSources][planes] table in BatchDev::src_inv
    DevSource src[kMaxSources];
};

struct DevProfile {
    int32_t cost;    // 0 ZSAD, 1 ZNCC
    int32_t radius;
    int32_t planes;  // the most depth hypotheses of any reference in the batch
    int32_t pad;
    double min_contrast, max_error, min_margin, margin_saturation, error_scale, min_variance;
};

// ---- exact f64 arithmetic (never contracted) ------------------------------
__device__ __forceinline__ double dadd(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double dsub(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dmul(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double ddiv(double a, double b) { return __ddiv_rn(a, b); }

struct D3 {
    double x, y, z;
};

__device__ __forceinline__ bool finite3(D3 v) {
    return isfinite(v.x) && isfinite(v.y) && isfinite(v.z);
}

// unproject (dense_legacy.rs:996-1011): R^T ((x - w/2)/f*d, (y - h/2)/f*d, d) - t)
__device__ __forceinline__ D3 unproject_exact(const DevCamera& c, double x, double y, double depth,
                                              uint32_t w, uint32_t h, double focal) {
    double cx = dmul(ddiv(dsub(x, dmul((double)w, 0.5)), focal), depth);
    double cy = dmul(ddiv(dsub(y, dmul((double)h, 0.5)), focal), depth);
    double dx = dsub(cx, c.t[0]), dy = dsub(cy, c.t[1]), dz = dsub(depth, c.t[2]);
    D3 r;
    r.x = dadd(dadd(dmul(c.R[0], dx), dmul(c.R[3], dy)), dmul(c.R[6], dz));
    r.y = dadd(dadd(dmul(c.R[1], dx), dmul(c.R[4], dy)), dmul(c.R[7], dz));
    r.z = dadd(dadd(dmul(c.R[2], dx), dmul(c.R[5], dy)), dmul(c.R[8], dz));
    return r;
}

// project (dense_legacy.rs:1013-1029); returns false where the reference returns None.
__device__ __forceinline__ bool project_exact(const DevCamera& c, D3 p, uint32_t w, uint32_t h,
                                              double focal, D3& out) {
    double x = dadd(dadd(dadd(dmul(c.R[0], p.x), dmul(c.R[1], p.y)), dmul(c.R[2], p.z)), c.t[0]);
    double y = dadd(dadd(dadd(dmul(c.R[3], p.x), dmul(c.R[4], p.y)), dmul(c.R[5], p.z)), c.t[1]);
    double z = dadd(dadd(dadd(dmul(c.R[6], p.x), dmul(c.R[7], p.y)), dmul(c.R[8], p.z)), c.t[2]);
    if (!(isfinite(x) && isfinite(y) && isfinite(z)) || z <= 1.0e-4) return false;
    out.x = dadd(ddiv(dmul(focal, x), z), dmul((double)w, 0.5));
    out.y = dadd(ddiv(dmul(focal, y), z), dmul((double)h, 0.5));
    out.z = z;
    return true;
}

__device__ __forceinline__ bool in_bilinear_bounds(double x, double y, uint32_t w, uint32_t h) {
    double wm = w > 0 ? (double)(w - 1) : 0.0;
    double hm = h > 0 ? (double)(h - 1) : 0.0;
    return isfinite(x) && isfinite(y) && x >= 0.0 && y >= 0.0 && x < wm && y < hm;
}

// hypothesis depth (dense_legacy.rs:286-293)
__device__ __forceinline__ double hypothesis_depth(int k, int count, double mn, double mx) {
    double t = count == 1 ? 0.0 : ddiv((double)k, (double)(count - 1));
    double inv = dadd(dmul(ddiv(1.0, mn), dsub(1.0, t)), dmul(ddiv(1.0, mx), t));
    return ddiv(1.0, inv);
}

__device__ __forceinline__ double clampd(double v, double lo, double hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}

// ---- pixel access -----------------------------------------------------------
template <class T>
__device__ __forceinline__ float pix(const T* p, size_t i);
template <>
__device__ __forceinline__ float pix<uint8_t>(const uint8_t* p, size_t i) {
    return (float)__ldg(p + i);
}
template <>
__device__ __forceinline__ float pix<float>(const float* p, size_t i) {
    return __ldg(p + i);
}
template <>
__device__ __forceinline__ float pix<__half>(const __half* p, size_t i) {
    return __half2float(__ldg(p + i));
}
template <>
__device__ __forceinline__ float pix<__nv_bfloat16>(const __nv_bfloat16* p, size_t i) {
    return __bfloat162float(__ldg(p + i));
}

// sample_bilinear (dense_legacy.rs:1113-1127) in exact f64.
template <class T>
__device__ __forceinline__ bool sample_exact(const DevImage& img, double x, double y, double& v) {
    if (!in_bilinear_bounds(x, y, img.width, img.height)) return false;
    const T* p = static_cast<const T*>(img.data);
    uint32_t x0 = (uint32_t)floor(x), y0 = (uint32_t)floor(y);
    double tx = dsub(x, (double)x0), ty = dsub(y, (double)y0);
    size_t r0 = (size_t)y0 * img.width, r1 = r0 + img.width;
    double v00 = pix<T>(p, r0 + x0), v10 = pix<T>(p, r0 + x0 + 1);
    double v01 = pix<T>(p, r1 + x0), v11 = pix<T>(p, r1 + x0 + 1);
    double top = dadd(dmul(v00, dsub(1.0, tx)), dmul(v10, tx));
    double bot = dadd(dmul(v01, dsub(1.0, tx)), dmul(v11, tx));
    v = dadd(dmul(top, dsub(1.0, ty)), dmul(bot, ty));
    return true;
}

// f32 bilinear sample; the caller guarantees 0 <= x < w-1, 0 <= y < h-1.
template <class T>
__device__ __forceinline__ float sample_fast(const T* p, uint32_t w, float x, float y) {
    float fx = floorf(x), fy = floorf(y);
    int x0 = (int)fx, y0 = (int)fy;
    float tx = x - fx, ty = y - fy;
    size_t r0 = (size_t)y0 * w + x0;
    float v00 = pix<T>(p, r0), v10 = pix<T>(p, r0 + 1);
    float v01 = pix<T>(p, r0 + w), v11 = pix<T>(p, r0 + w + 1);
    float top = fmaf(v10 - v00, tx, v00);
    float bot = fmaf(v11 - v01, tx, v01);
    return fmaf(bot - top, ty, top);
}

__device__ __forceinline__ bool in_bounds_fast(float x, float y, uint32_t w, uint32_t h) {
    // NaN fails every comparison
    return x >= 0.0f && y >= 0.0f && x < (float)(w - 1) && y < (float)(h - 1);
}

// patch_contrast (dense_legacy.rs:1097-1111) in exact f64: max - min of the
// (2r+1)^2 bilinear samples, 0 when any sample is out of bounds.
template <class T>
__device__ double patch_contrast_exact(const DevImage& img, double x, double y, int r) {
    double mn = __longlong_as_double(0x7ff0000000000000LL);
    double mx = -mn;
    for (int dy = -r; dy <= r; ++dy)
        for (int dx = -r; dx <= r; ++dx) {
            double v;
            if (!sample_exact<T>(img, dadd(x, (double)dx), dadd(y, (double)dy), v)) return 0.0;
            mn = fmin(mn, v);
            mx = fmax(mx, v);
        }
    return dsub(mx, mn);
}

// ---- exact window cost --------------------------------------------------------
// patch_error (dense_legacy.rs:1032-1095): ZSAD, or the profile's ZNCC cost
// 1 - cov/sqrt(var_r var_s) with the variance floor.  Two passes over the taps
// (sums, then centred sums) recompute the deterministic samples instead of
// storing them.
template <class T>
__device__ bool tap_exact(const DevCamera& rc, const DevImage& ri, const DevCamera& sc,
                          const DevImage& si, double focal, double x, double y, double depth,
                          int dx, int dy, double& rv, double& sv) {
    double rx = dadd(x, (double)dx), ry = dadd(y, (double)dy);
    D3 world = unproject_exact(rc, rx, ry, depth, ri.width, ri.height, focal);
    D3 s;
    if (!project_exact(sc, world, si.width, si.height, focal, s)) return false;
    if (!in_bilinear_bounds(s.x, s.y, si.width, si.height)) return false;
    if (!sample_exact<T>(ri, rx, ry, rv)) return false;
    if (!sample_exact<T>(si, s.x, s.y, sv)) return false;
    return true;
}

template <class T>
__device__ bool patch_error_exact(const DevProfile& prof, const DevCamera& rc, const DevImage& ri,
                                  const DevCamera& sc, const DevImage& si, double focal, double x,
                                  double y, double depth, double& cost) {
    const int r = prof.radius;
    double sr = 0.0, ss = 0.0;
    int n = 0;
    for (int dy = -r; dy <= r; ++dy)
        for (int dx = -r; dx <= r; ++dx) {
            double a, b;
            if (!tap_exact<T>(rc, ri, sc, si, focal, x, y, depth, dx, dy, a, b)) return false;
            sr = dadd(sr, a);
            ++n;
        }
    // second accumulation in the reference's order: all r first, then all s
    for (int dy = -r; dy <= r; ++dy)
        for (int dx = -r; dx <= r; ++dx) {
            double a, b;
            tap_exact<T>(rc, ri, sc, si, focal, x, y, depth, dx, dy, a, b);
            ss = dadd(ss, b);
        }
    double dn = (double)n;
    double mr = ddiv(sr, dn), ms = ddiv(ss, dn);
    if (prof.cost == 0) {
        double acc = 0.0;
        for (int dy = -r; dy <= r; ++dy)
            for (int dx = -r; dx <= r; ++dx) {
                double a, b;
                tap_exact<T>(rc, ri, sc, si, focal, x, y, depth, dx, dy, a, b);
                acc = dadd(acc, fabs(dsub(dsub(a, mr), dsub(b, ms))));
            }
        cost = ddiv(acc, dn);
        return true;
    }
    double cov = 0.0, vr = 0.0, vs = 0.0;
    for (int dy = -r; dy <= r; ++dy)
        for (int dx = -r; dx <= r; ++dx) {
            double a, b;
            tap_exact<T>(rc, ri, sc, si, focal, x, y, depth, dx, dy, a, b);
            double da = dsub(a, mr), db = dsub(b, ms);
            cov = dadd(cov, dmul(da, db));
            vr = dadd(vr, dmul(da, da));
            vs = dadd(vs, dmul(db, db));
        }
    if (!(vr > 0.0) || !(vs > 0.0) || ddiv(vr, dn) < prof.min_variance ||
        ddiv(vs, dn) < prof.min_variance)
        return false;
    cost = dsub(1.0, ddiv(cov, __dsqrt_rn(dmul(vr, vs))));
    return true;
}

// ---- running best / comparable-second state -------------------------------
// The reference sorts candidates by (support desc, error asc, depth asc) and
// takes the first candidate with the best's support after it
// (dense_legacy.rs:332-362).  Hypotheses are visited in increasing depth, so
// a running state with plane index as the final tie-break reproduces the
// sort; `merge` combines states over disjoint plane sets.
struct Rank {
    int support;    // -1: no candidate
    int plane;
    double error;
    double second;  // best error among the other candidates with the same support
};

__device__ __forceinline__ Rank rank_empty() {
    Rank r;
    r.support = -1;
    r.plane = 0x7fffffff;
    r.error = 0.0;
    r.second = __longlong_as_double(0x7ff0000000000000LL);
    return r;
}

__device__ __forceinline__ bool rank_before(const Rank& a, const Rank& b) {
    if (a.error != b.error) return a.error < b.error;
    return a.plane < b.plane;
}

__device__ __forceinline__ Rank rank_merge(const Rank& a, const Rank& b) {
    if (a.support > b.support) return a;
    if (b.support > a.support) return b;
    if (a.support < 0) return a;
    Rank w = rank_before(a, b) ? a : b;
    const Rank& l = rank_before(a, b) ? b : a;
    w.second = fmin(fmin(a.second, b.second), l.error);
    return w;
}

__device__ __forceinline__ Rank rank_shfl_merge(Rank r, int offset) {
    Rank o;
    o.support = __shfl_down_sync(0xffffffffu, r.support, offset);
    o.plane = __shfl_down_sync(0xffffffffu, r.plane, offset);
    o.error = __shfl_down_sync(0xffffffffu, r.error, offset);
    o.second = __shfl_down_sync(0xffffffffu, r.second, offset);
    return rank_merge(r, o);
}

// k-th smallest (k = n/2, the reference's quantile(., 0.5) index round((n-1)/2))
// of up to kMaxSources values held in a small array.
template <class F>
__device__ __forceinline__ F median_of(F* v, int n) {
    for (int i = 1; i < n; ++i) {
        F x = v[i];
        int j = i - 1;
        while (j >= 0 && v[j] > x) {
            v[j + 1] = v[j];
            --j;
        }
        v[j + 1] = x;
    }
    return v[n / 2];
}

}  // namespace v3d
