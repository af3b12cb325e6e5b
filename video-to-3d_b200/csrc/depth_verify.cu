// Geometric depth-grid verification on the device: the reference's
// verify_patch (colmap_surface.rs:175-275) of every reference grid sample
// against each of its source views, and verified_union
// (colmap_surface.rs:289-314) of the sources' verdicts, for many references in
// one pass, behind v3d_verify_depth_grids.
//
// A thread owns one reference grid sample and runs its source views in the
// grid's order, so the union needs no second pass: the point comes from the
// reference depth and colour (every verifying source agrees on it), the
// confidence is the largest agreement, and a bit per verifying source records
// which ones did.  Every f64 operation is an explicitly rounded intrinsic in the
// reference's order (nalgebra's left-to-right matrix-vector products, scalar
// chains left to right), rounding is half away from zero and float-to-integer
// casts saturate as Rust's do, so samples and funnel counts are the reference's
// bit for bit.  The outcome counts of each warp are reduced in registers and
// added with one atomic per counter.  Samples leave in grid order through an
// order-preserving compaction.
//
// The work is a gather: per (sample, source) a few dozen f64 operations, one
// depth read and two texel reads; frames and grids stay in L2.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/v3d_dense.h"
#include "host.hpp"
#include "pass_kernels.cuh"

namespace v3d {
namespace {

struct DevView {
    const uint8_t* rgba;
    const float* depth;
    double R[9];
    double t[3];
};

enum Outcome : int {
    kMissingReferenceDepth = 0,
    kInsufficientParallax,
    kBehindSource,
    kOutsideSource,
    kMissingSourceDepth,
    kDepthDisagreement,
    kColorDisagreement,
    kAccepted,
    kOutcomes
};

// nalgebra rotation * v and rotation.transpose() * v, rows left to right
__device__ __forceinline__ D3 rot(const double* R, D3 v) {
    return D3{dadd(dadd(dmul(R[0], v.x), dmul(R[1], v.y)), dmul(R[2], v.z)),
              dadd(dadd(dmul(R[3], v.x), dmul(R[4], v.y)), dmul(R[5], v.z)),
              dadd(dadd(dmul(R[6], v.x), dmul(R[7], v.y)), dmul(R[8], v.z))};
}
__device__ __forceinline__ D3 rot_t(const double* R, D3 v) {
    return D3{dadd(dadd(dmul(R[0], v.x), dmul(R[3], v.y)), dmul(R[6], v.z)),
              dadd(dadd(dmul(R[1], v.x), dmul(R[4], v.y)), dmul(R[7], v.z)),
              dadd(dadd(dmul(R[2], v.x), dmul(R[5], v.y)), dmul(R[8], v.z))};
}
// camera_center (multi_view.rs:92-94): the negated transpose times t
__device__ __forceinline__ D3 center_of(const DevView& v) {
    const double* R = v.R;
    return D3{dadd(dadd(dmul(-R[0], v.t[0]), dmul(-R[3], v.t[1])), dmul(-R[6], v.t[2])),
              dadd(dadd(dmul(-R[1], v.t[0]), dmul(-R[4], v.t[1])), dmul(-R[7], v.t[2])),
              dadd(dadd(dmul(-R[2], v.t[0]), dmul(-R[5], v.t[1])), dmul(-R[8], v.t[2]))};
}
__device__ __forceinline__ double dot3(D3 a, D3 b) {
    return dadd(dadd(dmul(a.x, b.x), dmul(a.y, b.y)), dmul(a.z, b.z));
}
__device__ __forceinline__ double norm3(D3 a) { return __dsqrt_rn(dot3(a, a)); }
__device__ __forceinline__ D3 sub3(D3 a, D3 b) { return D3{dsub(a.x, b.x), dsub(a.y, b.y), dsub(a.z, b.z)}; }
// Rust's `f64 as usize`: saturating, NaN to 0
__device__ __forceinline__ uint64_t as_usize(double v) {
    if (!(v > 0.0)) return 0;
    if (v >= 18446744073709551615.0) return ~0ull;
    return (uint64_t)v;
}

struct Params {
    const DevView* views;
    const uint32_t* ref_view;   // [n_refs]
    const int32_t* src_view;    // [n_refs][4]
    uint32_t n_refs, width, height, stride, rstride, cols, rows;
    double focal, cx, cy, min_cos;
};

// One reference grid sample against each of its sources (verify_patch), the
// union of the verdicts (verified_union).
__global__ void k_verify(Params p, v3d_verified_sample* __restrict__ slot, uint8_t* __restrict__ kept,
                         uint32_t* __restrict__ per_ref, unsigned long long* __restrict__ funnel) {
    const uint64_t cells = (uint64_t)p.cols * p.rows, total = cells * p.n_refs;
    uint32_t cnt[kOutcomes + 1] = {};  // [kOutcomes] = reference samples
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < total;
         g += (uint64_t)gridDim.x * blockDim.x) {
        kept[g] = 0;
        const uint32_t r = (uint32_t)(g / cells);
        const uint64_t i = g - (uint64_t)r * cells;
        const uint64_t x = (i % p.cols) * p.stride, y = (i / p.cols) * p.stride;
        if (x % p.rstride != 0 || y % p.rstride != 0) continue;
        const DevView& rv = p.views[p.ref_view[r]];
        const float z = rv.depth[i];
        const D3 ray{ddiv(dsub(dadd((double)x, 0.5), p.cx), p.focal),
                     ddiv(dsub(dadd((double)y, 0.5), p.cy), p.focal), 1.0};
        const double zd = (double)z;
        const D3 world = rot_t(rv.R, D3{dsub(dmul(ray.x, zd), rv.t[0]), dsub(dmul(ray.y, zd), rv.t[1]),
                                        dsub(dmul(ray.z, zd), rv.t[2])});
        const D3 ref_center = center_of(rv);
        const D3 direction = sub3(world, ref_center);
        const double dn = norm3(direction);
        const uint8_t* rp = rv.rgba + (y * p.width + x) * 4;
        const uchar4 rc = *reinterpret_cast<const uchar4*>(rp);
        float conf = 0.f;
        uint32_t mask = 0;
        for (int j = 0; j < 4; ++j) {
            const int32_t sv = p.src_view[4 * r + j];
            if (sv < 0) continue;
            ++cnt[kOutcomes];
            if (z <= 0.f) {
                ++cnt[kMissingReferenceDepth];
                continue;
            }
            const DevView& s = p.views[sv];
            const D3 from_source = sub3(world, center_of(s));
            if (dot3(direction, from_source) >= dmul(dmul(p.min_cos, dn), norm3(from_source))) {
                ++cnt[kInsufficientParallax];
                continue;
            }
            const D3 rq = rot(s.R, world);
            const D3 q{dadd(rq.x, s.t[0]), dadd(rq.y, s.t[1]), dadd(rq.z, s.t[2])};
            if (q.z <= 0.0) {
                ++cnt[kBehindSource];
                continue;
            }
            const double u = dsub(dadd(ddiv(dmul(p.focal, q.x), q.z), p.cx), 0.5);
            const double v = dsub(dadd(ddiv(dmul(p.focal, q.y), q.z), p.cy), 0.5);
            const uint64_t col = as_usize(round(ddiv(u, (double)p.stride)));
            const uint64_t row = as_usize(round(ddiv(v, (double)p.stride)));
            if (!(u >= 0.0 && u < (double)p.width) || !(v >= 0.0 && v < (double)p.height) ||
                col >= p.cols || row >= p.rows) {
                ++cnt[kOutsideSource];
                continue;
            }
            const double other = (double)s.depth[row * p.cols + col];
            if (other <= 0.0) {
                ++cnt[kMissingSourceDepth];
                continue;
            }
            const double diff = fabs(dsub(other, q.z));
            if (diff > dmul(0.02, q.z)) {
                ++cnt[kDepthDisagreement];
                continue;
            }
            const uint64_t sx = min(as_usize(round(u)), (uint64_t)p.width - 1);
            const uint64_t sy = min(as_usize(round(v)), (uint64_t)p.height - 1);
            const uchar4 sc = *reinterpret_cast<const uchar4*>(s.rgba + (sy * p.width + sx) * 4);
            const uint32_t err = (uint32_t)abs((int)rc.x - (int)sc.x) +
                                 (uint32_t)abs((int)rc.y - (int)sc.y) +
                                 (uint32_t)abs((int)rc.z - (int)sc.z);
            if (err > 105) {
                ++cnt[kColorDisagreement];
                continue;
            }
            ++cnt[kAccepted];
            const float c = (float)dsub(1.0, ddiv(diff, q.z));
            conf = mask ? fmaxf(conf, c) : c;
            mask |= 1u << j;
        }
        if (!mask) continue;
        v3d_verified_sample out;
        out.point = v3d_point{(float)world.x, (float)world.y, (float)world.z, conf, rc.x, rc.y, rc.z, 0};
        out.site = v3d_grid_site{(uint32_t)x, (uint32_t)y};
        out.source_mask = mask;
        slot[g] = out;
        kept[g] = 1;
        atomicAdd(&per_ref[r], 1u);
    }
    // the warp's counts, then one atomic per counter
#pragma unroll
    for (int k = 0; k <= kOutcomes; ++k) {
        uint32_t v = cnt[k];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0 && v) atomicAdd(&funnel[k], (unsigned long long)v);
    }
}

__global__ void k_gather_samples(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ count,
                                 const v3d_verified_sample* __restrict__ slot,
                                 v3d_verified_sample* __restrict__ out) {
    const uint32_t m = *count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
        out[k] = slot[idx[k]];
}

unsigned grid_of(uint64_t n) {
    uint64_t b = (n + 255) / 256;
    if (b > 148ull * 16) b = 148ull * 16;
    return (unsigned)std::max<uint64_t>(b, 1);
}

struct Carve {
    size_t off = 0;
    template <class T>
    size_t take(uint64_t count) {
        const size_t at = (off + 255) & ~size_t(255);
        off = at + sizeof(T) * std::max<uint64_t>(count, 1);
        return at;
    }
};

}  // namespace
}  // namespace v3d

using namespace v3d;


extern "C" int32_t v3d_verify_depth_grids(
    v3d_context* ctx, const v3d_depth_view* views, uint64_t n_views, const uint32_t* reference_views,
    uint64_t n_references, const int32_t* source_views, uint32_t stride, uint32_t reference_stride,
    double focal, v3d_verified_sample* samples, uint64_t capacity, uint64_t* sample_offsets,
    v3d_verification_funnel* funnel) {
    if (!ctx || !views || !n_views || (n_references && (!reference_views || !source_views)) ||
        !sample_offsets || !funnel || stride == 0 || reference_stride == 0 ||
        reference_stride % stride != 0)
        return V3D_ERR_INVALID_ARGUMENT;
    const uint32_t width = views[0].width, height = views[0].height;
    if (width == 0 || height == 0) return V3D_ERR_INVALID_ARGUMENT;
    for (uint64_t v = 0; v < n_views; ++v)
        if (views[v].width != width || views[v].height != height || !views[v].rgba || !views[v].depth)
            return V3D_ERR_INVALID_ARGUMENT;
    for (uint64_t r = 0; r < n_references; ++r) {
        if (reference_views[r] >= n_views) return V3D_ERR_INVALID_ARGUMENT;
        for (int j = 0; j < 4; ++j)
            if (source_views[4 * r + j] >= (int64_t)n_views) return V3D_ERR_INVALID_ARGUMENT;
    }
    const uint32_t cols = (width + stride - 1) / stride, rows = (height + stride - 1) / stride;
    const uint64_t cells = (uint64_t)cols * rows, total = cells * n_references;
    if (total >= 0xFFFFFFFFull) {
        ctx->last_error = "depth-grid verification takes fewer than 2^32 reference grid samples a call";
        return V3D_ERR_INVALID_ARGUMENT;
    }
    std::memset(funnel, 0, sizeof(*funnel));
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(ctx->stream);
    const uint64_t frame_bytes = (uint64_t)width * height * 4;

    Carve cv;
    std::vector<size_t> o_rgba(n_views), o_depth(n_views);
    for (uint64_t v = 0; v < n_views; ++v) {
        o_rgba[v] = cv.take<uint8_t>(frame_bytes);
        o_depth[v] = cv.take<float>(cells);
    }
    const size_t o_views = cv.take<DevView>(n_views), o_ref = cv.take<uint32_t>(n_references),
                 o_src = cv.take<int32_t>(4 * n_references),
                 o_slot = cv.take<v3d_verified_sample>(total), o_kept = cv.take<uint8_t>(total),
                 o_idx = cv.take<uint32_t>(total), o_out = cv.take<v3d_verified_sample>(total),
                 o_perref = cv.take<uint32_t>(n_references), o_funnel = cv.take<unsigned long long>(16),
                 o_count = cv.take<uint32_t>(4),
                 o_scratch = cv.take<uint8_t>(compaction_scratch_bytes(total));
    if (!ensure_arena(ctx, cv.off + 256)) {
        ctx->last_error = "device arena allocation failed";
        return V3D_ERR_OUT_OF_MEMORY;
    }
    char* base = static_cast<char*>(ctx->arena);
    auto at = [&](size_t o) { return base + o; };
    std::vector<DevView> hv(n_views);
    for (uint64_t v = 0; v < n_views; ++v) {
        V3D_CTX_CK(cudaMemcpyAsync(at(o_rgba[v]), views[v].rgba, frame_bytes, cudaMemcpyHostToDevice, st));
        V3D_CTX_CK(cudaMemcpyAsync(at(o_depth[v]), views[v].depth, sizeof(float) * cells,
                                cudaMemcpyHostToDevice, st));
        hv[v].rgba = reinterpret_cast<const uint8_t*>(at(o_rgba[v]));
        hv[v].depth = reinterpret_cast<const float*>(at(o_depth[v]));
        std::memcpy(hv[v].R, views[v].camera.rotation, sizeof(hv[v].R));
        std::memcpy(hv[v].t, views[v].camera.translation, sizeof(hv[v].t));
    }
    V3D_CTX_CK(cudaMemcpyAsync(at(o_views), hv.data(), sizeof(DevView) * n_views, cudaMemcpyHostToDevice, st));
    if (n_references) {
        V3D_CTX_CK(cudaMemcpyAsync(at(o_ref), reference_views, sizeof(uint32_t) * n_references,
                                cudaMemcpyHostToDevice, st));
        V3D_CTX_CK(cudaMemcpyAsync(at(o_src), source_views, sizeof(int32_t) * 4 * n_references,
                                cudaMemcpyHostToDevice, st));
    }
    auto* d_slot = reinterpret_cast<v3d_verified_sample*>(at(o_slot));
    auto* d_kept = reinterpret_cast<uint8_t*>(at(o_kept));
    auto* d_idx = reinterpret_cast<uint32_t*>(at(o_idx));
    auto* d_out = reinterpret_cast<v3d_verified_sample*>(at(o_out));
    auto* d_perref = reinterpret_cast<uint32_t*>(at(o_perref));
    auto* d_funnel = reinterpret_cast<unsigned long long*>(at(o_funnel));
    auto* d_count = reinterpret_cast<uint32_t*>(at(o_count));
    V3D_CTX_CK(cudaMemsetAsync(d_perref, 0, sizeof(uint32_t) * std::max<uint64_t>(n_references, 1), st));
    V3D_CTX_CK(cudaMemsetAsync(d_funnel, 0, sizeof(unsigned long long) * 16, st));
    V3D_CTX_CK(cudaMemsetAsync(d_count, 0, sizeof(uint32_t) * 4, st));

    Params p;
    p.views = reinterpret_cast<const DevView*>(at(o_views));
    p.ref_view = reinterpret_cast<const uint32_t*>(at(o_ref));
    p.src_view = reinterpret_cast<const int32_t*>(at(o_src));
    p.n_refs = (uint32_t)n_references;
    p.width = width;
    p.height = height;
    p.stride = stride;
    p.rstride = reference_stride;
    p.cols = cols;
    p.rows = rows;
    p.focal = focal;
    p.cx = (double)width / 2.0;
    p.cy = (double)height / 2.0;
    p.min_cos = std::cos(0.5 * (3.141592653589793 / 180.0));  // 0.5_f64.to_radians().cos()

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
    if (total) {
        V3D_COUNTED k_verify<<<grid_of(total), 256, 0, st>>>(p, d_slot, d_kept, d_perref, d_funnel);
        V3D_CTX_CK(cudaGetLastError());
    }
    V3D_CTX_CK(launch_compact(d_kept, 1, total, d_idx, d_count, at(o_scratch), st));
    V3D_COUNTED k_gather_samples<<<grid_of(total), 256, 0, st>>>(d_idx, d_count, d_slot, d_out);
    V3D_CTX_CK(cudaGetLastError());
    cudaEventRecord(ev1, st);
    std::vector<uint32_t> per_ref(std::max<uint64_t>(n_references, 1));
    unsigned long long f[16];
    uint32_t n_out = 0;
    V3D_CTX_CK(cudaMemcpyAsync(per_ref.data(), d_perref, sizeof(uint32_t) * per_ref.size(),
                            cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaMemcpyAsync(f, d_funnel, sizeof(f), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaMemcpyAsync(&n_out, d_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaStreamSynchronize(st));
    if (n_out > capacity) {
        ctx->last_error = "verified samples exceed the caller's capacity";
        return V3D_ERR_INVALID_ARGUMENT;
    }
    if (n_out) {
        if (!samples) return V3D_ERR_INVALID_ARGUMENT;
        V3D_CTX_CK(cudaMemcpyAsync(samples, d_out, sizeof(v3d_verified_sample) * n_out,
                                cudaMemcpyDeviceToHost, st));
        V3D_CTX_CK(cudaStreamSynchronize(st));
    }
    uint64_t k = 0;
    for (uint64_t r = 0; r < n_references; ++r) {
        sample_offsets[r] = k;
        k += per_ref[r];
    }
    sample_offsets[n_references] = k;
    funnel->reference_samples = f[kOutcomes];
    funnel->missing_reference_depth = f[kMissingReferenceDepth];
    funnel->insufficient_parallax = f[kInsufficientParallax];
    funnel->behind_source = f[kBehindSource];
    funnel->outside_source = f[kOutsideSource];
    funnel->missing_source_depth = f[kMissingSourceDepth];
    funnel->depth_disagreement = f[kDepthDisagreement];
    funnel->color_disagreement = f[kColorDisagreement];
    funnel->accepted = f[kAccepted];
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess) ctx->last_ms = ms;
    ctx->last_launches = g_kernel_launches - launches0;
    return V3D_OK;
}
