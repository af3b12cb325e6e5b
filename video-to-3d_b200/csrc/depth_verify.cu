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
#include <cub/device/device_radix_sort.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/v3d_dense.h"
#include "host.hpp"
#include "mesh_batch.cuh"
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
                         unsigned long long* __restrict__ funnel) {
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

// Samples per reference from the compacted slot list: slots are numbered
// reference by reference, so a reference's samples are the run between two
// lower bounds of the sorted list.
__global__ void k_ref_counts(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ count,
                             uint64_t cells, uint32_t n_refs, uint32_t* __restrict__ per_ref) {
    const uint32_t r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= n_refs) return;
    const uint32_t n = *count;
    auto lower = [&](uint64_t key) {
        uint32_t lo = 0, hi = n;
        while (lo < hi) {
            const uint32_t mid = lo + (hi - lo) / 2;
            if (idx[mid] < key) lo = mid + 1;
            else hi = mid;
        }
        return lo;
    };
    per_ref[r] = lower((uint64_t)(r + 1) * cells) - lower((uint64_t)r * cells);
}

__global__ void k_gather_samples(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ count,
                                 const v3d_verified_sample* __restrict__ slot,
                                 v3d_verified_sample* __restrict__ out) {
    const uint32_t m = *count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
        out[k] = slot[idx[k]];
}

// ---- the export's meshing of verified samples (colmap_surface.rs:380-471) ----

constexpr unsigned long long kUnused = ~0ull;  // first use of an input no triangle names
constexpr int kFirstUseBits = 40;              // keys 3 * triangle + corner stay below 2^34
constexpr uint32_t kNoRegion = 0xFFFFFFFFu;

struct SplitTables {
    const uint64_t* off;         // [n_refs + 1] first sample of each reference
    const int32_t* patch_of_ref; // [n_refs] meshed patch, -1 for none
    const uint64_t* moff;        // [n_patches] first mesh input of each patch
    uint32_t n_refs;
};

// The meshed references' samples as mesh inputs (point, site, patch,
// patch-local index, source bits), and the samples more than one source
// verified (every reference's, as the export counts them).
__global__ void k_split_samples(const v3d_verified_sample* __restrict__ s, const uint32_t* __restrict__ count,
                                SplitTables t, v3d_point* __restrict__ mp, v3d_grid_site* __restrict__ ms,
                                uint32_t* __restrict__ mpatch, uint32_t* __restrict__ mlocal,
                                uint32_t* __restrict__ mmask, unsigned long long* __restrict__ multiply) {
    const uint32_t n = *count;
    unsigned mult = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = t.n_refs;  // the last reference whose first sample is at or before i
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) / 2;
            if (t.off[mid] <= i) lo = mid;
            else hi = mid;
        }
        const v3d_verified_sample v = s[i];
        mult += __popc(v.source_mask) > 1 ? 1u : 0u;
        const int32_t p = t.patch_of_ref[lo];
        if (p >= 0) {
            const uint64_t local = i - t.off[lo], dst = t.moff[p] + local;
            mp[dst] = v.point;
            ms[dst] = v.site;
            mpatch[dst] = (uint32_t)p;
            mlocal[dst] = (uint32_t)local;
            mmask[dst] = v.source_mask;
        }
    }
    mult = __reduce_add_sync(0xFFFFFFFFu, mult);
    if ((threadIdx.x & 31) == 0 && mult) atomicAdd(multiply, (unsigned long long)mult);
}

// The first (triangle, corner) that names each mesh input; triangles are in
// patch order and each patch's in the reference's order.
__global__ void k_first_use(const v3d_mesh_triangle* __restrict__ tris, const uint32_t* __restrict__ tpatch,
                            uint64_t nt, const uint64_t* __restrict__ moff, unsigned long long* __restrict__ first) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nt;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const v3d_mesh_triangle tri = tris[t];
        const uint64_t base = moff[tpatch[t]];
        atomicMin(&first[base + tri.a], 3ull * t);
        atomicMin(&first[base + tri.b], 3ull * t + 1);
        atomicMin(&first[base + tri.c], 3ull * t + 2);
    }
}

__global__ void k_iota_retained(const unsigned long long* __restrict__ first, uint64_t n,
                                uint32_t* __restrict__ vals, unsigned long long* __restrict__ retained) {
    unsigned c = 0;
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < n; g += (uint64_t)gridDim.x * blockDim.x) {
        vals[g] = (uint32_t)g;
        c += first[g] != kUnused ? 1u : 0u;
    }
    c = __reduce_add_sync(0xFFFFFFFFu, c);
    if ((threadIdx.x & 31) == 0 && c) atomicAdd(retained, (unsigned long long)c);
}

// The retained inputs in first-use order become the exported points; each
// patch's run of them is its region.
__global__ void k_place(const uint32_t* __restrict__ order, const unsigned long long* __restrict__ retained,
                        const v3d_point* __restrict__ mp, const v3d_grid_site* __restrict__ ms,
                        const uint32_t* __restrict__ mpatch, const uint32_t* __restrict__ mmask,
                        uint32_t* __restrict__ new_index, v3d_point* __restrict__ out_p,
                        v3d_grid_site* __restrict__ out_s, uint32_t* __restrict__ mask_sorted,
                        uint32_t* __restrict__ region_first, uint32_t* __restrict__ region_end) {
    const uint64_t n = *retained;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < n; j += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t g = order[j], p = mpatch[g];
        new_index[g] = (uint32_t)j;
        out_p[j] = mp[g];
        out_s[j] = ms[g];
        mask_sorted[j] = mmask[g];
        if (j == 0 || mpatch[order[j - 1]] != p) region_first[p] = (uint32_t)j;
        if (j + 1 == n || mpatch[order[j + 1]] != p) region_end[p] = (uint32_t)(j + 1);
    }
}

// One block per patch: the union of the source bits of its region.
__global__ void __launch_bounds__(256) k_region_masks(const uint32_t* __restrict__ region_first,
                                                      const uint32_t* __restrict__ region_end,
                                                      const uint32_t* __restrict__ mask_sorted,
                                                      uint32_t* __restrict__ region_mask) {
    __shared__ uint32_t part[8];
    const uint32_t p = blockIdx.x, first = region_first[p];
    uint32_t m = 0;
    if (first != kNoRegion)
        for (uint32_t j = first + threadIdx.x; j < region_end[p]; j += blockDim.x) m |= mask_sorted[j];
    m = __reduce_or_sync(0xFFFFFFFFu, m);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t all = 0;
        for (int w = 0; w < 8; ++w) all |= part[w];
        region_mask[p] = all;
    }
}

__global__ void k_reindex(v3d_mesh_triangle* __restrict__ tris, const uint32_t* __restrict__ tpatch, uint64_t nt,
                          const uint64_t* __restrict__ moff, const uint32_t* __restrict__ new_index) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nt;
         t += (uint64_t)gridDim.x * blockDim.x) {
        v3d_mesh_triangle tri = tris[t];
        const uint64_t base = moff[tpatch[t]];
        tri.a = new_index[base + tri.a];
        tri.b = new_index[base + tri.b];
        tri.c = new_index[base + tri.c];
        tris[t] = tri;
    }
}

// ---- one verification: checks, arena layout, enqueue, read-back ----------

struct VerifyArgs {
    const v3d_depth_view* views;
    uint64_t n_views;
    const uint32_t* refs;
    uint64_t n_refs;
    const int32_t* srcs;
    uint32_t stride, rstride;
    double focal;
    uint32_t width = 0, height = 0, cols = 0, rows = 0;
    uint64_t cells = 0, total = 0;
};

int32_t verify_check(v3d_context* ctx, VerifyArgs& a) {
    if (!a.views || !a.n_views || (a.n_refs && (!a.refs || !a.srcs)) || a.stride == 0 || a.rstride == 0 ||
        a.rstride % a.stride != 0)
        return V3D_ERR_INVALID_ARGUMENT;
    a.width = a.views[0].width;
    a.height = a.views[0].height;
    if (a.width == 0 || a.height == 0) return V3D_ERR_INVALID_ARGUMENT;
    for (uint64_t v = 0; v < a.n_views; ++v)
        if (a.views[v].width != a.width || a.views[v].height != a.height || !a.views[v].rgba || !a.views[v].depth)
            return V3D_ERR_INVALID_ARGUMENT;
    for (uint64_t r = 0; r < a.n_refs; ++r) {
        if (a.refs[r] >= a.n_views) return V3D_ERR_INVALID_ARGUMENT;
        for (int j = 0; j < 4; ++j)
            if (a.srcs[4 * r + j] >= (int64_t)a.n_views) return V3D_ERR_INVALID_ARGUMENT;
    }
    a.cols = (a.width + a.stride - 1) / a.stride;
    a.rows = (a.height + a.stride - 1) / a.stride;
    a.cells = (uint64_t)a.cols * a.rows;
    a.total = a.cells * a.n_refs;
    if (a.total >= 0xFFFFFFFFull) {
        ctx->last_error = "depth-grid verification takes fewer than 2^32 reference grid samples a call";
        return V3D_ERR_INVALID_ARGUMENT;
    }
    return V3D_OK;
}

struct VerifyLayout {
    std::vector<size_t> o_rgba, o_depth;
    size_t o_views, o_ref, o_src, o_slot, o_kept, o_idx, o_out, o_perref, o_funnel, o_count, o_scratch;
};

void verify_layout(Carve& cv, const VerifyArgs& a, VerifyLayout& L) {
    const uint64_t frame_bytes = (uint64_t)a.width * a.height * 4;
    L.o_rgba.resize(a.n_views);
    L.o_depth.resize(a.n_views);
    for (uint64_t v = 0; v < a.n_views; ++v) {
        L.o_rgba[v] = cv.take<uint8_t>(frame_bytes);
        L.o_depth[v] = cv.take<float>(a.cells);
    }
    L.o_views = cv.take<DevView>(a.n_views);
    L.o_ref = cv.take<uint32_t>(a.n_refs);
    L.o_src = cv.take<int32_t>(4 * a.n_refs);
    L.o_slot = cv.take<v3d_verified_sample>(a.total);
    L.o_kept = cv.take<uint8_t>(a.total);
    L.o_idx = cv.take<uint32_t>(a.total);
    L.o_out = cv.take<v3d_verified_sample>(a.total);
    L.o_perref = cv.take<uint32_t>(a.n_refs);
    L.o_funnel = cv.take<unsigned long long>(16);
    L.o_count = cv.take<uint32_t>(4);
    L.o_scratch = cv.take<uint8_t>(compaction_scratch_bytes(a.total));
}

// Uploads the views and enqueues verify and union: the samples of every
// reference, in reference order and grid order, end compacted at o_out.
// `first_kernel` is recorded after the uploads.
int32_t verify_enqueue(v3d_context* ctx, char* base, const VerifyArgs& a, const VerifyLayout& L,
                       cudaEvent_t first_kernel, cudaStream_t st) {
    auto at = [&](size_t o) { return base + o; };
    const uint64_t frame_bytes = (uint64_t)a.width * a.height * 4;
    std::vector<DevView> hv(a.n_views);
    for (uint64_t v = 0; v < a.n_views; ++v) {
        V3D_CTX_CK(cudaMemcpyAsync(at(L.o_rgba[v]), a.views[v].rgba, frame_bytes, cudaMemcpyHostToDevice, st));
        V3D_CTX_CK(cudaMemcpyAsync(at(L.o_depth[v]), a.views[v].depth, sizeof(float) * a.cells,
                                   cudaMemcpyHostToDevice, st));
        hv[v].rgba = reinterpret_cast<const uint8_t*>(at(L.o_rgba[v]));
        hv[v].depth = reinterpret_cast<const float*>(at(L.o_depth[v]));
        std::memcpy(hv[v].R, a.views[v].camera.rotation, sizeof(hv[v].R));
        std::memcpy(hv[v].t, a.views[v].camera.translation, sizeof(hv[v].t));
    }
    V3D_CTX_CK(cudaMemcpyAsync(at(L.o_views), hv.data(), sizeof(DevView) * a.n_views, cudaMemcpyHostToDevice, st));
    if (a.n_refs) {
        V3D_CTX_CK(cudaMemcpyAsync(at(L.o_ref), a.refs, sizeof(uint32_t) * a.n_refs, cudaMemcpyHostToDevice, st));
        V3D_CTX_CK(cudaMemcpyAsync(at(L.o_src), a.srcs, sizeof(int32_t) * 4 * a.n_refs, cudaMemcpyHostToDevice, st));
    }
    auto* d_slot = reinterpret_cast<v3d_verified_sample*>(at(L.o_slot));
    auto* d_kept = reinterpret_cast<uint8_t*>(at(L.o_kept));
    auto* d_idx = reinterpret_cast<uint32_t*>(at(L.o_idx));
    auto* d_out = reinterpret_cast<v3d_verified_sample*>(at(L.o_out));
    auto* d_perref = reinterpret_cast<uint32_t*>(at(L.o_perref));
    auto* d_funnel = reinterpret_cast<unsigned long long*>(at(L.o_funnel));
    auto* d_count = reinterpret_cast<uint32_t*>(at(L.o_count));
    V3D_CTX_CK(cudaMemsetAsync(d_perref, 0, sizeof(uint32_t) * std::max<uint64_t>(a.n_refs, 1), st));
    V3D_CTX_CK(cudaMemsetAsync(d_funnel, 0, sizeof(unsigned long long) * 16, st));
    V3D_CTX_CK(cudaMemsetAsync(d_count, 0, sizeof(uint32_t) * 4, st));
    Params p;
    p.views = reinterpret_cast<const DevView*>(at(L.o_views));
    p.ref_view = reinterpret_cast<const uint32_t*>(at(L.o_ref));
    p.src_view = reinterpret_cast<const int32_t*>(at(L.o_src));
    p.n_refs = (uint32_t)a.n_refs;
    p.width = a.width;
    p.height = a.height;
    p.stride = a.stride;
    p.rstride = a.rstride;
    p.cols = a.cols;
    p.rows = a.rows;
    p.focal = a.focal;
    p.cx = (double)a.width / 2.0;
    p.cy = (double)a.height / 2.0;
    p.min_cos = std::cos(0.5 * (3.141592653589793 / 180.0));  // 0.5_f64.to_radians().cos()
    cudaEventRecord(first_kernel, st);
    if (a.total) {
        V3D_COUNTED k_verify<<<grid_of(a.total), 256, 0, st>>>(p, d_slot, d_kept, d_funnel);
        V3D_CTX_CK(cudaGetLastError());
    }
    V3D_CTX_CK(launch_compact(d_kept, 1, a.total, d_idx, d_count, at(L.o_scratch), st));
    if (a.n_refs) {
        V3D_COUNTED k_ref_counts<<<(unsigned)((a.n_refs + 255) / 256), 256, 0, st>>>(d_idx, d_count, a.cells,
                                                                                   (uint32_t)a.n_refs, d_perref);
        V3D_CTX_CK(cudaGetLastError());
    }
    V3D_COUNTED k_gather_samples<<<grid_of(a.total), 256, 0, st>>>(d_idx, d_count, d_slot, d_out);
    V3D_CTX_CK(cudaGetLastError());
    return V3D_OK;
}

struct VerifyCounts {
    std::vector<uint32_t> per_ref;
    uint32_t n_out = 0;
    v3d_verification_funnel funnel{};
};

int32_t verify_read(v3d_context* ctx, char* base, const VerifyArgs& a, const VerifyLayout& L, VerifyCounts& c,
                    cudaStream_t st) {
    c.per_ref.assign(std::max<uint64_t>(a.n_refs, 1), 0);
    unsigned long long f[16];
    V3D_CTX_CK(cudaMemcpyAsync(c.per_ref.data(), base + L.o_perref, sizeof(uint32_t) * c.per_ref.size(),
                               cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaMemcpyAsync(f, base + L.o_funnel, sizeof(f), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaMemcpyAsync(&c.n_out, base + L.o_count, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaStreamSynchronize(st));
    c.funnel.reference_samples = f[kOutcomes];
    c.funnel.missing_reference_depth = f[kMissingReferenceDepth];
    c.funnel.insufficient_parallax = f[kInsufficientParallax];
    c.funnel.behind_source = f[kBehindSource];
    c.funnel.outside_source = f[kOutsideSource];
    c.funnel.missing_source_depth = f[kMissingSourceDepth];
    c.funnel.depth_disagreement = f[kDepthDisagreement];
    c.funnel.color_disagreement = f[kColorDisagreement];
    c.funnel.accepted = f[kAccepted];
    return V3D_OK;
}

struct Events {
    cudaEvent_t a = nullptr, b = nullptr;
    Events() {
        cudaEventCreate(&a);
        cudaEventCreate(&b);
    }
    ~Events() {
        cudaEventDestroy(a);
        cudaEventDestroy(b);
    }
    float ms() const {
        float v = 0.f;
        return cudaEventElapsedTime(&v, a, b) == cudaSuccess ? v : 0.f;
    }
};

// VerificationFunnel::dominant_rejection (colmap_surface.rs:81-95): the
// largest count, ties to the smaller name; 1..7 in field order, 0 for none.
int32_t dominant_rejection(const v3d_verification_funnel& f) {
    const std::pair<const char*, uint64_t> c[7] = {
        {"missing_reference_depth", f.missing_reference_depth}, {"insufficient_parallax", f.insufficient_parallax},
        {"behind_source", f.behind_source},                     {"outside_source", f.outside_source},
        {"missing_source_depth", f.missing_source_depth},       {"depth_disagreement", f.depth_disagreement},
        {"color_disagreement", f.color_disagreement}};
    int32_t best = 0;
    for (int k = 0; k < 7; ++k) {
        if (c[k].second == 0) continue;
        if (!best || c[k].second > c[best - 1].second ||
            (c[k].second == c[best - 1].second && std::strcmp(c[k].first, c[best - 1].first) < 0))
            best = k + 1;
    }
    return best;
}

}  // namespace
}  // namespace v3d

using namespace v3d;

extern "C" int32_t v3d_verify_depth_grids(
    v3d_context* ctx, const v3d_depth_view* views, uint64_t n_views, const uint32_t* reference_views,
    uint64_t n_references, const int32_t* source_views, uint32_t stride, uint32_t reference_stride,
    double focal, v3d_verified_sample* samples, uint64_t capacity, uint64_t* sample_offsets,
    v3d_verification_funnel* funnel) {
    if (!ctx || !sample_offsets || !funnel) return V3D_ERR_INVALID_ARGUMENT;
    VerifyArgs a{views, n_views, reference_views, n_references, source_views, stride, reference_stride, focal};
    const int32_t checked = verify_check(ctx, a);
    if (checked != V3D_OK) return checked;
    std::memset(funnel, 0, sizeof(*funnel));
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(ctx->stream);
    Carve cv;
    VerifyLayout L;
    verify_layout(cv, a, L);
    if (!ensure_arena(ctx, cv.off + 256)) {
        ctx->last_error = "device arena allocation failed";
        return V3D_ERR_OUT_OF_MEMORY;
    }
    char* base = static_cast<char*>(ctx->arena);
    const uint64_t launches0 = g_kernel_launches;
    Events ev;
    int32_t status = verify_enqueue(ctx, base, a, L, ev.a, st);
    if (status != V3D_OK) return status;
    cudaEventRecord(ev.b, st);
    VerifyCounts c;
    status = verify_read(ctx, base, a, L, c, st);
    if (status != V3D_OK) return status;
    if (c.n_out > capacity) {
        ctx->last_error = "verified samples exceed the caller's capacity";
        return V3D_ERR_INVALID_ARGUMENT;
    }
    if (c.n_out) {
        if (!samples) return V3D_ERR_INVALID_ARGUMENT;
        V3D_CTX_CK(cudaMemcpyAsync(samples, base + L.o_out, sizeof(v3d_verified_sample) * c.n_out,
                                   cudaMemcpyDeviceToHost, st));
        V3D_CTX_CK(cudaStreamSynchronize(st));
    }
    uint64_t k = 0;
    for (uint64_t r = 0; r < n_references; ++r) {
        sample_offsets[r] = k;
        k += c.per_ref[r];
    }
    sample_offsets[n_references] = k;
    *funnel = c.funnel;
    ctx->last_ms = ev.ms();
    ctx->last_launches = g_kernel_launches - launches0;
    return V3D_OK;
}

extern "C" void v3d_verified_surface_bounds(uint32_t width, uint32_t height, uint32_t reference_stride,
                                            uint64_t n_references, uint64_t* max_points,
                                            uint64_t* max_triangles) {
    const uint32_t gw = reference_stride ? (width + reference_stride - 1) / reference_stride : 0;
    const uint32_t gh = reference_stride ? (height + reference_stride - 1) / reference_stride : 0;
    if (max_points) *max_points = n_references * gw * gh;
    if (max_triangles) *max_triangles = gw && gh ? n_references * mesh_slots(gw, gh) : 0;
}

extern "C" int32_t v3d_mesh_verified_depth_grids(
    v3d_context* ctx, const v3d_depth_view* views, uint64_t n_views, const uint32_t* reference_views,
    uint64_t n_references, const int32_t* source_views, uint32_t stride, uint32_t reference_stride,
    double focal, v3d_point* points, v3d_grid_site* sites, uint64_t point_capacity,
    v3d_mesh_triangle* triangles, uint64_t triangle_capacity, v3d_verified_surface_region* regions,
    v3d_verified_surface* out) {
    if (!ctx || !out) return V3D_ERR_INVALID_ARGUMENT;
    VerifyArgs a{views, n_views, reference_views, n_references, source_views, stride, reference_stride, focal};
    const int32_t checked = verify_check(ctx, a);
    if (checked != V3D_OK) return checked;
    for (uint64_t v = 0; v < n_views; ++v)
        for (uint64_t k = 0; k < v; ++k)
            if (views[k].camera.frame_index == views[v].camera.frame_index) {
                ctx->last_error = "views must have distinct camera frame indices";
                return V3D_ERR_INVALID_ARGUMENT;
            }
    std::memset(out, 0, sizeof(*out));
    const uint32_t gw = (a.width + reference_stride - 1) / reference_stride;
    const uint32_t gh = (a.height + reference_stride - 1) / reference_stride;
    const uint64_t cells_patch = (uint64_t)gw * gh, slots_patch = mesh_slots(gw, gh);
    const uint64_t ncap = n_references * cells_patch, total_cells = ncap, total_slots = n_references * slots_patch;
    // the radix sorts take int item counts: samples (and so n_mesh <= ncap) stay below 2^31
    if (ncap >= 0x7FFFFFFFull || 3 * total_slots >= (1ull << 34)) {
        ctx->last_error = "the verified surface takes fewer than 2^31 samples and 2^33 triangle slots a call";
        return V3D_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(ctx->stream);

    Carve cv;
    VerifyLayout L;
    verify_layout(cv, a, L);
    const size_t o_off = cv.take<uint64_t>(n_references + 1), o_por = cv.take<int32_t>(n_references),
                 o_moff = cv.take<uint64_t>(n_references + 1), o_mp = cv.take<v3d_point>(ncap),
                 o_ms = cv.take<v3d_grid_site>(ncap), o_mpatch = cv.take<uint32_t>(ncap),
                 o_mlocal = cv.take<uint32_t>(ncap), o_mmask = cv.take<uint32_t>(ncap),
                 o_ctr = cv.take<unsigned long long>(2),  // [0] multiply verified, [1] retained
                 o_mscr = cv.take<uint8_t>(mesh_scratch_layout(nullptr, (uint32_t)std::max<uint64_t>(n_references, 1),
                                                               ncap, total_cells, total_slots, nullptr)),
                 o_tris = cv.take<v3d_mesh_triangle>(total_slots), o_tpatch = cv.take<uint32_t>(total_slots),
                 o_first = cv.take<unsigned long long>(ncap), o_keys2 = cv.take<unsigned long long>(ncap),
                 o_vals = cv.take<uint32_t>(ncap), o_vals2 = cv.take<uint32_t>(ncap),
                 o_newidx = cv.take<uint32_t>(ncap), o_outp = cv.take<v3d_point>(ncap),
                 o_outs = cv.take<v3d_grid_site>(ncap), o_msort = cv.take<uint32_t>(ncap),
                 o_rfirst = cv.take<uint32_t>(n_references), o_rend = cv.take<uint32_t>(n_references),
                 o_rmask = cv.take<uint32_t>(n_references);
    size_t sort_bytes = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, sort_bytes, (const unsigned long long*)nullptr,
                                    (unsigned long long*)nullptr, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (int)std::max<uint64_t>(ncap, 1), 0, kFirstUseBits, st);
    const size_t o_sort = cv.take<uint8_t>(sort_bytes);
    if (!ensure_arena(ctx, cv.off + 256)) {
        ctx->last_error = "device arena allocation failed";
        return V3D_ERR_OUT_OF_MEMORY;
    }
    char* base = static_cast<char*>(ctx->arena);
    auto at = [&](size_t o) { return base + o; };
    const uint64_t launches0 = g_kernel_launches;

    // 1. verification and union
    Events ev_verify;
    int32_t status = verify_enqueue(ctx, base, a, L, ev_verify.a, st);
    if (status != V3D_OK) return status;
    cudaEventRecord(ev_verify.b, st);
    VerifyCounts c;
    status = verify_read(ctx, base, a, L, c, st);
    if (status != V3D_OK) return status;
    out->verification = c.funnel;
    out->meshing.depth_views = n_views;

    // 2. the union of every reference with at least three samples meshed as one
    //    patch (mesh_legacy.rs:162-168 skips smaller ones before the grid)
    std::vector<uint64_t> off(n_references + 1, 0), moff;
    std::vector<int32_t> por(std::max<uint64_t>(n_references, 1), -1);
    std::vector<uint64_t> patch_ref;
    const bool projectable = std::isfinite(focal) && focal > 0.0;
    uint64_t n_mesh = 0;
    for (uint64_t r = 0; r < n_references; ++r) {
        off[r + 1] = off[r] + c.per_ref[r];
        if (projectable && c.per_ref[r] >= 3) {
            por[r] = (int32_t)patch_ref.size();
            moff.push_back(n_mesh);
            n_mesh += c.per_ref[r];
            patch_ref.push_back(r);
        }
    }
    moff.push_back(n_mesh);
    const uint32_t n_patches = (uint32_t)patch_ref.size();
    std::vector<MeshPatchDev> mp(std::max<uint32_t>(n_patches, 1));
    for (uint32_t k = 0; k < n_patches; ++k) {
        const v3d_camera& cam = views[reference_views[patch_ref[k]]].camera;
        MeshPatchDev& m = mp[k];
        std::memset(&m, 0, sizeof(m));
        std::memcpy(m.cam.R, cam.rotation, sizeof(m.cam.R));
        std::memcpy(m.cam.t, cam.translation, sizeof(m.cam.t));
        m.focal = focal;
        m.width = a.width;
        m.height = a.height;
        m.border = 0;
        m.stride = reference_stride;
        m.gw = gw;
        m.gh = gh;
        m.grid_off = k * cells_patch;
        m.slot_off = k * slots_patch;
        m.n_points = c.per_ref[patch_ref[k]];
    }
    MeshScratch ms;
    mesh_scratch_layout(at(o_mscr), (uint32_t)std::max<uint64_t>(n_references, 1), ncap, total_cells, total_slots, &ms);
    auto* d_off = reinterpret_cast<uint64_t*>(at(o_off));
    auto* d_moff = reinterpret_cast<uint64_t*>(at(o_moff));
    auto* d_mp = reinterpret_cast<v3d_point*>(at(o_mp));
    auto* d_ms = reinterpret_cast<v3d_grid_site*>(at(o_ms));
    auto* d_mpatch = reinterpret_cast<uint32_t*>(at(o_mpatch));
    auto* d_mlocal = reinterpret_cast<uint32_t*>(at(o_mlocal));
    auto* d_mmask = reinterpret_cast<uint32_t*>(at(o_mmask));
    auto* d_ctr = reinterpret_cast<unsigned long long*>(at(o_ctr));
    auto* d_tris = reinterpret_cast<v3d_mesh_triangle*>(at(o_tris));
    auto* d_tpatch = reinterpret_cast<uint32_t*>(at(o_tpatch));
    V3D_CTX_CK(cudaMemcpyAsync(d_off, off.data(), sizeof(uint64_t) * off.size(), cudaMemcpyHostToDevice, st));
    V3D_CTX_CK(cudaMemcpyAsync(at(o_por), por.data(), sizeof(int32_t) * por.size(), cudaMemcpyHostToDevice, st));
    V3D_CTX_CK(cudaMemcpyAsync(d_moff, moff.data(), sizeof(uint64_t) * moff.size(), cudaMemcpyHostToDevice, st));
    V3D_CTX_CK(cudaMemcpyAsync(ms.patches, mp.data(), sizeof(MeshPatchDev) * mp.size(), cudaMemcpyHostToDevice, st));
    V3D_CTX_CK(cudaMemsetAsync(d_ctr, 0, sizeof(unsigned long long) * 2, st));
    Events ev_mesh;
    cudaEventRecord(ev_mesh.a, st);
    if (n_references) {
        SplitTables t{d_off, reinterpret_cast<const int32_t*>(at(o_por)), d_moff, (uint32_t)n_references};
        V3D_COUNTED k_split_samples<<<grid_of(c.n_out), 256, 0, st>>>(
            reinterpret_cast<const v3d_verified_sample*>(at(L.o_out)), reinterpret_cast<const uint32_t*>(at(L.o_count)),
            t, d_mp, d_ms, d_mpatch, d_mlocal, d_mmask, d_ctr);
        V3D_CTX_CK(cudaGetLastError());
    }
    if (n_patches)
        V3D_CTX_CK(mesh_batch_enqueue(ms, n_patches, n_patches * cells_patch, n_patches * slots_patch, d_mp, d_ms,
                                      d_mpatch, d_mlocal, n_mesh, d_tris, d_tpatch, st));
    cudaEventRecord(ev_mesh.b, st);
    uint32_t n_tris = 0;
    unsigned long long multiply = 0;
    std::vector<MeshCounters> mc(std::max<uint32_t>(n_patches, 1));
    if (n_patches) {
        V3D_CTX_CK(cudaMemcpyAsync(&n_tris, ms.count, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        V3D_CTX_CK(cudaMemcpyAsync(mc.data(), ms.counters, sizeof(MeshCounters) * n_patches, cudaMemcpyDeviceToHost, st));
    }
    V3D_CTX_CK(cudaMemcpyAsync(&multiply, d_ctr, sizeof(multiply), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaStreamSynchronize(st));
    out->meshing.multiply_verified_samples = multiply;
    for (uint32_t k = 0; k < n_patches; ++k) {
        out->meshing.candidate_cells += mc[k].candidate_cells;
        out->meshing.rejected_discontinuities += mc[k].discontinuities;
        out->meshing.rejected_degenerate += mc[k].degenerate;
    }
    float device_ms = ev_verify.ms() + ev_mesh.ms();
    if (n_tris == 0) {
        ctx->last_error = "COLMAP stereo produced no cross-view verified surface triangles";
        ctx->last_ms = device_ms;
        ctx->last_launches = g_kernel_launches - launches0;
        return V3D_SKIPPED;
    }

    // 3. the vertices the triangles use, in the order they first use them
    auto* d_first = reinterpret_cast<unsigned long long*>(at(o_first));
    auto* d_vals = reinterpret_cast<uint32_t*>(at(o_vals));
    auto* d_vals2 = reinterpret_cast<uint32_t*>(at(o_vals2));
    auto* d_newidx = reinterpret_cast<uint32_t*>(at(o_newidx));
    auto* d_outp = reinterpret_cast<v3d_point*>(at(o_outp));
    auto* d_outs = reinterpret_cast<v3d_grid_site*>(at(o_outs));
    auto* d_msort = reinterpret_cast<uint32_t*>(at(o_msort));
    auto* d_rfirst = reinterpret_cast<uint32_t*>(at(o_rfirst));
    auto* d_rend = reinterpret_cast<uint32_t*>(at(o_rend));
    auto* d_rmask = reinterpret_cast<uint32_t*>(at(o_rmask));
    V3D_CTX_CK(cudaMemsetAsync(d_first, 0xFF, sizeof(unsigned long long) * n_mesh, st));
    V3D_CTX_CK(cudaMemsetAsync(d_rfirst, 0xFF, sizeof(uint32_t) * n_patches, st));
    V3D_CTX_CK(cudaMemsetAsync(d_rend, 0, sizeof(uint32_t) * n_patches, st));
    Events ev_index;
    cudaEventRecord(ev_index.a, st);
    V3D_COUNTED k_first_use<<<grid_of(n_tris), 256, 0, st>>>(d_tris, d_tpatch, n_tris, d_moff, d_first);
    V3D_COUNTED k_iota_retained<<<grid_of(n_mesh), 256, 0, st>>>(d_first, n_mesh, d_vals, d_ctr + 1);
    V3D_CTX_CK(cudaGetLastError());
    // keys below 3 * n_tris; one bit more keeps the unused inputs' all-ones keys last
    int key_bits = 1;
    while (key_bits < kFirstUseBits - 1 && (3ull * n_tris) >> key_bits) ++key_bits;
    size_t sb = sort_bytes;
    V3D_CTX_CK(cub::DeviceRadixSort::SortPairs(at(o_sort), sb, d_first,
                                               reinterpret_cast<unsigned long long*>(at(o_keys2)), d_vals, d_vals2,
                                               (int)n_mesh, 0, key_bits + 1, st));
    V3D_COUNTED k_place<<<grid_of(n_mesh), 256, 0, st>>>(d_vals2, d_ctr + 1, d_mp, d_ms, d_mpatch, d_mmask, d_newidx,
                                                         d_outp, d_outs, d_msort, d_rfirst, d_rend);
    V3D_COUNTED k_region_masks<<<n_patches, 256, 0, st>>>(d_rfirst, d_rend, d_msort, d_rmask);
    V3D_COUNTED k_reindex<<<grid_of(n_tris), 256, 0, st>>>(d_tris, d_tpatch, n_tris, d_moff, d_newidx);
    V3D_CTX_CK(cudaGetLastError());
    cudaEventRecord(ev_index.b, st);
    unsigned long long retained = 0;
    std::vector<uint32_t> rfirst(n_patches), rend(n_patches), rmask(n_patches);
    V3D_CTX_CK(cudaMemcpyAsync(&retained, d_ctr + 1, sizeof(retained), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaMemcpyAsync(rfirst.data(), d_rfirst, sizeof(uint32_t) * n_patches, cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaMemcpyAsync(rend.data(), d_rend, sizeof(uint32_t) * n_patches, cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaMemcpyAsync(rmask.data(), d_rmask, sizeof(uint32_t) * n_patches, cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaStreamSynchronize(st));
    device_ms += ev_index.ms();
    out->n_points = retained;
    out->n_triangles = n_tris;
    out->meshing.exported_triangles = n_tris;
    out->dominant_rejection = dominant_rejection(c.funnel);
    std::vector<v3d_verified_surface_region> regs;
    for (uint32_t k = 0; k < n_patches; ++k) {
        if (rfirst[k] == kNoRegion) continue;
        const uint64_t r = patch_ref[k];
        v3d_verified_surface_region reg{};
        reg.reference_frame = views[reference_views[r]].camera.frame_index;
        reg.first_point = rfirst[k];
        reg.point_count = rend[k] - rfirst[k];
        std::vector<uint64_t> frames;
        for (int j = 0; j < 4; ++j) {
            const int32_t s = source_views[4 * r + j];
            if (s >= 0 && (rmask[k] >> j & 1u)) frames.push_back(views[s].camera.frame_index);
        }
        std::sort(frames.begin(), frames.end());
        frames.erase(std::unique(frames.begin(), frames.end()), frames.end());
        reg.n_source_frames = (uint32_t)frames.size();
        for (size_t q = 0; q < frames.size(); ++q) reg.source_frames[q] = frames[q];
        regs.push_back(reg);
    }
    out->n_regions = regs.size();
    out->meshing.meshed_reference_views = regs.size();
    if (retained > point_capacity || n_tris > triangle_capacity || !points || !sites || !triangles || !regions) {
        ctx->last_error = "the verified surface exceeds the caller's capacities";
        return V3D_ERR_INVALID_ARGUMENT;
    }
    V3D_CTX_CK(cudaMemcpyAsync(points, d_outp, sizeof(v3d_point) * retained, cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaMemcpyAsync(sites, d_outs, sizeof(v3d_grid_site) * retained, cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaMemcpyAsync(triangles, d_tris, sizeof(v3d_mesh_triangle) * n_tris, cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaStreamSynchronize(st));
    std::copy(regs.begin(), regs.end(), regions);

    // 4. topology of the exported mesh (colmap_surface.rs:467)
    float topo_ms = 0.f;
    uint64_t topo_launches = 0;
    status = surface_topology_locked(ctx, triangles, n_tris, retained, &out->topology, &topo_ms, &topo_launches);
    if (status != V3D_OK) return status;
    ctx->last_ms = device_ms + topo_ms;
    ctx->last_launches = g_kernel_launches - launches0;
    return V3D_OK;
}
