// The dense stage's working-set budget (dense.rs:354-605): which grid and how
// many reference views the Rust process can afford before the pass runs.  It
// is size arithmetic only, over the x86-64 layouts of the Rust containers the
// reference charges, so the host computes it and the device pass that follows
// is the ordinary v3d_estimate_depth_points_limited.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <string>

#include "host.hpp"

namespace v3d {
namespace {

// usize arithmetic with Rust's saturating_add / saturating_mul.
struct Sat {
    uint64_t v = 0;
    static uint64_t mul(uint64_t a, uint64_t b) {
        uint64_t r;
        return __builtin_mul_overflow(a, b, &r) ? UINT64_MAX : r;
    }
    static uint64_t add(uint64_t a, uint64_t b) {
        uint64_t r;
        return __builtin_add_overflow(a, b, &r) ? UINT64_MAX : r;
    }
    Sat& charge(uint64_t count, uint64_t bytes_each) {
        v = add(v, mul(count, bytes_each));
        return *this;
    }
};

// Sizes of the Rust types involved (rustc's repr(Rust) layout on x86-64).
namespace rs {
constexpr uint64_t usize = 8, f64 = 8, f32 = 4, u32 = 4, i32 = 4, i64 = 8, i16 = 2, u8 = 1,
                   boolean = 1;
constexpr uint64_t vec = 24;                 // Vec<T> header
constexpr uint64_t vector3 = 24;             // nalgebra::Vector3<f64>
constexpr uint64_t point3 = 20;              // Point3 (reconstruction/types.rs:69)
constexpr uint64_t grid_site = 8;            // DenseGridSite
constexpr uint64_t point_attributes = 8;     // EvidencePointAttributes
constexpr uint64_t mesh_triangle = 32;       // MeshTriangle (mesh_legacy.rs:18)
constexpr uint64_t option_usize = 16, option_f64 = 16, option_vector3 = 32;
constexpr uint64_t option_usize_f64 = 24;    // Option<(usize, f64)>
constexpr uint64_t option_origin = 1;        // Option<EvidenceOrigin>, niche-packed
constexpr uint64_t option_triangle_geometry = 128;  // surface_merge.rs:1137 (120 B) + tag
constexpr uint64_t image_removal = 24;       // surface_merge_stitch.rs:67
constexpr uint64_t projected_triangle = 72;  // [(Vector2<f64>, f64); 3]
constexpr uint64_t source_corners = 32;      // TriangleSourceCorners
constexpr uint64_t kept_triangle = 112;      // ([Vector3<f64>; 3], usize, [usize; 3], usize)
constexpr uint64_t half_edge = 16;           // surface_merge_stitch.rs:78
constexpr uint64_t option_seam = 32;         // Seam {[u32; 6], u8} (28 B) + tag
constexpr uint64_t edge_use = 8;
// a BTreeMap / HashMap entry as the reference charges it
constexpr uint64_t entry(uint64_t payload) { return payload + 4 * usize + 32; }
}  // namespace rs

constexpr uint64_t kMaxReferenceViews = 3;           // dense.rs:8
constexpr uint64_t kSourcesPerReference = 4;         // dense.rs:11
constexpr uint64_t kGridBorder = 3;                  // dense.rs:12
constexpr uint64_t kScaleSamples = 4096;             // surface_merge.rs:99
constexpr uint64_t kSeamVertices = 6;                // surface_merge_stitch.rs:51
constexpr uint64_t kSeamsPerVertex = 16;             // surface_merge_stitch.rs:54

uint64_t axis_samples(uint64_t extent, uint64_t stride) {
    const uint64_t usable = extent > 2 * kGridBorder ? extent - 2 * kGridBorder : 0;
    return Sat::add(usable, stride - 1) / stride;
}

// surface_merge_stitch.rs:128-152
uint64_t stitch_bytes(uint64_t vertices, uint64_t triangles) {
    using namespace rs;
    const uint64_t per_triangle = 3 * half_edge + option_seam + kSeamVertices * 2 * u32 +
                                  3 * u32 + mesh_triangle + 3 * entry(2 * u32 + edge_use) +
                                  usize + entry(4 * usize + vec);
    const uint64_t scratch =
        2 * kSeamsPerVertex * (entry(usize) + kSeamVertices * (entry(usize) + 2 * 4 * usize));
    return Sat{}.charge(vertices, boolean).charge(triangles, per_triangle).charge(1, scratch).v;
}

// surface_merge.rs:1080-1121
uint64_t merge_bytes(uint64_t vertices, uint64_t triangles) {
    using namespace rs;
    const uint64_t per_vertex = 3 * usize + boolean + option_origin + 2 * 2 * usize +
                                entry(2 * usize) + 2 * entry(2 * usize) +
                                entry(usize + 24 /* (Option<usize>, bool) */);
    const uint64_t per_triangle = usize + option_usize + boolean + option_triangle_geometry +
                                  2 * usize + image_removal + projected_triangle + usize +
                                  3 * usize + 2 * usize + entry(3 * usize + vec) +
                                  entry(4 * usize + vec) + entry(2 * usize) + 4 * usize +
                                  source_corners;
    const uint64_t ownership = Sat{}.charge(triangles, 3 * f64 + kept_triangle + entry(usize))
                                   .charge(kScaleSamples, f64)
                                   .v;
    return Sat{}
        .charge(vertices, per_vertex)
        .charge(triangles, per_triangle)
        .charge(1, std::max(ownership, stitch_bytes(vertices, triangles)))
        .v;
}

uint64_t frame_storage_bytes(const v3d_frame& f) {
    const uint64_t bpp = (f.format == V3D_PIXEL_RGBA8 || f.format == V3D_PIXEL_GRAY_F32) ? 4 : 2;
    return Sat::mul(Sat::mul(f.width, f.height), bpp);
}

}  // namespace

// dense.rs:423-605
v3d_working_set_estimate working_set(const v3d_frame* frames, uint64_t n_frames,
                                     uint64_t max_features, uint32_t descriptor_radius,
                                     uint64_t reference_views, bool fine_grid) {
    using namespace rs;
    v3d_working_set_estimate w;
    std::memset(&w, 0, sizeof(w));
    Sat luma_px;
    uint64_t largest = 0;
    for (uint64_t i = 0; i < n_frames; ++i) {
        w.frame_bytes = Sat::add(w.frame_bytes, frame_storage_bytes(frames[i]));
        const uint64_t px = Sat::mul(frames[i].width, frames[i].height);
        luma_px.charge(1, px);
        largest = std::max(largest, px);
    }
    uint64_t per_ref = 0;
    if (n_frames) {
        const uint64_t st = reference_grid_stride(frames[0].width, frames[0].height, fine_grid);
        per_ref = Sat::mul(axis_samples(frames[0].width, st), axis_samples(frames[0].height, st));
    }
    const uint64_t samples = Sat::mul(per_ref, reference_views);
    const uint64_t triangles = Sat::mul(samples, 8);  // cells and bridges: 8 candidates a sample
    w.retry_frame_bytes = w.frame_bytes;      // a retry's owned request clone
    w.remapped_frame_bytes = w.frame_bytes;   // the reference-first frame clones
    w.luminance_bytes = luma_px.charge(largest, 1 + kSourcesPerReference).v;
    const uint64_t side = Sat::add(Sat::mul(descriptor_radius, 2), 1);
    const uint64_t descriptor = Sat::mul(Sat::mul(side, side), i16);
    const uint64_t features = Sat::mul(n_frames, max_features);
    const uint64_t matches = Sat::mul(n_frames ? n_frames - 1 : 0, max_features);
    const uint64_t observations = Sat::mul(matches, 2);
    w.sparse_pipeline_bytes =
        Sat{}
            .charge(features, Sat::add(3 * u32 + vec, descriptor))   // features + descriptors
            .charge(matches, 3 * usize)                               // FeatureMatch
            .charge(matches, vec)                                     // track headers
            .charge(observations, 2 * usize)                          // track observations
            .charge(observations, entry(3 * usize))                   // membership hash
            .charge(matches, point3 + usize + f32 + vector3 + 2 * f64 + 4 * usize)
            .v;
    w.dense_sample_bytes =
        Sat::mul(Sat::mul(samples, point3 + grid_site + point_attributes + 2 * f64 + 3 * usize), 2);
    w.topology_bytes = Sat::mul(triangles, mesh_triangle);
    w.mesh_builder_bytes = Sat{}
                               .charge(samples, entry(2 * i32 + usize + 6 * f64 + f32))
                               .charge(Sat::mul(samples, 4), entry(2 * i32))
                               .charge(triangles, entry(3 * usize))
                               .charge(triangles, mesh_triangle)
                               .v;
    const uint64_t fusion_vertex = option_usize + vector3 + f64 + usize + vec + option_vector3 +
                                   option_f64 + option_usize_f64 + option_usize + 2 * boolean +
                                   3 * i64 + vec + 4 * usize + usize + 2 * usize + vector3;
    const uint64_t fusion_triangle = 6 * usize + 3 * f64 + boolean + usize;
    w.surface_fusion_bytes =
        std::max(Sat{}.charge(samples, fusion_vertex).charge(triangles, fusion_triangle).v,
                 merge_bytes(samples, triangles));
    // the retained best result is charged at the largest plan
    const uint64_t retained = Sat::mul(per_ref, kMaxReferenceViews);
    w.retained_candidate_bytes = Sat{}
                                     .charge(retained, point3 + grid_site + point_attributes)
                                     .charge(Sat::mul(retained, 8), mesh_triangle)
                                     .v;
    w.packed_output_bytes =
        Sat{}.charge(samples, 6 * f32 + 3 * u8 + 2 * u32).charge(triangles, 4 * u32).v;
    Sat total;
    for (uint64_t part : {w.frame_bytes, w.retry_frame_bytes, w.remapped_frame_bytes,
                          w.luminance_bytes, w.sparse_pipeline_bytes, w.dense_sample_bytes,
                          w.topology_bytes, w.mesh_builder_bytes, w.surface_fusion_bytes,
                          w.retained_candidate_bytes, w.packed_output_bytes})
        total.charge(1, part);
    w.total_bytes = total.v;
    return w;
}

}  // namespace v3d

using namespace v3d;

extern "C" int32_t v3d_estimate_working_set(const v3d_frame* frames, uint64_t n_frames,
                                            uint64_t max_features, uint32_t descriptor_radius,
                                            uint64_t reference_views, int32_t fine_grid,
                                            v3d_working_set_estimate* out) {
    if (!out || (n_frames && !frames)) return V3D_ERR_INVALID_ARGUMENT;
    *out = working_set(frames, n_frames, max_features, descriptor_radius, reference_views,
                       fine_grid != 0);
    return V3D_OK;
}

namespace {
// ReconstructionControl's sticky cancel shared by the landmark test and the pass
struct StickyCancel {
    v3d_cancel_fn fn;
    void* user;
    bool canceled = false;
    static int32_t poll(void* p) {
        auto* s = static_cast<StickyCancel*>(p);
        if (!s->canceled && s->fn && s->fn(s->user) != 0) s->canceled = true;
        return s->canceled ? 1 : 0;
    }
};
}  // namespace

extern "C" int32_t v3d_estimate_depth_points_with_budget_and_control(
    v3d_context* ctx, const v3d_frame* frames, uint64_t n_frames, const v3d_camera* cameras,
    uint64_t n_cameras, const double* sparse_xyz, uint64_t n_sparse, double focal,
    uint64_t budget_bytes, uint64_t max_features, uint32_t descriptor_radius,
    const v3d_profile* profile, v3d_cancel_fn cancel, void* cancel_user, v3d_dense_result* out,
    v3d_dense_budget* budget) {
    // dense.rs:355-420
    if (!out || !budget || (n_frames && !frames)) return V3D_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    std::memset(budget, 0, sizeof(*budget));
    budget->working_set_budget_bytes = budget_bytes;
    StickyCancel sc{cancel, cancel_user};
    v3d_cancel_fn poll = cancel ? &StickyCancel::poll : nullptr;
    auto estimate = [&](uint64_t views, bool fine) {
        return working_set(frames, n_frames, max_features, descriptor_radius, views, fine);
    };
    // the full set of reference views is kept before a finer grid is paid for
    const bool finer = n_frames &&
                       reference_grid_stride(frames[0].width, frames[0].height, true) <
                           reference_grid_stride(frames[0].width, frames[0].height, false);
    bool fine = false;
    v3d_working_set_estimate full;
    if (finer && v3d_has_distributed_landmarks(frames, n_frames, cameras, n_cameras, sparse_xyz,
                                               n_sparse, focal, poll, &sc) == 1) {
        full = estimate(kMaxReferenceViews, true);
        fine = full.total_bytes <= budget_bytes;
    }
    if (!fine) full = estimate(kMaxReferenceViews, false);
    budget->full_working_set_bytes = full.total_bytes;
    uint64_t views = 0;
    for (uint64_t v = kMaxReferenceViews; v >= 1 && !views; --v) {
        const v3d_working_set_estimate e = v == kMaxReferenceViews ? full : estimate(v, false);
        if (e.total_bytes <= budget_bytes) {
            views = v;
            budget->working_set_estimate = e;
        }
    }
    if (!views) {
        budget->working_set_estimate = estimate(1, false);
        out->stats.skip_code = V3D_SKIP_WORKING_SET_BUDGET;
        out->stats.has_skip_reason = 1;
        const std::string why = "estimated dense working set of " +
                                std::to_string(budget->working_set_estimate.total_bytes) +
                                " bytes exceeds the configured " + std::to_string(budget_bytes) +
                                " byte budget even for one reference view";
        std::strncpy(out->stats.skip_reason, why.c_str(), V3D_SKIP_REASON_BYTES - 1);
        return V3D_SKIPPED;
    }
    budget->fine_grid = fine ? 1 : 0;
    budget->reference_views = views;
    int32_t omitted = 0;
    const int32_t st = v3d_estimate_depth_points_limited(
        ctx, frames, n_frames, cameras, n_cameras, sparse_xyz, n_sparse, focal, views,
        fine ? 1 : 0, profile, poll, &sc, out, &omitted);
    if (st < 0) return st;
    // the limit is reported only when it left a reference candidate out
    if (views < kMaxReferenceViews && omitted) {
        out->stats.has_reference_view_limit = 1;
        out->stats.reference_view_limit = views;
    }
    return st;
}
