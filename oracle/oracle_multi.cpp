// TEST INFRASTRUCTURE — CPU oracle, multi-reference driver.
// Restates crates/video-to-3d-core/src/dense.rs:165-213 (has_distributed_landmarks),
// 250-330 (estimate_depth_points_limited), 620-747 (reference order and the
// remapped per-reference call) and 749-1082 (attempt stats, patch split,
// concatenation, legacy conversion).  The working-set budget of dense.rs:354-605
// sizes the Rust process's own heap and stays with the Rust caller; its outcome
// arrives here as (reference_views, fine_grid).
#include <algorithm>
#include <cmath>
#include <set>
#include <string>

#include "oracle.hpp"

namespace v3do {

namespace {
constexpr size_t kMaxReferenceAttempts = 6;  // dense.rs:9
constexpr size_t kMinReferencePatchPoints = 3;  // dense.rs:10
constexpr size_t kMinVisible = 8;  // dense_legacy.rs:8

size_t absdiff(size_t a, size_t b) { return a > b ? a - b : b - a; }

std::vector<Vec3> visible_sparse_points_for_reference(const Camera& c,
                                                      const std::vector<Vec3>& sparse,
                                                      uint32_t w, uint32_t h, double focal) {
    // dense.rs:36-51
    std::vector<Vec3> out;
    for (const Vec3& p : sparse) {
        auto q = project(c, p, w, h, focal);
        if (q && in_image_bounds(q->x, q->y, w, h)) out.push_back(p);
    }
    return out;
}

struct Patch {
    size_t reference_frame;
    LegacyStats stats;
    std::vector<Point3> pp, cp;
    std::vector<GridSite> ps, cs;
    std::vector<Attr> pa, ca;
};

Patch split_patch(size_t reference_frame, LegacyAnalysis a) {
    // dense.rs:816-840
    Patch p;
    p.reference_frame = reference_frame;
    size_t completion = std::min(a.stats.surface_completed_points, a.points.size());
    size_t primary = a.points.size() - completion;
    p.pp.assign(a.points.begin(), a.points.begin() + primary);
    p.cp.assign(a.points.begin() + primary, a.points.end());
    p.ps.assign(a.grid_sites.begin(), a.grid_sites.begin() + std::min(primary, a.grid_sites.size()));
    if (primary < a.grid_sites.size()) p.cs.assign(a.grid_sites.begin() + primary, a.grid_sites.end());
    p.pa.assign(a.point_attributes.begin(),
                a.point_attributes.begin() + std::min(primary, a.point_attributes.size()));
    if (primary < a.point_attributes.size())
        p.ca.assign(a.point_attributes.begin() + primary, a.point_attributes.end());
    p.stats = std::move(a.stats);
    return p;
}

DenseAnalysis combine_patches(std::vector<Patch> patches, std::vector<AttemptStats> attempts) {
    // dense.rs:842-995
    DenseAnalysis out;
    std::vector<size_t> primary_starts, completion_starts;
    for (const Patch& p : patches) {
        primary_starts.push_back(out.points.size());
        out.points.insert(out.points.end(), p.pp.begin(), p.pp.end());
        out.grid_sites.insert(out.grid_sites.end(), p.ps.begin(), p.ps.end());
        out.point_attributes.insert(out.point_attributes.end(), p.pa.begin(), p.pa.end());
    }
    size_t total_completion = 0;
    for (const Patch& p : patches) {
        completion_starts.push_back(out.points.size());
        total_completion += p.cp.size();
        out.points.insert(out.points.end(), p.cp.begin(), p.cp.end());
        out.grid_sites.insert(out.grid_sites.end(), p.cs.begin(), p.cs.end());
        out.point_attributes.insert(out.point_attributes.end(), p.ca.begin(), p.ca.end());
    }
    DenseStats& st = out.stats;
    for (const Patch& p : patches) st.reference_frames.push_back(p.reference_frame);
    size_t primary_reference = st.reference_frames[0];
    std::set<size_t> participating;
    for (const Patch& p : patches) {
        participating.insert(p.reference_frame);
        participating.insert(p.stats.source_frames.begin(), p.stats.source_frames.end());
    }
    participating.erase(primary_reference);
    st.source_frames.assign(participating.begin(), participating.end());
    for (size_t i = 0; i < patches.size(); ++i) {
        const Patch& p = patches[i];
        PatchStats ps;
        ps.reference_frame = p.reference_frame;
        ps.source_frames = p.stats.source_frames;
        ps.primary_start = primary_starts[i];
        ps.primary_points = p.pp.size();
        ps.completion_start = completion_starts[i];
        ps.completed_points = p.cp.size();
        ps.sampled_pixels = p.stats.sampled_pixels;
        ps.accepted_points = p.pp.size() + p.cp.size();
        ps.reciprocal_consistent_points = p.stats.reciprocal_consistent_points;
        ps.grid_stride = p.stats.grid_stride;
        ps.grid_border = p.stats.grid_border;
        ps.search_min_depth = p.stats.search_min_depth;
        ps.search_max_depth = p.stats.search_max_depth;
        st.reference_patches.push_back(ps);
    }
    const LegacyStats& first = patches[0].stats;
    bool single = patches.size() == 1;
    st.attempted = true;
    st.reference_frame = primary_reference;
    st.source_views = st.source_frames.size();
    for (const Patch& p : patches) {
        st.sampled_pixels += p.stats.sampled_pixels;
        st.depth_hypotheses = std::max(st.depth_hypotheses, p.stats.depth_hypotheses);
        st.surface_completion_proposals += p.stats.surface_completion_proposals;
        st.surface_completion_rejected_texture += p.stats.surface_completion_rejected_texture;
        st.surface_completion_rejected_cross_view += p.stats.surface_completion_rejected_cross_view;
        st.surface_completion_rejected_reciprocal += p.stats.surface_completion_rejected_reciprocal;
        st.surface_completion_rejected_fusion += p.stats.surface_completion_rejected_fusion;
        st.surface_completion_rejected_footprint += p.stats.surface_completion_rejected_footprint;
        st.reciprocal_checked_points += p.stats.reciprocal_checked_points;
        st.reciprocal_rejected_points += p.stats.reciprocal_rejected_points;
        st.reciprocal_consistent_points += p.stats.reciprocal_consistent_points;
        st.fusion_input_observations += p.stats.fusion_input_observations;
        st.fusion_rejected_observations += p.stats.fusion_rejected_observations;
        st.fusion_rejected_points += p.stats.fusion_rejected_points;
    }
    st.accepted_points = out.points.size();
    st.surface_completed_points = total_completion;
    st.grid_stride = first.grid_stride;
    st.grid_border = first.grid_border;
    if (single) {
        st.median_fusion_observations = first.median_fusion_observations;
        st.median_supporting_views = first.median_supporting_views;
        st.median_photometric_error = first.median_photometric_error;
        st.search_min_depth = first.search_min_depth;
        st.search_max_depth = first.search_max_depth;
    }
    st.reference_attempts = std::move(attempts);
    return out;
}
}  // namespace

bool has_distributed_landmarks(const std::vector<Frame>& frames,
                               const std::vector<Camera>& cameras,
                               const std::vector<Vec3>& sparse, double focal, Control& control) {
    // dense.rs:165-213
    size_t majority = cameras.size() / 2 + 1;
    size_t covered = 0;
    for (const Camera& c : cameras) {
        if (c.frame_index >= frames.size()) continue;
        const Frame& f = frames[c.frame_index];
        uint8_t tiles[4][4] = {};
        size_t supported = 0;
        bool stop = false;
        for (size_t start = 0; start < sparse.size() && !stop; start += 256) {
            if (control.is_canceled()) return false;
            size_t end = std::min(sparse.size(), start + 256);
            for (size_t i = start; i < end; ++i) {
                auto q = project(c, sparse[i], f.width, f.height, focal);
                if (!q) continue;
                double x = q->x, y = q->y;
                if (!(x >= 0.0 && x < static_cast<double>(f.width)) ||
                    !(y >= 0.0 && y < static_cast<double>(f.height)))
                    continue;
                size_t col = static_cast<size_t>(4.0 * x / static_cast<double>(f.width));
                size_t row = static_cast<size_t>(4.0 * y / static_cast<double>(f.height));
                uint8_t& tile = tiles[row][col];
                if (tile < 255) ++tile;
                if (tile == 2) {
                    ++supported;
                    if (supported >= 8) {
                        ++covered;
                        if (covered == majority) return true;
                        stop = true;
                        break;
                    }
                }
            }
        }
    }
    return false;
}

std::vector<size_t> reference_candidate_order(const std::vector<Frame>& frames,
                                              const std::vector<Camera>& cameras,
                                              const std::vector<Vec3>& sparse, double focal) {
    // dense.rs:620-672
    std::vector<std::pair<size_t, size_t>> cands;
    for (size_t i = 0; i < cameras.size(); ++i) {
        const Camera& c = cameras[i];
        if (c.frame_index >= frames.size()) continue;
        const Frame& f = frames[c.frame_index];
        size_t visible =
            visible_sparse_points_for_reference(c, sparse, f.width, f.height, focal).size();
        if (visible >= kMinVisible) cands.push_back({i, visible});
    }
    std::stable_sort(cands.begin(), cands.end(), [&](const auto& a, const auto& b) {
        if (a.second != b.second) return a.second > b.second;
        return cameras[a.first].frame_index < cameras[b.first].frame_index;
    });
    if (cands.empty()) return {};
    Vec3 pc = cameras[cands[0].first].center();
    std::stable_sort(cands.begin() + 1, cands.end(), [&](const auto& a, const auto& b) {
        double da = norm_squared(sub(cameras[a.first].center(), pc));
        double db = norm_squared(sub(cameras[b.first].center(), pc));
        if (da != db) return da > db;  // right.total_cmp(left): farthest first
        if (a.second != b.second) return a.second > b.second;
        return cameras[a.first].frame_index < cameras[b.first].frame_index;
    });
    std::vector<size_t> order;
    for (auto& c : cands) order.push_back(c.first);
    return order;
}

std::optional<LegacyAnalysis> reconstruct_reference_patch(const Profile& prof,
                                                          const std::vector<Frame>& frames,
                                                          const std::vector<Camera>& cameras,
                                                          const std::vector<Vec3>& sparse,
                                                          double focal, size_t camera_index,
                                                          bool fine_grid, Control& control,
                                                          const RowBand* band,
                                                          std::vector<ExplainRecord>* explain) {
    // dense.rs:674-747
    if (camera_index >= cameras.size()) return std::nullopt;
    const Camera& rc = cameras[camera_index];
    if (rc.frame_index >= frames.size()) return std::nullopt;
    const Frame& rf = frames[rc.frame_index];
    auto visible = visible_sparse_points_for_reference(rc, sparse, rf.width, rf.height, focal);
    if (visible.size() < kMinVisible) return std::nullopt;
    std::vector<size_t> src;
    for (size_t i = 0; i < cameras.size(); ++i)
        if (i != camera_index && cameras[i].frame_index < frames.size()) src.push_back(i);
    std::stable_sort(src.begin(), src.end(), [&](size_t a, size_t b) {
        size_t da = absdiff(cameras[a].frame_index, rc.frame_index);
        size_t db = absdiff(cameras[b].frame_index, rc.frame_index);
        if (da != db) return da < db;
        return cameras[a].frame_index < cameras[b].frame_index;
    });
    std::vector<size_t> order{camera_index};
    order.insert(order.end(), src.begin(), src.end());
    std::vector<const Frame*> rframes;
    std::vector<Camera> rcams;
    for (size_t k = 0; k < order.size(); ++k) {
        if (control.is_canceled()) return std::nullopt;
        const Camera& c = cameras[order[k]];
        rframes.push_back(&frames[c.frame_index]);
        Camera m = c;
        m.frame_index = k;
        rcams.push_back(m);
    }
    LegacyAnalysis a = estimate_depth_points_ptr(prof, rframes, rcams, visible, focal, fine_grid,
                                                 control, nullptr, band, explain);
    a.stats.reference_frame = rc.frame_index;
    std::vector<size_t> mapped;
    for (size_t r : a.stats.source_frames)
        if (r < order.size()) mapped.push_back(cameras[order[r]].frame_index);
    a.stats.source_frames = mapped;
    return a;
}

AttemptStats reference_attempt_stats(size_t reference_frame, const LegacyStats& s,
                                     size_t accepted_points, bool accepted) {
    // dense.rs:749-785
    AttemptStats a;
    if (!accepted) {
        if (s.skip_reason)
            a.skip_reason = s.skip_reason;
        else if (!s.attempted)
            a.skip_reason = "dense estimation did not run for this reference";
        else
            a.skip_reason = "reference produced " + std::to_string(accepted_points) +
                            " accepted dense points; at least 3 are required for a surface patch";
    }
    a.reference_frame = reference_frame;
    a.attempted = s.attempted;
    a.accepted = accepted;
    a.sampled_pixels = s.sampled_pixels;
    a.accepted_points = accepted_points;
    a.reciprocal_checked_points = s.reciprocal_checked_points;
    a.reciprocal_rejected_points = s.reciprocal_rejected_points;
    a.reciprocal_consistent_points = s.reciprocal_consistent_points;
    a.surface_completion_proposals = s.surface_completion_proposals;
    a.surface_completed_points = s.surface_completed_points;
    a.surface_completion_rejected_texture = s.surface_completion_rejected_texture;
    a.surface_completion_rejected_cross_view = s.surface_completion_rejected_cross_view;
    a.surface_completion_rejected_reciprocal = s.surface_completion_rejected_reciprocal;
    a.surface_completion_rejected_fusion = s.surface_completion_rejected_fusion;
    a.surface_completion_rejected_footprint = s.surface_completion_rejected_footprint;
    return a;
}

std::vector<AttemptStats> merge_fallback_attempts(std::vector<AttemptStats> attempts,
                                                  std::vector<AttemptStats> fallback) {
    // dense.rs:787-804
    for (AttemptStats& f : fallback) {
        auto it = std::find_if(attempts.begin(), attempts.end(), [&](const AttemptStats& a) {
            return a.reference_frame == f.reference_frame;
        });
        if (it != attempts.end()) {
            if (f.accepted && !it->accepted) *it = f;
        } else {
            attempts.push_back(f);
        }
    }
    return attempts;
}

DenseAnalysis from_legacy(LegacyAnalysis a) {
    // dense.rs:997-1082
    DenseAnalysis out;
    const LegacyStats& s = a.stats;
    size_t completion = std::min(s.surface_completed_points, a.points.size());
    size_t primary = a.points.size() - completion;
    static_cast<LegacyStats&>(out.stats) = s;
    if (s.reference_frame) {
        out.stats.reference_frames.push_back(*s.reference_frame);
        out.stats.reference_attempts.push_back(reference_attempt_stats(
            *s.reference_frame, s, a.points.size(),
            s.attempted && a.points.size() >= kMinReferencePatchPoints));
        if (s.attempted) {
            PatchStats ps;
            ps.reference_frame = *s.reference_frame;
            ps.source_frames = s.source_frames;
            ps.primary_start = 0;
            ps.primary_points = primary;
            ps.completion_start = primary;
            ps.completed_points = completion;
            ps.sampled_pixels = s.sampled_pixels;
            ps.accepted_points = a.points.size();
            ps.reciprocal_consistent_points = s.reciprocal_consistent_points;
            ps.grid_stride = s.grid_stride;
            ps.grid_border = s.grid_border;
            ps.search_min_depth = s.search_min_depth;
            ps.search_max_depth = s.search_max_depth;
            out.stats.reference_patches.push_back(ps);
        }
    }
    out.points = std::move(a.points);
    out.grid_sites = std::move(a.grid_sites);
    out.point_attributes = std::move(a.point_attributes);
    return out;
}

std::pair<DenseAnalysis, bool> estimate_depth_points_limited(const Profile& prof,
                                                             const std::vector<Frame>& frames,
                                                             const std::vector<Camera>& cameras,
                                                             const std::vector<Vec3>& sparse,
                                                             double focal, size_t reference_views,
                                                             bool fine_grid, Control& control) {
    // dense.rs:250-330
    auto order = reference_candidate_order(frames, cameras, sparse, focal);
    if (order.empty())
        return {from_legacy(estimate_depth_points_with_control(prof, frames, cameras, sparse,
                                                               focal, fine_grid, control)),
                false};
    std::vector<Patch> patches;
    std::vector<AttemptStats> attempts;
    bool omitted = false;
    size_t n = std::min(order.size(), kMaxReferenceAttempts);
    for (size_t i = 0; i < n; ++i) {
        if (control.is_canceled()) return {DenseAnalysis{}, false};
        size_t ci = order[i];
        auto a = reconstruct_reference_patch(prof, frames, cameras, sparse, focal, ci, fine_grid,
                                             control);
        if (!a) continue;
        size_t rf = cameras[ci].frame_index;
        bool accepted = a->stats.attempted && a->points.size() >= kMinReferencePatchPoints;
        attempts.push_back(reference_attempt_stats(rf, a->stats, a->points.size(), accepted));
        if (!accepted) continue;
        patches.push_back(split_patch(rf, std::move(*a)));
        if (patches.size() >= reference_views) {
            omitted = i + 1 < n;
            break;
        }
    }
    if (patches.empty()) {
        DenseAnalysis fb = from_legacy(
            estimate_depth_points_with_control(prof, frames, cameras, sparse, focal, fine_grid,
                                               control));
        auto fa = std::move(fb.stats.reference_attempts);
        fb.stats.reference_attempts = merge_fallback_attempts(std::move(attempts), std::move(fa));
        return {std::move(fb), false};
    }
    return {combine_patches(std::move(patches), std::move(attempts)), omitted};
}


// ---- the working-set budget (dense.rs:354-605) -------------------------------
//
// Pure size arithmetic over Rust type sizes.  Every size below is the
// x86-64 layout rustc gives the named type (repr(Rust): fields reordered by
// alignment, no niche in usize/f64/u8, so Option<T> adds an aligned tag).

namespace {

uint64_t sat_add(uint64_t a, uint64_t b) { return a + b < a ? UINT64_MAX : a + b; }
uint64_t sat_mul(uint64_t a, uint64_t b) {
    uint64_t r;
    return __builtin_mul_overflow(a, b, &r) ? UINT64_MAX : r;
}

constexpr uint64_t kUsize = 8, kF64 = 8, kF32 = 4, kU32 = 4, kI32 = 4, kI64 = 8, kI16 = 2,
                   kBool = 1, kU8 = 1;
constexpr uint64_t kVec = 24;                    // Vec<T>: pointer, capacity, length
constexpr uint64_t kVector3 = 24;                // nalgebra Vector3<f64>
constexpr uint64_t kPoint3 = 20;                 // reconstruction/types.rs:69: 4 x f32 + 3 x u8
constexpr uint64_t kGridSite = 8;                // DenseGridSite {u32, u32}
constexpr uint64_t kAttrs = 8;                   // EvidencePointAttributes {f32, f32}
constexpr uint64_t kMeshTriangle = 32;           // mesh_legacy.rs:18: 3 x usize + f32
constexpr uint64_t kOptUsize = 16, kOptF64 = 16, kOptVector3 = 32, kOptUsizeF64 = 24;
constexpr uint64_t kOptOrigin = 1;               // Option<EvidenceOrigin>: 4-variant enum, niche
constexpr uint64_t kOptTriangleGeometry = 128;   // surface_merge.rs:1137: 120 B + tag
constexpr uint64_t kImageRemoval = 24;           // surface_merge_stitch.rs:67
constexpr uint64_t kProjectedTriangle = 72;      // [(Vector2<f64>, f64); 3]
constexpr uint64_t kTriangleSourceCorners = 32;  // reconstruction_evidence.rs:125
constexpr uint64_t kKeptTriangle = 112;          // ([Vector3<f64>; 3], usize, [usize; 3], usize)
constexpr uint64_t kHalfEdge = 16;               // surface_merge_stitch.rs:78: 4 x u32
constexpr uint64_t kOptSeam = 32;                // [u32; 6] + u8 = 28 B, plus an aligned tag
constexpr uint64_t kEdgeUse = 8;                 // {u32, u32}
constexpr uint64_t kMaxScaleSamples = 4096;      // surface_merge.rs:99
constexpr uint64_t kMaxSeamVertices = 6;         // surface_merge_stitch.rs:51
constexpr uint64_t kMaxSeamsPerVertex = 16;      // surface_merge_stitch.rs:54
constexpr uint64_t kMaxReferenceViews = 3;       // dense.rs:8
constexpr uint64_t kMaxSourceViewsPerReference = 4;  // dense.rs:11
constexpr uint64_t kDenseGridBorder = 3;         // dense.rs:12

constexpr uint64_t entry(uint64_t payload) { return payload + 4 * kUsize + 32; }

uint64_t grid_axis_samples(uint64_t extent, uint64_t stride) {
    // dense.rs:615-618
    uint64_t usable = extent > 2 * kDenseGridBorder ? extent - 2 * kDenseGridBorder : 0;
    return sat_add(usable, stride ? stride - 1 : 0) / stride;
}

uint64_t stitch_working_set(uint64_t vertices, uint64_t triangles) {
    // surface_merge_stitch.rs:128-152
    const uint64_t per_vertex = kBool;
    const uint64_t per_triangle = 3 * kHalfEdge + kOptSeam + kMaxSeamVertices * 8 + 3 * kU32 +
                                  kMeshTriangle + 3 * entry(8 + kEdgeUse) + kUsize +
                                  entry(32 + kVec);
    const uint64_t scratch =
        2 * kMaxSeamsPerVertex * (entry(kUsize) + kMaxSeamVertices * (entry(kUsize) + 2 * 32));
    return sat_add(sat_add(sat_mul(vertices, per_vertex), sat_mul(triangles, per_triangle)),
                   scratch);
}

uint64_t merge_working_set(uint64_t vertices, uint64_t triangles) {
    // surface_merge.rs:1080-1121
    const uint64_t per_vertex = 3 * kUsize + kBool + kOptOrigin + 2 * 16 + entry(16) +
                                2 * entry(2 * kUsize) + entry(kUsize + 24);
    const uint64_t per_triangle = kUsize + kOptUsize + kBool + kOptTriangleGeometry + 2 * kUsize +
                                  kImageRemoval + kProjectedTriangle + kUsize + 24 + 2 * kUsize +
                                  entry(24 + kVec) + entry(32 + kVec) + entry(2 * kUsize) + 32 +
                                  kTriangleSourceCorners;
    const uint64_t ownership = sat_add(
        sat_mul(triangles, 3 * kF64 + kKeptTriangle + entry(kUsize)), kMaxScaleSamples * kF64);
    return sat_add(sat_add(sat_mul(vertices, per_vertex), sat_mul(triangles, per_triangle)),
                   std::max(ownership, stitch_working_set(vertices, triangles)));
}

}  // namespace

WorkingSet estimate_working_set(const std::vector<Frame>& frames, uint64_t max_features,
                                uint32_t descriptor_radius, uint64_t reference_views,
                                bool fine_grid) {
    // dense.rs:423-605
    WorkingSet w;
    uint64_t luminance_pixels = 0, largest = 0;
    for (const Frame& f : frames) {
        const uint64_t px = sat_mul(f.width, f.height);
        w.frame_bytes = sat_add(w.frame_bytes, f.bytes.size());
        luminance_pixels = sat_add(luminance_pixels, px);
        largest = std::max(largest, px);
    }
    uint64_t per_reference = 0;
    if (!frames.empty()) {
        const uint64_t stride = grid_stride(frames[0].width, frames[0].height, fine_grid);
        per_reference = sat_mul(grid_axis_samples(frames[0].width, stride),
                                grid_axis_samples(frames[0].height, stride));
    }
    const uint64_t samples = sat_mul(per_reference, reference_views);
    const uint64_t triangles = sat_mul(samples, 8);
    w.retry_frame_bytes = w.frame_bytes;
    w.remapped_frame_bytes = w.frame_bytes;
    w.luminance_bytes =
        sat_add(luminance_pixels, sat_mul(largest, 1 + kMaxSourceViewsPerReference));
    const uint64_t side = sat_add(sat_mul(descriptor_radius, 2), 1);
    const uint64_t descriptor_bytes = sat_mul(sat_mul(side, side), kI16);
    const uint64_t n = frames.size();
    const uint64_t features = sat_mul(n, max_features);
    const uint64_t matches = sat_mul(n ? n - 1 : 0, max_features);
    const uint64_t observations = sat_mul(matches, 2);
    const uint64_t feature_record = 3 * kU32 + kVec;
    w.sparse_pipeline_bytes = sat_add(
        sat_add(sat_add(sat_add(sat_add(sat_mul(features, sat_add(feature_record, descriptor_bytes)),
                                        sat_mul(matches, 3 * kUsize)),
                                sat_mul(matches, kVec)),
                        sat_mul(observations, 2 * kUsize)),
                sat_mul(observations, entry(3 * kUsize))),
        sat_mul(matches, kPoint3 + kUsize + kF32 + kVector3 + 2 * kF64 + 4 * kUsize));
    const uint64_t retained_sample = kPoint3 + kGridSite + kAttrs + 2 * kF64 + 3 * kUsize;
    w.dense_sample_bytes = sat_mul(sat_mul(samples, retained_sample), 2);
    w.topology_bytes = sat_mul(triangles, kMeshTriangle);
    w.mesh_builder_bytes = sat_add(
        sat_add(sat_add(sat_mul(samples, entry(2 * kI32 + kUsize + 6 * kF64 + kF32)),
                        sat_mul(sat_mul(samples, 4), entry(2 * kI32))),
                sat_mul(triangles, entry(3 * kUsize))),
        sat_mul(triangles, kMeshTriangle));
    const uint64_t per_vertex_fusion = kOptUsize + kVector3 + kF64 + kUsize + kVec + kOptVector3 +
                                       kOptF64 + kOptUsizeF64 + kOptUsize + 2 * kBool + 3 * kI64 +
                                       kVec + 4 * kUsize + kUsize + 2 * kUsize + kVector3;
    const uint64_t per_triangle_fusion = 6 * kUsize + 3 * kF64 + kBool + kUsize;
    w.surface_fusion_bytes = std::max(sat_add(sat_mul(samples, per_vertex_fusion),
                                              sat_mul(triangles, per_triangle_fusion)),
                                      merge_working_set(samples, triangles));
    const uint64_t retained = sat_mul(per_reference, kMaxReferenceViews);
    w.retained_candidate_bytes = sat_add(sat_mul(retained, kPoint3 + kGridSite + kAttrs),
                                         sat_mul(sat_mul(retained, 8), kMeshTriangle));
    w.packed_output_bytes = sat_add(sat_mul(samples, 6 * kF32 + 3 * kU8 + 2 * kU32),
                                    sat_mul(triangles, 4 * kU32));
    uint64_t t = 0;
    for (uint64_t v : {w.frame_bytes, w.retry_frame_bytes, w.remapped_frame_bytes,
                       w.luminance_bytes, w.sparse_pipeline_bytes, w.dense_sample_bytes,
                       w.topology_bytes, w.mesh_builder_bytes, w.surface_fusion_bytes,
                       w.retained_candidate_bytes, w.packed_output_bytes})
        t = sat_add(t, v);
    w.total_bytes = t;
    return w;
}

BudgetedAnalysis estimate_depth_points_with_budget(const Profile& prof,
                                                   const std::vector<Frame>& frames,
                                                   const std::vector<Camera>& cameras,
                                                   const std::vector<Vec3>& sparse, double focal,
                                                   uint64_t budget, uint64_t max_features,
                                                   uint32_t descriptor_radius, Control& control) {
    // dense.rs:355-420
    BudgetedAnalysis out;
    out.budget_bytes = budget;
    auto estimate = [&](uint64_t views, bool fine) {
        return estimate_working_set(frames, max_features, descriptor_radius, views, fine);
    };
    const bool finer = !frames.empty() && grid_stride(frames[0].width, frames[0].height, true) <
                                              grid_stride(frames[0].width, frames[0].height, false);
    std::optional<WorkingSet> fine_estimate;
    if (finer && has_distributed_landmarks(frames, cameras, sparse, focal, control)) {
        WorkingSet f = estimate(kMaxReferenceViews, true);
        if (f.total_bytes <= budget) fine_estimate = f;
    }
    const bool fine_grid = fine_estimate.has_value();
    const WorkingSet full = fine_estimate ? *fine_estimate : estimate(kMaxReferenceViews, false);
    out.full_bytes = full.total_bytes;
    uint64_t views = 0;
    WorkingSet plan;
    if (full.total_bytes <= budget) {
        views = kMaxReferenceViews;
        plan = full;
    } else {
        for (uint64_t v = kMaxReferenceViews - 1; v >= 1; --v) {
            WorkingSet l = estimate(v, false);
            if (l.total_bytes <= budget) {
                views = v;
                plan = l;
                break;
            }
        }
    }
    if (views == 0) {
        const WorkingSet single = estimate(1, false);
        out.estimate = single;
        out.analysis.stats.skip_reason =
            "estimated dense working set of " + std::to_string(single.total_bytes) +
            " bytes exceeds the configured " + std::to_string(budget) +
            " byte budget even for one reference view";
        return out;
    }
    auto [analysis, omitted] =
        estimate_depth_points_limited(prof, frames, cameras, sparse, focal, views, fine_grid,
                                      control);
    out.analysis = std::move(analysis);
    out.estimate = plan;
    out.fine_grid = fine_grid;
    out.reference_views = views;
    if (views < kMaxReferenceViews && omitted) out.analysis.stats.reference_view_limit = views;
    return out;
}

}  // namespace v3do
