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
                                                          const RowBand* band) {
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
                                                 control, nullptr, band);
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

}  // namespace v3do
