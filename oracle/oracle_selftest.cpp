// TEST INFRASTRUCTURE — the reference's own tests for the dense path, re-run
// against the CPU oracle.  Each test names the reference test it ports
// (file:line inside crates/video-to-3d-core/src).  These assertions are what
// pins the restatement: the reference has no golden output vectors.
//
// Budget-arithmetic tests (dense.rs:1270, 1430, 1475, and the byte assertions
// of 1115/1298/1361) test estimate_working_set, which stays with the Rust
// caller; their dense-pass halves are ported below.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <functional>
#include <string>

#include "oracle.hpp"

using namespace v3do;

namespace {

std::string g_report;
int g_failures = 0;
int g_checks = 0;
const char* g_test = "";

void check(bool ok, const char* what, int line) {
    ++g_checks;
    if (!ok) {
        ++g_failures;
        char buf[512];
        std::snprintf(buf, sizeof(buf), "FAIL %s:%d %s\n", g_test, line, what);
        g_report += buf;
    }
}
#define CHECK(cond) check((cond), #cond, __LINE__)

Camera camera(size_t frame_index, double center_x) {
    Camera c;
    c.frame_index = frame_index;
    c.t[0] = -center_x;
    return c;
}

uint8_t texture(double wx, double wy) {
    double v = 128.0 + 55.0 * std::sin(wx * 15.0 + wy * 2.7) + 40.0 * std::cos(wy * 17.0 - wx * 3.1) +
               25.0 * std::sin((wx + wy) * 11.0);
    v = std::round(v);
    if (v < 0) v = 0;
    if (v > 255) v = 255;
    return static_cast<uint8_t>(v);
}

Frame plane_frame(uint32_t w, uint32_t h, double focal, double cx, double depth) {
    Frame f;
    f.width = w;
    f.height = h;
    f.bytes.assign(static_cast<size_t>(w) * h * 4, 0);
    for (uint32_t y = 0; y < h; ++y)
        for (uint32_t x = 0; x < w; ++x) {
            double wx = cx + (x - w * 0.5) / focal * depth;
            double wy = (y - h * 0.5) / focal * depth;
            uint8_t v = texture(wx, wy);
            size_t i = (static_cast<size_t>(y) * w + x) * 4;
            f.bytes[i] = f.bytes[i + 1] = f.bytes[i + 2] = v;
            f.bytes[i + 3] = 255;
        }
    return f;
}

Frame flat_frame(uint32_t w, uint32_t h, uint8_t value) {
    Frame f;
    f.width = w;
    f.height = h;
    f.bytes.assign(static_cast<size_t>(w) * h * 4, value);
    return f;
}

std::vector<Vec3> plane_sparse_points(uint32_t w, uint32_t h, double focal, double depth) {
    std::vector<Vec3> pts;
    for (uint32_t y : {10u, 18u, 26u, 34u})
        for (uint32_t x : {12u, 24u, 36u, 48u, 56u})
            pts.push_back({(x - w * 0.5) / focal * depth, (y - h * 0.5) / focal * depth, depth});
    return pts;
}

Point3 point_at_pixel(const Camera& c, double x, double y, double depth, uint32_t w, uint32_t h,
                      double focal) {
    Vec3 p = unproject(c, x, y, depth, w, h, focal);
    return {static_cast<float>(p.x), static_cast<float>(p.y), static_cast<float>(p.z), 0.8f, 120,
            120, 120};
}

Profile reference_profile() { return Profile{}; }

Control never() { return Control{}; }

// dense.rs:222-244 (#[cfg(test)] estimate_depth_points)
DenseAnalysis dense_estimate(const std::vector<Frame>& frames, const std::vector<Camera>& cams,
                             const std::vector<Vec3>& sparse, double focal) {
    Control c1 = never(), c2 = never();
    bool fine = has_distributed_landmarks(frames, cams, sparse, focal, c1);
    return estimate_depth_points_limited(reference_profile(), frames, cams, sparse, focal, 3, fine,
                                         c2)
        .first;
}

// ---------------- dense_legacy.rs tests ----------------

void estimates_coarse_depth_on_textured_plane() {  // dense_legacy.rs:1261
    uint32_t w = 68, h = 48;
    double f = 60.0, depth = 4.0;
    std::vector<Frame> frames{plane_frame(w, h, f, 0.0, depth), plane_frame(w, h, f, 0.18, depth),
                              plane_frame(w, h, f, -0.16, depth)};
    std::vector<Camera> cams{camera(0, 0.0), camera(1, 0.18), camera(2, -0.16)};
    auto sparse = plane_sparse_points(w, h, f, depth);
    Control c = never();
    auto r = estimate_depth_points_with_control(reference_profile(), frames, cams, sparse, f, false, c);
    const LegacyStats& s = r.stats;
    CHECK(s.attempted);
    CHECK(!s.skip_reason);
    CHECK(s.reference_frame && *s.reference_frame == 0);
    CHECK(s.source_views == 2);
    CHECK((s.source_frames == std::vector<size_t>{1, 2}));
    CHECK(s.reciprocal_checked_points == s.reciprocal_consistent_points + s.reciprocal_rejected_points);
    CHECK(s.reciprocal_consistent_points + s.surface_completed_points ==
          s.accepted_points + s.fusion_rejected_points);
    CHECK(s.surface_completion_proposals ==
          s.surface_completed_points + s.surface_completion_rejected_texture +
              s.surface_completion_rejected_cross_view + s.surface_completion_rejected_reciprocal +
              s.surface_completion_rejected_fusion + s.surface_completion_rejected_footprint);
    CHECK(s.fusion_input_observations >= s.reciprocal_consistent_points * 2);
    CHECK(s.median_fusion_observations && *s.median_fusion_observations >= 2.0f);
    CHECK(r.points.size() >= 12);
    std::vector<double> depths;
    for (auto& p : r.points) depths.push_back(p.z);
    std::sort(depths.begin(), depths.end());
    double md = quantile(depths, 0.5);
    CHECK(std::fabs(md - depth) < 0.55);
}

void surface_completion_reports_texture_rejections() {  // dense_legacy.rs:1323
    uint32_t w = 68, h = 48;
    double f = 60.0;
    Frame frame = flat_frame(w, h, 120);
    std::vector<Camera> cams{camera(0, 0.0), camera(1, 0.2)};
    Plane luma = to_luma(frame);
    std::vector<SourceView> sources{{&cams[1], &frame, luma, 3.2, 5.0}};
    std::vector<Point3> points{point_at_pixel(cams[0], 3, 3, 4, w, h, f),
                               point_at_pixel(cams[0], 7, 3, 4, w, h, f),
                               point_at_pixel(cams[0], 3, 7, 4, w, h, f)};
    std::vector<GridSite> sites{{3, 3}, {7, 3}, {3, 7}};
    std::vector<Attr> attrs(3);
    std::vector<double> errors, supports;
    Control c = never();
    auto st = complete_surface_samples(reference_profile(), cams[0], frame, luma, sources, points,
                                       sites, attrs, errors, supports, w, h, 3, 4, f, c);
    CHECK(st.proposals > 0);
    CHECK(st.accepted == 0);
    CHECK(st.rejected_texture == st.proposals);
    CHECK(st.proposals == st.outcomes());
}

void surface_depth_prediction_requires_consistent_neighbors() {  // dense_legacy.rs:1379
    std::vector<double> smooth{4.0, 4.03, 3.98, 4.01};
    auto p = surface_depth_prediction(smooth);
    CHECK(p.has_value());
    CHECK(p && std::fabs(*p - 4.01) < 0.05);
    std::vector<double> disc{4.0, 4.02, 5.2};
    CHECK(!surface_depth_prediction(disc));
    std::vector<double> under{4.0, 4.01};
    CHECK(!surface_depth_prediction(under));
}

void reciprocal_depth_search_recovers_source_view_depth() {  // dense_legacy.rs:1392
    uint32_t w = 68, h = 48;
    double f = 60.0, depth = 4.0;
    Frame f0 = plane_frame(w, h, f, 0.0, depth), f1 = plane_frame(w, h, f, 0.18, depth);
    Camera c0 = camera(0, 0.0), c1 = camera(1, 0.18);
    auto sparse = plane_sparse_points(w, h, f, depth);
    auto b = depth_search_bounds(c1, sparse, w, h, f);
    CHECK(b.has_value());
    if (!b) return;
    auto q = project(c1, Vec3{0, 0, depth}, w, h, f);
    CHECK(q.has_value());
    if (!q) return;
    Plane sl = to_luma(f1), rl = to_luma(f0);
    auto est = estimate_single_view_depth(reference_profile(), c1, c0, sl, rl, q->x, q->y, b->first,
                                          b->second, f);
    CHECK(est.has_value());
    CHECK(est && reciprocal_depth_agrees(q->z, *est));
}

void fusion_rejects_spatially_inconsistent_reciprocal_observations() {  // dense_legacy.rs:1435
    Vec3 primary{0, 0, 4};
    std::vector<Vec3> rec{{0.02, -0.01, 4.04}, {0.9, 0.0, 4.0}};
    Fused fz = fuse_depth_observations(primary, rec, 4.0);
    CHECK(fz.observations == 2);
    CHECK(fz.rejected_observations == 1);
    CHECK(std::fabs(fz.position.z - 4.02) < 1.0e-9);
    CHECK(std::fabs(fz.position.x) < 0.02);
}

void reciprocal_consistency_rejects_wrong_depth() {  // dense_legacy.rs:1451
    CHECK(reciprocal_depth_agrees(4.0, 4.2));
    CHECK(!reciprocal_depth_agrees(4.0, 5.0));
}

void rejects_textureless_depth_hypotheses() {  // dense_legacy.rs:1457
    uint32_t w = 68, h = 48;
    double f = 60.0;
    Frame frame = flat_frame(w, h, 120);
    std::vector<Camera> cams{camera(0, 0.0), camera(1, 0.2)};
    auto sparse = plane_sparse_points(w, h, f, 4.0);
    Control c = never();
    auto r = estimate_depth_points_with_control(reference_profile(), {frame, frame}, cams, sparse, f,
                                                false, c);
    CHECK(r.stats.attempted);
    CHECK(!r.stats.skip_reason);
    CHECK(r.points.empty());
    CHECK(r.stats.accepted_points == 0);
    CHECK(r.stats.surface_completed_points == 0);
    CHECK(r.stats.surface_completion_proposals == 0);
}

void does_not_attempt_dense_depth_without_registered_baseline() {  // dense_legacy.rs:1480
    uint32_t w = 68, h = 48;
    double f = 60.0;
    auto sparse = plane_sparse_points(w, h, f, 4.0);
    Control c = never();
    auto r = estimate_depth_points_with_control(reference_profile(), {plane_frame(w, h, f, 0, 4)},
                                                {camera(0, 0.0)}, sparse, f, false, c);
    CHECK(!r.stats.attempted);
    CHECK(r.stats.skip_reason &&
          r.stats.skip_reason->find("two accepted registered cameras") != std::string::npos);
    CHECK(r.points.empty());
}

void visible_depths_ignore_offscreen_landmarks() {  // dense_legacy.rs:1499
    auto d = visible_depths(camera(0, 0.0), {{0, 0, 4}, {100, 0, 4}, {0, -100, 4}}, 68, 48, 60.0);
    CHECK((d == std::vector<double>{4.0}));
}

// ---------------- dense.rs tests ----------------

void clustered_landmark_scan_can_be_canceled_within_one_camera() {  // dense.rs:1089
    std::vector<Frame> frames(1);
    frames[0].width = 240;
    frames[0].height = 240;
    std::vector<Vec3> pts(4096, Vec3{0, 0, 4});
    int polls = 0;
    Control c;
    c.poll = [&]() { return ++polls == 3; };
    CHECK(!has_distributed_landmarks(frames, {camera(0, 0.0)}, pts, 200.0, c));
    CHECK(c.is_canceled());
    CHECK(polls == 3);
}

void finer_dense_grid_requires_distributed_landmarks() {  // dense.rs:1114 (dense-pass half)
    uint32_t w = 240, h = 240;
    double f = 200.0;
    Frame frame = flat_frame(w, h, 128);
    std::vector<Frame> frames{frame, frame};
    std::vector<Camera> cams{camera(0, 0.0), camera(1, 0.2)};
    auto world = [&](double x, double y) {
        return Vec3{(x - 120.0) / f * 4.0, (y - 120.0) / f * 4.0, 4.0};
    };
    std::vector<Vec3> distributed, concentrated;
    for (double y : {30.0, 90.0, 150.0, 210.0})
        for (double x : {30.0, 90.0, 150.0, 210.0}) {
            distributed.push_back(world(x, y));
            distributed.push_back(world(x + 2.0, y));
        }
    for (size_t i = 0; i < distributed.size(); ++i) concentrated.push_back(world(90.0 + i, 90.0));
    CHECK(grid_stride(w, h, true) < grid_stride(w, h, false));
    for (auto [sparse, expected] : {std::make_pair(&distributed, size_t(4)),
                                    std::make_pair(&concentrated, size_t(5))}) {
        Control c1 = never(), c2 = never();
        bool fine = has_distributed_landmarks(frames, cams, *sparse, f, c1);
        auto r = estimate_depth_points_limited(reference_profile(), frames, cams, *sparse, f, 3,
                                               fine, c2)
                     .first;
        CHECK(r.stats.grid_stride == expected);
        CHECK(r.points.empty());
    }
    // Third case: a budget that only fits the coarse plan runs with fine_grid=false.
    Control c3 = never();
    auto r = estimate_depth_points_limited(reference_profile(), frames, cams, distributed, f, 3,
                                           false, c3)
                 .first;
    CHECK(r.stats.grid_stride == 5);
}

void reconstructs_multiple_reference_patches_without_relaxing_dense_gates() {  // dense.rs:1210
    uint32_t w = 68, h = 48;
    double f = 60.0, depth = 4.0;
    std::vector<Frame> frames{plane_frame(w, h, f, 0.0, depth), plane_frame(w, h, f, 0.24, depth),
                              plane_frame(w, h, f, -0.22, depth)};
    std::vector<Camera> cams{camera(0, 0.0), camera(1, 0.24), camera(2, -0.22)};
    auto r = dense_estimate(frames, cams, plane_sparse_points(w, h, f, depth), f);
    const DenseStats& s = r.stats;
    CHECK(s.attempted);
    CHECK(s.reference_frames.size() >= 2);
    CHECK(s.reference_frames.size() == s.reference_patches.size());
    size_t accepted = 0;
    bool all = true;
    for (auto& a : s.reference_attempts) {
        accepted += a.accepted;
        all = all && (a.accepted || a.skip_reason);
    }
    CHECK(s.reference_patches.size() == accepted);
    CHECK(all);
    CHECK(r.points.size() == r.grid_sites.size());
    CHECK(r.points.size() == r.point_attributes.size());
    bool in_range = true;
    for (auto& a : r.point_attributes)
        in_range = in_range && a.reciprocal_consistency >= 0 && a.reciprocal_consistency <= 1 &&
                   a.depth_margin >= 0 && a.depth_margin <= 1;
    CHECK(in_range);
    CHECK(r.points.size() == s.accepted_points);
    CHECK(s.surface_completion_proposals ==
          s.surface_completed_points + s.surface_completion_rejected_texture +
              s.surface_completion_rejected_cross_view + s.surface_completion_rejected_reciprocal +
              s.surface_completion_rejected_fusion + s.surface_completion_rejected_footprint);
    CHECK(s.source_frames.size() == s.source_views);
    CHECK(s.reference_frame.has_value());
    CHECK(std::find(s.source_frames.begin(), s.source_frames.end(), *s.reference_frame) ==
          s.source_frames.end());
}

bool same_bits(const Point3& a, const Point3& b) {
    return std::memcmp(&a.x, &b.x, 4) == 0 && std::memcmp(&a.y, &b.y, 4) == 0 &&
           std::memcmp(&a.z, &b.z, 4) == 0 && std::memcmp(&a.confidence, &b.confidence, 4) == 0;
}

void a_tight_budget_keeps_the_leading_reference_patches_of_the_full_run() {  // dense.rs:1297
    uint32_t w = 68, h = 48;
    double f = 60.0, depth = 4.0;
    std::vector<Frame> frames{plane_frame(w, h, f, 0.0, depth), plane_frame(w, h, f, 0.24, depth),
                              plane_frame(w, h, f, -0.22, depth)};
    std::vector<Camera> cams{camera(0, 0.0), camera(1, 0.24), camera(2, -0.22)};
    auto sparse = plane_sparse_points(w, h, f, depth);
    auto full = dense_estimate(frames, cams, sparse, f);
    CHECK(full.stats.reference_patches.size() >= 2);
    // 68x48 has equal fine and coarse strides, so the budget plan runs coarse.
    Control c = never();
    auto lim = estimate_depth_points_limited(reference_profile(), frames, cams, sparse, f, 1, false, c);
    CHECK(lim.first.stats.attempted);
    CHECK(lim.second);  // a candidate remained: reference_view_limit = Some(1)
    CHECK(lim.first.stats.reference_patches.size() == 1);
    if (full.stats.reference_patches.empty() || lim.first.stats.reference_patches.empty()) return;
    const PatchStats& kept = lim.first.stats.reference_patches[0];
    const PatchStats& lead = full.stats.reference_patches[0];
    CHECK(kept.reference_frame == lead.reference_frame);
    std::vector<Point3> expected(full.points.begin() + lead.primary_start,
                                 full.points.begin() + lead.primary_start + lead.primary_points);
    expected.insert(expected.end(), full.points.begin() + lead.completion_start,
                    full.points.begin() + lead.completion_start + lead.completed_points);
    CHECK(lim.first.points.size() == expected.size());
    bool same = lim.first.points.size() == expected.size();
    for (size_t i = 0; same && i < expected.size(); ++i) same = same_bits(expected[i], lim.first.points[i]);
    CHECK(same);
    Control c2 = never();
    auto wider = estimate_depth_points_limited(reference_profile(), frames, cams, sparse, f, 2, false, c2);
    CHECK(wider.second);  // reference_view_limit = Some(2)
    CHECK(wider.first.stats.reference_patches.size() ==
          std::min<size_t>(full.stats.reference_patches.size(), 2));
}

void budget_above_estimate_preserves_dense_output() {  // dense.rs:1360 (dense-pass half)
    uint32_t w = 68, h = 48;
    double f = 60.0, depth = 4.0;
    std::vector<Frame> frames{plane_frame(w, h, f, 0.0, depth), plane_frame(w, h, f, 0.24, depth),
                              plane_frame(w, h, f, -0.22, depth)};
    std::vector<Camera> cams{camera(0, 0.0), camera(1, 0.24), camera(2, -0.22)};
    auto sparse = plane_sparse_points(w, h, f, depth);
    auto base = dense_estimate(frames, cams, sparse, f);
    Control c = never();
    auto budgeted =
        estimate_depth_points_limited(reference_profile(), frames, cams, sparse, f, 3, false, c).first;
    CHECK(base.points.size() == budgeted.points.size());
    CHECK(base.grid_sites.size() == budgeted.grid_sites.size());
    bool same = base.points.size() == budgeted.points.size();
    for (size_t i = 0; same && i < base.points.size(); ++i)
        same = same_bits(base.points[i], budgeted.points[i]) && base.points[i].r == budgeted.points[i].r &&
               base.grid_sites[i].x == budgeted.grid_sites[i].x &&
               base.grid_sites[i].y == budgeted.grid_sites[i].y &&
               base.point_attributes[i].reciprocal_consistency ==
                   budgeted.point_attributes[i].reciprocal_consistency &&
               base.point_attributes[i].depth_margin == budgeted.point_attributes[i].depth_margin;
    CHECK(same);
}

void a_limit_that_omits_no_reference_is_not_reported() {  // dense.rs:1451
    uint32_t w = 68, h = 48;
    double f = 60.0, depth = 4.0;
    std::vector<Frame> frames{plane_frame(w, h, f, 0.0, depth), plane_frame(w, h, f, 0.24, depth)};
    std::vector<Camera> cams{camera(0, 0.0), camera(1, 0.24)};
    Control c = never();
    auto lim = estimate_depth_points_limited(reference_profile(), frames, cams,
                                             plane_sparse_points(w, h, f, depth), f, 2, false, c);
    CHECK(!lim.second);
}

void rejected_reference_attempt_keeps_its_diagnostics() {  // dense.rs:1489
    LegacyStats s;
    s.attempted = true;
    s.sampled_pixels = 41;
    s.reciprocal_checked_points = 2;
    s.reciprocal_rejected_points = 1;
    s.reciprocal_consistent_points = 1;
    s.surface_completion_proposals = 3;
    s.surface_completed_points = 1;
    s.surface_completion_rejected_cross_view = 2;
    AttemptStats a = reference_attempt_stats(7, s, 2, false);
    CHECK(a.attempted);
    CHECK(!a.accepted);
    CHECK(a.reference_frame == 7);
    CHECK(a.sampled_pixels == 41);
    CHECK(a.accepted_points == 2);
    CHECK(a.reciprocal_checked_points == 2);
    CHECK(a.reciprocal_rejected_points == 1);
    CHECK(a.reciprocal_consistent_points == 1);
    CHECK(a.surface_completion_proposals == 3);
    CHECK(a.surface_completed_points == 1);
    CHECK(a.surface_completion_rejected_cross_view == 2);
    CHECK(a.skip_reason && a.skip_reason->find("at least 3") != std::string::npos);
}

void successful_fallback_evidence_replaces_rejected_attempt() {  // dense.rs:1522
    AttemptStats rejected;
    rejected.reference_frame = 3;
    rejected.attempted = true;
    rejected.skip_reason = "remapped reference rejected";
    rejected.accepted_points = 1;
    AttemptStats other;
    other.reference_frame = 5;
    other.attempted = true;
    other.skip_reason = "another reference rejected";
    AttemptStats fb;
    fb.reference_frame = 3;
    fb.attempted = true;
    fb.accepted = true;
    fb.accepted_points = 9;
    auto merged = merge_fallback_attempts({rejected, other}, {fb});
    CHECK(merged.size() == 2);
    const AttemptStats* acc = nullptr;
    for (auto& m : merged)
        if (m.reference_frame == 3) acc = &m;
    CHECK(acc && acc->accepted && acc->accepted_points == 9 && !acc->skip_reason);
    bool five = false;
    for (auto& m : merged) five = five || (m.reference_frame == 5 && !m.accepted);
    CHECK(five);
}

// ---------------- surface_completion_tests.rs ----------------

void verified_surface_completion_adds_expected_plane_geometry() {  // surface_completion_tests.rs:55
    uint32_t w = 68, h = 48;
    double f = 60.0, depth = 4.0;
    std::vector<Frame> frames{plane_frame(w, h, f, 0.0, depth), plane_frame(w, h, f, 0.25, depth),
                              plane_frame(w, h, f, -0.22, depth)};
    std::vector<Camera> cams{camera(0, 0.0), camera(1, 0.25), camera(2, -0.22)};
    auto r = dense_estimate(frames, cams, plane_sparse_points(w, h, f, depth), f);
    const DenseStats& s = r.stats;
    CHECK(s.attempted);
    CHECK(s.surface_completion_proposals > 0);
    CHECK(s.surface_completed_points > 0);
    CHECK(s.surface_completion_proposals ==
          s.surface_completed_points + s.surface_completion_rejected_texture +
              s.surface_completion_rejected_cross_view + s.surface_completion_rejected_reciprocal +
              s.surface_completion_rejected_fusion + s.surface_completion_rejected_footprint);
    CHECK(r.points.size() >= s.surface_completed_points);
    size_t primary = r.points.size() - s.surface_completed_points;
    bool ok = true;
    for (size_t i = primary; i < r.points.size(); ++i)
        ok = ok && std::fabs(static_cast<double>(r.points[i].z) - depth) < 0.55 &&
             r.points[i].confidence >= 0.05f && r.points[i].confidence <= 0.9f;
    CHECK(ok);
}

// ---------------- mesh_legacy.rs tests ----------------

Point3 mesh_point(double x, double y, double depth, uint32_t w, uint32_t h, double f, float conf) {
    return {static_cast<float>((x - w * 0.5) / f * depth), static_cast<float>((y - h * 0.5) / f * depth),
            static_cast<float>(depth), conf, 120, 140, 160};
}

MeshDenseInput mesh_dense() {
    MeshDenseInput d;
    d.attempted = true;
    d.reference_frame = 0;
    d.grid_stride = 4;
    d.grid_border = 3;
    return d;
}

// mesh_legacy.rs:111-148 (#[cfg(test)] reconstruct_dense_mesh)
MeshAnalysis legacy_mesh(const std::vector<Point3>& p, const std::vector<GridSite>& s) {
    Camera c;
    MeshDenseInput d = mesh_dense();
    if (p.size() < 3) {
        MeshAnalysis m;
        m.stats.reference_frame = d.reference_frame;
        m.stats.skip_reason = "fewer than three accepted fused dense points are available";
        return m;
    }
    Control ctl = never();
    return reconstruct_dense_mesh_samples(p, s, d, {c}, 68, 48, 60.0, ctl);
}

std::vector<GridSite> four_sites() { return {{3, 3}, {7, 3}, {3, 7}, {7, 7}}; }

bool has_triangle(const MeshAnalysis& m, size_t a, size_t b, size_t c) {
    for (auto& t : m.triangles) {
        size_t i[3] = {t.a, t.b, t.c};
        std::sort(i, i + 3);
        if (i[0] == a && i[1] == b && i[2] == c) return true;
    }
    return false;
}

void mesh_tests() {
    const uint32_t w = 68, h = 48;
    const double f = 60.0;
    {
        g_test = "preserves_admission_stats_when_too_few_grid_vertices_survive";  // :609
        auto m = legacy_mesh({mesh_point(3, 3, 4, w, h, f, 0.8f), mesh_point(7, 3, 4, w, h, f, 0.7f),
                              mesh_point(6, 7, 4, w, h, f, 0.9f)},
                             {{3, 3}, {7, 3}, {3, 7}});
        CHECK(m.stats.attempted);
        CHECK(m.stats.skip_reason.has_value());
        CHECK(m.stats.grid_vertices == 2);
        CHECK(m.stats.rejected_grid_vertices == 1);
        CHECK(m.triangles.empty());
    }
    {
        g_test = "triangulates_a_smooth_reference_grid_quad";  // :642
        auto m = legacy_mesh({mesh_point(3, 3, 4, w, h, f, 0.8f), mesh_point(7, 3, 4, w, h, f, 0.7f),
                              mesh_point(3, 7, 4, w, h, f, 0.9f), mesh_point(7, 7, 4, w, h, f, 0.6f)},
                             four_sites());
        CHECK(m.stats.attempted);
        CHECK(m.stats.grid_vertices == 4);
        CHECK(m.stats.candidate_cells == 1);
        CHECK(m.stats.candidate_triangles == 2);
        CHECK(m.stats.accepted_triangles == 2);
        CHECK(m.stats.rejected_discontinuities == 0);
        CHECK(m.stats.rejected_degenerate == 0);
        CHECK(m.triangles.size() == 2);
        bool ok = true;
        for (auto& t : m.triangles) ok = ok && t.a < 4 && t.b < 4 && t.c < 4 && t.confidence <= 0.8f;
        CHECK(ok);
    }
    std::vector<GridSite> bridge_sites{{3, 3}, {11, 3}, {3, 7}, {11, 7}, {7, 7}};
    {
        g_test = "bridges_one_missing_grid_sample_on_a_smooth_surface";  // :682
        std::vector<Point3> p;
        for (auto& s : bridge_sites) p.push_back(mesh_point(s.x, s.y, 4, w, h, f, 0.8f));
        auto m = legacy_mesh(p, bridge_sites);
        CHECK(m.stats.attempted);
        CHECK(m.stats.grid_vertices == 5);
        CHECK(m.stats.accepted_triangles == 3);
        CHECK(has_triangle(m, 0, 1, 4));
    }
    {
        g_test = "does_not_bridge_a_missing_sample_across_a_depth_discontinuity";  // :719
        auto m = legacy_mesh({mesh_point(3, 3, 4, w, h, f, 0.8f), mesh_point(11, 3, 5, w, h, f, 0.8f),
                              mesh_point(3, 7, 4, w, h, f, 0.8f), mesh_point(11, 7, 5, w, h, f, 0.8f),
                              mesh_point(7, 7, 4, w, h, f, 0.8f)},
                             bridge_sites);
        CHECK(m.stats.attempted);
        CHECK(m.stats.rejected_discontinuities > 0);
        CHECK(!has_triangle(m, 0, 1, 4));
    }
    {
        g_test = "rejects_triangles_that_bridge_a_depth_discontinuity";  // :758
        auto m = legacy_mesh({mesh_point(3, 3, 4, w, h, f, 0.8f), mesh_point(7, 3, 4, w, h, f, 0.8f),
                              mesh_point(3, 7, 4, w, h, f, 0.8f), mesh_point(7, 7, 7, w, h, f, 0.8f)},
                             four_sites());
        CHECK(m.stats.attempted);
        CHECK(m.stats.candidate_triangles == 2);
        CHECK(m.stats.accepted_triangles < m.stats.candidate_triangles);
        CHECK(m.stats.rejected_discontinuities > 0);
        CHECK(m.stats.accepted_triangles > 0);
    }
    {
        g_test = "preserves_original_grid_site_after_fusion_shifts_reprojection";  // :787
        auto m = legacy_mesh({mesh_point(4.8, 3, 4, w, h, f, 0.8f), mesh_point(7, 3, 4, w, h, f, 0.8f),
                              mesh_point(3, 7, 4, w, h, f, 0.8f)},
                             {{3, 3}, {7, 3}, {3, 7}});
        CHECK(m.stats.attempted);
        CHECK(m.stats.grid_vertices == 3);
        CHECK(m.stats.accepted_triangles == 1);
    }
    {
        g_test = "rejects_fused_vertex_that_leaves_original_grid_footprint";  // :818
        auto m = legacy_mesh({mesh_point(5.4, 3, 4, w, h, f, 0.8f), mesh_point(7, 3, 4, w, h, f, 0.8f),
                              mesh_point(3, 7, 4, w, h, f, 0.8f), mesh_point(7, 7, 4, w, h, f, 0.8f)},
                             four_sites());
        CHECK(m.stats.attempted);
        CHECK(m.stats.grid_vertices == 3);
        CHECK(m.stats.accepted_triangles == 1);
        bool ok = true;
        for (auto& t : m.triangles) ok = ok && t.a != 0 && t.b != 0 && t.c != 0;
        CHECK(ok);
    }
    {
        g_test = "rejects_triangle_that_flips_reference_projection_winding";  // :848
        auto m = legacy_mesh({mesh_point(4.9, 1.1, 4, w, h, f, 0.8f), mesh_point(5.1, 4.9, 4, w, h, f, 0.8f),
                              mesh_point(8.9, 5.1, 4, w, h, f, 0.8f)},
                             {{3, 3}, {7, 3}, {7, 7}});
        CHECK(m.stats.attempted);
        CHECK(m.stats.grid_vertices == 3);
        CHECK(m.stats.candidate_triangles == 1);
        CHECK(m.stats.accepted_triangles == 0);
        CHECK(m.stats.rejected_degenerate == 1);
    }
    {
        g_test = "does_not_attempt_mesh_without_enough_dense_points";  // :881
        auto m = legacy_mesh({mesh_point(3, 3, 4, w, h, f, 0.8f), mesh_point(7, 3, 4, w, h, f, 0.8f)},
                             four_sites());
        CHECK(!m.stats.attempted);
        CHECK(m.triangles.empty());
        CHECK(m.stats.skip_reason &&
              m.stats.skip_reason->find("three accepted fused dense points") != std::string::npos);
    }
    {
        g_test = "combines_reference_meshes_using_global_dense_point_indices";  // mesh.rs:310
        std::vector<GridSite> sites = four_sites();
        std::vector<Point3> p;
        for (auto& s : sites) p.push_back(mesh_point(s.x, s.y, 4, w, h, f, 0.8f));
        std::vector<Point3> pts = p;
        pts.insert(pts.end(), p.begin(), p.end());
        std::vector<GridSite> gs = sites;
        gs.insert(gs.end(), sites.begin(), sites.end());
        MeshDenseInput d = mesh_dense();
        PatchStats a, b;
        a.reference_frame = 0;
        a.primary_start = 0;
        a.primary_points = 4;
        a.completion_start = 4;
        a.grid_stride = 4;
        a.grid_border = 3;
        a.accepted_points = 4;
        b = a;
        b.reference_frame = 1;
        b.primary_start = 4;
        b.completion_start = 8;
        d.reference_patches = {a, b};
        Camera c0, c1;
        c1.frame_index = 1;
        Control ctl = never();
        auto m = reconstruct_dense_mesh_with_control(pts, gs, d, {c0, c1}, w, h, f, ctl);
        CHECK(m.stats.attempted);
        CHECK((m.reference_frames == std::vector<size_t>{0, 1}));
        CHECK(m.reference_patches.size() == 2);
        CHECK(m.stats.accepted_triangles == 4);
        CHECK(m.triangles.size() == 4);
        bool second = false;
        for (auto& t : m.triangles) second = second || (t.a >= 4 && t.b >= 4 && t.c >= 4);
        CHECK(second);
    }
}

// ---- surface_fusion.rs:891-1070 and fusion_prepass_acceptance_tests.rs ----
Point3 fpoint(float x, float y, float z, float c) { return Point3{x, y, z, c, 128, 128, 128}; }
MeshTriangle ftri(size_t a, size_t b, size_t c) { return MeshTriangle{a, b, c, 0.9f}; }

// surface_fusion.rs:891-915
void groups_evidence_regions_by_camera_support_instead_of_dense_patch_identity() {
    std::vector<EvidenceRegion> regions = {
        {0, {2, 1}, 0, 2}, {0, {1, 2}, 2, 1}, {3, {4}, 3, 1}, {std::nullopt, {}, 4, 1}};
    auto [membership, groups] = evidence_support_membership(regions, 5);
    CHECK(groups == 2);
    CHECK((membership == std::vector<int64_t>{0, 0, 0, 1, -1}));
}

// surface_fusion.rs:917-940
void aligns_mutually_nearest_vertices_from_consistent_evidence_groups() {
    std::vector<Point3> pts = {fpoint(0, 0, 0, 1), fpoint(1, 0, 0, 1), fpoint(0, 1, 0, 1),
                               fpoint(0, 0, 0.06f, 1), fpoint(1, 0, 0.06f, 1),
                               fpoint(0, 1, 0.06f, 1)};
    std::vector<MeshTriangle> tris = {ftri(0, 1, 2), ftri(3, 4, 5)};
    std::vector<int64_t> mem = {0, 0, 0, 1, 1, 1};
    Control ctl = never();
    FusionStats st = fuse_mutually_supported_vertices(pts, tris, mem, ctl).stats;
    CHECK(st.fused_pairs == 3);
    CHECK(st.rejected_normal_pairs == 0);
    CHECK(st.rejected_topology_pairs == 0);
    for (auto [l, r] : {std::pair<int, int>{0, 3}, {1, 4}, {2, 5}}) {
        CHECK(std::fabs(pts[l].z - 0.03f) < 1.0e-6f);
        CHECK(std::fabs(pts[l].z - pts[r].z) < 1.0e-6f);
    }
}

// surface_fusion.rs:942-961
void rejects_nearby_vertices_when_surface_normals_disagree() {
    std::vector<Point3> pts = {fpoint(0, 0, 0, 1), fpoint(1, 0, 0, 1), fpoint(0, 1, 0, 1),
                               fpoint(0, 0, 0.05f, 1), fpoint(1, 0, 0.05f, 1),
                               fpoint(0, 0.05f, 1, 1)};
    std::vector<MeshTriangle> tris = {ftri(0, 1, 2), ftri(3, 4, 5)};
    std::vector<int64_t> mem = {0, 0, 0, 1, 1, 1};
    Control ctl = never();
    FusionStats st = fuse_mutually_supported_vertices(pts, tris, mem, ctl).stats;
    CHECK(st.fused_pairs == 0);
    CHECK(st.rejected_normal_pairs >= 2);
    CHECK(pts[0].z == 0.0f);
    CHECK(pts[3].z == 0.05f);
}

// surface_fusion.rs:963-982
void rejects_a_seam_move_that_would_weaken_an_accepted_triangle() {
    std::vector<Point3> pts = {fpoint(0, 0, 0, 1), fpoint(1, 0, 0, 1), fpoint(0.9f, 0.01f, 0, 1),
                               fpoint(0, 0.12f, 0, 1), fpoint(1, 0.12f, 0, 1),
                               fpoint(0, 1.12f, 0, 1)};
    std::vector<MeshTriangle> tris = {ftri(0, 1, 2), ftri(3, 4, 5)};
    std::vector<int64_t> mem = {0, 0, 0, 1, 1, 1};
    Control ctl = never();
    FusionStats st = fuse_mutually_supported_vertices(pts, tris, mem, ctl).stats;
    CHECK(st.fused_pairs == 0);
    CHECK(st.rejected_topology_pairs > 0);
    CHECK(pts[0].y == 0.0f);
    CHECK(pts[3].y == 0.12f);
}

// surface_fusion.rs:984-1010
void validates_the_complete_move_set_against_original_topology() {
    std::vector<Point3> pts = {fpoint(0, 0, 0, 1), fpoint(1, 0, 0, 1), fpoint(0, 1, 0, 1),
                               fpoint(0.2f, 0, 0, 1), fpoint(0.8f, 0, 0, 1)};
    std::vector<MeshTriangle> tris = {ftri(0, 1, 2)};
    std::vector<std::vector<size_t>> incident = {{0}, {0}, {0}, {}, {}};
    std::vector<FusionMove> moves = {FusionMove{0, 3, Vec3{0.2, 0, 0}},
                                     FusionMove{1, 4, Vec3{0.8, 0, 0}}};
    Control ctl = never();
    auto [accepted, rejected] = topology_safe_moves(pts, tris, incident, moves, ctl);
    CHECK(accepted.empty());
    CHECK(rejected == 2);
}

// surface_fusion.rs:1012-1027
void never_fuses_vertices_from_the_same_evidence_group() {
    std::vector<Point3> pts = {fpoint(0, 0, 0, 1), fpoint(1, 0, 0, 1), fpoint(0, 1, 0, 1)};
    std::vector<MeshTriangle> tris = {ftri(0, 1, 2)};
    std::vector<int64_t> mem = {0, 0, 0};
    Control ctl = never();
    FusionStats st = fuse_mutually_supported_vertices(pts, tris, mem, ctl).stats;
    CHECK(st.fused_pairs == 0);
    CHECK(st.candidate_pairs == 0);
}

// fusion_prepass_acceptance_tests.rs:31-57 and :59-79 (evidence of 4096
// repeated triangles; a cancellation after entry yields no partial evidence)
void controlled_fusion_prepass_preserves_actual_geometry_evidence() {
    std::vector<Point3> pts = {fpoint(0, 0, 0, 0.9f), fpoint(1, 0, 0, 0.9f), fpoint(0, 1, 0, 0.9f)};
    std::vector<MeshTriangle> tris(4096, ftri(0, 1, 2));
    int polls = 0;
    Control ctl;
    ctl.poll = [&] {
        ++polls;
        return false;
    };
    auto ev = vertex_surface_evidence(pts, tris, ctl);
    CHECK(ev.has_value());
    if (!ev) return;
    CHECK(polls > 4);
    CHECK(ev->global_edge_scale.has_value() && *ev->global_edge_scale == 1.0);
    bool normals = ev->normals.size() == 3;
    for (auto& n : ev->normals) normals = normals && n && n->x == 0 && n->y == 0 && n->z == 1;
    CHECK(normals);
    std::vector<size_t> all(tris.size());
    for (size_t i = 0; i < all.size(); ++i) all[i] = i;
    CHECK((ev->incident == std::vector<std::vector<size_t>>(3, all)));
    for (int cancel_at : {2, 4}) {
        int k = 0;
        Control c2;
        c2.poll = [&] { return ++k >= cancel_at; };
        CHECK(!vertex_surface_evidence(pts, tris, c2).has_value());
        CHECK(k >= cancel_at);
    }
}

// ---- colmap_surface.rs:548-759 ----
// colmap_surface.rs:548-631
void sources_verifying_one_sample_share_one_vertex() {
    auto sample = [](uint32_t x, uint32_t y, float c) {
        return std::make_pair(Point3{(float)x, (float)y, 5.f, c, 1, 2, 3}, GridSite{x, y});
    };
    std::vector<std::pair<size_t, std::vector<std::pair<Point3, GridSite>>>> cand = {
        {7, {sample(0, 0, 0.9f), sample(4, 0, 0.9f), sample(0, 4, 0.9f), sample(4, 4, 0.9f)}},
        {3, {sample(4, 0, 0.95f), sample(8, 0, 0.95f), sample(4, 4, 0.8f), sample(8, 4, 0.95f)}}};
    auto u = verified_union(cand);
    std::vector<std::pair<uint32_t, uint32_t>> sites;
    for (auto& v : u) sites.emplace_back(v.site.x, v.site.y);
    CHECK((sites == std::vector<std::pair<uint32_t, uint32_t>>{{0, 0}, {4, 0}, {8, 0}, {0, 4}, {4, 4}, {8, 4}}));
    std::vector<std::vector<size_t>> srcs;
    for (auto& v : u) srcs.push_back(v.sources);
    CHECK((srcs == std::vector<std::vector<size_t>>{{7}, {3, 7}, {3}, {7}, {3, 7}, {3}}));
    CHECK(u.size() == 6 && u[1].point.confidence == 0.95f && u[4].point.confidence == 0.9f);
    if (u.size() != 6) return;
    std::vector<Camera> cams(3);
    cams[0].frame_index = 0;
    cams[1].frame_index = 3;
    cams[2].frame_index = 7;
    std::vector<Point3> pts;
    std::vector<GridSite> gs;
    for (auto& v : u) {
        Point3 p = v.point;
        p.x = ((float)v.site.x + 0.5f - 6.f) / 20.f * 5.f;
        p.y = ((float)v.site.y + 0.5f - 4.f) / 20.f * 5.f;
        pts.push_back(p);
        gs.push_back(v.site);
    }
    MeshDenseInput d;
    d.attempted = true;
    d.reference_frame = 0;
    d.grid_stride = 4;
    Control ctl = never();
    auto m = reconstruct_dense_mesh_with_control(pts, gs, d, cams, 12, 8, 20.0, ctl);
    CHECK(m.triangles.size() == 4);
    CHECK(surface_topology(pts.size(), m.triangles).islands == 1);
}

// colmap_surface.rs:633-730
void plane_requires_agreeing_depth_color_and_camera_baseline() {
    std::vector<uint8_t> frame(24 * 16 * 4, 100), other_color(24 * 16 * 4, 200);
    std::vector<float> map(24, 5.f), wrong(24, 8.f);
    Camera first, second;
    second.frame_index = 1;
    second.t[0] = -1.0;
    DepthView reference{24, 16, frame.data(), map.data(), first};
    DepthView source{24, 16, frame.data(), map.data(), second};
    Funnel f;
    CHECK(verify_patch(reference, source, 4, 4, 20.0, f).size() == 20);
    CHECK(f.reference_samples == 24 && f.outside_source == 4 && f.accepted == 20 &&
          f.missing_reference_depth == 0 && f.insufficient_parallax == 0 && f.behind_source == 0 &&
          f.missing_source_depth == 0 && f.depth_disagreement == 0 && f.color_disagreement == 0);
    Funnel g;
    auto coarse = verify_patch(reference, source, 4, 8, 20.0, g);
    CHECK(coarse.size() == 4);
    bool on = true;
    for (auto& [p, site] : coarse) on = on && site.x % 8 == 0 && site.y % 8 == 0;
    CHECK(on);
    DepthView w = source;
    w.depth = wrong.data();
    DepthView c = source;
    c.rgba = other_color.data();
    DepthView pa = source;
    pa.camera = first;
    const std::pair<DepthView, const char*> cases[] = {
        {w, "depth_disagreement"}, {c, "color_disagreement"}, {pa, "insufficient_parallax"}};
    for (auto& [view, expected] : cases) {
        Funnel h;
        CHECK(verify_patch(reference, view, 4, 4, 20.0, h).empty());
        CHECK(h.accepted == 0);
        const char* dom = dominant_rejection(h);
        CHECK(dom && std::string(dom) == expected);
    }
}

// colmap_surface.rs:732-759
void topology_counts_islands_and_open_boundaries() {
    auto face = [](size_t a, size_t b, size_t c) { return MeshTriangle{a, b, c, 1.f}; };
    std::vector<MeshTriangle> tris = {face(0, 1, 2), face(1, 3, 2), face(4, 5, 6), face(5, 7, 6)};
    Topology t = surface_topology(8, tris);
    CHECK(t.islands == 2 && t.small_islands == 2 && t.small_island_triangles == 4 &&
          t.largest_island_triangles == 2 && t.boundary_edges == 8);
    std::vector<MeshTriangle> large;
    for (size_t i = 0; i < 32; ++i) large.push_back(face(i, i + 1, i + 2));
    Topology l = surface_topology(34, large);
    CHECK(l.islands == 1 && l.small_islands == 0 && l.largest_island_triangles == 32);
}

struct Test {
    const char* name;
    void (*fn)();
};

}  // namespace

extern "C" int32_t v3do_selftest(char* report, uint64_t capacity, int32_t* checks) {
    g_report.clear();
    g_failures = 0;
    g_checks = 0;
    const Test tests[] = {
        {"estimates_coarse_depth_on_textured_plane", estimates_coarse_depth_on_textured_plane},
        {"surface_completion_reports_texture_rejections", surface_completion_reports_texture_rejections},
        {"surface_depth_prediction_requires_consistent_neighbors",
         surface_depth_prediction_requires_consistent_neighbors},
        {"reciprocal_depth_search_recovers_source_view_depth",
         reciprocal_depth_search_recovers_source_view_depth},
        {"fusion_rejects_spatially_inconsistent_reciprocal_observations",
         fusion_rejects_spatially_inconsistent_reciprocal_observations},
        {"reciprocal_consistency_rejects_wrong_depth", reciprocal_consistency_rejects_wrong_depth},
        {"rejects_textureless_depth_hypotheses", rejects_textureless_depth_hypotheses},
        {"does_not_attempt_dense_depth_without_registered_baseline",
         does_not_attempt_dense_depth_without_registered_baseline},
        {"visible_depths_ignore_offscreen_landmarks", visible_depths_ignore_offscreen_landmarks},
        {"clustered_landmark_scan_can_be_canceled_within_one_camera",
         clustered_landmark_scan_can_be_canceled_within_one_camera},
        {"finer_dense_grid_requires_distributed_landmarks", finer_dense_grid_requires_distributed_landmarks},
        {"reconstructs_multiple_reference_patches_without_relaxing_dense_gates",
         reconstructs_multiple_reference_patches_without_relaxing_dense_gates},
        {"a_tight_budget_keeps_the_leading_reference_patches_of_the_full_run",
         a_tight_budget_keeps_the_leading_reference_patches_of_the_full_run},
        {"budget_above_estimate_preserves_dense_output", budget_above_estimate_preserves_dense_output},
        {"a_limit_that_omits_no_reference_is_not_reported", a_limit_that_omits_no_reference_is_not_reported},
        {"rejected_reference_attempt_keeps_its_diagnostics", rejected_reference_attempt_keeps_its_diagnostics},
        {"successful_fallback_evidence_replaces_rejected_attempt",
         successful_fallback_evidence_replaces_rejected_attempt},
        {"verified_surface_completion_adds_expected_plane_geometry",
         verified_surface_completion_adds_expected_plane_geometry},
        {"mesh_legacy_and_mesh_tests", mesh_tests},
        {"groups_evidence_regions_by_camera_support_instead_of_dense_patch_identity",
         groups_evidence_regions_by_camera_support_instead_of_dense_patch_identity},
        {"aligns_mutually_nearest_vertices_from_consistent_evidence_groups",
         aligns_mutually_nearest_vertices_from_consistent_evidence_groups},
        {"rejects_nearby_vertices_when_surface_normals_disagree",
         rejects_nearby_vertices_when_surface_normals_disagree},
        {"rejects_a_seam_move_that_would_weaken_an_accepted_triangle",
         rejects_a_seam_move_that_would_weaken_an_accepted_triangle},
        {"validates_the_complete_move_set_against_original_topology",
         validates_the_complete_move_set_against_original_topology},
        {"never_fuses_vertices_from_the_same_evidence_group",
         never_fuses_vertices_from_the_same_evidence_group},
        {"controlled_fusion_prepass_preserves_actual_geometry_evidence",
         controlled_fusion_prepass_preserves_actual_geometry_evidence},
        {"sources_verifying_one_sample_share_one_vertex", sources_verifying_one_sample_share_one_vertex},
        {"plane_requires_agreeing_depth_color_and_camera_baseline",
         plane_requires_agreeing_depth_color_and_camera_baseline},
        {"topology_counts_islands_and_open_boundaries", topology_counts_islands_and_open_boundaries},
    };
    std::string names;
    for (const Test& t : tests) {
        g_test = t.name;
        int before = g_failures;
        t.fn();
        names += (g_failures == before ? "ok   " : "FAIL ");
        names += t.name;
        names += "\n";
    }
    std::string full = names + g_report;
    if (report && capacity) {
        std::strncpy(report, full.c_str(), capacity - 1);
        report[capacity - 1] = 0;
    }
    if (checks) *checks = g_checks;
    return g_failures;
}
