// TEST INFRASTRUCTURE — the CPU oracle of the dense plane-sweep pass.
//
// A literal f64 restatement of video-to-3d-core's dense pass
// (crates/video-to-3d-core/src/dense_legacy.rs:1-1182), its multi-reference
// driver (dense.rs:165-330, 620-1082) and the reference-grid triangle gates
// (mesh_legacy.rs:150-555, mesh.rs:74-260).  It keeps the reference's
// evaluation order: stable sorts, quantile() with round-half-away-from-zero,
// IEEE f64 without fused multiply-add, nalgebra's left-to-right 3x3 products
// and dot products, and the f32 casts of the outputs.
//
// Only tests/, the smoke check and bench.py's CPU-baseline leg may load this
// code, and only as the checker or the timed CPU baseline.  The product path
// (video-to-3d_b200/) never links it.
//
// Parity pin: the reference ships no golden output vectors for this path and
// cannot be compiled here (Rust toolchain and crates.io dependencies absent).
// The restatement is pinned by re-running every assertion of the reference's
// own tests for the path (dense_legacy.rs:1261-1514, dense.rs:1089-1562,
// surface_completion_tests.rs:56-113, mesh_legacy.rs:609-908,
// mesh.rs:311-380) in oracle/oracle_selftest.cpp.  Cross-reference surface
// fusion (surface_fusion.rs:316-852, oracle_fusion.cpp) is pinned the same way
// by surface_fusion.rs:891-1070 and fusion_prepass_acceptance_tests.rs:31-57,
// and the geometric depth-grid verification (colmap_surface.rs:56-314,
// oracle_colmap.cpp) by colmap_surface.rs:548-759.
#pragma once

#include <cstdint>
#include <functional>
#include <optional>
#include <string>
#include <vector>

#include "../include/v3d_dense.h"

namespace v3do {

struct Vec3 {
    double x = 0, y = 0, z = 0;
};

inline Vec3 sub(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 add(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
// nalgebra norm_squared: ((x*x + y*y) + z*z)
double norm_squared(Vec3 v);
double norm(Vec3 v);
Vec3 cross(Vec3 a, Vec3 b);

// RegisteredCamera (multi_view.rs:85-94); R row-major.
struct Camera {
    size_t frame_index = 0;
    double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
    double t[3] = {0, 0, 0};
    Vec3 center() const;  // -R^T t
};

// FrameInput plus the other storage formats of the profiles.
struct Frame {
    uint32_t width = 0, height = 0;
    int format = V3D_PIXEL_RGBA8;
    std::vector<uint8_t> bytes;  // raw storage as handed in
};

// Intensity plane read by the sweep: u8 luma, or the decoded gray values.
struct Plane {
    uint32_t width = 0, height = 0;
    std::vector<double> v;
};

struct Profile {
    int cost = V3D_COST_ZSAD;
    int patch_radius = 1;
    int depth_hypotheses = 24;
    int max_source_views = 4;
    int grid_stride = 0;  // 0: dense.rs:215-218
    double min_reference_contrast = 14.0;
    double max_photometric_error = 18.0;
    double min_ambiguity_margin = 1.0;
    double depth_margin_saturation = 6.0;
    double error_confidence_scale = 8.0;
    double min_window_variance = 0.0;
    static Profile from_c(const v3d_profile& p);
};

struct Point3 {
    float x, y, z, confidence;
    uint8_t r, g, b;
};
struct GridSite {
    uint32_t x, y;
};
struct Attr {
    float reciprocal_consistency = 0, depth_margin = 0;
};

// DenseStats (dense_legacy.rs:23-53)
struct LegacyStats {
    bool attempted = false;
    std::optional<std::string> skip_reason;
    int skip_code = 0;
    std::optional<size_t> reference_frame;
    size_t source_views = 0;
    std::vector<size_t> source_frames;
    size_t sampled_pixels = 0, depth_hypotheses = 0, accepted_points = 0;
    size_t surface_completion_proposals = 0, surface_completed_points = 0;
    size_t surface_completion_rejected_texture = 0, surface_completion_rejected_cross_view = 0;
    size_t surface_completion_rejected_reciprocal = 0, surface_completion_rejected_fusion = 0;
    size_t surface_completion_rejected_footprint = 0;
    size_t grid_stride = 0;
    uint32_t grid_border = 0;
    size_t reciprocal_checked_points = 0, reciprocal_rejected_points = 0,
           reciprocal_consistent_points = 0;
    size_t fusion_input_observations = 0, fusion_rejected_observations = 0,
           fusion_rejected_points = 0;
    std::optional<float> median_fusion_observations, median_supporting_views,
        median_photometric_error, search_min_depth, search_max_depth;
};

struct LegacyAnalysis {
    LegacyStats stats;
    std::vector<Point3> points;
    std::vector<GridSite> grid_sites;
    std::vector<Attr> point_attributes;
};

// dense.rs:63-80
struct AttemptStats {
    size_t reference_frame = 0;
    bool attempted = false, accepted = false;
    std::optional<std::string> skip_reason;
    size_t sampled_pixels = 0, accepted_points = 0, reciprocal_checked_points = 0,
           reciprocal_rejected_points = 0, reciprocal_consistent_points = 0,
           surface_completion_proposals = 0, surface_completed_points = 0,
           surface_completion_rejected_texture = 0, surface_completion_rejected_cross_view = 0,
           surface_completion_rejected_reciprocal = 0, surface_completion_rejected_fusion = 0,
           surface_completion_rejected_footprint = 0;
};

// dense.rs:83-97
struct PatchStats {
    size_t reference_frame = 0;
    std::vector<size_t> source_frames;
    size_t primary_start = 0, primary_points = 0, completion_start = 0, completed_points = 0,
           sampled_pixels = 0, accepted_points = 0, reciprocal_consistent_points = 0,
           grid_stride = 0;
    uint32_t grid_border = 0;
    std::optional<float> search_min_depth, search_max_depth;
};

// dense.rs DenseStats/DenseAnalysis (99-148)
struct DenseStats : LegacyStats {
    std::vector<size_t> reference_frames;
    std::vector<AttemptStats> reference_attempts;
    std::vector<PatchStats> reference_patches;
    std::optional<size_t> reference_view_limit;
};
struct DenseAnalysis {
    DenseStats stats;
    std::vector<Point3> points;
    std::vector<GridSite> grid_sites;
    std::vector<Attr> point_attributes;
};

// ReconstructionControl (reconstruction/control.rs:35-57): sticky cancel.
struct Control {
    std::function<bool()> poll;
    bool canceled = false;
    bool is_canceled() {
        if (!canceled && poll && poll()) canceled = true;
        return canceled;
    }
};

struct SourceView {
    const Camera* camera;
    const Frame* frame;
    Plane luma;
    double search_min_depth, search_max_depth;
};

// ---- dense_legacy.rs helpers (exposed for the ported tests) ----
Plane to_luma(const Frame& frame);
double quantile(const std::vector<double>& sorted, double q);
std::optional<double> median_option(std::vector<double>& values);
Vec3 unproject(const Camera& c, double x, double y, double depth, uint32_t w, uint32_t h,
               double focal);
std::optional<Vec3> project(const Camera& c, Vec3 p, uint32_t w, uint32_t h, double focal);
std::optional<double> sample_bilinear(const Plane& img, double x, double y);
bool in_bilinear_bounds(double x, double y, uint32_t w, uint32_t h);
bool in_image_bounds(double x, double y, uint32_t w, uint32_t h);
double patch_contrast(const Plane& img, double x, double y, int radius);
std::optional<double> patch_error(const Profile& prof, const Camera& ref_cam,
                                  const Camera& src_cam, const Plane& ref_img,
                                  const Plane& src_img, double x, double y, double depth,
                                  double focal);
std::vector<double> visible_depths(const Camera& c, const std::vector<Vec3>& sparse, uint32_t w,
                                   uint32_t h, double focal);
std::optional<std::pair<double, double>> depth_search_bounds(const Camera& c,
                                                             const std::vector<Vec3>& sparse,
                                                             uint32_t w, uint32_t h,
                                                             double focal);
std::optional<double> surface_depth_prediction(std::vector<double>& depths);
bool reciprocal_depth_agrees(double expected, double estimated);
struct Fused {
    Vec3 position;
    size_t observations, rejected_observations;
};
Fused fuse_depth_observations(Vec3 primary, const std::vector<Vec3>& reciprocal,
                              double reference_depth);
// `gap`, when given, receives the smallest distance of a cost-based decision of
// the call to the point where it would go the other way (see ExplainRecord).
std::optional<double> estimate_single_view_depth(const Profile& prof, const Camera& ref_cam,
                                                 const Camera& src_cam, const Plane& ref_img,
                                                 const Plane& src_img, double x, double y,
                                                 double search_min, double search_max,
                                                 double focal, double* gap = nullptr);
std::vector<Vec3> reciprocal_depth_observations(const Profile& prof, Vec3 position,
                                                const Camera& ref_cam, const Frame& ref_frame,
                                                const Plane& ref_luma,
                                                const std::vector<SourceView>& sources,
                                                double focal, double* gap = nullptr);

// Parity diagnostic (no counterpart in the reference): for every sampled
// primary grid site and every completion proposal of a pass, how close its
// cost-based decisions came to going the other way.  A device policy that
// computes window costs with a bounded error can only decide differently
// where one of these gaps is within twice that bound, so the parity tests
// attribute every differing output site to a gap, to a moved hypothesis or to
// a differing neighbour.
//  * sweep_gap: primary sites: min(|best cost - photometric gate|,
//    |margin - ambiguity gate|), or for sites without a candidate the smallest
//    |cost - photometric gate| of any window; completion proposals: the
//    smallest |direct cost - photometric gate| over the sources.
//  * recip_gap: over the reciprocal check of every source: |direct cost -
//    photometric gate|, and in the single-view sweep the distance between the
//    best and second-best passing costs (a near tie moves the arg-min) and
//    |best cost - photometric gate| (or, with no passing hypothesis, the
//    smallest |cost - photometric gate|).
struct ExplainRecord {
    uint32_t x, y;
    int32_t stage;    // 0 primary sweep, 1 and 2 the completion passes
    int32_t outcome;  // primary: sweep status 2..4, 5 reciprocal rejected, 6 fusion rejected,
                      // 7 kept; completion: 0 kept, 1 texture, 2 cross view, 3 reciprocal,
                      // 4 fusion, 5 footprint
    int32_t plane;
    int32_t support;
    double error;   // primary: the best candidate's cost; completion: the median direct cost
    double margin;  // primary: the ambiguity margin (infinite without a comparable second)
    double sweep_gap;
    double recip_gap;
};
struct CompletionStats {
    size_t proposals = 0, accepted = 0, rejected_texture = 0, rejected_cross_view = 0,
           rejected_reciprocal = 0, rejected_fusion = 0, rejected_footprint = 0;
    size_t outcomes() const {
        return accepted + rejected_texture + rejected_cross_view + rejected_reciprocal +
               rejected_fusion + rejected_footprint;
    }
};
CompletionStats complete_surface_samples(const Profile& prof, const Camera& ref_cam,
                                         const Frame& ref_frame, const Plane& ref_luma,
                                         const std::vector<SourceView>& sources,
                                         std::vector<Point3>& points,
                                         std::vector<GridSite>& grid_sites,
                                         std::vector<Attr>& attrs, std::vector<double>& errors,
                                         std::vector<double>& supports, uint32_t width,
                                         uint32_t height, uint32_t border, size_t stride,
                                         double focal, Control& control,
                                         std::vector<ExplainRecord>* explain = nullptr);

// dense_legacy.rs:149-470
LegacyAnalysis estimate_depth_points_with_control(const Profile& prof,
                                                  const std::vector<Frame>& frames,
                                                  const std::vector<Camera>& cameras,
                                                  const std::vector<Vec3>& sparse, double focal,
                                                  bool fine_grid, Control& control);

// A band of grid rows [begin, end) for bounded CPU-baseline timing: only
// those rows are swept, checked and fused, completion is skipped, and `units`
// counts sites x hypotheses x source views of the band.
struct RowBand {
    uint32_t begin = 0, end = 0;
    mutable uint64_t units = 0;
};

// `sweep_records`, when given, receives the per-site sweep outcome in raster
// order and the pass stops after the sweep (a parity diagnostic); `explain`
// receives the ExplainRecords of the primary sites in raster order, then of
// each completion pass's proposals.  Sites are independent, so the grid is
// swept by OpenMP threads and reduced in raster order; the cancellation
// callback is polled once per grid row, in row order, before the rows run.
LegacyAnalysis estimate_depth_points_ptr(const Profile& prof,
                                         const std::vector<const Frame*>& frames,
                                         const std::vector<Camera>& cameras,
                                         const std::vector<Vec3>& sparse, double focal,
                                         bool fine_grid, Control& control,
                                         std::vector<v3d_site_record>* sweep_records = nullptr,
                                         const RowBand* band = nullptr,
                                         std::vector<ExplainRecord>* explain = nullptr);

// ---- dense.rs ----
size_t grid_stride(uint32_t width, uint32_t height, bool fine_grid);
size_t profile_grid_stride(const Profile& prof, uint32_t width, uint32_t height, bool fine_grid);
bool has_distributed_landmarks(const std::vector<Frame>& frames,
                               const std::vector<Camera>& cameras,
                               const std::vector<Vec3>& sparse, double focal, Control& control);
std::vector<size_t> reference_candidate_order(const std::vector<Frame>& frames,
                                              const std::vector<Camera>& cameras,
                                              const std::vector<Vec3>& sparse, double focal);
std::optional<LegacyAnalysis> reconstruct_reference_patch(const Profile& prof,
                                                          const std::vector<Frame>& frames,
                                                          const std::vector<Camera>& cameras,
                                                          const std::vector<Vec3>& sparse,
                                                          double focal, size_t camera_index,
                                                          bool fine_grid, Control& control,
                                                          const RowBand* band = nullptr,
                                                          std::vector<ExplainRecord>* explain = nullptr);
AttemptStats reference_attempt_stats(size_t reference_frame, const LegacyStats& stats,
                                     size_t accepted_points, bool accepted);
std::vector<AttemptStats> merge_fallback_attempts(std::vector<AttemptStats> attempts,
                                                  std::vector<AttemptStats> fallback);
DenseAnalysis from_legacy(LegacyAnalysis analysis);
std::pair<DenseAnalysis, bool> estimate_depth_points_limited(const Profile& prof,
                                                             const std::vector<Frame>& frames,
                                                             const std::vector<Camera>& cameras,
                                                             const std::vector<Vec3>& sparse,
                                                             double focal, size_t reference_views,
                                                             bool fine_grid, Control& control);

// ---- the working-set budget (dense.rs:15-28, 354-605) ----
struct WorkingSet {  // DenseWorkingSetEstimate
    uint64_t frame_bytes = 0, retry_frame_bytes = 0, remapped_frame_bytes = 0,
             luminance_bytes = 0, sparse_pipeline_bytes = 0, dense_sample_bytes = 0,
             topology_bytes = 0, mesh_builder_bytes = 0, surface_fusion_bytes = 0,
             retained_candidate_bytes = 0, packed_output_bytes = 0, total_bytes = 0;
};
// estimate_working_set (dense.rs:423-605); a frame's bytes are its storage as
// handed in (the reference's RGBA frames: width x height x 4).
WorkingSet estimate_working_set(const std::vector<Frame>& frames, uint64_t max_features,
                                uint32_t descriptor_radius, uint64_t reference_views,
                                bool fine_grid);
struct BudgetedAnalysis {
    DenseAnalysis analysis;
    WorkingSet estimate;          // stats.working_set_estimate
    uint64_t budget_bytes = 0;    // stats.working_set_budget_bytes
    uint64_t full_bytes = 0;      // stats.full_working_set_bytes
    bool fine_grid = false;       // the plan that ran
    uint64_t reference_views = 0; // 0: the budget skip
};
// estimate_depth_points_with_budget_and_control (dense.rs:355-420)
BudgetedAnalysis estimate_depth_points_with_budget(const Profile& prof,
                                                   const std::vector<Frame>& frames,
                                                   const std::vector<Camera>& cameras,
                                                   const std::vector<Vec3>& sparse, double focal,
                                                   uint64_t budget, uint64_t max_features,
                                                   uint32_t descriptor_radius, Control& control);

// ---- mesh_legacy.rs / mesh.rs ----
struct MeshTriangle {
    size_t a, b, c;
    float confidence;
};
struct MeshStats {
    bool attempted = false;
    std::optional<std::string> skip_reason;
    std::optional<size_t> reference_frame;
    size_t point_count = 0, grid_vertices = 0, rejected_grid_vertices = 0, candidate_cells = 0,
           candidate_triangles = 0, accepted_triangles = 0, rejected_discontinuities = 0,
           rejected_degenerate = 0;
};
struct MeshAnalysis {
    MeshStats stats;
    std::vector<MeshTriangle> triangles;
    std::vector<size_t> reference_frames;
    std::vector<MeshStats> reference_patches;
};
struct MeshDenseInput {
    bool attempted = false;
    std::optional<size_t> reference_frame;
    size_t grid_stride = 0;
    uint32_t grid_border = 0;
    std::vector<PatchStats> reference_patches;
};
MeshAnalysis reconstruct_dense_mesh_samples(const std::vector<Point3>& points,
                                            const std::vector<GridSite>& sites,
                                            const MeshDenseInput& dense,
                                            const std::vector<Camera>& cameras, uint32_t width,
                                            uint32_t height, double focal, Control& control);
MeshAnalysis reconstruct_dense_mesh_with_control(const std::vector<Point3>& points,
                                                 const std::vector<GridSite>& sites,
                                                 const MeshDenseInput& dense,
                                                 const std::vector<Camera>& cameras,
                                                 uint32_t width, uint32_t height, double focal,
                                                 Control& control);

// Half / bfloat16 decoding (exact).
double half_to_double(uint16_t h);
double bf16_to_double(uint16_t b);

// ---- surface_fusion.rs (oracle_fusion.cpp) ----
// SurfaceEvidenceRegion (reconstruction_evidence.rs), the fields that
// evidence_support_membership reads.
struct EvidenceRegion {
    std::optional<size_t> reference_frame;
    std::vector<size_t> source_frames;
    size_t start = 0, count = 0;
};
// VertexSurfaceEvidence (surface_fusion.rs:47-52)
struct VertexEvidence {
    std::vector<std::optional<Vec3>> normals;
    std::vector<std::optional<double>> local_scales;
    std::vector<std::vector<size_t>> incident;
    std::optional<double> global_edge_scale;
};
// FusionMove (surface_fusion.rs:40-45)
struct FusionMove {
    size_t first, second;
    Vec3 position;
};
// FusionStats, FusionOutcome (surface_fusion.rs:17-32)
struct FusionStats {
    size_t eligible_vertices = 0, candidate_pairs = 0, rejected_normal_pairs = 0,
           rejected_topology_pairs = 0, fused_pairs = 0;
};
struct FusionOutcome {
    FusionStats stats;
    std::vector<std::pair<size_t, size_t>> pairs;
    std::vector<size_t> moved_indices;
};
std::pair<std::vector<int64_t>, size_t> evidence_support_membership(
    const std::vector<EvidenceRegion>& regions, size_t point_count);
std::optional<VertexEvidence> vertex_surface_evidence(const std::vector<Point3>& points,
                                                      const std::vector<MeshTriangle>& triangles,
                                                      Control& control);
std::pair<std::vector<FusionMove>, size_t> topology_safe_moves(
    const std::vector<Point3>& points, const std::vector<MeshTriangle>& triangles,
    const std::vector<std::vector<size_t>>& incident, std::vector<FusionMove> moves,
    Control& control);
// membership: support group per point, negative = none
FusionOutcome fuse_mutually_supported_vertices(std::vector<Point3>& points,
                                               const std::vector<MeshTriangle>& triangles,
                                               const std::vector<int64_t>& membership,
                                               Control& control);

// ---- colmap_surface.rs (oracle_colmap.cpp) ----
// View (colmap_surface.rs:158-162): a frame, its depth grid and its camera
struct DepthView {
    uint32_t width = 0, height = 0;
    const uint8_t* rgba = nullptr;
    const float* depth = nullptr;
    Camera camera;
};
// VerificationFunnel (colmap_surface.rs:56-79)
struct Funnel {
    size_t reference_samples = 0, missing_reference_depth = 0, insufficient_parallax = 0,
           behind_source = 0, outside_source = 0, missing_source_depth = 0,
           depth_disagreement = 0, color_disagreement = 0, accepted = 0;
    void add(const Funnel& o) {
        reference_samples += o.reference_samples;
        missing_reference_depth += o.missing_reference_depth;
        insufficient_parallax += o.insufficient_parallax;
        behind_source += o.behind_source;
        outside_source += o.outside_source;
        missing_source_depth += o.missing_source_depth;
        depth_disagreement += o.depth_disagreement;
        color_disagreement += o.color_disagreement;
        accepted += o.accepted;
    }
};
// VerifiedSample (colmap_surface.rs:277-283)
struct VerifiedSample {
    Point3 point;
    GridSite site;
    std::vector<size_t> sources;
};
// SurfaceTopology (colmap_surface.rs:114-121)
struct Topology {
    size_t islands = 0, small_islands = 0, small_island_triangles = 0,
           largest_island_triangles = 0, boundary_edges = 0;
};
double min_parallax_cos();
const char* dominant_rejection(const Funnel& f);
std::vector<std::pair<Point3, GridSite>> verify_patch(const DepthView& ref, const DepthView& src,
                                                      size_t stride, size_t reference_stride,
                                                      double focal, Funnel& funnel);
std::vector<VerifiedSample> verified_union(
    const std::vector<std::pair<size_t, std::vector<std::pair<Point3, GridSite>>>>& candidates);
Topology surface_topology(size_t vertex_count, const std::vector<MeshTriangle>& triangles);

}  // namespace v3do
