// TEST INFRASTRUCTURE — the CPU oracle of the connected-surface merge.
//
// A literal f64 restatement of video-to-3d-core's surface merge
// (crates/video-to-3d-core/src/surface_merge.rs, surface_merge_clip.rs,
// surface_merge_stitch.rs): shared vertices from fusion-accepted pairs,
// ownership of overlapping triangles in the higher-priority reference's
// image (and the 3D fallback), seam stitching over existing vertices,
// clipping of retained overlap seams with derived vertices, and the
// edge-conforming split.  Evaluation order follows nalgebra's (3-vectors:
// (x*x + y*y) + z*z; 3x3 products column by column, left to right), sets and
// maps are ordered where the reference's are (BTreeSet/BTreeMap), and no
// multiply-add is contracted (-ffp-contract=off).
//
// Parity pin: the reference cannot be compiled here; every assertion of its
// own tests for this module (surface_merge_tests.rs,
// surface_merge_derived_acceptance_tests.rs) is re-run against this
// restatement in oracle_merge_selftest.cpp.
#pragma once

#include <array>
#include <cmath>
#include <cstdint>
#include <functional>
#include <map>
#include <optional>
#include <set>
#include <string>
#include <utility>
#include <vector>

#include "oracle.hpp"

namespace v3do {
namespace merge {

struct V2 {
    double x = 0, y = 0;
};
inline V2 operator+(V2 a, V2 b) { return {a.x + b.x, a.y + b.y}; }
inline V2 operator-(V2 a, V2 b) { return {a.x - b.x, a.y - b.y}; }
inline V2 operator*(V2 a, double s) { return {a.x * s, a.y * s}; }
inline V2 operator/(V2 a, double s) { return {a.x / s, a.y / s}; }
inline double dot2(V2 a, V2 b) { return a.x * b.x + a.y * b.y; }
inline double norm2(V2 a) { return std::sqrt(a.x * a.x + a.y * a.y); }
inline double cross2(V2 a, V2 b) { return a.x * b.y - a.y * b.x; }

inline Vec3 scale3(Vec3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline double dot3(Vec3 a, Vec3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

// f64::signum: 1.0 for +0.0 and positives, -1.0 for -0.0 and negatives.
double signum(double v);
// f64::total_cmp as a strict weak order.
bool total_less(double a, double b);

// EvidenceOrigin (reconstruction_evidence.rs:74-79); -1 = None.
constexpr int kOriginNone = -1;

// ReferenceCamera (surface_merge.rs:103-132).
struct RefCamera {
    double R[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};  // row-major
    double t[3] = {0, 0, 0};
    Vec3 to_camera(Vec3 p) const;
    struct Projection {
        V2 image;
        double depth;
    };
    std::optional<Projection> project(Vec3 p) const;
    std::optional<std::pair<Vec3, double>> plane(const std::array<Vec3, 3>& corners) const;
    std::optional<std::array<Projection, 3>> project_triangle(
        const std::array<Vec3, 3>& corners) const;
};
using PC = RefCamera::Projection;
using ProjTri = std::array<PC, 3>;
using Polygon = std::vector<V2>;

double polygon_area(const Polygon& p);
std::pair<Polygon, Polygon> split_polygon(const Polygon& polygon, V2 a, V2 b, double orientation);
double image_area(const ProjTri& t);
std::optional<double> inverse_depth(const ProjTri& t, V2 point);

// Coverage (surface_merge.rs:1293-1302).
enum class Coverage { Full, Partial, Uncovered, BudgetExhausted };
struct CoverageResult {
    Coverage kind;
    bool partially_covered;  // BudgetExhausted only
};

// TriangleGeometry (surface_merge.rs:1137-1291).
struct TriangleGeometry {
    std::array<Vec3, 3> corners;
    Vec3 normal;
    double edges[3];
    static std::optional<TriangleGeometry> make(const std::array<Vec3, 3>& corners);
    double area() const;
    void aabb(double padding, double low[3], double high[3]) const;
    CoverageResult coverage(const std::vector<const TriangleGeometry*>& surfaces,
                            double tolerance) const;
    // (covered, partially covered): surface_merge.rs:1198-1211
    std::pair<bool, bool> covered_by(const std::vector<const TriangleGeometry*>& surfaces,
                                     double tolerance) const;
};

// QueryLimit / PostingBudget / PostingTally (surface_merge.rs:1817-1869).
enum class QueryLimit { None, Cells, Postings };
struct PostingBudget {
    size_t limit, used = 0;
    explicit PostingBudget(size_t l) : limit(l) {}
    static PostingBudget per_query();
    QueryLimit take_into(const std::vector<size_t>& items, std::set<size_t>& out);
};
struct PostingTally {
    size_t max_postings = 0, bound_hits = 0;
    void record(const PostingBudget& b, QueryLimit result);
};

// LevelGrid<D> (surface_merge.rs:1678-1815).
template <int D>
struct LevelGrid {
    double cell;
    std::map<std::pair<int32_t, std::array<int64_t, D>>, std::vector<size_t>> cells;
    int32_t levels = 0;
    std::vector<size_t> unindexed;
    explicit LevelGrid(double c) : cell(c) {}
    bool range(const double* low, const double* high, int32_t level,
               std::array<std::pair<int64_t, int64_t>, D>& out) const;
    void insert(size_t item, const double* low, const double* high);
    QueryLimit query_bounded(const double* low, const double* high, size_t max_cells,
                             PostingBudget& budget, std::set<size_t>& out) const;
    bool query(const double* low, const double* high, size_t max_cells,
               std::set<size_t>& out) const;
};

// KeptTriangle (surface_merge.rs:1313-1315).
struct KeptTriangle {
    std::array<Vec3, 3> corners;
    size_t component;
    std::array<size_t, 3> vertices;
    size_t mesh_index;
};

enum class Unjudged { None, Unprojectable, TooManyCells, PostingBound };
struct Ownership {
    double image_share = 0.0, surface_area = 0.0;
};

// Footprint (surface_merge.rs:1317-1592).
struct Footprint {
    size_t patch;
    RefCamera camera;
    std::vector<ProjTri> triangles;
    std::vector<size_t> components;
    std::vector<std::array<size_t, 3>> vertices;
    std::vector<size_t> mesh_indices;
    LevelGrid<2> grid{1.0};
    std::vector<std::pair<size_t, size_t>> omitted;

    static std::optional<Footprint> make(size_t patch, const RefCamera& camera,
                                         const std::vector<KeptTriangle>& kept);
    std::optional<ProjTri> project_candidate(const std::array<Vec3, 3>& corners) const;
    // visit(polygon, index) -> continue?
    QueryLimit visit_overlaps(const ProjTri& candidate, const std::function<bool(size_t)>& include,
                              const std::function<bool(Polygon&&, size_t)>& visit,
                              PostingTally& tally) const;
    std::vector<double> depth_ratios_tallied(
        const std::array<Vec3, 3>& corners, const std::function<bool(size_t)>& linked,
        const std::function<bool(const std::array<size_t, 3>&)>& anchored, size_t limit,
        PostingTally& tally) const;
    Unjudged ownership_tallied(const std::array<Vec3, 3>& corners, double scale,
                               const std::function<bool(size_t)>& linked, PostingTally& tally,
                               Ownership& owned, std::vector<size_t>& unjudged) const;
};

// DerivedVertexSource (reconstruction_evidence.rs:144-153).
struct DerivedVertexSource {
    size_t point_index, source_triangle;
    std::array<size_t, 3> source_corners;
    std::array<double, 3> barycentric;
};
// TriangleSourceCorners (reconstruction_evidence.rs:125-130).
struct TriangleSourceCorners {
    size_t triangle;
    std::array<size_t, 3> corners;
};

// MergeStats (surface_merge.rs:131-202).
struct MergeStats {
    size_t fused_pairs = 0, shared_vertices = 0, cross_reference_triangles = 0,
           removed_duplicate_triangles = 0, remaining_overlap_triangles = 0,
           provenance_separated_pairs = 0, trimmed_seam_triangles = 0;
    double trimmed_seam_area_share = 0.0;
    size_t stitched_seam_triangles = 0;
    std::vector<std::pair<size_t, size_t>> uncalibrated_patch_pairs;
    std::vector<size_t> retained_by_group;
    size_t patch_components = 0, meshed_patches = 0, max_postings_per_query = 0,
           posting_bound_hits = 0, clipping_budget_exhausted = 0, clipped_overlap_triangles = 0,
           clip_pieces = 0, derived_vertices = 0, unclipped_overlap_triangles = 0,
           conformed_triangles = 0, conformance_failures = 0;
    std::vector<TriangleSourceCorners> triangle_sources;
    bool operator==(const MergeStats& o) const;
    std::string diagnostic(size_t support_groups) const;
};

struct MergeInputs {
    const std::vector<Point3>* points;
    const std::vector<int64_t>* membership;                // negative = None
    const std::vector<std::pair<size_t, size_t>>* pairs;
    const std::vector<std::optional<RefCamera>>* cameras;  // per support group
    const std::vector<int>* origins;                       // per point, kOriginNone = None
};

// merge_fused_patches_with_control (surface_merge.rs:246-270): triangles
// re-indexed and filtered in place.
MergeStats merge_fused_patches(const MergeInputs& in, std::vector<MeshTriangle>& triangles,
                               Control& control);

// merge_fused_patches_owned_with_control (surface_merge.rs:312-353).
struct OwnedMerge {
    std::vector<Point3> points;
    std::vector<MeshTriangle> triangles;
    std::vector<DerivedVertexSource> derived_vertices;
    MergeStats stats;
};
// Returns false with `error` set where the reference returns Err.
bool merge_fused_patches_owned(std::vector<Point3> points, std::vector<MeshTriangle> triangles,
                               const MergeInputs& in, Control& control, OwnedMerge& out,
                               std::string& error);

// surface_merge_clip.rs:220-257 (tests use it directly)
std::optional<std::vector<std::array<size_t, 3>>> ear_clip(const Polygon& polygon,
                                                          double tolerance);

int merge_selftest(std::string& failure);

}  // namespace merge
}  // namespace v3do
