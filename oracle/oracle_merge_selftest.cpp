// TEST INFRASTRUCTURE — the reference's own tests of the connected-surface
// merge, re-run against the oracle (oracle_merge.cpp): every assertion of
// surface_merge_tests.rs and surface_merge_derived_acceptance_tests.rs, with
// the same fixtures, restated in C++.  merge_selftest() returns the number of
// checks that passed, or -1 with the first failing check in `failure`.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <tuple>

#include "oracle_merge.hpp"

namespace v3do {
namespace merge {
namespace {

struct Fail {
    std::string what;
};
int g_checks = 0;
#define MCHECK(cond)                                                                        \
    do {                                                                                    \
        if (!(cond)) throw Fail{std::string("oracle_merge_selftest.cpp:") +                 \
                                std::to_string(__LINE__) + ": " #cond};                     \
        ++g_checks;                                                                         \
    } while (0)

constexpr int kGeometric = 0;  // EvidenceOrigin::GeometricMultiView
constexpr int kRevalidated = 1;  // EvidenceOrigin::RevalidatedCompletion
constexpr size_t kPostingBound = 512;   // MAX_POSTINGS_PER_QUERY
constexpr size_t kUncoveredPieces = 128;  // MAX_UNCOVERED_PIECES
constexpr size_t kGridCells = 1728;     // MAX_GRID_CELLS
constexpr size_t kImageGridCells = 4096;  // MAX_IMAGE_GRID_CELLS

Point3 point(float x, float y, float z) { return Point3{x, y, z, 1.0f, 40, 80, 120}; }
MeshTriangle triangle(size_t a, size_t b, size_t c) { return MeshTriangle{a, b, c, 0.9f}; }
std::array<Vec3, 3> corners(std::array<std::array<double, 3>, 3> v) {
    return {Vec3{v[0][0], v[0][1], v[0][2]}, Vec3{v[1][0], v[1][1], v[1][2]},
            Vec3{v[2][0], v[2][1], v[2][2]}};
}
TriangleGeometry geometry(std::array<std::array<double, 3>, 3> v) {
    return *TriangleGeometry::make(corners(v));
}
using Sig = std::vector<std::tuple<size_t, size_t, size_t>>;
Sig signature(const std::vector<MeshTriangle>& t) {
    Sig s;
    for (const auto& x : t) s.push_back({x.a, x.b, x.c});
    return s;
}
bool has_sig(const std::vector<MeshTriangle>& t, size_t a, size_t b, size_t c) {
    for (const auto& x : t)
        if (x.a == a && x.b == b && x.c == c) return true;
    return false;
}
bool has_bc(const std::vector<MeshTriangle>& t, size_t b, size_t c) {
    for (const auto& x : t)
        if (x.b == b && x.c == c) return true;
    return false;
}
RefCamera identity_camera(double x) {
    RefCamera c;
    c.t[0] = -x;
    c.t[1] = 0.0;
    c.t[2] = 0.0;
    return c;
}
std::vector<int64_t> groups(const std::vector<int>& g) {
    return std::vector<int64_t>(g.begin(), g.end());
}
using Cameras = std::vector<std::optional<RefCamera>>;
using Pairs = std::vector<std::pair<size_t, size_t>>;

MergeStats merge(const std::vector<Point3>& points, std::vector<MeshTriangle>& triangles,
                 const std::vector<int64_t>& membership, const Pairs& pairs, const Cameras& cameras,
                 const std::vector<int>& origins) {
    MergeInputs in{&points, &membership, &pairs, &cameras, &origins};
    Control control;
    return merge_fused_patches(in, triangles, control);
}

bool owned_merge(std::vector<Point3> points, std::vector<MeshTriangle> triangles,
                 const std::vector<int64_t>& membership, const Pairs& pairs, const Cameras& cameras,
                 const std::vector<int>& origins, Control& control, OwnedMerge& out) {
    MergeInputs in{nullptr, &membership, &pairs, &cameras, &origins};
    std::string error;
    return merge_fused_patches_owned(std::move(points), std::move(triangles), in, control, out,
                                     error);
}

std::set<size_t> query(const LevelGrid<3>& g, std::array<double, 3> lo, std::array<double, 3> hi,
                       bool& ok) {
    std::set<size_t> found;
    ok = g.query(lo.data(), hi.data(), kGridCells, found);
    return found;
}

// Footprint::ownership / depth_ratios (test forms, unbounded tally)
std::optional<std::pair<Ownership, std::vector<size_t>>> ownership(
    const Footprint& f, const std::array<Vec3, 3>& c, double scale,
    const std::function<bool(size_t)>& linked) {
    PostingTally tally;
    Ownership o;
    std::vector<size_t> unjudged;
    if (f.ownership_tallied(c, scale, linked, tally, o, unjudged) != Unjudged::None)
        return std::nullopt;
    return std::make_pair(o, unjudged);
}
double share_or_zero(const Footprint& f, const std::array<Vec3, 3>& c, double scale) {
    auto o = ownership(f, c, scale, [](size_t) { return true; });
    return o ? o->first.image_share : 0.0;
}
std::vector<double> depth_ratios(const Footprint& f, const std::array<Vec3, 3>& c,
                                 const std::function<bool(const std::array<size_t, 3>&)>& anchored,
                                 size_t limit) {
    PostingTally tally;
    return f.depth_ratios_tallied(c, [](size_t) { return true; }, anchored, limit, tally);
}
bool all_anchored(const std::array<size_t, 3>&) { return true; }

// A 2 x 2 square at depth 5 split into two kept triangles (surface_merge_tests.rs:242-262).
Footprint square_footprint(const RefCamera& camera) {
    std::vector<KeptTriangle> kept{
        {corners({{{-1.0, -1.0, 5.0}, {1.0, -1.0, 5.0}, {1.0, 1.0, 5.0}}}), 0, {0, 1, 2}, 101},
        {corners({{{-1.0, -1.0, 5.0}, {1.0, 1.0, 5.0}, {-1.0, 1.0, 5.0}}}), 0, {0, 2, 3}, 102}};
    return *Footprint::make(0, camera, kept);
}

bool contains_str(const std::string& hay, const std::string& needle) {
    return hay.find(needle) != std::string::npos;
}

// ---- surface_merge_tests.rs:33-229 ----------------------------------------------------
void union_coverage_handles_a_different_diagonal_and_large_triangles() {
    auto left = geometry({{{0.0, 0.0, 0.0}, {2.0, 0.0, 0.0}, {0.0, 2.0, 0.0}}});
    auto right = geometry({{{2.0, 0.0, 0.0}, {2.0, 2.0, 0.0}, {0.0, 2.0, 0.0}}});
    auto inner = geometry({{{0.2, 0.2, 0.05}, {1.8, 0.3, 0.05}, {1.4, 1.7, 0.05}}});
    MCHECK(inner.covered_by({&left, &right}, 0.1) == std::make_pair(true, true));
}

void never_discards_an_unsupported_hole_or_partial_boundary() {
    auto left = geometry({{{0.0, 0.0, 0.0}, {0.9, 0.0, 0.0}, {0.0, 1.0, 0.0}}});
    auto right = geometry({{{1.1, 0.0, 0.0}, {2.0, 0.0, 0.0}, {2.0, 1.0, 0.0}}});
    auto spanning = geometry({{{0.0, 0.0, 0.0}, {2.0, 0.0, 0.0}, {1.0, 0.8, 0.0}}});
    MCHECK(!spanning.covered_by({&left, &right}, 0.1).first);
    auto accepted = geometry({{{0.0, 0.0, 0.0}, {1.0, 0.0, 0.0}, {0.0, 1.0, 0.0}}});
    auto outside = geometry({{{0.7, 0.1, 0.0}, {1.4, 0.1, 0.0}, {1.1, 0.8, 0.0}}});
    MCHECK(!outside.covered_by({&accepted}, 0.1).first);
}

void normal_and_depth_disagreement_are_not_coverage() {
    auto kept = geometry({{{0.0, 0.0, 0.0}, {2.0, 0.0, 0.0}, {0.0, 2.0, 0.0}}});
    auto distant = geometry({{{0.1, 0.1, 1.0}, {1.0, 0.1, 1.0}, {0.1, 1.0, 1.0}}});
    MCHECK(distant.covered_by({&kept}, 0.1) == std::make_pair(false, false));
    auto orthogonal = geometry({{{0.0, 0.0, 0.0}, {0.0, 0.0, 1.0}, {0.0, 1.0, 0.0}}});
    MCHECK(orthogonal.covered_by({&kept}, 0.1) == std::make_pair(false, false));
}

void no_accepted_fusion_pair_means_no_dedup_even_for_coincident_sheets() {
    std::vector<Point3> points{point(0, 0, 0), point(1, 0, 0), point(0, 1, 0),
                               point(0, 0, 0), point(1, 0, 0), point(0, 1, 0)};
    std::vector<MeshTriangle> original{triangle(0, 1, 2), triangle(3, 4, 5)};
    auto triangles = original;
    auto stats = merge(points, triangles, groups({0, 0, 0, 1, 1, 1}), {}, {}, {});
    MCHECK(stats.removed_duplicate_triangles == 0);
    MCHECK(stats.cross_reference_triangles == 0);
    MCHECK(stats.patch_components == 2);
    MCHECK(signature(triangles) == signature(original));
}

void a_fusion_link_does_not_erase_an_unrelated_island_of_the_same_camera_pair() {
    std::vector<Point3> points{point(0, 0, 0),  point(1, 0, 0),  point(0, 1, 0),
                               point(10, 0, 0), point(11, 0, 0), point(10, 1, 0),
                               point(0, 0, 0),  point(1, 0, 0),  point(0, 1, 0),
                               point(10, 0, 0), point(11, 0, 0), point(10, 1, 0)};
    std::vector<MeshTriangle> triangles{triangle(0, 1, 2), triangle(3, 4, 5), triangle(6, 7, 8),
                                        triangle(9, 10, 11)};
    auto stats = merge(points, triangles, groups({0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, 1}), {{0, 6}},
                       {}, {});
    MCHECK(stats.fused_pairs == 1);
    MCHECK(stats.removed_duplicate_triangles == 1);
    MCHECK(has_sig(triangles, 9, 10, 11));
    MCHECK(has_sig(triangles, 3, 4, 5));
}

// Two adjacent camera grids: A covers x=0..2, B x=1..3, fused at x=2.
void adjacent_grids_fixture(std::vector<Point3>& points, std::vector<MeshTriangle>& triangles,
                            std::vector<int64_t>& membership) {
    points.clear();
    triangles.clear();
    membership.clear();
    const std::tuple<float, float, int> patches[2] = {{0.0f, 0.0f, 0}, {1.0f, 0.06f, 1}};
    for (const auto& p : patches) {
        for (int y = 0; y <= 1; ++y)
            for (int x = 0; x <= 2; ++x) {
                bool shared = std::get<2>(p) == 1 && x == 1;
                points.push_back(point(std::get<0>(p) + (float)x, (float)y,
                                       shared ? 0.0f : std::get<1>(p)));
                membership.push_back(std::get<2>(p));
            }
    }
    for (size_t offset : {0, 6})
        for (size_t x = 0; x < 2; ++x) {
            size_t start = offset + x;
            triangles.push_back(triangle(start, start + 1, start + 3));
            triangles.push_back(triangle(start + 1, start + 4, start + 3));
        }
}

void a_confirmed_seam_deduplicates_overlap_but_keeps_the_uncovered_extension() {
    std::vector<Point3> points;
    std::vector<MeshTriangle> triangles;
    std::vector<int64_t> membership;
    adjacent_grids_fixture(points, triangles, membership);
    const auto original = triangles;
    auto stats = merge(points, triangles, membership, {{2, 7}, {5, 10}}, {}, {});
    MCHECK(stats.fused_pairs == 2);
    MCHECK(stats.patch_components == 1);
    MCHECK(stats.cross_reference_triangles > 0);
    MCHECK(stats.removed_duplicate_triangles == 2);
    MCHECK(triangles.size() == original.size() - 2);
    bool uses8 = false;
    for (const auto& t : triangles) uses8 |= t.a == 8 || t.b == 8 || t.c == 8;
    MCHECK(uses8);
    auto first = signature(triangles);
    auto again_t = original;
    auto again = merge(points, again_t, membership, {{2, 7}, {5, 10}}, {}, {});
    MCHECK(stats == again);
    auto replay = original;
    merge(points, replay, membership, {{2, 7}, {5, 10}}, {}, {});
    MCHECK(first == signature(replay));
}

void large_triangles_are_indexed_across_their_interior() {
    auto surface = geometry({{{0.0, 0.0, 0.0}, {60.0, 0.0, 0.0}, {0.0, 60.0, 0.0}}});
    LevelGrid<3> grid(1.0);
    double low[3], high[3];
    surface.aabb(0.0, low, high);
    grid.insert(7, low, high);
    MCHECK(grid.cells.size() == 1);
    for (const auto& kv : grid.cells) MCHECK(kv.first.first > 0);
    bool ok;
    auto found = query(grid, {4.0, 4.0, 0.0}, {5.0, 5.0, 0.0}, ok);
    MCHECK(ok);
    MCHECK(found.count(7));
    auto small = geometry({{{4.0, 4.0, 0.0}, {5.0, 4.0, 0.0}, {4.0, 5.0, 0.0}}});
    MCHECK(small.covered_by({&surface}, 0.1).first);
}

// ---- surface_merge_tests.rs:264-369: image ownership --------------------------------------
void image_ownership_tolerates_reference_scale_but_not_another_surface() {
    auto footprint = square_footprint(identity_camera(0.0));
    auto same = corners({{{-0.5, -0.5, 5.05}, {0.6, -0.4, 5.05}, {0.1, 0.7, 5.05}}});
    MCHECK(std::fabs(share_or_zero(footprint, same, 1.0) - 1.0) < 1.0e-9);
    auto layer = corners({{{-0.5, -0.5, 4.8}, {0.6, -0.4, 4.8}, {0.1, 0.7, 4.8}}});
    MCHECK(share_or_zero(footprint, layer, 1.0) == 0.0);
    auto ratios = depth_ratios(footprint, layer, all_anchored, SIZE_MAX);
    MCHECK(!ratios.empty());
    for (double r : ratios) MCHECK(std::fabs(r - 0.96) < 1.0e-9);
    MCHECK(std::fabs(share_or_zero(footprint, layer, 0.96) - 1.0) < 1.0e-9);
    auto behind = corners({{{-0.5, -0.5, 5.6}, {0.6, -0.4, 5.6}, {0.1, 0.7, 5.6}}});
    MCHECK(share_or_zero(footprint, behind, 1.0) == 0.0);
    auto flipped = corners({{{-0.5, -0.5, -5.0}, {0.6, -0.4, -5.0}, {0.1, 0.7, -5.0}}});
    MCHECK(!ownership(footprint, flipped, 1.0, [](size_t) { return true; }));
}

void image_ownership_measures_the_share_on_the_footprint() {
    auto footprint = square_footprint(identity_camera(0.0));
    auto seam = corners({{{0.0, -0.5, 5.0}, {2.0, -0.5, 5.0}, {1.0, 0.5, 5.0}}});
    auto owned = ownership(footprint, seam, 1.0, [](size_t) { return true; });
    MCHECK(owned);
    MCHECK(std::fabs(owned->first.image_share - 0.5) < 1.0e-9);
    MCHECK(std::fabs(owned->first.surface_area - 0.5) < 1.0e-9);
    auto tilted = corners({{{0.0, -0.5, 4.9}, {2.0, -0.5, 5.1}, {1.0, 0.5, 5.0}}});
    auto t = ownership(footprint, tilted, 1.0, [](size_t) { return true; });
    MCHECK(t);
    double full = norm(cross(sub(tilted[1], tilted[0]), sub(tilted[2], tilted[0]))) * 0.5;
    MCHECK(t->first.image_share > 0.4 && t->first.image_share < 0.6);
    MCHECK(t->first.surface_area > 0.0 && t->first.surface_area < full);
    auto outside = corners({{{1.5, -0.5, 5.0}, {2.5, -0.5, 5.0}, {2.0, 0.5, 5.0}}});
    MCHECK(share_or_zero(footprint, outside, 1.0) == 0.0);
}

struct OwnedOverlapFixture {
    std::vector<Point3> points;
    std::vector<int64_t> membership;
    std::vector<MeshTriangle> original;
    Pairs link;
    Cameras cameras;
};

// surface_merge_tests.rs:370-410
OwnedOverlapFixture owned_overlap_fixture() {
    OwnedOverlapFixture f;
    f.points = {point(-1.0f, -1.0f, 5.0f),  point(1.0f, -1.0f, 5.0f),   point(1.0f, 1.0f, 5.0f),
                point(-1.0f, 1.0f, 5.0f),   point(-4.0f, -1.0f, 5.0f),  point(-3.0f, -1.0f, 5.0f),
                point(-3.5f, 0.0f, 5.0f),   point(-0.5f, -0.5f, 5.05f), point(0.6f, -0.4f, 5.05f),
                point(0.1f, 0.7f, 5.05f),   point(3.0f, -0.5f, 5.0f),   point(3.5f, 0.5f, 5.0f),
                point(-0.5f, -0.5f, 5.05f), point(-0.6f, 0.2f, 5.0f),   point(-0.2f, 0.2f, 5.0f),
                point(-0.4f, 0.6f, 5.0f)};
    for (size_t i = 0; i < f.points.size(); ++i)
        f.membership.push_back(((i >= 7 && i < 12) || i >= 13) ? 1 : 0);
    f.original = {triangle(0, 1, 2), triangle(0, 2, 3),  triangle(4, 5, 6),  triangle(0, 1, 12),
                  triangle(7, 8, 9), triangle(8, 10, 11), triangle(13, 14, 15)};
    f.link = {{12, 7}};
    f.cameras = {identity_camera(0.0), identity_camera(0.4)};
    return f;
}

void owned_overlap_is_removed_and_unique_surface_is_kept() {
    auto f = owned_overlap_fixture();
    auto triangles = f.original;
    auto stats = merge(f.points, triangles, f.membership, f.link, f.cameras, {});
    MCHECK(stats.removed_duplicate_triangles == 1);
    MCHECK(stats.retained_by_group == (std::vector<size_t>{4, 2}));
    MCHECK(has_sig(triangles, 13, 14, 15));
    MCHECK(has_bc(triangles, 10, 11));
    MCHECK(!has_bc(triangles, 8, 9));
    for (const Cameras& cameras : {f.cameras, Cameras{}}) {
        auto t = f.original;
        auto s = merge(f.points, t, f.membership, {}, cameras, {});
        MCHECK(s.removed_duplicate_triangles == 0);
        MCHECK(t.size() == f.original.size());
    }
}

void a_depth_rejection_in_the_image_is_not_overturned_by_the_3d_test() {
    std::vector<Point3> points{
        point(-1.0f, -1.0f, 5.0f), point(1.0f, -1.0f, 5.0f), point(1.0f, 1.0f, 5.0f),
        point(-1.0f, 1.0f, 5.0f),  point(-4.0f, -1.0f, 5.0f), point(-3.0f, -1.0f, 5.0f),
        point(-3.5f, 0.0f, 5.0f),  point(-0.5f, -0.5f, 4.8f), point(0.9f, -0.9f, 5.0f),
        point(-0.5f, -0.5f, 4.8f), point(0.0f, -0.4f, 4.8f),  point(-0.3f, 0.0f, 4.8f),
        point(0.9f, -0.9f, 5.0f),  point(0.9f, 0.9f, 5.0f),   point(0.2f, -0.9f, 5.0f),
        point(0.2f, 0.9f, 5.0f),   point(0.5f, 0.0f, 5.0f)};
    std::vector<int64_t> membership;
    for (size_t i = 0; i < points.size(); ++i) membership.push_back(i >= 9 ? 1 : 0);
    std::vector<MeshTriangle> triangles{triangle(0, 1, 2),   triangle(0, 2, 3),   triangle(4, 5, 6),
                                        triangle(0, 1, 7),   triangle(1, 2, 8),   triangle(9, 10, 11),
                                        triangle(12, 13, 16), triangle(12, 16, 14),
                                        triangle(13, 15, 16)};
    Cameras cameras{identity_camera(0.0), identity_camera(0.4)};
    auto stats = merge(points, triangles, membership, {{7, 9}, {8, 12}}, cameras, {});
    MCHECK(stats.removed_duplicate_triangles == 3);
    MCHECK(has_bc(triangles, 10, 11));
}

void the_relative_scale_is_anchored_at_fusion_accepted_seam_vertices() {
    std::vector<Point3> points{point(-1.0f, -1.0f, 5.0f), point(1.0f, -1.0f, 5.0f),
                               point(1.0f, 1.0f, 5.0f),   point(-1.0f, 1.0f, 5.0f),
                               point(-4.0f, -1.0f, 5.0f), point(-3.0f, -1.0f, 5.0f),
                               point(-3.5f, 0.0f, 5.0f),  point(0.9f, -0.9f, 5.0f),
                               point(0.9f, -0.9f, 5.0f),  point(0.9f, -0.2f, 5.0f),
                               point(0.4f, -0.9f, 5.0f),  point(0.4f, -0.2f, 5.0f)};
    for (int row = 0; row < 3; ++row)
        for (int column = 0; column < 3; ++column)
            points.push_back(point(-0.9f + (float)column * 0.5f, -0.9f + (float)row * 0.5f, 4.8f));
    std::vector<int64_t> membership;
    for (size_t i = 0; i < points.size(); ++i) membership.push_back(i >= 8 ? 1 : 0);
    auto grid = [](size_t row, size_t column) { return 12 + row * 3 + column; };
    std::vector<MeshTriangle> original{triangle(0, 1, 2),  triangle(0, 2, 3),  triangle(4, 5, 6),
                                       triangle(1, 2, 7),  triangle(8, 9, 10), triangle(9, 11, 10),
                                       triangle(11, 9, grid(2, 2))};
    for (int i = 0; i < 12; ++i) original.push_back(triangle(4, 5, 6));
    for (size_t row = 0; row < 2; ++row)
        for (size_t column = 0; column < 2; ++column) {
            original.push_back(triangle(grid(row, column), grid(row, column + 1),
                                        grid(row + 1, column + 1)));
            original.push_back(
                triangle(grid(row, column), grid(row + 1, column + 1), grid(row + 1, column)));
        }
    Cameras cameras{identity_camera(0.0), identity_camera(0.4)};
    auto layer_kept = [](const std::vector<MeshTriangle>& t) {
        size_t n = 0;
        for (const auto& x : t)
            if (x.a >= 12 && x.a < 21 && x.b >= 12 && x.b < 21 && x.c >= 12 && x.c < 21) ++n;
        return n;
    };
    auto triangles = original;
    auto stats = merge(points, triangles, membership, {{7, 8}}, cameras, {});
    MCHECK(layer_kept(triangles) == 8);
    MCHECK(stats.uncalibrated_patch_pairs == (Pairs{{0, 1}}));
    MCHECK(contains_str(stats.diagnostic(2),
                        "1 linked patch pair(s) had too few anchored overlap samples"));
    const size_t third = points.size();
    Pairs pairs{{7, 8}};
    for (size_t row = 0; row < 3; ++row)
        for (size_t column = 0; column < 3; ++column) {
            pairs.push_back({grid(row, column), points.size()});
            points.push_back(point(-0.9f + (float)column * 0.5f, -0.9f + (float)row * 0.5f, 4.8f));
            membership.push_back(2);
        }
    points.push_back(point(-6.0f, 3.0f, 4.8f));
    membership.push_back(2);
    original.push_back(triangle(third, third + 1, points.size() - 1));
    Cameras cameras3{identity_camera(0.0), identity_camera(0.4), identity_camera(0.8)};
    triangles = original;
    stats = merge(points, triangles, membership, pairs, cameras3, {});
    MCHECK(layer_kept(triangles) == 8);
}

void pairs_across_evidence_origins_link_patches_but_keep_their_vertices() {
    std::vector<Point3> points{point(-1.0f, -1.0f, 5.0f), point(1.0f, -1.0f, 5.0f),
                               point(1.0f, 1.0f, 5.0f),   point(-1.0f, 1.0f, 5.0f),
                               point(-4.0f, -1.0f, 5.0f), point(-3.0f, -1.0f, 5.0f),
                               point(-3.5f, 0.0f, 5.0f),  point(-0.5f, -0.5f, 5.0f),
                               point(0.6f, -0.4f, 5.0f),  point(0.1f, 0.7f, 5.0f),
                               point(-3.0f, 1.0f, 5.0f),  point(-2.0f, 1.0f, 5.0f),
                               point(-0.5f, -0.5f, 5.0f)};
    std::vector<int64_t> membership;
    for (size_t i = 0; i < points.size(); ++i) membership.push_back(i >= 7 && i < 10 ? 1 : 0);
    std::vector<int> origins(points.size(), kGeometric);
    origins[7] = kRevalidated;
    std::vector<MeshTriangle> original{triangle(0, 1, 2),  triangle(0, 2, 3),  triangle(4, 5, 6),
                                       triangle(4, 10, 11), triangle(0, 1, 12), triangle(7, 8, 9)};
    Cameras cameras{identity_camera(0.0), identity_camera(0.4)};
    auto triangles = original;
    auto stats = merge(points, triangles, membership, {{12, 7}}, cameras, origins);
    MCHECK(stats.fused_pairs == 0);
    MCHECK(stats.provenance_separated_pairs == 1);
    MCHECK(stats.shared_vertices == 0);
    MCHECK(stats.removed_duplicate_triangles == 1);
    MCHECK(!has_bc(triangles, 8, 9));
    std::vector<int> same(points.size(), kGeometric);
    triangles = original;
    stats = merge(points, triangles, membership, {{12, 7}}, cameras, same);
    MCHECK(stats.fused_pairs == 1);
    MCHECK(stats.provenance_separated_pairs == 0);
}

void only_vertices_referenced_by_two_patches_count_as_shared() {
    std::vector<Point3> points{point(0, 0, 0), point(1, 0, 0),  point(0, 1, 0),
                               point(0, 1, 0), point(-1, 2, 0), point(-1, 1, 0)};
    std::vector<MeshTriangle> triangles{triangle(0, 1, 2), triangle(3, 4, 5)};
    auto stats = merge(points, triangles, groups({0, 0, 0, 1, 1, 1}), {{2, 3}}, {}, {});
    MCHECK(stats.fused_pairs == 1);
    MCHECK(stats.cross_reference_triangles == 1);
    MCHECK(stats.shared_vertices == 1);
}

void oversized_owner_triangles_are_checked_exactly() {
    std::vector<KeptTriangle> kept{
        {corners({{{-1.0, -1.0, 5.0}, {1.0, -1.0, 5.0}, {1.0, 1.0, 5.0}}}), 0, {0, 1, 2}, 103}};
    for (int step = 0; step < 4; ++step) {
        double x = 3.0 + (double)step * 0.02;
        kept.push_back({corners({{{x, 3.0, 5.0}, {x + 0.01, 3.0, 5.0}, {x, 3.01, 5.0}}}), 0,
                        {3 + (size_t)step, 9, 10}, 104});
    }
    auto footprint = *Footprint::make(0, identity_camera(0.0), kept);
    MCHECK(footprint.grid.levels > 1);
    auto inside = corners({{{0.5, -0.8, 5.0}, {0.8, -0.8, 5.0}, {0.8, -0.5, 5.0}}});
    auto owned = ownership(footprint, inside, 1.0, [](size_t) { return true; });
    MCHECK(owned);
    MCHECK(std::fabs(owned->first.image_share - 1.0) < 1.0e-9);
}

void scale_samples_need_an_anchored_owner_triangle() {
    auto footprint = square_footprint(identity_camera(0.0));
    auto layer = corners({{{-0.5, -0.5, 4.8}, {0.6, -0.4, 4.8}, {0.1, 0.7, 4.8}}});
    auto has = [](size_t v) {
        return [v](const std::array<size_t, 3>& vs) {
            return std::find(vs.begin(), vs.end(), v) != vs.end();
        };
    };
    MCHECK(depth_ratios(footprint, layer, has(99), SIZE_MAX).empty());
    MCHECK(depth_ratios(footprint, layer, has(1), SIZE_MAX).size() == 1);
}

void unprojectable_linked_owners_leave_the_image_unable_to_judge() {
    std::vector<KeptTriangle> kept{
        {corners({{{-1.0, -1.0, 5.0}, {1.0, -1.0, 5.0}, {1.0, 1.0, 5.0}}}), 0, {0, 1, 2}, 105},
        {corners({{{-1.0, -1.0, 5.0}, {1.0, 1.0, 5.0}, {-1.0, 1.0, 5.0}}}), 0, {0, 2, 3}, 106},
        {corners({{{3.0, 3.0, -1.0}, {4.0, 3.0, -1.0}, {3.0, 4.0, -1.0}}}), 1, {4, 5, 6}, 107}};
    auto footprint = *Footprint::make(0, identity_camera(0.0), kept);
    auto outside = corners({{{2.0, 2.0, 5.0}, {2.5, 2.0, 5.0}, {2.0, 2.5, 5.0}}});
    auto judged = ownership(footprint, outside, 1.0, [](size_t) { return true; });
    MCHECK(judged);
    MCHECK(judged->first.image_share == 0.0);
    MCHECK(judged->second.size() == 1);
    auto linked0 = ownership(footprint, outside, 1.0, [](size_t c) { return c == 0; });
    MCHECK(linked0);
    MCHECK(linked0->second.empty());
}

void scale_samples_stop_at_the_limit() {
    auto footprint = square_footprint(identity_camera(0.0));
    auto layer = corners({{{-0.5, -0.5, 4.8}, {0.6, -0.4, 4.8}, {0.1, 0.7, 4.8}}});
    MCHECK(depth_ratios(footprint, layer, all_anchored, SIZE_MAX).size() == 2);
    MCHECK(depth_ratios(footprint, layer, all_anchored, 1).size() == 1);
    MCHECK(depth_ratios(footprint, layer, all_anchored, 0).empty());
}

void an_owner_without_an_image_judgement_still_gets_the_3d_test() {
    std::vector<Point3> points{point(-1.0f, -1.0f, 5.0f), point(1.0f, -1.0f, 5.0f),
                               point(1.0f, 1.0f, 5.0f),   point(-1.0f, 1.0f, 5.0f),
                               point(-9.0f, -9.0f, 5.0f), point(-8.0f, -9.0f, 5.0f),
                               point(-9.0f, -8.0f, 5.0f), point(10.0f, 0.0f, 5.0f),
                               point(11.0f, 0.0f, 5.0f),  point(10.0f, 1.0f, 5.0f),
                               point(-1.0f, -1.0f, 5.0f), point(0.0f, -1.0f, 5.0f),
                               point(-1.0f, 0.0f, 5.0f)};
    std::vector<int64_t> membership;
    for (size_t i = 0; i < points.size(); ++i) membership.push_back(i < 7 ? 0 : i < 10 ? 1 : 2);
    std::vector<int> origins(points.size(), kGeometric);
    origins[7] = kRevalidated;
    std::vector<MeshTriangle> triangles{triangle(0, 1, 2), triangle(0, 2, 3)};
    for (int i = 0; i < 12; ++i) triangles.push_back(triangle(4, 5, 6));
    triangles.push_back(triangle(7, 8, 9));
    triangles.push_back(triangle(7, 8, 9));
    triangles.push_back(triangle(10, 11, 12));
    Cameras cameras{std::nullopt, identity_camera(0.0), std::nullopt};
    merge(points, triangles, membership, {{0, 10}, {7, 11}}, cameras, origins);
    bool survived = false;
    for (const auto& t : triangles)
        for (size_t v : {t.a, t.b, t.c}) survived |= v == 11 || v == 12;
    MCHECK(!survived);
}

void large_items_far_away_are_not_scanned_by_small_queries() {
    LevelGrid<2> grid(1.0);
    for (size_t item = 0; item < 100; ++item) {
        double y = 1000.0 + (double)item * 50.0;
        double lo[2] = {0.0, y}, hi[2] = {500.0, y + 1.0};
        grid.insert(item, lo, hi);
    }
    double lo[2] = {0.2, 0.2}, hi[2] = {0.8, 0.8};
    grid.insert(500, lo, hi);
    std::set<size_t> found;
    double qlo[2] = {0.0, 0.0}, qhi[2] = {1.0, 1.0};
    MCHECK(grid.query(qlo, qhi, kImageGridCells, found));
    MCHECK(found == (std::set<size_t>{500}));
}

// ---- surface_merge_tests.rs:912-1181: posting bound and clipping budget -------------------
std::string bound_hits_phrase(const MergeStats& s) {
    return std::to_string(s.posting_bound_hits) + " candidate lookup(s) hit the posting bound";
}
std::string clipping_budget_phrase(const MergeStats& s) {
    return std::to_string(s.clipping_budget_exhausted) +
           " triangle(s) exhausted the clipping budget";
}

void the_posting_bound_leaves_the_clipping_budget_reachable() {
    MCHECK(kPostingBound >= 2 * kUncoveredPieces);
    MCHECK(kPostingBound <= 1024);
}

struct Strips {
    std::vector<Point3> points;
    std::vector<int64_t> membership;
    std::vector<MeshTriangle> triangles;
    Pairs pairs;
    size_t left_end, right_end;
};

// surface_merge_tests.rs:948-1008
Strips crossing_strips(size_t bound) {
    Strips s;
    const size_t columns = 2 * bound + 4;
    auto comb = [&](size_t row, size_t column) { return row * (columns + 1) + column; };
    for (size_t row = 0; row < 3; ++row)
        for (size_t column = 0; column <= columns; ++column)
            s.points.push_back(point(-1.0f + 2.0f * (float)column / (float)columns,
                                     (float)row - 1.0f, 5.0f));
    for (size_t row = 0; row < 2; ++row)
        for (size_t column = 0; column < columns; ++column) {
            s.triangles.push_back(
                triangle(comb(row, column), comb(row, column + 1), comb(row + 1, column + 1)));
            s.triangles.push_back(
                triangle(comb(row, column), comb(row + 1, column + 1), comb(row + 1, column)));
        }
    const size_t base = s.points.size();
    const float xs[5] = {-1.5f, -1.0f, 0.0f, 1.0f, 1.5f};
    for (float y : {0.0f, 0.05f})
        for (float x : xs) s.points.push_back(point(x, y, 5.0f));
    auto bottom = [&](size_t k) { return base + k; };
    auto top = [&](size_t k) { return base + 5 + k; };
    for (size_t k = 0; k < 4; ++k) {
        s.triangles.push_back(triangle(bottom(k), bottom(k + 1), top(k + 1)));
        s.triangles.push_back(triangle(bottom(k), top(k + 1), top(k)));
    }
    for (size_t i = 0; i < s.points.size(); ++i) s.membership.push_back(i >= base ? 1 : 0);
    s.pairs = {{comb(1, 0), bottom(1)}};
    s.left_end = bottom(0);
    s.right_end = top(4);
    return s;
}

void crossing_strip_triangulations_keep_per_query_postings_bounded() {
    auto s = crossing_strips(kPostingBound);
    Cameras with_cameras{identity_camera(0.0), identity_camera(0.0)};
    for (const Cameras& cameras : {with_cameras, Cameras{}}) {
        auto triangles = s.triangles;
        auto stats = merge(s.points, triangles, s.membership, s.pairs, cameras, {});
        MCHECK(stats.fused_pairs == 1);
        MCHECK(stats.max_postings_per_query > 0);
        MCHECK(stats.max_postings_per_query <= kPostingBound);
        MCHECK(stats.posting_bound_hits > 0);
        MCHECK(contains_str(stats.diagnostic(2), bound_hits_phrase(stats)));
        size_t ends = 0;
        for (const auto& t : triangles)
            for (size_t v : {t.a, t.b, t.c})
                if (v == s.left_end || v == s.right_end) {
                    ++ends;
                    break;
                }
        MCHECK(ends == 4);
        MCHECK(stats.retained_by_group[0] == s.triangles.size() - 8);
    }
}

struct Fan {
    std::vector<Point3> points;
    std::vector<int64_t> membership;
    std::vector<MeshTriangle> triangles;
    size_t candidate;
};

// surface_merge_tests.rs:1058-1083
Fan sliver_fan(size_t slivers) {
    Fan f;
    f.points = {point(0.0f, -100.0f, 0.0f), point(-2.0f, 0.0f, 0.0f), point(-2.0f, -1.0f, 0.0f)};
    f.triangles = {triangle(0, 1, 2)};
    for (size_t sliver = 0; sliver < slivers; ++sliver) {
        float x = -2.0f + 4.0f * ((float)sliver + 0.5f) / (float)slivers;
        size_t index = f.points.size();
        f.points.push_back(point(x, 100.0f, 0.0f));
        f.points.push_back(point(x + 0.01f, 100.0f, 0.0f));
        f.triangles.push_back(triangle(0, index, index + 1));
    }
    f.candidate = f.points.size();
    f.points.push_back(point(-2.0f, 0.0f, 0.0f));
    f.points.push_back(point(2.0f, 0.0f, 0.0f));
    f.points.push_back(point(0.0f, 2.0f, 0.0f));
    f.triangles.push_back(triangle(f.candidate, f.candidate + 1, f.candidate + 2));
    for (size_t i = 0; i < f.points.size(); ++i) f.membership.push_back(i >= f.candidate ? 1 : 0);
    return f;
}

void a_seam_beyond_the_fragment_budget_is_reported_as_budget_exhausted() {
    const size_t slivers = kUncoveredPieces + 32;
    auto f = sliver_fan(slivers);
    auto stats = merge(f.points, f.triangles, f.membership, {{1, f.candidate}}, {}, {});
    MCHECK(stats.fused_pairs == 1);
    MCHECK(stats.posting_bound_hits == 0);
    MCHECK(stats.removed_duplicate_triangles == 0);
    MCHECK(stats.retained_by_group == (std::vector<size_t>{slivers + 1, 1}));
    MCHECK(stats.clipping_budget_exhausted == 1);
    MCHECK(stats.remaining_overlap_triangles == 0);
    MCHECK(contains_str(stats.diagnostic(2), clipping_budget_phrase(stats)));
}

void ordinary_overlaps_report_no_bound_hits_and_keep_their_results() {
    auto f = sliver_fan(8);
    auto stats = merge(f.points, f.triangles, f.membership, {{1, f.candidate}}, {}, {});
    MCHECK(stats.removed_duplicate_triangles == 0);
    MCHECK(stats.remaining_overlap_triangles == 1);
    MCHECK(stats.clipping_budget_exhausted == 0);
    MCHECK(stats.posting_bound_hits == 0);
    MCHECK(stats.max_postings_per_query > 0);
    MCHECK(contains_str(stats.diagnostic(2), clipping_budget_phrase(stats)));

    auto o = owned_overlap_fixture();
    auto triangles = o.original;
    stats = merge(o.points, triangles, o.membership, o.link, o.cameras, {});
    MCHECK(stats.removed_duplicate_triangles == 1);
    MCHECK(stats.retained_by_group == (std::vector<size_t>{4, 2}));
    MCHECK(stats.posting_bound_hits == 0);
    MCHECK(stats.clipping_budget_exhausted == 0);
    MCHECK(stats.max_postings_per_query > 0);
    MCHECK(stats.max_postings_per_query <= o.original.size());

    std::vector<Point3> points;
    std::vector<int64_t> membership;
    adjacent_grids_fixture(points, triangles, membership);
    const size_t total = triangles.size();
    stats = merge(points, triangles, membership, {{2, 7}, {5, 10}}, {}, {});
    MCHECK(stats.removed_duplicate_triangles == 2);
    MCHECK(triangles.size() == total - 2);
    MCHECK(stats.posting_bound_hits == 0);
    MCHECK(stats.clipping_budget_exhausted == 0);
    MCHECK(stats.max_postings_per_query > 0);
    MCHECK(stats.max_postings_per_query <= total);
    MCHECK(contains_str(stats.diagnostic(2), bound_hits_phrase(stats)));
}

// ---- surface_merge_tests.rs:1170-1450: seam fixtures ------------------------------------
const float kOwnerXs[5] = {-1.84f, -1.38f, -0.92f, -0.46f, 0.0f};
const std::vector<float> kSeamRows = {-1.0f, 0.0f, 1.0f};
const std::vector<float> kOwnerXsV(kOwnerXs, kOwnerXs + 5);

struct SeamFixture {
    std::vector<Point3> points;
    std::vector<int64_t> membership;
    std::vector<MeshTriangle> triangles;
    Pairs pairs;
    Cameras cameras;
    std::vector<int> origins;

    std::pair<std::vector<MeshTriangle>, MergeStats> run() const {
        auto t = triangles;
        auto s = merge(points, t, membership, pairs, cameras, origins);
        return {t, s};
    }
    std::optional<size_t> group(size_t v) const {
        return membership[v] < 0 ? std::nullopt : std::optional<size_t>((size_t)membership[v]);
    }
    // Output triangles that are neither an input triangle nor one re-indexed
    // through an accepted pair (either direction).
    std::vector<MeshTriangle> new_triangles(const std::vector<MeshTriangle>& output) const {
        auto key = [](std::array<size_t, 3> c) {
            std::sort(c.begin(), c.end());
            return c;
        };
        std::set<std::array<size_t, 3>> known;
        for (const auto& t : triangles) {
            std::array<size_t, 3> c{t.a, t.b, t.c};
            known.insert(key(c));
            for (const auto& p : pairs) {
                auto swap = [&](size_t from, size_t to) {
                    std::array<size_t, 3> r = c;
                    for (auto& v : r)
                        if (v == from) v = to;
                    return r;
                };
                known.insert(key(swap(p.first, p.second)));
                known.insert(key(swap(p.second, p.first)));
            }
        }
        std::vector<MeshTriangle> out;
        for (const auto& t : output)
            if (!known.count(key({t.a, t.b, t.c}))) out.push_back(t);
        return out;
    }
};

std::vector<std::vector<size_t>> push_grid(SeamFixture& f, const std::vector<float>& xs,
                                           const std::vector<float>& ys, float z, int64_t group) {
    std::vector<std::vector<size_t>> grid;
    for (float y : ys) {
        std::vector<size_t> row;
        for (float x : xs) {
            f.points.push_back(point(x, y, z));
            f.membership.push_back(group);
            f.origins.push_back(kGeometric);
            row.push_back(f.points.size() - 1);
        }
        grid.push_back(row);
    }
    for (size_t row = 0; row + 1 < ys.size(); ++row)
        for (size_t column = 0; column + 1 < xs.size(); ++column) {
            size_t p00 = grid[row][column], p10 = grid[row][column + 1];
            size_t p01 = grid[row + 1][column], p11 = grid[row + 1][column + 1];
            f.triangles.push_back(triangle(p00, p10, p01));
            f.triangles.push_back(triangle(p10, p11, p01));
        }
    return grid;
}

using Grid = std::vector<std::vector<size_t>>;
void trimmed_seam_fixture(SeamFixture& f, Grid& owner, Grid& lower) {
    owner = push_grid(f, kOwnerXsV, kSeamRows, 5.0f, 0);
    lower = push_grid(f, {-0.46f, 0.04f, 0.54f, 1.04f}, kSeamRows, 5.0f, 1);
    for (size_t row = 0; row < kSeamRows.size(); ++row) f.pairs.push_back({owner[row][3], lower[row][0]});
    f.cameras = {identity_camera(0.0), identity_camera(0.4)};
}

size_t tfind(std::vector<size_t>& parent, size_t index) {
    size_t root = index;
    while (parent[root] != root) root = parent[root];
    size_t node = index;
    while (parent[node] != root) {
        size_t next = parent[node];
        parent[node] = root;
        node = next;
    }
    return root;
}

std::pair<size_t, std::vector<size_t>> vertex_components(const std::vector<MeshTriangle>& t,
                                                         size_t vertices) {
    std::vector<size_t> parent(vertices);
    for (size_t i = 0; i < vertices; ++i) parent[i] = i;
    std::vector<char> used(vertices, 0);
    for (const auto& x : t) {
        used[x.a] = used[x.b] = used[x.c] = 1;
        size_t root = tfind(parent, x.a);
        for (size_t v : {x.b, x.c}) {
            size_t other = tfind(parent, v);
            parent[other] = root;
        }
    }
    std::vector<size_t> roots(vertices);
    for (size_t v = 0; v < vertices; ++v) roots[v] = tfind(parent, v);
    size_t count = 0;
    for (size_t v = 0; v < vertices; ++v)
        if (used[v] && roots[v] == v) ++count;
    return {count, roots};
}

double signed_area_2d(const std::vector<V2>& c) {
    double s = -0.0;
    for (size_t i = 0; i < c.size(); ++i) s += cross2(c[i], c[(i + 1) % c.size()]);
    return s * 0.5;
}

// the test's own convex clip (surface_merge_tests.rs:1330-1353)
double test_intersection_area(const std::vector<V2>& subject, const std::vector<V2>& clip) {
    double orientation = signum(signed_area_2d(clip));
    std::vector<V2> polygon = subject;
    for (size_t index = 0; index < 3; ++index) {
        V2 a = clip[index], b = clip[(index + 1) % 3];
        auto side = [&](V2 p) { return orientation * cross2(b - a, p - a); };
        std::vector<V2> next;
        for (size_t current = 0; current < polygon.size(); ++current) {
            V2 p = polygon[current], q = polygon[(current + 1) % polygon.size()];
            double sp = side(p), sq = side(q);
            if (sp >= 0.0) next.push_back(p);
            if ((sp >= 0.0) != (sq >= 0.0)) next.push_back(p + (q - p) * (sp / (sp - sq)));
        }
        polygon = next;
        if (polygon.size() < 3) return 0.0;
    }
    return std::fabs(signed_area_2d(polygon));
}

std::vector<std::vector<V2>> project_all(const SeamFixture& f, const std::vector<Point3>& points,
                                         const std::vector<MeshTriangle>& triangles) {
    const RefCamera camera = *f.cameras[0];
    std::vector<std::vector<V2>> out;
    for (const auto& t : triangles) {
        std::vector<V2> c;
        for (size_t v : {t.a, t.b, t.c}) {
            auto p = camera.project(Vec3{(double)points[v].x, (double)points[v].y, (double)points[v].z});
            MCHECK(p.has_value());
            c.push_back(p->image);
        }
        out.push_back(c);
    }
    return out;
}

void assert_tiles_owner_image_over(const SeamFixture& f, const std::vector<Point3>& points,
                                   const std::vector<MeshTriangle>& triangles, double left,
                                   double right) {
    auto projected = project_all(f, points, triangles);
    for (const auto& c : projected) MCHECK(signed_area_2d(c) > 0.0);
    for (size_t first = 0; first < projected.size(); ++first)
        for (size_t second = first + 1; second < projected.size(); ++second)
            MCHECK(test_intersection_area(projected[first], projected[second]) < 1.0e-9);
    const double rectangle = (right - left) / 5.0 * (2.0 / 5.0);
    double total = -0.0;
    for (const auto& c : projected) total += signed_area_2d(c);
    MCHECK(std::fabs(total - rectangle) < 1.0e-6 * rectangle);
}

void assert_tiles_owner_image(const SeamFixture& f, const std::vector<MeshTriangle>& t,
                              double left, double right) {
    assert_tiles_owner_image_over(f, f.points, t, left, right);
}

void a_trimmed_seam_is_stitched_into_one_connected_surface() {
    SeamFixture f;
    Grid owner, lower;
    trimmed_seam_fixture(f, owner, lower);
    auto [triangles, stats] = f.run();
    MCHECK(stats.removed_duplicate_triangles == 4);
    MCHECK(stats.trimmed_seam_triangles == 4);
    for (const auto& t : triangles)
        MCHECK(t.a < f.points.size() && t.b < f.points.size() && t.c < f.points.size());
    MCHECK(vertex_components(triangles, f.points.size()).first == 1);
    MCHECK(stats.patch_components == 1);
    auto stitches = f.new_triangles(triangles);
    MCHECK(!stitches.empty());
    MCHECK(stats.stitched_seam_triangles > 0);
    MCHECK(stats.stitched_seam_triangles == stitches.size());
    for (const auto& t : stitches) {
        std::set<std::optional<size_t>> g{f.group(t.a), f.group(t.b), f.group(t.c)};
        MCHECK(g == (std::set<std::optional<size_t>>{size_t(0), size_t(1)}));
    }
    MCHECK(contains_str(stats.diagnostic(2), std::to_string(stats.stitched_seam_triangles) +
                                                 " seam stitch triangle(s)"));
    assert_tiles_owner_image(f, triangles, (double)f.points[owner[0][0]].x,
                             (double)f.points[lower[0][3]].x);
}

void the_seam_contract_is_satisfiable_by_a_strip_over_existing_vertices() {
    SeamFixture f;
    Grid owner, lower;
    trimmed_seam_fixture(f, owner, lower);
    std::set<size_t> seam_column;
    for (const auto& row : lower) seam_column.insert(row[0]);
    std::vector<MeshTriangle> triangles;
    for (const auto& t : f.triangles)
        if (!seam_column.count(t.a) && !seam_column.count(t.b) && !seam_column.count(t.c))
            triangles.push_back(t);
    MCHECK(triangles.size() == f.triangles.size() - 4);
    MCHECK(vertex_components(triangles, f.points.size()).first == 2);
    for (size_t row = 0; row + 1 < kSeamRows.size(); ++row) {
        triangles.push_back(triangle(owner[row][4], lower[row][1], owner[row + 1][4]));
        triangles.push_back(triangle(lower[row][1], lower[row + 1][1], owner[row + 1][4]));
    }
    MCHECK(vertex_components(triangles, f.points.size()).first == 1);
    MCHECK(f.new_triangles(triangles).size() == 4);
    assert_tiles_owner_image(f, triangles, (double)f.points[owner[0][0]].x,
                             (double)f.points[lower[0][3]].x);
}

void seam_stitching_is_deterministic() {
    SeamFixture f;
    Grid owner, lower;
    trimmed_seam_fixture(f, owner, lower);
    auto a = f.run();
    auto b = f.run();
    MCHECK(signature(a.first) == signature(b.first));
    MCHECK(a.second == b.second);
}

void an_unobserved_gap_between_linked_patches_is_never_bridged() {
    SeamFixture f;
    auto owner = push_grid(f, kOwnerXsV, kSeamRows, 5.0f, 0);
    auto lower = push_grid(f, {0.3f, 0.8f, 1.3f}, kSeamRows, 5.0f, 1);
    f.origins[lower[1][0]] = kRevalidated;
    f.pairs = {{owner[1][4], lower[1][0]}};
    f.cameras = {identity_camera(0.0), identity_camera(0.4)};
    auto [triangles, stats] = f.run();
    MCHECK(stats.provenance_separated_pairs == 1);
    MCHECK(stats.removed_duplicate_triangles == 0);
    MCHECK(stats.stitched_seam_triangles == 0);
    MCHECK(f.new_triangles(triangles).empty());
    MCHECK(signature(triangles) == signature(f.triangles));
    MCHECK(vertex_components(triangles, f.points.size()).first == 2);
}

void a_trimmed_seam_is_not_stitched_to_a_surface_at_another_depth() {
    SeamFixture f;
    auto owner = push_grid(f, kOwnerXsV, kSeamRows, 5.0f, 0);
    auto seam = push_grid(f, {-0.46f, 0.04f}, kSeamRows, 5.0f, 1);
    auto far = push_grid(f, {0.04f, 0.54f, 1.04f}, kSeamRows, 5.4f, 1);
    f.origins[far[1][0]] = kRevalidated;
    for (size_t row = 0; row < kSeamRows.size(); ++row) f.pairs.push_back({owner[row][3], seam[row][0]});
    f.pairs.push_back({owner[1][4], far[1][0]});
    f.cameras = {identity_camera(0.0), identity_camera(0.4)};
    std::set<size_t> far_vertices, owner_vertices;
    for (const auto& r : far) far_vertices.insert(r.begin(), r.end());
    for (const auto& r : owner) owner_vertices.insert(r.begin(), r.end());
    auto [triangles, stats] = f.run();
    MCHECK(stats.trimmed_seam_triangles == 4);
    size_t far_kept = 0;
    for (const auto& t : triangles)
        if (far_vertices.count(t.a) && far_vertices.count(t.b) && far_vertices.count(t.c)) ++far_kept;
    MCHECK(far_kept == 8);
    for (const auto& t : triangles) {
        bool o = owner_vertices.count(t.a) || owner_vertices.count(t.b) || owner_vertices.count(t.c);
        bool r = far_vertices.count(t.a) || far_vertices.count(t.b) || far_vertices.count(t.c);
        MCHECK(!(o && r));
    }
    auto roots = vertex_components(triangles, f.points.size()).second;
    MCHECK(roots[owner[1][4]] != roots[far[1][0]]);
    MCHECK(stats.stitched_seam_triangles == 0);
}

void patches_without_a_fusion_link_are_never_stitched() {
    SeamFixture f;
    Grid owner, lower;
    trimmed_seam_fixture(f, owner, lower);
    f.pairs.clear();
    auto [triangles, stats] = f.run();
    MCHECK(stats.removed_duplicate_triangles == 0);
    MCHECK(stats.stitched_seam_triangles == 0);
    MCHECK(f.new_triangles(triangles).empty());
    MCHECK(signature(triangles) == signature(f.triangles));
    MCHECK(vertex_components(triangles, f.points.size()).first == 2);
}

void only_the_linked_patch_of_three_is_stitched() {
    SeamFixture f;
    Grid owner, lower;
    trimmed_seam_fixture(f, owner, lower);
    auto third = push_grid(f, {-2.3f, -1.8f, -1.3f}, kSeamRows, 5.0f, 2);
    f.cameras.push_back(identity_camera(-1.5));
    std::set<size_t> third_vertices;
    for (const auto& r : third) third_vertices.insert(r.begin(), r.end());
    auto [triangles, stats] = f.run();
    MCHECK(stats.trimmed_seam_triangles == 4);
    MCHECK(stats.retained_by_group[2] == 8);
    auto [components, roots] = vertex_components(triangles, f.points.size());
    MCHECK(components == 2);
    MCHECK(roots[owner[1][4]] == roots[lower[1][1]]);
    MCHECK(roots[owner[1][0]] != roots[third[1][0]]);
    auto stitches = f.new_triangles(triangles);
    MCHECK(!stitches.empty());
    MCHECK(stats.stitched_seam_triangles == stitches.size());
    for (const auto& t : stitches)
        MCHECK(!third_vertices.count(t.a) && !third_vertices.count(t.b) && !third_vertices.count(t.c));
}

void partial_overlap(SeamFixture& f, bool sloped, Grid& owner, Grid& lower) {
    owner = push_grid(f, kOwnerXsV, kSeamRows, 5.0f, 0);
    lower = push_grid(f, {-0.46f, -0.04f, 0.46f, 0.96f}, kSeamRows, 5.0f, 1);
    if (sloped)
        for (auto& p : f.points) p.z = 5.0f + 0.25f * p.x + 0.15f * p.y;
    for (size_t row = 0; row < kSeamRows.size(); ++row) f.pairs.push_back({owner[row][3], lower[row][0]});
    f.cameras = {identity_camera(0.0), identity_camera(0.4)};
}

void a_partial_overlap_seam_preserves_the_union_without_double_coverage() {
    SeamFixture f;
    Grid owner, lower;
    partial_overlap(f, false, owner, lower);
    Control control;
    OwnedMerge out;
    MCHECK(owned_merge(f.points, f.triangles, f.membership, f.pairs, f.cameras, f.origins, control,
                       out));
    MCHECK(out.stats.fused_pairs > 0);
    MCHECK(out.points.size() >= f.points.size());
    for (size_t i = 0; i < f.points.size(); ++i)
        MCHECK(out.points[i].x == f.points[i].x && out.points[i].y == f.points[i].y &&
               out.points[i].z == f.points[i].z);
    MCHECK(out.derived_vertices.size() == out.points.size() - f.points.size());
    for (const auto& t : out.triangles)
        MCHECK(t.a < out.points.size() && t.b < out.points.size() && t.c < out.points.size());
    assert_tiles_owner_image_over(f, out.points, out.triangles, -1.84, 0.96);
    MCHECK(vertex_components(out.triangles, out.points.size()).first == 1);
}

// ---- surface_merge_derived_acceptance_tests.rs ----------------------------------------
Vec3 xyz(const Point3& p) { return {(double)p.x, (double)p.y, (double)p.z}; }

void assert_edge_conforming(const std::vector<Point3>& points,
                            const std::vector<MeshTriangle>& triangles) {
    std::set<size_t> referenced;
    for (const auto& t : triangles) referenced.insert({t.a, t.b, t.c});
    for (const auto& t : triangles) {
        const std::pair<size_t, size_t> es[3] = {{t.a, t.b}, {t.b, t.c}, {t.c, t.a}};
        for (const auto& e : es) {
            Vec3 start = xyz(points[e.first]);
            Vec3 direction = sub(xyz(points[e.second]), start);
            MCHECK(norm_squared(direction) > 1.0e-14);
            for (size_t v : referenced) {
                if (v == e.first || v == e.second) continue;
                Vec3 delta = sub(xyz(points[v]), start);
                double fraction = dot3(delta, direction) / norm_squared(direction);
                MCHECK(!(fraction > 1.0e-6 && fraction < 1.0 - 1.0e-6 &&
                         norm(sub(delta, scale3(direction, fraction))) < 1.0e-6));
            }
        }
    }
}

void owned_clip_contract(bool sloped) {
    SeamFixture f;
    Grid owner, lower;
    partial_overlap(f, sloped, owner, lower);
    const auto original_points = f.points;
    const auto original_triangles = f.triangles;
    std::vector<std::vector<V2>> source_image = project_all(f, f.points, f.triangles);
    double uni = -0.0;
    for (const auto& c : source_image) uni += signed_area_2d(c);
    for (size_t first = 0; first < original_triangles.size(); ++first)
        for (size_t second = first + 1; second < original_triangles.size(); ++second)
            if (f.membership[original_triangles[first].a] != f.membership[original_triangles[second].a])
                uni -= test_intersection_area(source_image[first], source_image[second]);
    std::vector<Point3> points = f.points;
    points.reserve(1024);
    const Point3* allocation = points.data();
    Control control;
    OwnedMerge out;
    MergeInputs in{nullptr, &f.membership, &f.pairs, &f.cameras, &f.origins};
    std::string error;
    MCHECK(merge_fused_patches_owned(std::move(points), f.triangles, in, control, out, error));
    MCHECK(out.points.data() == allocation);
    MCHECK(out.points.size() > original_points.size());
    MCHECK(out.derived_vertices.size() == out.points.size() - original_points.size());
    for (size_t i = 0; i < original_points.size(); ++i) {
        const Point3 &b = original_points[i], &a = out.points[i];
        MCHECK(b.x == a.x && b.y == a.y && b.z == a.z && b.confidence == a.confidence &&
               b.r == a.r && b.g == a.g && b.b == a.b);
    }
    std::set<size_t> derived;
    for (const auto& record : out.derived_vertices) {
        MCHECK(derived.insert(record.point_index).second);
        MCHECK(record.point_index >= original_points.size() &&
               record.point_index < out.points.size());
        MCHECK(record.source_triangle < original_triangles.size());
        const MeshTriangle& parent = original_triangles[record.source_triangle];
        MCHECK(record.source_corners == (std::array<size_t, 3>{parent.a, parent.b, parent.c}));
        double sum = -0.0;
        for (double w : record.barycentric) {
            MCHECK(std::isfinite(w) && w >= -1.0e-7 && w <= 1.0 + 1.0e-7);
            sum += w;
        }
        MCHECK(std::fabs(sum - 1.0) < 1.0e-7);
        Vec3 expected{0.0, 0.0, 0.0};
        const size_t pc[3] = {parent.a, parent.b, parent.c};
        for (int k = 0; k < 3; ++k)
            expected = add(expected, scale3(xyz(original_points[pc[k]]), record.barycentric[k]));
        MCHECK(norm(sub(expected, xyz(out.points[record.point_index]))) < 1.0e-6);
    }
    auto projected = project_all(f, out.points, out.triangles);
    double area = -0.0;
    for (const auto& c : projected) {
        MCHECK(signed_area_2d(c) > 0.0);
        area += signed_area_2d(c);
    }
    MCHECK(std::fabs(area - uni) < 1.0e-6 * uni);
    for (size_t first = 0; first < projected.size(); ++first)
        for (size_t second = first + 1; second < projected.size(); ++second)
            MCHECK(test_intersection_area(projected[first], projected[second]) < 1.0e-9);
    MCHECK(vertex_components(out.triangles, out.points.size()).first == 1);
    assert_edge_conforming(out.points, out.triangles);
}

void flat_overlap_uses_owned_buffers_and_sparse_source_triangle_lineage() {
    owned_clip_contract(false);
}

void sloped_overlap_reconstructs_derived_world_positions_from_immutable_parents() {
    owned_clip_contract(true);
}

bool same_owned(const OwnedMerge& a, const OwnedMerge& b) {
    if (a.points.size() != b.points.size() || a.triangles.size() != b.triangles.size() ||
        a.derived_vertices.size() != b.derived_vertices.size())
        return false;
    for (size_t i = 0; i < a.points.size(); ++i)
        if (std::memcmp(&a.points[i], &b.points[i], sizeof(Point3)) != 0) return false;
    for (size_t i = 0; i < a.triangles.size(); ++i)
        if (a.triangles[i].a != b.triangles[i].a || a.triangles[i].b != b.triangles[i].b ||
            a.triangles[i].c != b.triangles[i].c ||
            std::memcmp(&a.triangles[i].confidence, &b.triangles[i].confidence, 4) != 0)
            return false;
    for (size_t i = 0; i < a.derived_vertices.size(); ++i) {
        const auto &x = a.derived_vertices[i], &y = b.derived_vertices[i];
        if (x.point_index != y.point_index || x.source_triangle != y.source_triangle ||
            x.source_corners != y.source_corners ||
            std::memcmp(x.barycentric.data(), y.barycentric.data(), 24) != 0)
            return false;
    }
    return true;
}

void owned_overlap_cancellation_aborts_without_a_partial_result_and_noop_is_identical() {
    SeamFixture f;
    Grid owner, lower;
    partial_overlap(f, true, owner, lower);
    Control plain_control;
    OwnedMerge plain;
    MCHECK(owned_merge(f.points, f.triangles, f.membership, f.pairs, f.cameras, f.origins,
                       plain_control, plain));
    size_t polls = 0;
    Control never;
    never.poll = [&]() {
        ++polls;
        return false;
    };
    OwnedMerge controlled;
    MCHECK(owned_merge(f.points, f.triangles, f.membership, f.pairs, f.cameras, f.origins, never,
                       controlled));
    MCHECK(same_owned(plain, controlled));
    MCHECK(polls > 2);
    const size_t stop = std::max<size_t>(polls / 2, 2);
    size_t seen = 0;
    Control cancel;
    cancel.poll = [&]() {
        ++seen;
        return seen >= stop;
    };
    OwnedMerge result;
    MCHECK(!owned_merge(f.points, f.triangles, f.membership, f.pairs, f.cameras, f.origins, cancel,
                        result));
    MCHECK(seen >= stop);
}

}  // namespace

int merge_selftest(std::string& failure) {
    static void (*const tests[])() = {
        union_coverage_handles_a_different_diagonal_and_large_triangles,
        never_discards_an_unsupported_hole_or_partial_boundary,
        normal_and_depth_disagreement_are_not_coverage,
        no_accepted_fusion_pair_means_no_dedup_even_for_coincident_sheets,
        a_fusion_link_does_not_erase_an_unrelated_island_of_the_same_camera_pair,
        a_confirmed_seam_deduplicates_overlap_but_keeps_the_uncovered_extension,
        large_triangles_are_indexed_across_their_interior,
        image_ownership_tolerates_reference_scale_but_not_another_surface,
        image_ownership_measures_the_share_on_the_footprint,
        owned_overlap_is_removed_and_unique_surface_is_kept,
        a_depth_rejection_in_the_image_is_not_overturned_by_the_3d_test,
        the_relative_scale_is_anchored_at_fusion_accepted_seam_vertices,
        pairs_across_evidence_origins_link_patches_but_keep_their_vertices,
        only_vertices_referenced_by_two_patches_count_as_shared,
        oversized_owner_triangles_are_checked_exactly,
        scale_samples_need_an_anchored_owner_triangle,
        unprojectable_linked_owners_leave_the_image_unable_to_judge,
        scale_samples_stop_at_the_limit,
        an_owner_without_an_image_judgement_still_gets_the_3d_test,
        large_items_far_away_are_not_scanned_by_small_queries,
        the_posting_bound_leaves_the_clipping_budget_reachable,
        crossing_strip_triangulations_keep_per_query_postings_bounded,
        a_seam_beyond_the_fragment_budget_is_reported_as_budget_exhausted,
        ordinary_overlaps_report_no_bound_hits_and_keep_their_results,
        a_trimmed_seam_is_stitched_into_one_connected_surface,
        the_seam_contract_is_satisfiable_by_a_strip_over_existing_vertices,
        seam_stitching_is_deterministic,
        an_unobserved_gap_between_linked_patches_is_never_bridged,
        a_trimmed_seam_is_not_stitched_to_a_surface_at_another_depth,
        patches_without_a_fusion_link_are_never_stitched,
        only_the_linked_patch_of_three_is_stitched,
        a_partial_overlap_seam_preserves_the_union_without_double_coverage,
        flat_overlap_uses_owned_buffers_and_sparse_source_triangle_lineage,
        sloped_overlap_reconstructs_derived_world_positions_from_immutable_parents,
        owned_overlap_cancellation_aborts_without_a_partial_result_and_noop_is_identical,
    };
    g_checks = 0;
    try {
        for (auto t : tests) t();
    } catch (const Fail& f) {
        failure = f.what;
        return -1;
    }
    return g_checks;
}

}  // namespace merge
}  // namespace v3do
