// TEST INFRASTRUCTURE — CPU oracle of the connected-surface merge
// (surface_merge.rs, surface_merge_clip.rs, surface_merge_stitch.rs).
// See oracle_merge.hpp for the evaluation-order rules.
#include "oracle_merge.hpp"

#include <algorithm>
#include <cinttypes>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <limits>
#include <unordered_map>

namespace v3do {
namespace merge {

namespace {

constexpr double kGeometricEpsilon = 1.0e-9;            // surface_merge.rs:57
constexpr double kMaxOverlapDistanceFraction = 0.9;     // :60
constexpr size_t kMaxGridCells = 1728;                  // :63
constexpr size_t kMaxUncoveredPieces = 128;             // :65
constexpr size_t kMaxPostingsPerQuery = 512;            // :73
constexpr double kMinNormalAlignment = 0.94;            // :76
constexpr double kMinImageOwnershipShare = 0.8;         // :81
constexpr double kMaxRelativeDepthDisagreement = 0.035; // :89
constexpr double kMaxRelativeScaleSample = 0.1;         // :93
constexpr size_t kMinScaleSamples = 5;                  // :95
constexpr size_t kMaxScaleSamples = 4096;               // :99
constexpr double kOwnershipEpsilon = 1.0e-9;            // :1304
constexpr size_t kMaxImageGridCells = 4096;             // :1307
constexpr int64_t kMaxAnchorCellSpan = 3;               // :1311
constexpr int32_t kMaxGridLevels = 48;                  // :1678
// surface_merge_clip.rs:48-67
constexpr size_t kMaxClipOwnerTriangles = 48;
constexpr size_t kMaxClipNodes = 160;
constexpr double kMaxClipDepthDisagreement = 0.014;
constexpr double kRelativeTolerance = 1.0e-5;
constexpr double kAreaTolerance = 1.0e-4;
// surface_merge_stitch.rs:48-63
constexpr size_t kMaxSeamVertices = 6;
constexpr size_t kMaxSeamsPerVertex = 16;
constexpr double kMaxUnobservedStitchShare = 1.0e-6;
constexpr double kMaxStitchOverlapShare = 1.0e-6;
constexpr double kInsideTolerance = 1.0e-6;
constexpr double kF64Epsilon = std::numeric_limits<double>::epsilon();
constexpr double kF64MinPositive = std::numeric_limits<double>::min();

// Rust `as i64` from f64: saturating, NaN to 0.
int64_t sat_i64(double v) {
    if (std::isnan(v)) return 0;
    if (v >= 9223372036854775807.0) return INT64_MAX;
    if (v <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)v;
}
int64_t sat_sub(int64_t a, int64_t b) {
    int64_t r;
    if (__builtin_sub_overflow(a, b, &r)) return b < 0 ? INT64_MAX : INT64_MIN;
    return r;
}
size_t sat_mul(size_t a, size_t b) {
    size_t r;
    if (__builtin_mul_overflow(a, b, &r)) return SIZE_MAX;
    return r;
}
// Rust f64::max / f64::min (NaN-ignoring).
double fmax_(double a, double b) { return std::fmax(a, b); }
double fmin_(double a, double b) { return std::fmin(a, b); }
// f64::clamp
double clamp_(double v, double lo, double hi) {
    if (v < lo) v = lo;
    if (v > hi) v = hi;
    return v;
}

Vec3 to_v3(const Point3& p) { return {(double)p.x, (double)p.y, (double)p.z}; }
Vec3 normalize3(Vec3 v) {
    double n = norm(v);
    return {v.x / n, v.y / n, v.z / n};
}

size_t find(std::vector<size_t>& parent, size_t index) {
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

std::optional<size_t> group_of_vec(const std::vector<int64_t>& membership, size_t v) {
    if (v < membership.size() && membership[v] >= 0) return (size_t)membership[v];
    return std::nullopt;
}

// signed_area (surface_merge_clip.rs:761-766)
double signed_area(const Polygon& polygon) {
    double s = -0.0;
    const size_t n = polygon.size();
    for (size_t i = 0; i < n; ++i) s += cross2(polygon[i], polygon[(i + 1) % n]);
    return s * 0.5;
}

}  // namespace

double signum(double v) {
    if (std::isnan(v)) return v;
    return std::signbit(v) ? -1.0 : 1.0;
}

bool total_less(double a, double b) {
    int64_t l, r;
    std::memcpy(&l, &a, 8);
    std::memcpy(&r, &b, 8);
    l ^= (int64_t)(((uint64_t)(l >> 63)) >> 1);
    r ^= (int64_t)(((uint64_t)(r >> 63)) >> 1);
    return l < r;
}

// ---- ReferenceCamera --------------------------------------------------------
Vec3 RefCamera::to_camera(Vec3 p) const {
    // rotation * point (nalgebra: columns accumulated left to right) + translation
    Vec3 r;
    r.x = (R[0] * p.x + R[1] * p.y) + R[2] * p.z;
    r.y = (R[3] * p.x + R[4] * p.y) + R[5] * p.z;
    r.z = (R[6] * p.x + R[7] * p.y) + R[8] * p.z;
    return {r.x + t[0], r.y + t[1], r.z + t[2]};
}

std::optional<PC> RefCamera::project(Vec3 p) const {
    Vec3 c = to_camera(p);
    if (c.z > kGeometricEpsilon && std::isfinite(c.x) && std::isfinite(c.y) && std::isfinite(c.z))
        return PC{V2{c.x / c.z, c.y / c.z}, c.z};
    return std::nullopt;
}

std::optional<std::pair<Vec3, double>> RefCamera::plane(const std::array<Vec3, 3>& corners) const {
    Vec3 a = to_camera(corners[0]), b = to_camera(corners[1]), c = to_camera(corners[2]);
    Vec3 normal = cross(sub(b, a), sub(c, a));
    if (norm(normal) > kGeometricEpsilon) return std::make_pair(normal, dot3(normal, a));
    return std::nullopt;
}

std::optional<ProjTri> RefCamera::project_triangle(const std::array<Vec3, 3>& corners) const {
    auto a = project(corners[0]);
    auto b = project(corners[1]);
    auto c = project(corners[2]);
    if (!a || !b || !c) return std::nullopt;
    return ProjTri{*a, *b, *c};
}

// ---- polygon helpers (surface_merge.rs:1871-1917) -------------------------------
double polygon_area(const Polygon& points) {
    if (points.size() < 3) return 0.0;
    double s = -0.0;
    const size_t n = points.size();
    for (size_t i = 0; i < n; ++i) s += cross2(points[i], points[(i + 1) % n]);
    return std::fabs(s) * 0.5;
}

std::pair<Polygon, Polygon> split_polygon(const Polygon& polygon, V2 a, V2 b, double orientation) {
    Polygon included, excluded;
    if (polygon.empty()) return {included, excluded};
    const V2 ba = b - a;
    auto signed_ = [&](V2 p) { return orientation * cross2(ba, p - a); };
    const size_t n = polygon.size();
    for (size_t i = 0; i < n; ++i) {
        V2 previous = polygon[(i + n - 1) % n];
        V2 current = polygon[i];
        double before = signed_(previous), after = signed_(current);
        if ((before < 0.0 && after > 0.0) || (before > 0.0 && after < 0.0)) {
            V2 x = previous + (current - previous) * (before / (before - after));
            included.push_back(x);
            excluded.push_back(x);
        }
        if (after >= 0.0) included.push_back(current);
        if (after <= 0.0) excluded.push_back(current);
    }
    return {included, excluded};
}

double image_area(const ProjTri& t) {
    return std::fabs(cross2(t[1].image - t[0].image, t[2].image - t[0].image)) * 0.5;
}

std::optional<double> inverse_depth(const ProjTri& t, V2 point) {
    V2 a = t[0].image, b = t[1].image, c = t[2].image;
    double za = t[0].depth, zb = t[1].depth, zc = t[2].depth;
    double determinant = cross2(b - a, c - a);
    if (std::fabs(determinant) <= kGeometricEpsilon * kGeometricEpsilon) return std::nullopt;
    double wb = cross2(point - a, c - a) / determinant;
    double wc = cross2(b - a, point - a) / determinant;
    double inverse = (((1.0 - wb) - wc) / za + wb / zb) + wc / zc;
    if (std::isfinite(inverse) && inverse > 0.0) return inverse;
    return std::nullopt;
}

namespace {
void image_aabb(const ProjTri& t, double low[2], double high[2]) {
    low[0] = low[1] = INFINITY;
    high[0] = high[1] = -INFINITY;
    for (const auto& c : t) {
        low[0] = fmin_(low[0], c.image.x);
        high[0] = fmax_(high[0], c.image.x);
        low[1] = fmin_(low[1], c.image.y);
        high[1] = fmax_(high[1], c.image.y);
    }
}

// Area of an image polygon lifted onto a camera-space plane (surface_merge.rs:1628-1645).
double back_projected_area(const Polygon& polygon, const std::pair<Vec3, double>& plane) {
    const Vec3 normal = plane.first;
    const double offset = plane.second;
    std::vector<Vec3> lifted;
    lifted.reserve(polygon.size());
    for (const V2& p : polygon) {
        Vec3 ray{p.x, p.y, 1.0};
        double along = dot3(normal, ray);
        if (!(std::fabs(along) > kGeometricEpsilon)) return 0.0;
        lifted.push_back(scale3(ray, offset / along));
    }
    Vec3 sum{0.0, 0.0, 0.0};
    for (size_t i = 0; i < lifted.size(); ++i)
        sum = add(sum, cross(lifted[i], lifted[(i + 1) % lifted.size()]));
    return norm(sum) * 0.5;
}
}  // namespace

// ---- TriangleGeometry (surface_merge.rs:1137-1291) ------------------------------
std::optional<TriangleGeometry> TriangleGeometry::make(const std::array<Vec3, 3>& c) {
    for (const auto& p : c)
        if (!std::isfinite(p.x) || !std::isfinite(p.y) || !std::isfinite(p.z)) return std::nullopt;
    Vec3 n = cross(sub(c[1], c[0]), sub(c[2], c[0]));
    double length = norm(n);
    if (!std::isfinite(length) || length <= kGeometricEpsilon) return std::nullopt;
    TriangleGeometry g;
    g.corners = c;
    g.normal = {n.x / length, n.y / length, n.z / length};
    g.edges[0] = norm(sub(c[1], c[0]));
    g.edges[1] = norm(sub(c[2], c[1]));
    g.edges[2] = norm(sub(c[0], c[2]));
    return g;
}

double TriangleGeometry::area() const {
    return norm(cross(sub(corners[1], corners[0]), sub(corners[2], corners[0]))) * 0.5;
}

void TriangleGeometry::aabb(double padding, double low[3], double high[3]) const {
    for (int axis = 0; axis < 3; ++axis) {
        double lo = INFINITY, hi = -INFINITY;
        for (const auto& p : corners) {
            double v = axis == 0 ? p.x : axis == 1 ? p.y : p.z;
            lo = fmin_(lo, v);
            hi = fmax_(hi, v);
        }
        low[axis] = lo - padding;
        high[axis] = hi + padding;
    }
}

CoverageResult TriangleGeometry::coverage(const std::vector<const TriangleGeometry*>& surfaces,
                                          double tolerance) const {
    const Vec3 origin = corners[0];
    const Vec3 u = normalize3(sub(corners[1], origin));
    const Vec3 v = cross(normal, u);
    auto project = [&](Vec3 point) {
        Vec3 rel = sub(point, origin);
        return V2{dot3(rel, u), dot3(rel, v)};
    };
    double m = 1.0e-12;
    for (double e : edges) m = fmax_(m, e);
    const double area_epsilon = m * m * 1.0e-10;
    std::vector<Polygon> remaining{Polygon{project(corners[0]), project(corners[1]),
                                           project(corners[2])}};
    bool partially_covered = false;
    for (const TriangleGeometry* surface : surfaces) {
        if (std::fabs(dot3(normal, surface->normal)) < kMinNormalAlignment) continue;
        V2 projected[3] = {project(surface->corners[0]), project(surface->corners[1]),
                           project(surface->corners[2])};
        double winding = cross2(projected[1] - projected[0], projected[2] - projected[0]);
        if (std::fabs(winding) <= area_epsilon) continue;
        double orientation = signum(winding);
        std::vector<Polygon> next;
        for (Polygon& polygon : remaining) {
            Polygon inside = std::move(polygon);
            std::vector<Polygon> outside;
            for (int edge = 0; edge < 3; ++edge) {
                auto split = split_polygon(inside, projected[edge], projected[(edge + 1) % 3],
                                           orientation);
                if (polygon_area(split.second) > area_epsilon) outside.push_back(split.second);
                inside = std::move(split.first);
                if (inside.empty()) break;
            }
            if (polygon_area(inside) > area_epsilon) {
                bool supported = true;
                for (const V2& p : inside) {
                    Vec3 point = add(add(origin, scale3(u, p.x)), scale3(v, p.y));
                    if (!(std::fabs(dot3(sub(point, surface->corners[0]), surface->normal)) <=
                          tolerance)) {
                        supported = false;
                        break;
                    }
                }
                if (supported)
                    partially_covered = true;
                else
                    outside.push_back(inside);
            }
            for (auto& o : outside) next.push_back(std::move(o));
            if (next.size() > kMaxUncoveredPieces)
                return {Coverage::BudgetExhausted, partially_covered};
        }
        remaining = std::move(next);
        if (remaining.empty()) return {Coverage::Full, false};
    }
    return {partially_covered ? Coverage::Partial : Coverage::Uncovered, false};
}

std::pair<bool, bool> TriangleGeometry::covered_by(
    const std::vector<const TriangleGeometry*>& surfaces, double tolerance) const {
    CoverageResult r = coverage(surfaces, tolerance);
    switch (r.kind) {
        case Coverage::Full: return {true, true};
        case Coverage::Partial: return {false, true};
        case Coverage::Uncovered: return {false, false};
        default: return {false, r.partially_covered};
    }
}

// ---- postings ----------------------------------------------------------------
PostingBudget PostingBudget::per_query() { return PostingBudget(kMaxPostingsPerQuery); }

QueryLimit PostingBudget::take_into(const std::vector<size_t>& items, std::set<size_t>& out) {
    size_t room = limit - used;
    if (items.size() <= room) {
        used += items.size();
        out.insert(items.begin(), items.end());
        return QueryLimit::None;
    }
    used = limit;
    out.insert(items.begin(), items.begin() + room);
    return QueryLimit::Postings;
}

void PostingTally::record(const PostingBudget& b, QueryLimit result) {
    max_postings = std::max(max_postings, b.used);
    if (result == QueryLimit::Postings) bound_hits += 1;
}

// ---- LevelGrid ----------------------------------------------------------------
template <int D>
bool LevelGrid<D>::range(const double* low, const double* high, int32_t level,
                         std::array<std::pair<int64_t, int64_t>, D>& out) const {
    // 2.0_f64.powi(level): exact for the levels used
    const double size = cell * std::ldexp(1.0, level);
    for (int axis = 0; axis < D; ++axis) {
        double first = std::floor(low[axis] / size), last = std::floor(high[axis] / size);
        if (!std::isfinite(first) || !std::isfinite(last) || first > last) return false;
        out[axis] = {sat_i64(first), sat_i64(last)};
    }
    return true;
}

template <int D>
void LevelGrid<D>::insert(size_t item, const double* low, const double* high) {
    for (int32_t level = 0; level < kMaxGridLevels; ++level) {
        std::array<std::pair<int64_t, int64_t>, D> r;
        if (!range(low, high, level, r)) break;
        bool fits = true;
        for (int axis = 0; axis < D; ++axis)
            if (sat_sub(r[axis].second, r[axis].first) > kMaxAnchorCellSpan) fits = false;
        if (fits) {
            std::array<int64_t, D> key;
            for (int axis = 0; axis < D; ++axis) key[axis] = r[axis].first;
            cells[{level, key}].push_back(item);
            levels = std::max(levels, level + 1);
            return;
        }
    }
    unindexed.push_back(item);
}

template <int D>
QueryLimit LevelGrid<D>::query_bounded(const double* low, const double* high, size_t max_cells,
                                       PostingBudget& budget, std::set<size_t>& out) const {
    std::vector<std::pair<int32_t, std::array<std::pair<int64_t, int64_t>, D>>> ranges;
    for (int32_t level = 0; level < levels; ++level) {
        std::array<std::pair<int64_t, int64_t>, D> r;
        if (!range(low, high, level, r)) return QueryLimit::Cells;
        for (int axis = 0; axis < D; ++axis) r[axis].first = sat_sub(r[axis].first, kMaxAnchorCellSpan);
        size_t count = 1;
        for (int axis = 0; axis < D; ++axis) {
            int64_t span;
            if (__builtin_sub_overflow(r[axis].second, r[axis].first, &span)) return QueryLimit::Cells;
            if (span < 0) return QueryLimit::Cells;
            uint64_t s1;
            if (__builtin_add_overflow((uint64_t)span, (uint64_t)1, &s1)) return QueryLimit::Cells;
            count = sat_mul(count, (size_t)s1);
        }
        if (count > max_cells) return QueryLimit::Cells;
        ranges.push_back({level, r});
    }
    QueryLimit q = budget.take_into(unindexed, out);
    if (q != QueryLimit::None) return q;
    for (const auto& lr : ranges) {
        const auto& r = lr.second;
        std::array<int64_t, D> key;
        for (int axis = 0; axis < D; ++axis) key[axis] = r[axis].first;
        for (;;) {
            auto it = cells.find({lr.first, key});
            if (it != cells.end()) {
                q = budget.take_into(it->second, out);
                if (q != QueryLimit::None) return q;
            }
            int axis = 0;
            for (;;) {
                if (axis == D) break;
                if (key[axis] < r[axis].second) {
                    key[axis] += 1;
                    break;
                }
                key[axis] = r[axis].first;
                axis += 1;
            }
            if (axis == D) break;
        }
    }
    return QueryLimit::None;
}

template <int D>
bool LevelGrid<D>::query(const double* low, const double* high, size_t max_cells,
                         std::set<size_t>& out) const {
    PostingBudget budget(SIZE_MAX);
    return query_bounded(low, high, max_cells, budget, out) == QueryLimit::None;
}

template struct LevelGrid<2>;
template struct LevelGrid<3>;

// ---- Footprint (surface_merge.rs:1339-1592) --------------------------------------
std::optional<Footprint> Footprint::make(size_t patch, const RefCamera& camera,
                                         const std::vector<KeptTriangle>& kept) {
    Footprint f;
    f.patch = patch;
    f.camera = camera;
    for (const KeptTriangle& k : kept) {
        auto projected = camera.project_triangle(k.corners);
        if (projected && image_area(*projected) > kGeometricEpsilon * kGeometricEpsilon) {
            f.triangles.push_back(*projected);
            f.components.push_back(k.component);
            f.vertices.push_back(k.vertices);
            f.mesh_indices.push_back(k.mesh_index);
        } else {
            f.omitted.push_back({k.component, k.mesh_index});
        }
    }
    std::vector<double> edges;
    for (const ProjTri& t : f.triangles)
        for (int i = 0; i < 3; ++i) edges.push_back(norm2(t[(i + 1) % 3].image - t[i].image));
    std::stable_sort(edges.begin(), edges.end(), total_less);
    if (edges.empty()) return std::nullopt;
    const double cell = fmax_(edges[edges.size() / 2] * 2.0, kGeometricEpsilon);
    f.grid = LevelGrid<2>(cell);
    for (size_t i = 0; i < f.triangles.size(); ++i) {
        double low[2], high[2];
        image_aabb(f.triangles[i], low, high);
        f.grid.insert(i, low, high);
    }
    return f;
}

std::optional<ProjTri> Footprint::project_candidate(const std::array<Vec3, 3>& corners) const {
    auto c = camera.project_triangle(corners);
    if (c && image_area(*c) > kGeometricEpsilon * kGeometricEpsilon) return c;
    return std::nullopt;
}

QueryLimit Footprint::visit_overlaps(const ProjTri& candidate,
                                     const std::function<bool(size_t)>& include,
                                     const std::function<bool(Polygon&&, size_t)>& visit,
                                     PostingTally& tally) const {
    std::set<size_t> nearby;
    double low[2], high[2];
    image_aabb(candidate, low, high);
    PostingBudget budget = PostingBudget::per_query();
    QueryLimit found = grid.query_bounded(low, high, kMaxImageGridCells, budget, nearby);
    tally.record(budget, found);
    if (found != QueryLimit::None) return found;
    const Polygon polygon{candidate[0].image, candidate[1].image, candidate[2].image};
    for (size_t index : nearby) {
        if (!include(index)) continue;
        const ProjTri& kept = triangles[index];
        double winding = cross2(kept[1].image - kept[0].image, kept[2].image - kept[0].image);
        Polygon inside = polygon;
        for (int edge = 0; edge < 3; ++edge) {
            inside = split_polygon(inside, kept[edge].image, kept[(edge + 1) % 3].image,
                                   signum(winding))
                         .first;
            if (inside.empty()) break;
        }
        if (polygon_area(inside) > 0.0 && !visit(std::move(inside), index)) break;
    }
    return QueryLimit::None;
}

std::vector<double> Footprint::depth_ratios_tallied(
    const std::array<Vec3, 3>& corners, const std::function<bool(size_t)>& linked,
    const std::function<bool(const std::array<size_t, 3>&)>& anchored, size_t limit,
    PostingTally& tally) const {
    std::vector<double> ratios;
    auto candidate = project_candidate(corners);
    if (!candidate) return ratios;
    if (limit == 0) return ratios;
    (void)visit_overlaps(
        *candidate,
        [&](size_t index) { return linked(components[index]) && anchored(vertices[index]); },
        [&](Polygon&& polygon, size_t index) {
            const ProjTri& kept = triangles[index];
            V2 sum{0.0, 0.0};
            for (const V2& p : polygon) sum = sum + p;
            V2 centroid = sum / (double)polygon.size();
            auto owner = inverse_depth(kept, centroid);
            auto own = inverse_depth(*candidate, centroid);
            if (owner && own) {
                double ratio = *owner / *own;
                if (std::fabs(ratio - 1.0) <= kMaxRelativeScaleSample) ratios.push_back(ratio);
            }
            return ratios.size() < limit;
        },
        tally);
    return ratios;
}

Unjudged Footprint::ownership_tallied(const std::array<Vec3, 3>& corners, double scale,
                                      const std::function<bool(size_t)>& linked,
                                      PostingTally& tally, Ownership& owned,
                                      std::vector<size_t>& unjudged) const {
    auto candidate = project_candidate(corners);
    if (!candidate) return Unjudged::Unprojectable;
    std::vector<std::pair<Polygon, size_t>> overlaps;
    QueryLimit q = visit_overlaps(
        *candidate, [&](size_t index) { return linked(components[index]); },
        [&](Polygon&& polygon, size_t index) {
            overlaps.push_back({std::move(polygon), index});
            return true;
        },
        tally);
    if (q == QueryLimit::Cells) return Unjudged::TooManyCells;
    if (q == QueryLimit::Postings) return Unjudged::PostingBound;
    const double total = image_area(*candidate);
    auto plane = camera.plane(corners);
    double image = 0.0, surface = 0.0;
    for (const auto& ov : overlaps) {
        const ProjTri& kept = triangles[ov.second];
        bool agrees = true;
        for (const V2& point : ov.first) {
            auto c = inverse_depth(*candidate, point);
            auto k = inverse_depth(kept, point);
            if (!c || !k) {
                agrees = false;
                break;
            }
            double cd = 1.0 / *c, kd = scale / *k;
            if (!(std::fabs(cd - kd) <= kMaxRelativeDepthDisagreement * kd)) {
                agrees = false;
                break;
            }
        }
        if (agrees) {
            image += polygon_area(ov.first);
            surface += plane ? back_projected_area(ov.first, *plane) : 0.0;
        }
    }
    const double image_share = fmin_(image / total, 1.0);
    unjudged.clear();
    if (image_share < kMinImageOwnershipShare)
        for (const auto& om : omitted)
            if (linked(om.first)) unjudged.push_back(om.second);
    owned.image_share = image_share;
    owned.surface_area = surface;
    return Unjudged::None;
}

// ---- clip (surface_merge_clip.rs) ----------------------------------------------------
namespace {

using EdgeKey = std::pair<size_t, size_t>;
EdgeKey ekey(size_t a, size_t b) { return {std::min(a, b), std::max(a, b)}; }

struct DerivedPoint {
    Point3 point;
    std::optional<size_t> group;
    DerivedVertexSource source;
};

struct ClipState {
    size_t base;
    std::vector<DerivedPoint> derived;
    std::map<std::pair<EdgeKey, EdgeKey>, size_t> crossings;
    std::map<EdgeKey, std::vector<std::pair<double, size_t>>> carriers;
    std::unordered_map<size_t, std::vector<EdgeKey>> vertex_carriers;
    explicit ClipState(size_t b) : base(b) {}
    void record(EdgeKey edge, double parameter, size_t vertex) {
        if (edge.first == vertex || edge.second == vertex) return;
        auto& entries = carriers[edge];
        for (const auto& e : entries)
            if (e.second == vertex) return;
        entries.push_back({parameter, vertex});
        auto& list = vertex_carriers[vertex];
        if (std::find(list.begin(), list.end(), edge) == list.end()) list.push_back(edge);
    }
    bool has_records() const { return !carriers.empty(); }
};

struct ClipJob {
    size_t triangle, footprint;
    double scale;
};

struct ClipInputs {
    const std::vector<Point3>* points;
    const std::vector<MeshTriangle>* triangles;
    std::function<std::optional<std::array<Vec3, 3>>(size_t)> corners;
    const std::vector<Footprint>* footprints;
    const std::vector<int>* point_origins;
    std::function<std::optional<size_t>(size_t)> group_of;
    std::function<std::array<size_t, 3>(size_t)> source_corners;
    std::function<bool(size_t, size_t)> linked;
};

double distance_to_line(V2 a, V2 b, V2 p) {
    V2 direction = b - a;
    double length = norm2(direction);
    if (length <= 0.0) return norm2(p - a);
    return cross2(direction, p - a) / length;
}

double parameter(V2 a, V2 b, V2 p) {
    V2 direction = b - a;
    return dot2(p - a, direction) / (direction.x * direction.x + direction.y * direction.y);
}

double world_parameter(double t, const double depths[2]) {
    double numerator = t * depths[0];
    double denominator = numerator + (1.0 - t) * depths[1];
    if (std::fabs(denominator) <= kF64MinPositive) return t;
    return clamp_(numerator / denominator, 0.0, 1.0);
}

bool strictly_inside(const V2 tri[3], V2 point, double tolerance) {
    double orientation = signum(cross2(tri[1] - tri[0], tri[2] - tri[0]));
    for (int edge = 0; edge < 3; ++edge)
        if (!(orientation * distance_to_line(tri[edge], tri[(edge + 1) % 3], point) > tolerance))
            return false;
    return true;
}

enum class ClipFailure { None, NothingOwned, Bounded, Unverified, MixedOrigins };

struct NodeKind {
    bool vertex;
    size_t id;                  // vertex
    EdgeKey subject_ids;        // crossing: (p, q) as on the subject segment
    double subject_t;
    std::pair<size_t, size_t> owner_ids;  // (a, b) as on the owner segment
    double owner_t;
    size_t owner_triangle;
};
struct Node {
    V2 position;
    NodeKind kind;
};
struct Segment {
    size_t nodes[2];
    size_t ids[2];
    double depths[2];
    std::vector<std::pair<double, size_t>> inside;
};

int origin_flat(const std::vector<int>& origins, size_t i) {
    return i < origins.size() ? origins[i] : kOriginNone;
}

// clip_overlap (surface_merge_clip.rs:294-759)
ClipFailure clip_overlap(const ClipInputs& in, ClipState& state, const ClipJob& job,
                         PostingTally& tally, std::vector<std::array<size_t, 3>>& out) {
    const Footprint& footprint = (*in.footprints)[job.footprint];
    const MeshTriangle& triangle = (*in.triangles)[job.triangle];
    auto world = in.corners(job.triangle);
    if (!world) return ClipFailure::Unverified;
    auto candidate_opt = footprint.project_candidate(*world);
    if (!candidate_opt) return ClipFailure::Unverified;
    const ProjTri candidate = *candidate_opt;
    std::vector<std::pair<size_t, double>> owned;
    bool overflow = false;
    QueryLimit q = footprint.visit_overlaps(
        candidate, [&](size_t index) { return in.linked(job.triangle, footprint.components[index]); },
        [&](Polygon&& polygon, size_t index) {
            const ProjTri& kept = footprint.triangles[index];
            bool agrees = true;
            for (const V2& point : polygon) {
                auto own = inverse_depth(candidate, point);
                auto owner = inverse_depth(kept, point);
                if (!own || !owner) {
                    agrees = false;
                    break;
                }
                double o = 1.0 / *own, w = job.scale / *owner;
                if (!(std::fabs(o - w) <= kMaxClipDepthDisagreement * w)) {
                    agrees = false;
                    break;
                }
            }
            if (agrees) {
                owned.push_back({index, polygon_area(polygon)});
                if (owned.size() > kMaxClipOwnerTriangles) {
                    overflow = true;
                    return false;
                }
            }
            return true;
        },
        tally);
    if (q != QueryLimit::None) return ClipFailure::Bounded;
    if (overflow) return ClipFailure::Bounded;
    if (owned.empty()) return ClipFailure::NothingOwned;
    double owned_area = -0.0;
    for (const auto& o : owned) owned_area += o.second;

    const size_t subject_ids[3] = {triangle.a, triangle.b, triangle.c};
    const double signed_ = cross2(candidate[1].image - candidate[0].image,
                                  candidate[2].image - candidate[0].image);
    const bool flipped = signed_ < 0.0;
    const int order[3] = {0, flipped ? 2 : 1, flipped ? 1 : 2};
    struct SubjectCorner {
        V2 position;
        double depth;
        size_t id;
    } subject[3];
    for (int i = 0; i < 3; ++i)
        subject[i] = {candidate[order[i]].image, candidate[order[i]].depth, subject_ids[order[i]]};
    double extent = 0.0;
    for (int edge = 0; edge < 3; ++edge)
        extent = fmax_(extent, norm2(subject[(edge + 1) % 3].position - subject[edge].position));
    const double tolerance = extent * kRelativeTolerance;
    const double subject_area = std::fabs(signed_) * 0.5;

    std::vector<Node> nodes;
    std::unordered_map<size_t, size_t> by_id;
    for (int i = 0; i < 3; ++i) {
        by_id[subject[i].id] = nodes.size();
        NodeKind k{};
        k.vertex = true;
        k.id = subject[i].id;
        nodes.push_back({subject[i].position, k});
    }
    std::unordered_map<size_t, double> owner_depth;
    for (const auto& o : owned) {
        for (int corner = 0; corner < 3; ++corner) {
            size_t id = footprint.vertices[o.first][corner];
            V2 position = footprint.triangles[o.first][corner].image;
            owner_depth[id] = footprint.triangles[o.first][corner].depth;
            if (by_id.count(id)) continue;
            size_t node = SIZE_MAX;
            for (int s = 0; s < 3; ++s)
                if (norm2(subject[s].position - position) <= tolerance) {
                    node = (size_t)s;
                    break;
                }
            if (node == SIZE_MAX) {
                NodeKind k{};
                k.vertex = true;
                k.id = id;
                nodes.push_back({position, k});
                node = nodes.size() - 1;
            }
            by_id[id] = node;
        }
    }
    std::vector<Segment> segments;
    for (int edge = 0; edge < 3; ++edge) {
        int next = (edge + 1) % 3;
        Segment s;
        s.nodes[0] = (size_t)edge;
        s.nodes[1] = (size_t)next;
        s.ids[0] = subject[edge].id;
        s.ids[1] = subject[next].id;
        s.depths[0] = subject[edge].depth;
        s.depths[1] = subject[next].depth;
        segments.push_back(std::move(s));
    }
    struct OwnerEdge {
        size_t a, b, index;
    };
    std::map<EdgeKey, OwnerEdge> owner_edges;
    for (const auto& o : owned) {
        const auto& ids = footprint.vertices[o.first];
        for (int corner = 0; corner < 3; ++corner) {
            size_t a = ids[corner], b = ids[(corner + 1) % 3];
            owner_edges.emplace(ekey(a, b), OwnerEdge{a, b, o.first});
        }
    }
    const size_t owner_first = segments.size();
    std::vector<size_t> owner_triangle_of_segment;
    for (const auto& kv : owner_edges) {
        size_t na = by_id.at(kv.second.a), nb = by_id.at(kv.second.b);
        if (na == nb) continue;
        Segment s;
        s.nodes[0] = na;
        s.nodes[1] = nb;
        s.ids[0] = kv.second.a;
        s.ids[1] = kv.second.b;
        s.depths[0] = owner_depth.at(kv.second.a);
        s.depths[1] = owner_depth.at(kv.second.b);
        segments.push_back(std::move(s));
        owner_triangle_of_segment.push_back(kv.second.index);
    }
    std::set<size_t> owner_nodes;
    for (const auto& kv : by_id)
        if (kv.second > 2) owner_nodes.insert(kv.second);
    for (int edge = 0; edge < 3; ++edge) {
        V2 a = nodes[segments[edge].nodes[0]].position, b = nodes[segments[edge].nodes[1]].position;
        double length = norm2(b - a);
        for (size_t node : owner_nodes) {
            V2 p = nodes[node].position;
            double t = parameter(a, b, p);
            if (std::fabs(distance_to_line(a, b, p)) <= tolerance && t * length > tolerance &&
                (1.0 - t) * length > tolerance)
                segments[edge].inside.push_back({t, node});
        }
    }
    for (size_t sg = owner_first; sg < segments.size(); ++sg) {
        size_t from = segments[sg].nodes[0], to = segments[sg].nodes[1];
        V2 a = nodes[from].position, b = nodes[to].position;
        double length = norm2(b - a);
        for (size_t node = 0; node < 3; ++node) {
            if (node == from || node == to) continue;
            V2 p = nodes[node].position;
            double t = parameter(a, b, p);
            if (std::fabs(distance_to_line(a, b, p)) <= tolerance && t * length > tolerance &&
                (1.0 - t) * length > tolerance)
                segments[sg].inside.push_back({t, node});
        }
    }
    for (int edge = 0; edge < 3; ++edge) {
        for (size_t sg = owner_first; sg < segments.size(); ++sg) {
            size_t p = segments[edge].nodes[0], qn = segments[edge].nodes[1];
            size_t a = segments[sg].nodes[0], b = segments[sg].nodes[1];
            if (p == a || p == b || qn == a || qn == b) continue;
            V2 pp = nodes[p].position, qp = nodes[qn].position, ap = nodes[a].position,
               bp = nodes[b].position;
            double da = distance_to_line(pp, qp, ap), db = distance_to_line(pp, qp, bp);
            double dp = distance_to_line(ap, bp, pp), dq = distance_to_line(ap, bp, qp);
            if (std::fabs(da) <= tolerance || std::fabs(db) <= tolerance ||
                std::fabs(dp) <= tolerance || std::fabs(dq) <= tolerance)
                continue;
            if (signum(da) == signum(db) || signum(dp) == signum(dq)) continue;
            double subject_t = dp / (dp - dq);
            double owner_t = da / (da - db);
            if (nodes.size() >= kMaxClipNodes) return ClipFailure::Bounded;
            size_t node = nodes.size();
            NodeKind k{};
            k.vertex = false;
            k.subject_ids = {segments[edge].ids[0], segments[edge].ids[1]};
            k.subject_t = subject_t;
            k.owner_ids = {segments[sg].ids[0], segments[sg].ids[1]};
            k.owner_t = owner_t;
            k.owner_triangle = owner_triangle_of_segment[sg - owner_first];
            nodes.push_back({pp + (qp - pp) * subject_t, k});
            segments[edge].inside.push_back({subject_t, node});
            segments[sg].inside.push_back({owner_t, node});
        }
    }
    if (nodes.size() > kMaxClipNodes) return ClipFailure::Bounded;

    const V2 subject_polygon[3] = {subject[0].position, subject[1].position, subject[2].position};
    std::set<std::pair<size_t, size_t>> edges;
    for (size_t index = 0; index < segments.size(); ++index) {
        Segment& segment = segments[index];
        std::stable_sort(segment.inside.begin(), segment.inside.end(),
                         [](const auto& x, const auto& y) { return total_less(x.first, y.first); });
        std::vector<size_t> chain{segment.nodes[0]};
        for (const auto& in_ : segment.inside) chain.push_back(in_.second);
        chain.push_back(segment.nodes[1]);
        chain.erase(std::unique(chain.begin(), chain.end()), chain.end());
        for (size_t i = 0; i + 1 < chain.size(); ++i) {
            size_t from = chain[i], to = chain[i + 1];
            if (from == to) continue;
            if (index >= owner_first) {
                V2 middle = (nodes[from].position + nodes[to].position) * 0.5;
                if (!strictly_inside(subject_polygon, middle, tolerance)) continue;
            }
            edges.insert({std::min(from, to), std::max(from, to)});
        }
    }
    std::vector<std::vector<size_t>> neighbours(nodes.size());
    for (const auto& e : edges) {
        neighbours[e.first].push_back(e.second);
        neighbours[e.second].push_back(e.first);
    }
    std::vector<size_t> parent(nodes.size());
    for (size_t i = 0; i < nodes.size(); ++i) parent[i] = i;
    for (const auto& e : edges) {
        size_t a = find(parent, e.first), b = find(parent, e.second);
        parent[a] = b;
    }
    std::vector<size_t> used;
    for (size_t node = 0; node < nodes.size(); ++node)
        if (!neighbours[node].empty()) used.push_back(node);
    // used[0] exists: the subject's three edges are always in the graph
    const size_t root = find(parent, used[0]);
    for (size_t node : used)
        if (find(parent, node) != root || neighbours[node].size() < 2) return ClipFailure::Unverified;
    for (size_t node = 0; node < nodes.size(); ++node) {
        V2 origin = nodes[node].position;
        std::stable_sort(neighbours[node].begin(), neighbours[node].end(), [&](size_t a, size_t b) {
            V2 da = nodes[a].position - origin, db = nodes[b].position - origin;
            return total_less(std::atan2(da.y, da.x), std::atan2(db.y, db.x));
        });
    }
    std::set<std::pair<size_t, size_t>> visited;
    std::vector<std::vector<size_t>> faces;
    size_t outer = 0;
    const size_t limit = 2 * edges.size() + 2;
    for (const auto& e : edges) {
        const std::pair<size_t, size_t> starts[2] = {{e.first, e.second}, {e.second, e.first}};
        for (const auto& st : starts) {
            if (visited.count(st)) continue;
            std::vector<size_t> face;
            size_t from = st.first, to = st.second;
            for (;;) {
                if (!visited.insert({from, to}).second || face.size() > limit)
                    return ClipFailure::Unverified;
                face.push_back(from);
                const auto& around = neighbours[to];
                size_t back = SIZE_MAX;
                for (size_t i = 0; i < around.size(); ++i)
                    if (around[i] == from) {
                        back = i;
                        break;
                    }
                if (back == SIZE_MAX) return ClipFailure::Unverified;
                size_t following = around[(back + around.size() - 1) % around.size()];
                from = to;
                to = following;
                if (from == st.first && to == st.second) break;
            }
            Polygon polygon;
            for (size_t node : face) polygon.push_back(nodes[node].position);
            if (signed_area(polygon) > 0.0)
                faces.push_back(std::move(face));
            else
                outer += 1;
        }
    }
    if (outer != 1) return ClipFailure::Unverified;
    std::vector<std::array<V2, 3>> owner_polygons;
    for (const auto& o : owned)
        owner_polygons.push_back({footprint.triangles[o.first][0].image,
                                  footprint.triangles[o.first][1].image,
                                  footprint.triangles[o.first][2].image});
    std::vector<std::array<size_t, 3>> kept;
    double kept_area = 0.0, removed_area = 0.0;
    for (const auto& face : faces) {
        Polygon polygon;
        for (size_t node : face) polygon.push_back(nodes[node].position);
        auto ears = ear_clip(polygon, tolerance);
        if (!ears) return ClipFailure::Unverified;
        V2 largest{0.0, 0.0};
        double best = -INFINITY;
        for (const auto& ear : *ears) {
            V2 a = polygon[ear[0]], b = polygon[ear[1]], c = polygon[ear[2]];
            V2 centroid = ((a + b) + c) / 3.0;
            double area = cross2(b - a, c - a);
            if (area > best) {
                best = area;
                largest = centroid;
            }
        }
        double area = signed_area(polygon);
        bool removed = false;
        for (const auto& owner : owner_polygons)
            if (strictly_inside(owner.data(), largest, 0.0)) {
                removed = true;
                break;
            }
        if (removed) {
            removed_area += area;
            continue;
        }
        kept_area += area;
        for (const auto& ear : *ears) kept.push_back({face[ear[0]], face[ear[1]], face[ear[2]]});
    }
    const double balance = kAreaTolerance * subject_area;
    if (std::fabs((kept_area + removed_area) - subject_area) > balance ||
        std::fabs(removed_area - owned_area) > balance)
        return ClipFailure::Unverified;

    std::set<size_t> used_nodes;
    for (const auto& k : kept)
        for (size_t n : k) used_nodes.insert(n);
    std::unordered_map<size_t, size_t> ids;
    struct Fresh {
        size_t id;
        DerivedPoint point;
        std::pair<EdgeKey, EdgeKey> crossing;
    };
    std::vector<Fresh> fresh;
    size_t next_index = state.base + state.derived.size();
    for (size_t node : used_nodes) {
        const NodeKind& k = nodes[node].kind;
        size_t id;
        if (k.vertex) {
            id = k.id;
        } else {
            const size_t a = k.owner_ids.first, b = k.owner_ids.second;
            auto crossing = std::make_pair(ekey(k.subject_ids.first, k.subject_ids.second), ekey(a, b));
            auto it = state.crossings.find(crossing);
            if (it != state.crossings.end()) {
                id = it->second;
            } else {
                int origin = origin_flat(*in.point_origins, a);
                if (origin != origin_flat(*in.point_origins, b)) return ClipFailure::MixedOrigins;
                const double depths[2] = {owner_depth.at(a), owner_depth.at(b)};
                const double s = world_parameter(k.owner_t, depths);
                const size_t mesh_index = footprint.mesh_indices[k.owner_triangle];
                const auto& current = footprint.vertices[k.owner_triangle];
                std::array<double, 3> barycentric;
                for (int c = 0; c < 3; ++c)
                    barycentric[c] = current[c] == a ? 1.0 - s : current[c] == b ? s : 0.0;
                const Point3 pa = (*in.points)[a], pb = (*in.points)[b];
                auto lerp = [&](float x, float y) {
                    return (float)((double)x * (1.0 - s) + (double)y * s);
                };
                auto lerp8 = [&](uint8_t x, uint8_t y) {
                    double v = clamp_(std::round((double)x * (1.0 - s) + (double)y * s), 0.0, 255.0);
                    return std::isnan(v) ? (uint8_t)0 : (uint8_t)v;
                };
                Point3 point{lerp(pa.x, pb.x), lerp(pa.y, pb.y), lerp(pa.z, pb.z),
                             lerp(pa.confidence, pb.confidence), lerp8(pa.r, pb.r),
                             lerp8(pa.g, pb.g), lerp8(pa.b, pb.b)};
                id = next_index++;
                DerivedPoint dp{point, in.group_of(a),
                                DerivedVertexSource{id, mesh_index, in.source_corners(mesh_index),
                                                    barycentric}};
                fresh.push_back({id, dp, crossing});
            }
        }
        ids[node] = id;
    }
    for (auto& f : fresh) {
        state.crossings[f.crossing] = f.id;
        state.derived.push_back(f.point);
    }
    for (const Segment& segment : segments) {
        EdgeKey edge = ekey(segment.ids[0], segment.ids[1]);
        bool forward = edge.first == segment.ids[0];
        for (const auto& in_ : segment.inside) {
            auto it = ids.find(in_.second);
            if (it == ids.end()) continue;
            double s = world_parameter(in_.first, segment.depths);
            state.record(edge, forward ? s : 1.0 - s, it->second);
        }
    }
    out.clear();
    for (const auto& k : kept) {
        std::array<size_t, 3> c{ids.at(k[0]), ids.at(k[1]), ids.at(k[2])};
        if (flipped) out.push_back({c[0], c[2], c[1]});
        else out.push_back(c);
    }
    return ClipFailure::None;
}

// conform_edges (surface_merge_clip.rs:775-879); false when canceled.
bool conform_edges(const ClipState& state, std::vector<MeshTriangle>& triangles,
                   const std::function<Vec3(size_t)>& position, Control& control,
                   std::vector<size_t>& split, size_t& failures) {
    auto parameter_on = [&](const EdgeKey& edge, size_t vertex) -> std::optional<double> {
        if (vertex == edge.first) return 0.0;
        if (vertex == edge.second) return 1.0;
        auto it = state.carriers.find(edge);
        if (it == state.carriers.end()) return std::nullopt;
        for (const auto& e : it->second)
            if (e.second == vertex) return e.first;
        return std::nullopt;
    };
    split.clear();
    failures = 0;
    std::vector<MeshTriangle> appended;
    const V2 frame[3] = {V2{0.0, 0.0}, V2{1.0, 0.0}, V2{0.0, 1.0}};
    const size_t n = triangles.size();
    for (size_t slot = 0; slot < n; ++slot) {
        if (slot % 256 == 0 && control.is_canceled()) return false;
        const MeshTriangle triangle = triangles[slot];
        const size_t corners[3] = {triangle.a, triangle.b, triangle.c};
        std::vector<std::pair<size_t, V2>> boundary;
        bool inserted = false;
        for (int edge = 0; edge < 3; ++edge) {
            size_t u = corners[edge], v = corners[(edge + 1) % 3];
            boundary.push_back({u, frame[edge]});
            std::vector<EdgeKey> carriers{ekey(u, v)};
            for (size_t endpoint : {u, v}) {
                auto it = state.vertex_carriers.find(endpoint);
                if (it != state.vertex_carriers.end())
                    carriers.insert(carriers.end(), it->second.begin(), it->second.end());
            }
            std::optional<EdgeKey> carrier;
            for (const auto& c : carriers)
                if (state.carriers.count(c) && parameter_on(c, u) && parameter_on(c, v)) {
                    carrier = c;
                    break;
                }
            if (!carrier) continue;
            double tu = *parameter_on(*carrier, u), tv = *parameter_on(*carrier, v);
            if (std::fabs(tv - tu) <= kF64Epsilon) continue;
            std::vector<std::pair<double, size_t>> between;
            for (const auto& e : state.carriers.at(*carrier)) {
                if (e.second == u || e.second == v) continue;
                double relative = (e.first - tu) / (tv - tu);
                if (relative > 1.0e-9 && relative < 1.0 - 1.0e-9) between.push_back({relative, e.second});
            }
            std::stable_sort(between.begin(), between.end(),
                             [](const auto& x, const auto& y) { return total_less(x.first, y.first); });
            between.erase(std::unique(between.begin(), between.end(),
                                      [](const auto& x, const auto& y) { return x.second == y.second; }),
                          between.end());
            V2 start = frame[edge], end = frame[(edge + 1) % 3];
            for (const auto& b : between) {
                boundary.push_back({b.second, start + (end - start) * b.first});
                inserted = true;
            }
        }
        if (!inserted) continue;
        Polygon polygon;
        for (const auto& b : boundary) polygon.push_back(b.second);
        auto ears = ear_clip(polygon, 1.0e-12);
        if (!ears) {
            failures += 1;
            continue;
        }
        bool degenerate = false;
        for (const auto& ear : *ears) {
            Vec3 a = position(boundary[ear[0]].first), b = position(boundary[ear[1]].first),
                 c = position(boundary[ear[2]].first);
            if (norm(cross(sub(b, a), sub(c, a))) <= kF64Epsilon) {
                degenerate = true;
                break;
            }
        }
        if (degenerate) {
            failures += 1;
            continue;
        }
        bool first = true;
        for (const auto& ear : *ears) {
            MeshTriangle t{boundary[ear[0]].first, boundary[ear[1]].first, boundary[ear[2]].first,
                           triangle.confidence};
            if (first) {
                triangles[slot] = t;
                first = false;
            } else {
                appended.push_back(t);
            }
        }
        split.push_back(slot);
    }
    triangles.insert(triangles.end(), appended.begin(), appended.end());
    return true;
}

// ---- stitch (surface_merge_stitch.rs) ------------------------------------------------
struct ImageRemoval {
    size_t triangle, footprint;
    double scale;
};

struct HalfEdge {
    uint32_t low, high, from, triangle;
    bool operator<(const HalfEdge& o) const {
        if (low != o.low) return low < o.low;
        if (high != o.high) return high < o.high;
        if (from != o.from) return from < o.from;
        return triangle < o.triangle;
    }
};
struct EdgeUse {
    uint32_t count, from;
};
struct Seam {
    uint32_t vertices[kMaxSeamVertices];
    uint8_t len;
};

struct Edges {
    std::vector<HalfEdge> retained;
    std::unordered_map<uint64_t, EdgeUse> stitched;
    static std::pair<uint32_t, uint32_t> key(uint32_t a, uint32_t b) {
        return {std::min(a, b), std::max(a, b)};
    }
    std::pair<size_t, size_t> retained_range(uint32_t a, uint32_t b) const {
        auto k = key(a, b);
        auto lo = std::partition_point(retained.begin(), retained.end(), [&](const HalfEdge& e) {
            return std::make_pair(e.low, e.high) < k;
        });
        auto hi = std::partition_point(retained.begin(), retained.end(), [&](const HalfEdge& e) {
            return std::make_pair(e.low, e.high) <= k;
        });
        return {(size_t)(lo - retained.begin()), (size_t)(hi - retained.begin())};
    }
    std::optional<EdgeUse> usage(uint32_t a, uint32_t b) const {
        auto k = key(a, b);
        auto it = stitched.find(((uint64_t)k.first << 32) | k.second);
        if (it != stitched.end()) return it->second;
        auto r = retained_range(a, b);
        if (r.first == r.second) return std::nullopt;
        return EdgeUse{(uint32_t)(r.second - r.first), retained[r.first].from};
    }
    void add(uint32_t from, uint32_t to) {
        auto u = usage(from, to);
        EdgeUse e = u ? EdgeUse{u->count + 1, u->from} : EdgeUse{1, from};
        auto k = key(from, to);
        stitched[((uint64_t)k.first << 32) | k.second] = e;
    }
};

double signed_image_area(const ProjTri& t) {
    return cross2(t[1].image - t[0].image, t[2].image - t[0].image) * 0.5;
}

bool contains(const ProjTri& t, V2 point) {
    V2 a = t[0].image, b = t[1].image, c = t[2].image;
    double determinant = cross2(b - a, c - a);
    if (std::fabs(determinant) <= kF64Epsilon) return false;
    double wb = cross2(point - a, c - a) / determinant;
    double wc = cross2(b - a, point - a) / determinant;
    return ((1.0 - wb) - wc) >= -kInsideTolerance && wb >= -kInsideTolerance &&
           wc >= -kInsideTolerance;
}

Polygon polygon_of(const ProjTri& t) { return {t[0].image, t[1].image, t[2].image}; }

double intersection_area(const Polygon& polygon, const ProjTri& triangle) {
    double orientation = signum(signed_image_area(triangle));
    Polygon inside = polygon;
    for (int edge = 0; edge < 3; ++edge) {
        inside = split_polygon(inside, triangle[edge].image, triangle[(edge + 1) % 3].image,
                               orientation)
                     .first;
        if (inside.empty()) return 0.0;
    }
    return polygon_area(inside);
}

std::optional<double> unobserved_area(const ProjTri& stitch, const std::vector<ProjTri>& seams) {
    const double area_epsilon = std::fabs(signed_image_area(stitch)) * 1.0e-12;
    std::vector<Polygon> remaining{polygon_of(stitch)};
    for (const ProjTri& seam : seams) {
        double orientation = signum(signed_image_area(seam));
        std::vector<Polygon> next;
        for (Polygon& polygon : remaining) {
            Polygon inside = std::move(polygon);
            std::vector<Polygon> outside;
            for (int edge = 0; edge < 3; ++edge) {
                auto sp = split_polygon(inside, seam[edge].image, seam[(edge + 1) % 3].image,
                                        orientation);
                if (polygon_area(sp.second) > area_epsilon) outside.push_back(sp.second);
                inside = std::move(sp.first);
                if (inside.empty()) break;
            }
            if (polygon_area(inside) > area_epsilon) {
                bool agrees = true;
                for (const V2& point : inside) {
                    auto s = inverse_depth(stitch, point);
                    auto m = inverse_depth(seam, point);
                    if (!s || !m) {
                        agrees = false;
                        break;
                    }
                    double sd = 1.0 / *s, md = 1.0 / *m;
                    if (!(std::fabs(sd - md) <= kMaxRelativeDepthDisagreement * md)) {
                        agrees = false;
                        break;
                    }
                }
                if (!agrees) outside.push_back(std::move(inside));
            }
            for (auto& o : outside) next.push_back(std::move(o));
            if (next.size() > kMaxUncoveredPieces) return std::nullopt;
        }
        remaining = std::move(next);
        if (remaining.empty()) break;
    }
    double total = -0.0;
    for (const auto& p : remaining) total += polygon_area(p);
    return total;
}

struct SeamInputs {
    size_t vertices;
    const std::vector<MeshTriangle>* triangles;
    const std::vector<char>* keep;
    const std::vector<std::optional<TriangleGeometry>>* geometry;
    const std::vector<int64_t>* membership;
    const std::vector<std::optional<size_t>>* patch_of;
    const std::vector<Footprint>* footprints;
    const std::vector<ImageRemoval>* removals;
    const LevelGrid<3>* kept_grid;
    const std::vector<size_t>* all_kept;
    double tolerance, cell;
};

void seams_of(const std::vector<std::pair<uint32_t, uint32_t>>& by_vertex, size_t vertex,
              std::vector<size_t>& out) {
    uint32_t v = (uint32_t)vertex;
    auto it = std::partition_point(by_vertex.begin(), by_vertex.end(),
                                   [&](const auto& e) { return e.first < v; });
    size_t taken = 0;
    for (; it != by_vertex.end() && it->first == v && taken < kMaxSeamsPerVertex; ++it, ++taken)
        out.push_back(it->second);
}

std::vector<MeshTriangle> stitch_trimmed_seams(const SeamInputs& in,
                                               const std::function<Vec3(size_t)>& position,
                                               const std::function<bool(size_t, size_t)>& linked,
                                               PostingTally& tally) {
    const auto& triangles = *in.triangles;
    const auto& removals = *in.removals;
    const auto& patch_of = *in.patch_of;
    const auto& footprints = *in.footprints;
    const auto& geometry = *in.geometry;
    std::vector<MeshTriangle> output;
    if (removals.empty() || in.vertices > UINT32_MAX || triangles.size() > UINT32_MAX ||
        removals.size() > UINT32_MAX)
        return output;
    auto group_of = [&](size_t v) { return group_of_vec(*in.membership, v); };

    std::vector<HalfEdge> retained;
    retained.reserve(3 * triangles.size());
    for (size_t index = 0; index < triangles.size(); ++index) {
        if (!(*in.keep)[index]) continue;
        const uint32_t a = (uint32_t)triangles[index].a, b = (uint32_t)triangles[index].b,
                       c = (uint32_t)triangles[index].c;
        const std::pair<uint32_t, uint32_t> es[3] = {{a, b}, {b, c}, {c, a}};
        for (const auto& e : es)
            if (e.first != e.second) {
                auto k = Edges::key(e.first, e.second);
                retained.push_back({k.first, k.second, e.first, (uint32_t)index});
            }
    }
    std::sort(retained.begin(), retained.end());
    Edges edges;
    edges.retained = std::move(retained);
    std::vector<char> on_boundary(in.vertices, 0);
    std::vector<uint32_t> boundary;
    size_t start = 0;
    while (start < edges.retained.size()) {
        const HalfEdge e = edges.retained[start];
        size_t end = start;
        while (end < edges.retained.size() && edges.retained[end].low == e.low &&
               edges.retained[end].high == e.high)
            ++end;
        if (end - start == 1) {
            on_boundary[e.low] = 1;
            on_boundary[e.high] = 1;
            boundary.push_back((uint32_t)start);
        }
        start = end;
    }

    std::vector<std::optional<Seam>> seams;
    seams.reserve(removals.size());
    std::vector<std::pair<uint32_t, uint32_t>> seams_by_vertex;
    for (size_t slot = 0; slot < removals.size(); ++slot) {
        const ImageRemoval& removal = removals[slot];
        auto seam = [&]() -> std::optional<Seam> {
            if (removal.footprint >= footprints.size()) return std::nullopt;
            const Footprint& footprint = footprints[removal.footprint];
            if (!geometry[removal.triangle]) return std::nullopt;
            auto projected = footprint.project_candidate(geometry[removal.triangle]->corners);
            if (!projected) return std::nullopt;
            const auto lower = patch_of[removal.triangle];
            const MeshTriangle& removed = triangles[removal.triangle];
            std::set<size_t> stitchable;
            for (size_t v : {removed.a, removed.b, removed.c})
                if (on_boundary[v] && group_of(v)) stitchable.insert(v);
            std::set<size_t> nearby;
            double low[2], high[2];
            image_aabb(*projected, low, high);
            PostingBudget budget = PostingBudget::per_query();
            QueryLimit found =
                footprint.grid.query_bounded(low, high, kMaxImageGridCells, budget, nearby);
            tally.record(budget, found);
            if (found != QueryLimit::None) return std::nullopt;
            for (size_t kept : nearby) {
                if (!linked(removal.triangle, footprint.components[kept])) continue;
                for (size_t vertex : footprint.vertices[kept]) {
                    if (!on_boundary[vertex] || !group_of(vertex) || group_of(vertex) == lower ||
                        stitchable.count(vertex))
                        continue;
                    auto p = footprint.camera.project(position(vertex));
                    if (p && contains(*projected, p->image)) stitchable.insert(vertex);
                }
            }
            if (stitchable.size() > kMaxSeamVertices) return std::nullopt;
            Seam s{};
            s.len = (uint8_t)stitchable.size();
            size_t i = 0;
            for (size_t v : stitchable) s.vertices[i++] = (uint32_t)v;
            return s;
        }();
        if (seam)
            for (size_t i = 0; i < seam->len; ++i)
                seams_by_vertex.push_back({seam->vertices[i], (uint32_t)slot});
        seams.push_back(seam);
    }
    std::sort(seams_by_vertex.begin(), seams_by_vertex.end());

    auto project_seam = [&](const ImageRemoval& r) -> std::optional<ProjTri> {
        if (r.footprint >= footprints.size()) return std::nullopt;
        if (!geometry[r.triangle]) return std::nullopt;
        return footprints[r.footprint].project_candidate(geometry[r.triangle]->corners);
    };
    auto length = [&](size_t a, size_t b) { return norm(sub(position(a), position(b))); };
    LevelGrid<3> stitch_grid(in.cell);

    // StitchContext::check (surface_merge_stitch.rs:567-660)
    auto check = [&](const std::array<size_t, 3>& corners, size_t removal_slot, size_t adjacent,
                     double low[3], double high[3]) -> bool {
        const size_t a = corners[0], b = corners[1], c = corners[2];
        const std::pair<size_t, size_t> es[3] = {{a, b}, {b, c}, {c, a}};
        for (const auto& e : es) {
            auto u = edges.usage((uint32_t)e.first, (uint32_t)e.second);
            if (u && !(u->count < 2 && u->from != (uint32_t)e.first)) return false;
        }
        auto surface = TriangleGeometry::make({position(a), position(b), position(c)});
        if (!surface) return false;
        const ImageRemoval& removal = removals[removal_slot];
        const Footprint& footprint = footprints[removal.footprint];
        const auto lower = patch_of[removal.triangle];
        auto projected_opt = footprint.camera.project_triangle(surface->corners);
        if (!projected_opt) return false;
        ProjTri projected = *projected_opt;
        double area = signed_image_area(projected);
        if (!geometry[adjacent]) return false;
        auto adj = footprint.camera.project_triangle(geometry[adjacent]->corners);
        if (!adj) return false;
        const double adjacent_area = signed_image_area(*adj);
        if (std::fabs(area) <= kF64Epsilon * kF64Epsilon || signum(adjacent_area) != signum(area))
            return false;
        area = std::fabs(area);
        for (int i = 0; i < 3; ++i)
            if (group_of(corners[i]) != lower) projected[i].depth *= removal.scale;
        std::set<size_t> cover_slots;
        for (size_t v : corners) {
            std::vector<size_t> s;
            seams_of(seams_by_vertex, v, s);
            for (size_t slot : s)
                if (seams[slot] && removals[slot].footprint == removal.footprint &&
                    patch_of[removals[slot].triangle] == lower)
                    cover_slots.insert(slot);
        }
        std::vector<ProjTri> cover;
        for (size_t slot : cover_slots) {
            auto p = project_seam(removals[slot]);
            if (p) cover.push_back(*p);
        }
        auto unobserved = unobserved_area(projected, cover);
        if (!unobserved) return false;
        if (*unobserved > kMaxUnobservedStitchShare * area) return false;
        const Polygon polygon = polygon_of(projected);
        surface->aabb(in.tolerance, low, high);
        std::set<size_t> nearby;
        PostingBudget budget = PostingBudget::per_query();
        QueryLimit found = in.kept_grid->query_bounded(low, high, kMaxGridCells, budget, nearby);
        if (found == QueryLimit::Cells) found = budget.take_into(*in.all_kept, nearby);
        tally.record(budget, found);
        if (found != QueryLimit::None) return false;
        double overlap = 0.0;
        for (size_t other : nearby) {
            if (!geometry[other]) continue;
            auto p = footprint.camera.project_triangle(geometry[other]->corners);
            if (!p) return false;
            overlap += intersection_area(polygon, *p);
        }
        std::set<size_t> near2;
        PostingBudget budget2 = PostingBudget::per_query();
        QueryLimit found2 = stitch_grid.query_bounded(low, high, kMaxGridCells, budget2, near2);
        tally.record(budget2, found2);
        if (found2 != QueryLimit::None) return false;
        for (size_t other : near2) {
            const MeshTriangle& o = output[other];
            auto p = footprint.camera.project_triangle({position(o.a), position(o.b), position(o.c)});
            if (!p) return false;
            overlap += intersection_area(polygon, *p);
        }
        return overlap <= kMaxStitchOverlapShare * area;
    };

    for (uint32_t edge_index : boundary) {
        if (output.size() >= removals.size()) break;
        const HalfEdge edge = edges.retained[edge_index];
        const size_t adjacent = edge.triangle;
        const size_t from = edge.from;
        const size_t to = edge.from == edge.low ? edge.high : edge.low;
        if (group_of(from) != group_of(to)) continue;
        std::set<size_t> slots;
        {
            std::vector<size_t> s;
            seams_of(seams_by_vertex, from, s);
            seams_of(seams_by_vertex, to, s);
            slots.insert(s.begin(), s.end());
        }
        std::set<size_t> seen;
        std::vector<std::pair<double, std::array<size_t, 4>>> candidates;
        for (size_t slot : slots) {
            if (!seams[slot]) continue;
            const auto lower = patch_of[removals[slot].triangle];
            const bool edge_is_lower = group_of(from) == lower;
            for (size_t i = 0; i < seams[slot]->len; ++i) {
                const size_t vertex = seams[slot]->vertices[i];
                if (vertex == from || vertex == to || (group_of(vertex) == lower) == edge_is_lower)
                    continue;
                if (!seen.insert(vertex).second) continue;
                double perimeter = (length(from, to) + length(to, vertex)) + length(vertex, from);
                candidates.push_back({perimeter, {to, from, vertex, slot}});
            }
        }
        std::stable_sort(candidates.begin(), candidates.end(), [](const auto& l, const auto& r) {
            if (total_less(l.first, r.first)) return true;
            if (total_less(r.first, l.first)) return false;
            return l.second < r.second;
        });
        for (const auto& cand : candidates) {
            const size_t a = cand.second[0], b = cand.second[1], c = cand.second[2],
                         slot = cand.second[3];
            double low[3], high[3];
            if (!check({a, b, c}, slot, adjacent, low, high)) continue;
            const std::pair<size_t, size_t> es[3] = {{a, b}, {b, c}, {c, a}};
            for (const auto& e : es) edges.add((uint32_t)e.first, (uint32_t)e.second);
            stitch_grid.insert(output.size(), low, high);
            output.push_back({a, b, c,
                              std::fmin(triangles[adjacent].confidence,
                                        triangles[removals[slot].triangle].confidence)});
            break;
        }
    }
    return output;
}

// ---- merge_impl (surface_merge.rs:355-1078) -----------------------------------------
// Returns false when canceled (the reference's Default::default() return),
// with `stats` default and `derived` empty.
bool merge_impl(const MergeInputs& in, std::vector<MeshTriangle>& triangles, Control& control,
                bool clip_overlaps, MergeStats& stats, std::vector<DerivedPoint>& derived_out) {
    const auto& points = *in.points;
    const auto& membership = *in.membership;
    const auto& pairs = *in.pairs;
    const auto& cameras = *in.cameras;
    const auto& origins = *in.origins;
    stats = MergeStats();
    derived_out.clear();
    auto group_of = [&](size_t v) { return group_of_vec(membership, v); };
    if (points.size() != membership.size()) return true;
    for (const auto& t : triangles)
        if (t.a >= points.size() || t.b >= points.size() || t.c >= points.size()) return true;

    std::vector<size_t> component_parent(points.size());
    for (size_t i = 0; i < points.size(); ++i) component_parent[i] = i;
    for (const auto& t : triangles) {
        if (control.is_canceled()) return false;
        if (!group_of(t.a) || group_of(t.a) != group_of(t.b) || group_of(t.a) != group_of(t.c))
            continue;
        size_t representative = find(component_parent, t.a);
        for (size_t v : {t.b, t.c}) {
            size_t root = find(component_parent, v);
            component_parent[root] = representative;
        }
    }
    std::vector<size_t> component_by_vertex(points.size());
    for (size_t v = 0; v < points.size(); ++v) component_by_vertex[v] = find(component_parent, v);
    std::vector<size_t> component_by_triangle(triangles.size());
    for (size_t i = 0; i < triangles.size(); ++i)
        component_by_triangle[i] = component_by_vertex[triangles[i].a];

    std::vector<std::optional<size_t>> patch_of(triangles.size());
    std::map<size_t, size_t> triangle_counts;
    for (size_t i = 0; i < triangles.size(); ++i) {
        patch_of[i] = group_of(triangles[i].a);
        if (patch_of[i]) triangle_counts[*patch_of[i]] += 1;
    }
    std::vector<size_t> order;
    for (const auto& kv : triangle_counts) order.push_back(kv.first);
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        if (triangle_counts[a] != triangle_counts[b]) return triangle_counts[a] > triangle_counts[b];
        return a < b;
    });
    std::map<size_t, size_t> rank;
    for (size_t r = 0; r < order.size(); ++r) rank[order[r]] = r;
    auto rank_of = [&](size_t v) -> size_t {
        auto g = group_of(v);
        if (!g) return SIZE_MAX;
        auto it = rank.find(*g);
        return it == rank.end() ? SIZE_MAX : it->second;
    };

    // point_origins.get(i): None beyond the slice, Some(origin) inside it
    auto origin_get = [&](size_t i) -> int { return i < origins.size() ? origins[i] : -2; };
    std::vector<size_t> canonical(points.size());
    for (size_t i = 0; i < points.size(); ++i) canonical[i] = i;
    std::vector<char> claimed(points.size(), 0);
    std::vector<std::pair<size_t, size_t>> accepted_pairs;
    size_t fused_pairs = 0, provenance_separated_pairs = 0;
    for (const auto& pr : pairs) {
        if (control.is_canceled()) return false;
        const size_t first = pr.first, second = pr.second;
        if (first >= points.size() || second >= points.size() || !group_of(first) ||
            group_of(first) == group_of(second) || claimed[first] || claimed[second])
            continue;
        claimed[first] = claimed[second] = 1;
        accepted_pairs.push_back({first, second});
        if (origin_get(first) != origin_get(second)) {
            provenance_separated_pairs += 1;
            continue;
        }
        const auto rf = std::make_pair(rank_of(first), first), rs = std::make_pair(rank_of(second), second);
        size_t keep_v, drop_v;
        if (rf <= rs) {
            keep_v = first;
            drop_v = second;
        } else {
            keep_v = second;
            drop_v = first;
        }
        canonical[drop_v] = keep_v;
        fused_pairs += 1;
    }
    std::set<std::pair<size_t, size_t>> linked_components;
    std::set<std::pair<size_t, size_t>> linked_patches;
    std::map<std::pair<size_t, size_t>, std::set<size_t>> scale_anchors;
    for (const auto& pr : accepted_pairs) {
        auto ga = group_of(pr.first), gb = group_of(pr.second);
        if (ga && gb && *ga != *gb) {
            size_t a = component_by_vertex[pr.first], b = component_by_vertex[pr.second];
            linked_components.insert({std::min(a, b), std::max(a, b)});
            linked_patches.insert({std::min(*ga, *gb), std::max(*ga, *gb)});
        }
        if (ga && gb) {
            auto& s = scale_anchors[{std::min(*ga, *gb), std::max(*ga, *gb)}];
            s.insert(pr.first);
            s.insert(pr.second);
        }
    }
    std::vector<std::pair<size_t, std::array<size_t, 3>>> reindexed;
    for (size_t index = 0; index < triangles.size(); ++index) {
        if (control.is_canceled()) return false;
        MeshTriangle& t = triangles[index];
        const std::array<size_t, 3> original{t.a, t.b, t.c};
        const std::array<size_t, 3> mapped{canonical[t.a], canonical[t.b], canonical[t.c]};
        if (mapped != original && mapped[0] != mapped[1] && mapped[1] != mapped[2] &&
            mapped[0] != mapped[2]) {
            t.a = mapped[0];
            t.b = mapped[1];
            t.c = mapped[2];
            reindexed.push_back({index, original});
        }
    }

    auto position = [&](size_t v) { return to_v3(points[v]); };
    std::vector<std::optional<TriangleGeometry>> geometry(triangles.size());
    for (size_t i = 0; i < triangles.size(); ++i)
        geometry[i] = TriangleGeometry::make(
            {position(triangles[i].a), position(triangles[i].b), position(triangles[i].c)});
    double median_edge;
    {
        std::vector<double> edges;
        for (const auto& g : geometry)
            if (g) edges.insert(edges.end(), g->edges, g->edges + 3);
        std::stable_sort(edges.begin(), edges.end(), total_less);
        if (edges.empty()) return true;
        median_edge = edges[edges.size() / 2];
    }
    const double tolerance = median_edge * kMaxOverlapDistanceFraction;
    const double cell = fmax_(median_edge * 2.0, kGeometricEpsilon);
    std::vector<char> keep(triangles.size(), 1);
    LevelGrid<3> kept_grid(cell);
    std::vector<size_t> all_kept;
    size_t removed_duplicate_triangles = 0, remaining_overlap_triangles = 0,
           clipping_budget_exhausted = 0, trimmed_seam_triangles = 0;
    PostingTally tally;
    double trimmed_seam_area = 0.0;
    std::vector<std::pair<size_t, size_t>> uncalibrated_patch_pairs;
    std::vector<ImageRemoval> image_removals;
    std::vector<ClipJob> clip_jobs;
    double total_area = -0.0;
    for (const auto& g : geometry)
        if (g) total_area += g->area();
    std::vector<Footprint> footprints;

    // components joined by linked pairs: only equality of the classes matters
    std::map<size_t, size_t> cluster_parent;
    auto cluster_root = [&](size_t node) {
        size_t root = node;
        for (;;) {
            auto it = cluster_parent.find(root);
            if (it == cluster_parent.end() || it->second == root) break;
            root = it->second;
        }
        cluster_parent[node] = root;
        return root;
    };
    for (const auto& lr : linked_components) {
        size_t l = cluster_root(lr.first), r = cluster_root(lr.second);
        cluster_parent[l] = r;
    }
    std::map<size_t, size_t> cluster_of;
    {
        std::vector<size_t> keys;
        for (const auto& kv : cluster_parent) keys.push_back(kv.first);
        for (size_t k : keys) cluster_of[k] = cluster_root(k);
    }
    auto components_linked = [&](size_t candidate, size_t component) {
        size_t own = component_by_triangle[candidate];
        if (own == component) return false;
        auto a = cluster_of.find(own);
        if (a == cluster_of.end()) return false;
        auto b = cluster_of.find(component);
        return b != cluster_of.end() && b->second == a->second;
    };

    for (size_t patch_rank = 0; patch_rank < order.size(); ++patch_rank) {
        const size_t patch = order[patch_rank];
        if (control.is_canceled()) return false;
        std::vector<size_t> members;
        for (size_t i = 0; i < patch_of.size(); ++i)
            if (patch_of[i] && *patch_of[i] == patch) members.push_back(i);
        if (patch_rank > 0) {
            struct Owner {
                size_t slot;
                const Footprint* footprint;
                double scale;
            };
            std::vector<Owner> owners;
            for (size_t slot = 0; slot < footprints.size(); ++slot) {
                const Footprint& fp = footprints[slot];
                const auto key = std::make_pair(std::min(fp.patch, patch), std::max(fp.patch, patch));
                if (!linked_patches.count(key)) continue;
                auto anchors_it = scale_anchors.find(key);
                const std::set<size_t>* anchors =
                    anchors_it == scale_anchors.end() ? nullptr : &anchors_it->second;
                auto anchored = [&](const std::array<size_t, 3>& vs) {
                    if (!anchors) return false;
                    for (size_t v : vs)
                        if (anchors->count(v)) return true;
                    return false;
                };
                std::vector<double> ratios;
                for (size_t index : members) {
                    if (ratios.size() >= kMaxScaleSamples) break;
                    const MeshTriangle& t = triangles[index];
                    if (!geometry[index]) continue;
                    if (anchored({t.a, t.b, t.c})) {
                        auto r = fp.depth_ratios_tallied(
                            geometry[index]->corners,
                            [&](size_t component) { return components_linked(index, component); },
                            anchored, kMaxScaleSamples - ratios.size(), tally);
                        ratios.insert(ratios.end(), r.begin(), r.end());
                    }
                }
                std::stable_sort(ratios.begin(), ratios.end(), total_less);
                double scale;
                if (ratios.size() >= kMinScaleSamples) {
                    scale = ratios[ratios.size() / 2];
                } else {
                    uncalibrated_patch_pairs.push_back({fp.patch, patch});
                    scale = 1.0;
                }
                owners.push_back({slot, &fp, scale});
            }
            bool imageless_owner = false;
            for (size_t r = 0; r < patch_rank; ++r) {
                const size_t owner = order[r];
                if (!linked_patches.count({std::min(owner, patch), std::max(owner, patch)})) continue;
                bool has = false;
                for (const auto& fp : footprints)
                    if (fp.patch == owner) has = true;
                if (!has) {
                    imageless_owner = true;
                    break;
                }
            }
            for (size_t index : members) {
                if (control.is_canceled()) return false;
                if (!geometry[index]) continue;
                const TriangleGeometry& candidate = *geometry[index];
                std::set<size_t> judged_patches;
                std::map<size_t, std::vector<size_t>> unjudged_triangles;
                struct Judged {
                    Ownership ownership;
                    size_t slot;
                    double scale;
                };
                std::vector<Judged> judged;
                bool cut_off = false;
                for (const Owner& o : owners) {
                    Ownership own;
                    std::vector<size_t> unjudged;
                    Unjudged u = o.footprint->ownership_tallied(
                        candidate.corners, o.scale,
                        [&](size_t component) { return components_linked(index, component); },
                        tally, own, unjudged);
                    if (u == Unjudged::None) {
                        if (unjudged.empty())
                            judged_patches.insert(o.footprint->patch);
                        else
                            unjudged_triangles[o.footprint->patch] = unjudged;
                        judged.push_back({own, o.slot, o.scale});
                    } else if (u == Unjudged::PostingBound) {
                        cut_off = true;
                        break;
                    }
                }
                if (cut_off) continue;
                Judged best{Ownership{}, SIZE_MAX, 1.0};
                for (const Judged& j : judged)
                    if (j.ownership.image_share > best.ownership.image_share) best = j;
                const Ownership owned = best.ownership;
                if (owned.image_share >= kMinImageOwnershipShare) {
                    keep[index] = 0;
                    removed_duplicate_triangles += 1;
                    image_removals.push_back({index, best.slot, best.scale});
                    if (owned.image_share < 1.0 - kOwnershipEpsilon) {
                        trimmed_seam_triangles += 1;
                        trimmed_seam_area += fmax_(candidate.area() - owned.surface_area, 0.0);
                    }
                    continue;
                }
                if (judged_patches.size() == owners.size() && !imageless_owner) {
                    if (owned.image_share > kOwnershipEpsilon) {
                        remaining_overlap_triangles += 1;
                        if (clip_overlaps) clip_jobs.push_back({index, best.slot, best.scale});
                    }
                    continue;
                }
                std::set<size_t> nearby;
                double low[3], high[3];
                candidate.aabb(0.0, low, high);
                PostingBudget budget = PostingBudget::per_query();
                QueryLimit found = kept_grid.query_bounded(low, high, kMaxGridCells, budget, nearby);
                if (found == QueryLimit::Cells) found = budget.take_into(all_kept, nearby);
                tally.record(budget, found);
                if (found != QueryLimit::None) continue;
                std::vector<const TriangleGeometry*> candidates;
                for (size_t other : nearby) {
                    if (!components_linked(index, component_by_triangle[other])) continue;
                    bool ok;
                    if (patch_of[other]) {
                        size_t owner = *patch_of[other];
                        if (judged_patches.count(owner)) {
                            ok = false;
                        } else {
                            auto it = unjudged_triangles.find(owner);
                            ok = it == unjudged_triangles.end() ||
                                 std::find(it->second.begin(), it->second.end(), other) !=
                                     it->second.end();
                        }
                    } else {
                        ok = true;
                    }
                    if (ok && geometry[other]) candidates.push_back(&*geometry[other]);
                }
                CoverageResult cov = candidate.coverage(candidates, tolerance);
                switch (cov.kind) {
                    case Coverage::Full:
                        keep[index] = 0;
                        removed_duplicate_triangles += 1;
                        break;
                    case Coverage::BudgetExhausted: clipping_budget_exhausted += 1; break;
                    case Coverage::Partial: remaining_overlap_triangles += 1; break;
                    case Coverage::Uncovered:
                        if (owned.image_share > kOwnershipEpsilon) remaining_overlap_triangles += 1;
                        break;
                }
            }
        }
        if (patch < cameras.size() && cameras[patch]) {
            std::vector<KeptTriangle> kept;
            for (size_t index : members) {
                if (!keep[index] || !geometry[index]) continue;
                const MeshTriangle& t = triangles[index];
                kept.push_back({geometry[index]->corners, component_by_triangle[index],
                                {t.a, t.b, t.c}, index});
            }
            auto fp = Footprint::make(patch, *cameras[patch], kept);
            if (fp) footprints.push_back(std::move(*fp));
        }
        for (size_t index : members) {
            if (!keep[index] || !geometry[index]) continue;
            all_kept.push_back(index);
            double low[3], high[3];
            geometry[index]->aabb(tolerance, low, high);
            kept_grid.insert(index, low, high);
        }
    }
    SeamInputs seam_inputs{points.size(), &triangles, &keep, &geometry, &membership, &patch_of,
                           &footprints, &image_removals, &kept_grid, &all_kept, tolerance, cell};
    std::vector<MeshTriangle> stitches = stitch_trimmed_seams(
        seam_inputs, position, [&](size_t t, size_t c) { return components_linked(t, c); }, tally);

    ClipState clip_state(points.size());
    std::vector<std::pair<size_t, std::vector<std::array<size_t, 3>>>> clipped;
    size_t clip_failures = 0;
    if (!clip_jobs.empty()) {
        ClipInputs ci;
        ci.points = &points;
        ci.triangles = &triangles;
        ci.corners = [&](size_t index) -> std::optional<std::array<Vec3, 3>> {
            if (!geometry[index]) return std::nullopt;
            return geometry[index]->corners;
        };
        ci.footprints = &footprints;
        ci.point_origins = &origins;
        ci.group_of = group_of;
        ci.source_corners = [&](size_t mesh_index) -> std::array<size_t, 3> {
            auto it = std::lower_bound(reindexed.begin(), reindexed.end(), mesh_index,
                                       [](const auto& e, size_t v) { return e.first < v; });
            if (it != reindexed.end() && it->first == mesh_index) return it->second;
            const MeshTriangle& t = triangles[mesh_index];
            return {t.a, t.b, t.c};
        };
        ci.linked = [&](size_t t, size_t c) { return components_linked(t, c); };
        for (const ClipJob& job : clip_jobs) {
            if (control.is_canceled()) return false;
            std::vector<std::array<size_t, 3>> pieces;
            if (clip_overlap(ci, clip_state, job, tally, pieces) == ClipFailure::None)
                clipped.push_back({job.triangle, std::move(pieces)});
            else
                clip_failures += 1;
        }
    }
    for (const auto& c : clipped) keep[c.first] = 0;
    const size_t stitched_seam_triangles = stitches.size();
    size_t group_count = 0;
    for (int64_t g : membership)
        if (g >= 0) group_count = std::max(group_count, (size_t)g + 1);
    std::vector<size_t> retained_by_group(group_count, 0);
    for (size_t index = 0; index < patch_of.size(); ++index)
        if (keep[index] && patch_of[index]) retained_by_group[*patch_of[index]] += 1;
    for (const auto& c : clipped)
        if (patch_of[c.first]) retained_by_group[*patch_of[c.first]] += c.second.size();
    size_t shared_vertices = 0;
    {
        std::unordered_map<size_t, std::pair<std::optional<size_t>, bool>> vertex_owner;
        for (size_t index = 0; index < triangles.size(); ++index) {
            if (!keep[index]) continue;
            for (size_t v : {triangles[index].a, triangles[index].b, triangles[index].c}) {
                auto it = vertex_owner.emplace(v, std::make_pair(patch_of[index], false)).first;
                if (it->second.first != patch_of[index]) it->second.second = true;
            }
        }
        for (const auto& kv : vertex_owner)
            if (kv.second.second) shared_vertices += 1;
    }
    std::map<size_t, float> original_confidence;
    for (const auto& c : clipped) original_confidence[c.first] = triangles[c.first].confidence;
    {
        size_t w = 0;
        for (size_t i = 0; i < triangles.size(); ++i)
            if (keep[i]) triangles[w++] = triangles[i];
        triangles.resize(w);
    }
    std::vector<TriangleSourceCorners> triangle_sources;
    {
        size_t retained_before = 0, next = 0;
        for (size_t original = 0; original < keep.size(); ++original) {
            if (next < reindexed.size() && reindexed[next].first == original) {
                if (keep[original]) triangle_sources.push_back({retained_before, reindexed[next].second});
                ++next;
            }
            retained_before += keep[original] ? 1 : 0;
        }
    }
    triangles.insert(triangles.end(), stitches.begin(), stitches.end());
    const size_t clipped_overlap_triangles = clipped.size();
    size_t clip_pieces = 0;
    for (const auto& c : clipped) {
        const float confidence = original_confidence.at(c.first);
        clip_pieces += c.second.size();
        for (const auto& p : c.second) triangles.push_back({p[0], p[1], p[2], confidence});
    }
    size_t conformed_triangles = 0, conformance_failures = 0;
    if (clip_state.has_records()) {
        auto derived_position = [&](size_t v) -> Vec3 {
            if (v < points.size()) return position(v);
            return to_v3(clip_state.derived[v - points.size()].point);
        };
        std::vector<size_t> split;
        size_t failures = 0;
        if (!conform_edges(clip_state, triangles, derived_position, control, split, failures))
            return false;
        conformance_failures = failures;
        conformed_triangles = split.size();
        std::set<size_t> split_set(split.begin(), split.end());
        triangle_sources.erase(std::remove_if(triangle_sources.begin(), triangle_sources.end(),
                                              [&](const TriangleSourceCorners& s) {
                                                  return split_set.count(s.triangle) > 0;
                                              }),
                               triangle_sources.end());
    }
    auto group_all = [&](size_t v) -> std::optional<size_t> {
        if (v < points.size()) return group_of(v);
        size_t d = v - points.size();
        return d < clip_state.derived.size() ? clip_state.derived[d].group : std::nullopt;
    };
    std::set<size_t> patches;
    size_t cross_reference_triangles = 0;
    std::vector<std::pair<size_t, size_t>> links;
    for (const auto& t : triangles) {
        if (control.is_canceled()) return false;
        std::optional<size_t> groups[3] = {group_all(t.a), group_all(t.b), group_all(t.c)};
        for (const auto& g : groups)
            if (g) patches.insert(*g);
        if (groups[1] != groups[0] || groups[2] != groups[0]) {
            cross_reference_triangles += 1;
            std::vector<size_t> present;
            for (const auto& g : groups)
                if (g) present.push_back(*g);
            for (size_t i = 0; i + 1 < present.size(); ++i) links.push_back({present[i], present[i + 1]});
        }
    }
    std::vector<size_t> patch_list(patches.begin(), patches.end());
    std::vector<size_t> parent(patch_list.size());
    for (size_t i = 0; i < parent.size(); ++i) parent[i] = i;
    auto slot = [&](size_t g) -> std::optional<size_t> {
        auto it = std::lower_bound(patch_list.begin(), patch_list.end(), g);
        if (it != patch_list.end() && *it == g) return (size_t)(it - patch_list.begin());
        return std::nullopt;
    };
    for (const auto& l : links) {
        auto a = slot(l.first), b = slot(l.second);
        if (a && b) {
            size_t ra = find(parent, *a), rb = find(parent, *b);
            parent[ra] = rb;
        }
    }
    size_t patch_components = 0;
    for (size_t i = 0; i < patch_list.size(); ++i)
        if (find(parent, i) == i) patch_components += 1;

    stats.clipped_overlap_triangles = clipped_overlap_triangles;
    stats.clip_pieces = clip_pieces;
    stats.derived_vertices = clip_state.derived.size();
    stats.unclipped_overlap_triangles = clip_failures;
    stats.conformed_triangles = conformed_triangles;
    stats.conformance_failures = conformance_failures;
    stats.fused_pairs = fused_pairs;
    stats.shared_vertices = shared_vertices;
    stats.cross_reference_triangles = cross_reference_triangles;
    stats.removed_duplicate_triangles = removed_duplicate_triangles;
    stats.remaining_overlap_triangles = remaining_overlap_triangles;
    stats.provenance_separated_pairs = provenance_separated_pairs;
    stats.trimmed_seam_triangles = trimmed_seam_triangles;
    stats.trimmed_seam_area_share = total_area > 0.0 ? trimmed_seam_area / total_area : 0.0;
    stats.stitched_seam_triangles = stitched_seam_triangles;
    stats.uncalibrated_patch_pairs = uncalibrated_patch_pairs;
    stats.retained_by_group = retained_by_group;
    stats.patch_components = patch_components;
    stats.meshed_patches = patch_list.size();
    stats.max_postings_per_query = tally.max_postings;
    stats.posting_bound_hits = tally.bound_hits;
    stats.clipping_budget_exhausted = clipping_budget_exhausted;
    stats.triangle_sources = triangle_sources;
    derived_out = std::move(clip_state.derived);
    return true;
}

}  // namespace

// ---- ear_clip (surface_merge_clip.rs:220-257) ------------------------------------------
std::optional<std::vector<std::array<size_t, 3>>> ear_clip(const Polygon& polygon,
                                                          double tolerance) {
    std::vector<size_t> remaining(polygon.size());
    for (size_t i = 0; i < polygon.size(); ++i) remaining[i] = i;
    std::vector<std::array<size_t, 3>> triangles;
    const double area_floor = tolerance * tolerance;
    while (remaining.size() > 3) {
        const size_t count = remaining.size();
        std::optional<size_t> found;
        for (size_t slot = 0; slot < count; ++slot) {
            const size_t previous = remaining[(slot + count - 1) % count], current = remaining[slot],
                         next = remaining[(slot + 1) % count];
            const V2 a = polygon[previous], b = polygon[current], c = polygon[next];
            if (cross2(b - a, c - a) <= area_floor) continue;
            const V2 ear[3] = {a, b, c};
            bool blocked = false;
            for (size_t other : remaining) {
                if (other == previous || other == current || other == next) continue;
                const V2 p = polygon[other];
                if (norm2(p - a) <= tolerance || norm2(p - b) <= tolerance ||
                    norm2(p - c) <= tolerance)
                    continue;
                bool inside = true;
                for (int edge = 0; edge < 3; ++edge)
                    if (!(distance_to_line(ear[edge], ear[(edge + 1) % 3], p) >= -tolerance)) {
                        inside = false;
                        break;
                    }
                if (inside) {
                    blocked = true;
                    break;
                }
            }
            if (!blocked) {
                found = slot;
                break;
            }
        }
        if (!found) return std::nullopt;
        const size_t slot = *found;
        const size_t cnt = remaining.size();
        triangles.push_back(
            {remaining[(slot + cnt - 1) % cnt], remaining[slot], remaining[(slot + 1) % cnt]});
        remaining.erase(remaining.begin() + (ptrdiff_t)slot);
    }
    if (remaining.size() < 3) return std::nullopt;
    const size_t a = remaining[0], b = remaining[1], c = remaining[2];
    if (cross2(polygon[b] - polygon[a], polygon[c] - polygon[a]) <= area_floor) return std::nullopt;
    triangles.push_back({a, b, c});
    return triangles;
}

bool MergeStats::operator==(const MergeStats& o) const {
    auto sources_equal = [&]() {
        if (triangle_sources.size() != o.triangle_sources.size()) return false;
        for (size_t i = 0; i < triangle_sources.size(); ++i)
            if (triangle_sources[i].triangle != o.triangle_sources[i].triangle ||
                triangle_sources[i].corners != o.triangle_sources[i].corners)
                return false;
        return true;
    };
    return fused_pairs == o.fused_pairs && shared_vertices == o.shared_vertices &&
           cross_reference_triangles == o.cross_reference_triangles &&
           removed_duplicate_triangles == o.removed_duplicate_triangles &&
           remaining_overlap_triangles == o.remaining_overlap_triangles &&
           provenance_separated_pairs == o.provenance_separated_pairs &&
           trimmed_seam_triangles == o.trimmed_seam_triangles &&
           trimmed_seam_area_share == o.trimmed_seam_area_share &&
           stitched_seam_triangles == o.stitched_seam_triangles &&
           uncalibrated_patch_pairs == o.uncalibrated_patch_pairs &&
           retained_by_group == o.retained_by_group && patch_components == o.patch_components &&
           meshed_patches == o.meshed_patches &&
           max_postings_per_query == o.max_postings_per_query &&
           posting_bound_hits == o.posting_bound_hits &&
           clipping_budget_exhausted == o.clipping_budget_exhausted &&
           clipped_overlap_triangles == o.clipped_overlap_triangles &&
           clip_pieces == o.clip_pieces && derived_vertices == o.derived_vertices &&
           unclipped_overlap_triangles == o.unclipped_overlap_triangles &&
           conformed_triangles == o.conformed_triangles &&
           conformance_failures == o.conformance_failures && sources_equal();
}

// MergeStats::diagnostic (surface_merge.rs:205-234); {:.2} of a percentage.
std::string MergeStats::diagnostic(size_t support_groups) const {
    char share[64];
    std::snprintf(share, sizeof share, "%.2f", trimmed_seam_area_share * 100.0);
    auto u = [](size_t v) { return std::to_string(v); };
    return "Overlapping reference patches: " + u(fused_pairs) +
           " fused seam pair(s) became shared vertices (" + u(shared_vertices) +
           " shared vertices, " + u(cross_reference_triangles) +
           " cross-reference triangles) and " + u(provenance_separated_pairs) +
           " kept separate vertices because their endpoints carry different evidence origins; " +
           u(removed_duplicate_triangles) +
           " duplicated overlap triangle(s) were dropped in favour of the patch already meshing "
           "that surface, " +
           u(trimmed_seam_triangles) + " of them seam triangles owned only in part, trimming " +
           share + "% of the accepted mesh area; " + u(stitched_seam_triangles) +
           " seam stitch triangle(s) over existing vertices closed the gaps trimmed seams left, "
           "only where the removed triangles observed the surface at the owner's depth; and " +
           u(remaining_overlap_triangles) +
           " partially overlapping triangle(s) were retained to preserve supported geometry. " +
           u(uncalibrated_patch_pairs.size()) +
           " linked patch pair(s) had too few anchored overlap samples to calibrate their "
           "relative depth scale and were compared uncalibrated. " +
           u(posting_bound_hits) + " candidate lookup(s) hit the posting bound of " +
           u(kMaxPostingsPerQuery) + " owner triangles (at most " + u(max_postings_per_query) +
           " processed by one lookup) and " + u(clipping_budget_exhausted) +
           " triangle(s) exhausted the clipping budget of " + u(kMaxUncoveredPieces) +
           " fragments; both were retained unjudged. " + u(meshed_patches) + " of " +
           u(support_groups) + " camera-support group(s) carry triangles, forming " +
           u(patch_components) + " connected patch component(s). " +
           u(clipped_overlap_triangles) +
           " partially owned overlap triangle(s) were clipped against their owner at the same "
           "depth into " +
           u(clip_pieces) + " remainder triangle(s), deriving " + u(derived_vertices) +
           " vertex(es) on owner edges with source-triangle and barycentric lineage (derived "
           "geometry, not new observations) and splitting " +
           u(conformed_triangles) +
           " triangle(s) at them so no vertex lies inside another edge; " +
           u(unclipped_overlap_triangles) +
           " could not be clipped verifiably and were kept whole. Only fusion-accepted pairs were "
           "merged; no observed vertex was created or moved, and gaps no patch observed stay open.";
}

MergeStats merge_fused_patches(const MergeInputs& in, std::vector<MeshTriangle>& triangles,
                               Control& control) {
    MergeStats stats;
    std::vector<DerivedPoint> derived;
    if (!merge_impl(in, triangles, control, false, stats, derived)) return MergeStats();
    return stats;
}

bool merge_fused_patches_owned(std::vector<Point3> points, std::vector<MeshTriangle> triangles,
                               const MergeInputs& in_, Control& control, OwnedMerge& out,
                               std::string& error) {
    if (control.is_canceled()) {
        error = "reconstruction canceled";
        return false;
    }
    MergeInputs in = in_;
    in.points = &points;
    MergeStats stats;
    std::vector<DerivedPoint> derived;
    if (!merge_impl(in, triangles, control, true, stats, derived)) {
        stats = MergeStats();
        derived.clear();
    }
    if (control.is_canceled()) {
        error = "reconstruction canceled";
        return false;
    }
    if (stats.conformance_failures > 0) {
        error = "surface merge could not split " + std::to_string(stats.conformance_failures) +
                " triangle(s) at clipped seam vertices; the merge is rejected rather than "
                "published with T-junctions";
        return false;
    }
    out.derived_vertices.clear();
    out.derived_vertices.reserve(derived.size());
    for (auto& d : derived) {
        points.push_back(d.point);
        out.derived_vertices.push_back(d.source);
    }
    out.points = std::move(points);
    out.triangles = std::move(triangles);
    out.stats = std::move(stats);
    return true;
}

}  // namespace merge
}  // namespace v3do

// ---- extern "C" surface (test infrastructure) -----------------------------------------
using namespace v3do;
using namespace v3do::merge;

namespace {
thread_local std::string g_merge_error;
}

extern "C" const char* v3do_merge_last_error(void) { return g_merge_error.c_str(); }

extern "C" void v3do_merge_result_free(v3d_merge_result* r) {
    if (!r) return;
    std::free(r->points);
    std::free(r->triangles);
    std::free(r->derived_vertices);
    std::free(r->uncalibrated_patch_pairs);
    std::free(r->retained_by_group);
    std::free(r->triangle_sources);
    std::free(r);
}

// Same arguments as v3d_merge_fused_patches_owned, without the context.
extern "C" int32_t v3do_merge_fused_patches_owned(
    const v3d_point* points, uint64_t n_points, const v3d_mesh_triangle* triangles,
    uint64_t n_triangles, const int64_t* membership, const v3d_fusion_pair* pairs,
    uint64_t n_pairs, const v3d_reference_camera* cameras, uint64_t n_cameras,
    const int32_t* origins, uint64_t n_origins, v3d_cancel_fn cancel, void* cancel_user,
    v3d_merge_result** out) {
    if (!out || (n_points && (!points || !membership)) || (n_triangles && !triangles) ||
        (n_pairs && !pairs) || (n_cameras && !cameras) || (n_origins && !origins))
        return V3D_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    std::vector<Point3> pts(n_points);
    for (uint64_t i = 0; i < n_points; ++i)
        pts[i] = Point3{points[i].x, points[i].y, points[i].z, points[i].confidence, points[i].r,
                        points[i].g, points[i].b};
    std::vector<MeshTriangle> tris(n_triangles);
    for (uint64_t i = 0; i < n_triangles; ++i)
        tris[i] = MeshTriangle{(size_t)triangles[i].a, (size_t)triangles[i].b,
                               (size_t)triangles[i].c, triangles[i].confidence};
    std::vector<int64_t> mem(membership, membership + n_points);
    std::vector<std::pair<size_t, size_t>> prs(n_pairs);
    for (uint64_t i = 0; i < n_pairs; ++i) prs[i] = {(size_t)pairs[i].first, (size_t)pairs[i].second};
    std::vector<std::optional<RefCamera>> cams(n_cameras);
    for (uint64_t i = 0; i < n_cameras; ++i)
        if (cameras[i].present) {
            RefCamera c;
            std::memcpy(c.R, cameras[i].rotation, sizeof c.R);
            std::memcpy(c.t, cameras[i].translation, sizeof c.t);
            cams[i] = c;
        }
    std::vector<int> orgs(origins, origins + n_origins);
    Control control;
    if (cancel) control.poll = [=] { return cancel(cancel_user) != 0; };
    MergeInputs in{nullptr, &mem, &prs, &cams, &orgs};
    OwnedMerge merged;
    std::string error;
    if (!merge_fused_patches_owned(std::move(pts), std::move(tris), in, control, merged, error)) {
        g_merge_error = error;
        return V3D_REJECTED;
    }
    auto* r = (v3d_merge_result*)std::calloc(1, sizeof(v3d_merge_result));
    const MergeStats& s = merged.stats;
    r->stats = v3d_merge_stats{s.fused_pairs, s.shared_vertices, s.cross_reference_triangles,
                               s.removed_duplicate_triangles, s.remaining_overlap_triangles,
                               s.provenance_separated_pairs, s.trimmed_seam_triangles,
                               s.trimmed_seam_area_share, s.stitched_seam_triangles,
                               s.patch_components, s.meshed_patches, s.max_postings_per_query,
                               s.posting_bound_hits, s.clipping_budget_exhausted,
                               s.clipped_overlap_triangles, s.clip_pieces, s.derived_vertices,
                               s.unclipped_overlap_triangles, s.conformed_triangles,
                               s.conformance_failures};
    auto alloc = [](size_t n, size_t size) { return std::calloc(n ? n : 1, size); };
    r->n_points = merged.points.size();
    r->points = (v3d_point*)alloc(r->n_points, sizeof(v3d_point));
    for (size_t i = 0; i < merged.points.size(); ++i) {
        const Point3& p = merged.points[i];
        r->points[i] = v3d_point{p.x, p.y, p.z, p.confidence, p.r, p.g, p.b, 0};
    }
    r->n_triangles = merged.triangles.size();
    r->triangles = (v3d_mesh_triangle*)alloc(r->n_triangles, sizeof(v3d_mesh_triangle));
    for (size_t i = 0; i < merged.triangles.size(); ++i) {
        const MeshTriangle& t = merged.triangles[i];
        r->triangles[i].a = t.a;
        r->triangles[i].b = t.b;
        r->triangles[i].c = t.c;
        r->triangles[i].confidence = t.confidence;
    }
    r->n_derived_vertices = merged.derived_vertices.size();
    r->derived_vertices =
        (v3d_derived_vertex_source*)alloc(r->n_derived_vertices, sizeof(v3d_derived_vertex_source));
    for (size_t i = 0; i < merged.derived_vertices.size(); ++i) {
        const DerivedVertexSource& d = merged.derived_vertices[i];
        auto& o = r->derived_vertices[i];
        o.point_index = d.point_index;
        o.source_triangle = d.source_triangle;
        for (int k = 0; k < 3; ++k) {
            o.source_corners[k] = d.source_corners[k];
            o.barycentric[k] = d.barycentric[k];
        }
    }
    r->n_uncalibrated_patch_pairs = s.uncalibrated_patch_pairs.size();
    r->uncalibrated_patch_pairs =
        (v3d_fusion_pair*)alloc(r->n_uncalibrated_patch_pairs, sizeof(v3d_fusion_pair));
    for (size_t i = 0; i < s.uncalibrated_patch_pairs.size(); ++i)
        r->uncalibrated_patch_pairs[i] =
            v3d_fusion_pair{s.uncalibrated_patch_pairs[i].first, s.uncalibrated_patch_pairs[i].second};
    r->n_retained_by_group = s.retained_by_group.size();
    r->retained_by_group = (uint64_t*)alloc(r->n_retained_by_group, sizeof(uint64_t));
    for (size_t i = 0; i < s.retained_by_group.size(); ++i) r->retained_by_group[i] = s.retained_by_group[i];
    r->n_triangle_sources = s.triangle_sources.size();
    r->triangle_sources = (v3d_triangle_source*)alloc(r->n_triangle_sources, sizeof(v3d_triangle_source));
    for (size_t i = 0; i < s.triangle_sources.size(); ++i) {
        r->triangle_sources[i].triangle = s.triangle_sources[i].triangle;
        for (int k = 0; k < 3; ++k) r->triangle_sources[i].corners[k] = s.triangle_sources[i].corners[k];
    }
    *out = r;
    return V3D_OK;
}

// The reference's own tests of this module (oracle_merge_selftest.cpp): the
// number of checks passed, or -1 with the failing check in `failure`.
extern "C" int32_t v3do_merge_selftest(char* failure, uint64_t capacity) {
    std::string f;
    int n = merge_selftest(f);
    if (failure && capacity) {
        std::snprintf(failure, capacity, "%s", f.c_str());
    }
    return n;
}

// MergeStats::diagnostic (surface_merge.rs:205-234) of a result's stats.
extern "C" uint64_t v3do_merge_diagnostic(const v3d_merge_result* r, uint64_t support_groups,
                                          char* out, uint64_t capacity) {
    MergeStats s;
    const v3d_merge_stats& c = r->stats;
    s.fused_pairs = c.fused_pairs;
    s.shared_vertices = c.shared_vertices;
    s.cross_reference_triangles = c.cross_reference_triangles;
    s.removed_duplicate_triangles = c.removed_duplicate_triangles;
    s.remaining_overlap_triangles = c.remaining_overlap_triangles;
    s.provenance_separated_pairs = c.provenance_separated_pairs;
    s.trimmed_seam_triangles = c.trimmed_seam_triangles;
    s.trimmed_seam_area_share = c.trimmed_seam_area_share;
    s.stitched_seam_triangles = c.stitched_seam_triangles;
    s.uncalibrated_patch_pairs.resize(r->n_uncalibrated_patch_pairs);
    s.patch_components = c.patch_components;
    s.meshed_patches = c.meshed_patches;
    s.max_postings_per_query = c.max_postings_per_query;
    s.posting_bound_hits = c.posting_bound_hits;
    s.clipping_budget_exhausted = c.clipping_budget_exhausted;
    s.clipped_overlap_triangles = c.clipped_overlap_triangles;
    s.clip_pieces = c.clip_pieces;
    s.derived_vertices = c.derived_vertices;
    s.unclipped_overlap_triangles = c.unclipped_overlap_triangles;
    s.conformed_triangles = c.conformed_triangles;
    s.conformance_failures = c.conformance_failures;
    std::string d = s.diagnostic(support_groups);
    if (out && capacity) std::snprintf(out, capacity, "%s", d.c_str());
    return d.size();
}
