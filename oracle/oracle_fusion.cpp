// TEST INFRASTRUCTURE — CPU oracle of cross-reference surface fusion.
//
// A literal f64 restatement of video-to-3d-core's surface_fusion.rs:316-852
// (evidence_support_membership, fuse_mutually_supported_vertices_with_control,
// topology_safe_moves_with_control, triangle_preserved_with_moves,
// vertex_surface_evidence_with_control and their helpers), in the reference's
// evaluation order: triangles in index order, per-vertex sums in triangle
// order, neighbour cells dz-dy-dx from -1 to 1 with each cell's vertices in
// index order, nalgebra's left-to-right dot and norm, no fused multiply-add
// (the Makefile builds with -ffp-contract=off).
//
// Only tests/ and bench.py's CPU-baseline leg load this code, as the checker
// or the timed CPU baseline; the product (video-to-3d_b200/) never links it.
//
// Parity pin: the reference's own tests of this module
// (surface_fusion.rs:891-1070, fusion_prepass_acceptance_tests.rs:31-57) are
// re-run against it in oracle_selftest.cpp.
#include <algorithm>
#include <cmath>
#include <map>
#include <optional>
#include <tuple>
#include <vector>

#include "oracle.hpp"

namespace v3do {

namespace {

constexpr double kGeometricEpsilon = 1.0e-9;       // surface_fusion.rs:6
constexpr double kMaxLocalEdgeFraction = 0.28;     // :7
constexpr double kMaxGlobalEdgeFraction = 0.35;    // :8
constexpr double kMinNormalAlignment = 0.94;       // :9
constexpr double kMinIncidentNormalAlignment = 0.985;  // :10
constexpr double kMinIncidentAreaRatio = 0.75;     // :11
constexpr double kMinConfidenceWeight = 0.05;      // :12

// point_position (surface_fusion.rs:824-830)
std::optional<Vec3> point_position(const Point3& p) {
    Vec3 v{(double)p.x, (double)p.y, (double)p.z};
    if (!std::isfinite(v.x) || !std::isfinite(v.y) || !std::isfinite(v.z)) return std::nullopt;
    return v;
}

// nalgebra dot of two 3-vectors: ((x x' + y y') + z z')
double dot(Vec3 a, Vec3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

// Rust's `f64 as i64`: saturating, NaN to 0
int64_t as_i64(double v) {
    if (std::isnan(v)) return 0;
    if (v >= 9223372036854775807.0) return INT64_MAX;
    if (v <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)v;
}

// spatial_cell (surface_fusion.rs:816-822)
std::tuple<int64_t, int64_t, int64_t> spatial_cell(Vec3 p, double cell) {
    return {as_i64(std::floor(p.x / cell)), as_i64(std::floor(p.y / cell)),
            as_i64(std::floor(p.z / cell))};
}

// median (surface_fusion.rs:838-849) of sorted values
std::optional<double> median_sorted(const std::vector<double>& v) {
    if (v.empty()) return std::nullopt;
    const size_t mid = v.size() / 2;
    if (v.size() % 2 == 0) return (v[mid - 1] + v[mid]) * 0.5;
    return v[mid];
}

// proposed_position (surface_fusion.rs:698-712)
std::optional<Vec3> proposed_position(size_t vertex, const std::vector<Point3>& points,
                                      const std::vector<FusionMove>& moves,
                                      const std::vector<char>& active,
                                      const std::vector<int64_t>& move_by_vertex) {
    if (vertex < move_by_vertex.size() && move_by_vertex[vertex] >= 0) {
        const size_t m = (size_t)move_by_vertex[vertex];
        if (m < active.size() && active[m]) return moves[m].position;
    }
    if (vertex >= points.size()) return std::nullopt;
    return point_position(points[vertex]);
}

// triangle_preserved_with_moves (surface_fusion.rs:652-696)
bool triangle_preserved(const std::vector<Point3>& points, const MeshTriangle& t,
                        const std::vector<FusionMove>& moves, const std::vector<char>& active,
                        const std::vector<int64_t>& move_by_vertex) {
    const size_t n = points.size();
    if (t.a >= n || t.b >= n || t.c >= n) return false;
    auto a = point_position(points[t.a]), b = point_position(points[t.b]),
         c = point_position(points[t.c]);
    if (!a || !b || !c) return false;
    const Vec3 on = cross(sub(*b, *a), sub(*c, *a));
    const double oa = norm(on);
    if (!std::isfinite(oa) || oa <= kGeometricEpsilon) return false;
    auto pa = proposed_position(t.a, points, moves, active, move_by_vertex);
    if (!pa) return false;
    auto pb = proposed_position(t.b, points, moves, active, move_by_vertex);
    if (!pb) return false;
    auto pc = proposed_position(t.c, points, moves, active, move_by_vertex);
    if (!pc) return false;
    const Vec3 pn = cross(sub(*pb, *pa), sub(*pc, *pa));
    const double ps = norm(pn);
    if (!std::isfinite(ps) || ps < oa * kMinIncidentAreaRatio) return false;
    return dot(on, pn) / (oa * ps) >= kMinIncidentNormalAlignment;
}

}  // namespace

// evidence_support_membership (surface_fusion.rs:316-345)
std::pair<std::vector<int64_t>, size_t> evidence_support_membership(
    const std::vector<EvidenceRegion>& regions, size_t point_count) {
    std::vector<int64_t> membership(point_count, -1);
    std::map<std::pair<size_t, std::vector<size_t>>, size_t> groups;
    for (const EvidenceRegion& r : regions) {
        if (!r.reference_frame) continue;
        std::vector<size_t> src = r.source_frames;
        std::sort(src.begin(), src.end());
        auto key = std::make_pair(*r.reference_frame, src);
        const size_t next = groups.size();
        auto it = groups.emplace(key, next).first;
        const size_t group = it->second;
        if (r.start > SIZE_MAX - r.count) continue;
        const size_t end = r.start + r.count;
        if (r.start > end || end > point_count) continue;
        for (size_t i = r.start; i < end; ++i) membership[i] = (int64_t)group;
    }
    return {membership, groups.size()};
}

// vertex_surface_evidence_with_control (surface_fusion.rs:723-814)
std::optional<VertexEvidence> vertex_surface_evidence(const std::vector<Point3>& points,
                                                      const std::vector<MeshTriangle>& triangles,
                                                      Control& control) {
    if (control.is_canceled()) return std::nullopt;
    const size_t n = points.size();
    std::vector<Vec3> normal_sums(n);
    std::vector<double> edge_sums(n, 0.0);
    std::vector<size_t> edge_counts(n, 0);
    VertexEvidence ev;
    ev.incident.assign(n, {});
    std::vector<double> edge_lengths;
    edge_lengths.reserve(triangles.size() * 3);
    for (size_t ti = 0; ti < triangles.size(); ++ti) {
        if (control.is_canceled()) return std::nullopt;
        const MeshTriangle& t = triangles[ti];
        if (t.a == t.b || t.b == t.c || t.c == t.a || t.a >= n || t.b >= n || t.c >= n) continue;
        auto a = point_position(points[t.a]), b = point_position(points[t.b]),
             c = point_position(points[t.c]);
        if (!a || !b || !c) continue;
        const Vec3 ab = sub(*b, *a), ac = sub(*c, *a), bc = sub(*c, *b);
        const double lab = norm(ab), lac = norm(ac), lbc = norm(bc);
        bool bad = false;
        for (double l : {lab, lac, lbc}) bad = bad || !std::isfinite(l) || l <= kGeometricEpsilon;
        if (bad) continue;
        const Vec3 nrm = cross(ab, ac);
        const double nl = norm(nrm);
        if (!std::isfinite(nl) || nl <= kGeometricEpsilon) continue;
        const double conf = std::clamp((double)t.confidence, kMinConfidenceWeight, 1.0);
        const Vec3 wn{nrm.x / nl * conf, nrm.y / nl * conf, nrm.z / nl * conf};
        for (size_t idx : {t.a, t.b, t.c}) {
            normal_sums[idx] = add(normal_sums[idx], wn);
            ev.incident[idx].push_back(ti);
        }
        edge_sums[t.a] += lab + lac;
        edge_counts[t.a] += 2;
        edge_sums[t.b] += lab + lbc;
        edge_counts[t.b] += 2;
        edge_sums[t.c] += lac + lbc;
        edge_counts[t.c] += 2;
        edge_lengths.push_back(lab);
        edge_lengths.push_back(lac);
        edge_lengths.push_back(lbc);
    }
    if (control.is_canceled()) return std::nullopt;
    std::sort(edge_lengths.begin(), edge_lengths.end());  // finite and positive: total order
    if (control.is_canceled()) return std::nullopt;
    ev.global_edge_scale = median_sorted(edge_lengths);
    ev.normals.resize(n);
    ev.local_scales.resize(n);
    for (size_t i = 0; i < n; ++i) {
        if (control.is_canceled()) return std::nullopt;
        const double len = norm(normal_sums[i]);
        if (std::isfinite(len) && len > kGeometricEpsilon)
            ev.normals[i] = Vec3{normal_sums[i].x / len, normal_sums[i].y / len,
                                 normal_sums[i].z / len};
    }
    for (size_t i = 0; i < n; ++i) {
        if (control.is_canceled()) return std::nullopt;
        if (edge_counts[i] > 0 && std::isfinite(edge_sums[i]))
            ev.local_scales[i] = edge_sums[i] / (double)edge_counts[i];
    }
    return ev;
}

// topology_safe_moves_with_control (surface_fusion.rs:566-650)
std::pair<std::vector<FusionMove>, size_t> topology_safe_moves(
    const std::vector<Point3>& points, const std::vector<MeshTriangle>& triangles,
    const std::vector<std::vector<size_t>>& incident, std::vector<FusionMove> moves,
    Control& control) {
    if (moves.empty()) return {moves, 0};
    std::vector<char> active(moves.size(), 1);
    std::vector<int64_t> move_by_vertex(points.size(), -1);
    for (size_t m = 0; m < moves.size(); ++m) {
        if (control.is_canceled()) return {{}, 0};
        if (moves[m].first >= points.size() || moves[m].second >= points.size()) {
            active[m] = 0;
            continue;
        }
        move_by_vertex[moves[m].first] = (int64_t)m;
        move_by_vertex[moves[m].second] = (int64_t)m;
    }
    for (;;) {
        if (control.is_canceled()) return {{}, 0};
        std::vector<char> touched(triangles.size(), 0);
        std::vector<size_t> touched_list;
        for (size_t m = 0; m < moves.size(); ++m) {
            if (control.is_canceled()) return {{}, 0};
            if (!active[m]) continue;
            for (size_t v : {moves[m].first, moves[m].second}) {
                if (v >= incident.size()) continue;
                for (size_t ti : incident[v])
                    if (ti < triangles.size() && !touched[ti]) {
                        touched[ti] = 1;
                        touched_list.push_back(ti);
                    }
            }
        }
        std::vector<char> reject(moves.size(), 0);
        for (size_t ti : touched_list) {
            const MeshTriangle& t = triangles[ti];
            if (triangle_preserved(points, t, moves, active, move_by_vertex)) continue;
            for (size_t v : {t.a, t.b, t.c}) {
                if (v >= move_by_vertex.size() || move_by_vertex[v] < 0) continue;
                const size_t m = (size_t)move_by_vertex[v];
                if (active[m]) reject[m] = 1;
            }
        }
        bool any = false;
        for (char r : reject) any = any || r;
        if (!any) break;
        for (size_t m = 0; m < moves.size(); ++m)
            if (reject[m]) active[m] = 0;
    }
    size_t rejected = 0;
    std::vector<FusionMove> accepted;
    for (size_t m = 0; m < moves.size(); ++m) {
        if (active[m])
            accepted.push_back(moves[m]);
        else
            ++rejected;
    }
    return {accepted, rejected};
}

// fuse_mutually_supported_vertices_with_control (surface_fusion.rs:369-549)
FusionOutcome fuse_mutually_supported_vertices(std::vector<Point3>& points,
                                               const std::vector<MeshTriangle>& triangles,
                                               const std::vector<int64_t>& membership,
                                               Control& control) {
    if (points.size() != membership.size()) return {};
    auto evo = vertex_surface_evidence(points, triangles, control);
    if (!evo) return {};
    const VertexEvidence& ev = *evo;
    if (!ev.global_edge_scale) return {};
    const double global = *ev.global_edge_scale;
    const double cell_size = std::max(global * kMaxGlobalEdgeFraction, kGeometricEpsilon);
    const size_t n = points.size();

    std::map<std::tuple<int64_t, int64_t, int64_t>, std::vector<size_t>> buckets;
    size_t eligible = 0;
    for (size_t i = 0; i < n; ++i) {
        if (control.is_canceled()) return {};
        if (membership[i] < 0 || !ev.normals[i] || !ev.local_scales[i]) continue;
        auto p = point_position(points[i]);
        if (!p) continue;
        buckets[spatial_cell(*p, cell_size)].push_back(i);
        ++eligible;
    }

    std::vector<std::optional<std::pair<size_t, double>>> nearest(n);
    size_t candidate_pairs = 0, rejected_normal = 0;
    for (size_t i = 0; i < n; ++i) {
        if (control.is_canceled()) return {};
        if (membership[i] < 0 || !ev.normals[i] || !ev.local_scales[i]) continue;
        auto p = point_position(points[i]);
        if (!p) continue;
        const int64_t group = membership[i];
        const Vec3 normal = *ev.normals[i];
        const double scale = *ev.local_scales[i];
        const auto cell = spatial_cell(*p, cell_size);
        for (int64_t dz = -1; dz <= 1; ++dz)
            for (int64_t dy = -1; dy <= 1; ++dy)
                for (int64_t dx = -1; dx <= 1; ++dx) {
                    auto it = buckets.find({std::get<0>(cell) + dx, std::get<1>(cell) + dy,
                                            std::get<2>(cell) + dz});
                    if (it == buckets.end()) continue;
                    for (size_t o : it->second) {
                        if (o == i || membership[o] == group) continue;
                        if (!ev.normals[o] || !ev.local_scales[o]) continue;
                        auto q = point_position(points[o]);
                        if (!q) continue;
                        const double maxd =
                            std::min(std::min(scale, *ev.local_scales[o]) * kMaxLocalEdgeFraction,
                                     global * kMaxGlobalEdgeFraction);
                        const double d = norm(sub(*q, *p));
                        if (!std::isfinite(d) || d > maxd) continue;
                        if (i < o) ++candidate_pairs;
                        const double align = std::fabs(dot(normal, *ev.normals[o]));
                        if (align < kMinNormalAlignment) {
                            if (i < o) ++rejected_normal;
                            continue;
                        }
                        bool replace = !nearest[i];
                        if (!replace) {
                            const size_t ci = nearest[i]->first;
                            const double cd = nearest[i]->second;
                            replace = d < cd - kGeometricEpsilon ||
                                      (std::fabs(d - cd) <= kGeometricEpsilon && o < ci);
                        }
                        if (replace) nearest[i] = std::make_pair(o, d);
                    }
                }
    }

    std::vector<FusionMove> proposed;
    for (size_t i = 0; i < n; ++i) {
        if (control.is_canceled()) return {};
        if (!nearest[i]) continue;
        const size_t o = nearest[i]->first;
        if (i >= o || !nearest[o] || nearest[o]->first != i) continue;
        auto p = point_position(points[i]), q = point_position(points[o]);
        if (!p || !q) continue;
        const double w = std::fmax((double)points[i].confidence, kMinConfidenceWeight);
        const double ow = std::fmax((double)points[o].confidence, kMinConfidenceWeight);
        const double ws = w + ow;
        proposed.push_back(FusionMove{i, o,
                                      Vec3{(p->x * w + q->x * ow) / ws, (p->y * w + q->y * ow) / ws,
                                           (p->z * w + q->z * ow) / ws}});
    }

    auto [accepted, rejected_topology] =
        topology_safe_moves(points, triangles, ev.incident, std::move(proposed), control);
    if (control.is_canceled()) return {};
    FusionOutcome out;
    for (const FusionMove& m : accepted)
        for (size_t idx : {m.first, m.second}) {
            const Point3 original = points[idx];
            points[idx].x = (float)m.position.x;
            points[idx].y = (float)m.position.y;
            points[idx].z = (float)m.position.z;
            const Point3& now = points[idx];
            const bool same = now.x == original.x && now.y == original.y && now.z == original.z &&
                              now.confidence == original.confidence && now.r == original.r &&
                              now.g == original.g && now.b == original.b;
            if (!same) out.moved_indices.push_back(idx);
        }
    std::sort(out.moved_indices.begin(), out.moved_indices.end());
    out.stats.eligible_vertices = eligible;
    out.stats.candidate_pairs = candidate_pairs;
    out.stats.rejected_normal_pairs = rejected_normal;
    out.stats.rejected_topology_pairs = rejected_topology;
    out.stats.fused_pairs = accepted.size();
    for (const FusionMove& m : accepted) out.pairs.emplace_back(m.first, m.second);
    return out;
}

}  // namespace v3do

using namespace v3do;

extern "C" int32_t v3do_fuse_mutually_supported_vertices(
    v3d_point* points, uint64_t n_points, const v3d_mesh_triangle* triangles, uint64_t n_triangles,
    const int64_t* membership, v3d_cancel_fn cancel, void* cancel_user, v3d_fusion_stats* stats,
    v3d_fusion_pair* pairs, uint64_t* n_pairs, uint64_t* moved, uint64_t* n_moved) {
    if ((n_points && (!points || !membership)) || (n_triangles && !triangles) || !stats ||
        !n_pairs || !n_moved || (n_points && (!pairs || !moved)))
        return V3D_ERR_INVALID_ARGUMENT;
    std::vector<Point3> pts(n_points);
    for (uint64_t i = 0; i < n_points; ++i)
        pts[i] = Point3{points[i].x, points[i].y, points[i].z, points[i].confidence, points[i].r,
                        points[i].g, points[i].b};
    std::vector<MeshTriangle> tris(n_triangles);
    for (uint64_t i = 0; i < n_triangles; ++i)
        tris[i] = MeshTriangle{(size_t)triangles[i].a, (size_t)triangles[i].b,
                               (size_t)triangles[i].c, triangles[i].confidence};
    std::vector<int64_t> mem(membership, membership + n_points);
    Control control;
    if (cancel) control.poll = [=] { return cancel(cancel_user) != 0; };
    FusionOutcome out = fuse_mutually_supported_vertices(pts, tris, mem, control);
    for (uint64_t i = 0; i < n_points; ++i) {
        points[i].x = pts[i].x;
        points[i].y = pts[i].y;
        points[i].z = pts[i].z;
    }
    stats->eligible_vertices = out.stats.eligible_vertices;
    stats->candidate_pairs = out.stats.candidate_pairs;
    stats->rejected_normal_pairs = out.stats.rejected_normal_pairs;
    stats->rejected_topology_pairs = out.stats.rejected_topology_pairs;
    stats->fused_pairs = out.stats.fused_pairs;
    *n_pairs = out.pairs.size();
    for (size_t k = 0; k < out.pairs.size(); ++k)
        pairs[k] = v3d_fusion_pair{out.pairs[k].first, out.pairs[k].second};
    *n_moved = out.moved_indices.size();
    for (size_t k = 0; k < out.moved_indices.size(); ++k) moved[k] = out.moved_indices[k];
    return V3D_OK;
}
