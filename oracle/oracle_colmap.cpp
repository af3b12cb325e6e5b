// TEST INFRASTRUCTURE — CPU oracle of the geometric depth-grid verification.
//
// A literal f64 restatement of video-to-3d-core's colmap_surface.rs:56-95
// (VerificationFunnel and its dominant rejection), :125-157 (surface_topology),
// :175-275 (verify_patch) and :289-314 (verified_union), in the reference's
// evaluation order: nalgebra's left-to-right matrix-vector products, scalar
// chains left to right, no fused multiply-add (-ffp-contract=off), Rust's
// round-half-away-from-zero and saturating float-to-integer casts.  The
// parallax threshold cos(0.5 degrees) is taken from the C library's cos, as
// the reference's f64::cos is on Linux.
//
// Only tests/ and bench.py's CPU-baseline leg load this code, as the checker
// or the timed CPU baseline; the product (video-to-3d_b200/) never links it.
//
// Parity pin: the reference's own tests of this module
// (colmap_surface.rs:548-759) are re-run against it in oracle_selftest.cpp.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <vector>

#include "oracle.hpp"

namespace v3do {

namespace {

// Rust's `f64 as usize`: saturating, NaN to 0
size_t as_usize(double v) {
    if (!(v > 0.0)) return 0;
    if (v >= 18446744073709551615.0) return SIZE_MAX;
    return (size_t)v;
}

// nalgebra rotation * v, row by row left to right
Vec3 rotate(const double R[9], Vec3 v) {
    return {(R[0] * v.x + R[1] * v.y) + R[2] * v.z, (R[3] * v.x + R[4] * v.y) + R[5] * v.z,
            (R[6] * v.x + R[7] * v.y) + R[8] * v.z};
}
// nalgebra rotation.transpose() * v
Vec3 rotate_t(const double R[9], Vec3 v) {
    return {(R[0] * v.x + R[3] * v.y) + R[6] * v.z, (R[1] * v.x + R[4] * v.y) + R[7] * v.z,
            (R[2] * v.x + R[5] * v.y) + R[8] * v.z};
}
double dot3(Vec3 a, Vec3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }

}  // namespace

double min_parallax_cos() { return std::cos(0.5 * (3.141592653589793 / 180.0)); }

// VerificationFunnel::dominant_rejection (colmap_surface.rs:81-95)
const char* dominant_rejection(const Funnel& f) {
    const std::pair<const char*, size_t> c[] = {
        {"missing_reference_depth", f.missing_reference_depth},
        {"insufficient_parallax", f.insufficient_parallax},
        {"behind_source", f.behind_source},
        {"outside_source", f.outside_source},
        {"missing_source_depth", f.missing_source_depth},
        {"depth_disagreement", f.depth_disagreement},
        {"color_disagreement", f.color_disagreement}};
    const char* best = nullptr;
    size_t best_n = 0;
    for (auto& [name, n] : c) {
        if (n == 0) continue;
        // max_by_key((count, Reverse(name))): the larger count, then the smaller name; last max wins
        if (!best || n > best_n || (n == best_n && std::strcmp(name, best) <= 0)) {
            best = name;
            best_n = n;
        }
    }
    return best;
}

// verify_patch (colmap_surface.rs:175-275)
std::vector<std::pair<Point3, GridSite>> verify_patch(const DepthView& ref, const DepthView& src,
                                                      size_t stride, size_t reference_stride,
                                                      double focal, Funnel& funnel) {
    const size_t width = ref.width, height = ref.height;
    const size_t cols = (width + stride - 1) / stride, rows = (height + stride - 1) / stride;
    const double cx = (double)width / 2.0, cy = (double)height / 2.0;
    std::vector<std::pair<Point3, GridSite>> points;
    const Vec3 source_center = src.camera.center(), ref_center = ref.camera.center();
    const double min_cos = min_parallax_cos();
    for (size_t i = 0; i < cols * rows; ++i) {
        const size_t x = (i % cols) * stride, y = (i / cols) * stride;
        if (x % reference_stride != 0 || y % reference_stride != 0) continue;
        ++funnel.reference_samples;
        const float z = ref.depth[i];
        if (z <= 0.f) {
            ++funnel.missing_reference_depth;
            continue;
        }
        const Vec3 ray{((double)x + 0.5 - cx) / focal, ((double)y + 0.5 - cy) / focal, 1.0};
        const double zd = (double)z;
        const Vec3 cam{ray.x * zd - ref.camera.t[0], ray.y * zd - ref.camera.t[1],
                       ray.z * zd - ref.camera.t[2]};
        const Vec3 world = rotate_t(ref.camera.R, cam);
        const Vec3 direction = sub(world, ref_center), from_source = sub(world, source_center);
        if (dot3(direction, from_source) >= min_cos * norm(direction) * norm(from_source)) {
            ++funnel.insufficient_parallax;
            continue;
        }
        const Vec3 r = rotate(src.camera.R, world);
        const Vec3 q{r.x + src.camera.t[0], r.y + src.camera.t[1], r.z + src.camera.t[2]};
        if (q.z <= 0.0) {
            ++funnel.behind_source;
            continue;
        }
        const double u = focal * q.x / q.z + cx - 0.5, v = focal * q.y / q.z + cy - 0.5;
        const size_t col = as_usize(std::round(u / (double)stride));
        const size_t row = as_usize(std::round(v / (double)stride));
        if (!(u >= 0.0 && u < (double)width) || !(v >= 0.0 && v < (double)height) || col >= cols ||
            row >= rows) {
            ++funnel.outside_source;
            continue;
        }
        const double other = (double)src.depth[row * cols + col];
        if (other <= 0.0) {
            ++funnel.missing_source_depth;
            continue;
        }
        if (std::fabs(other - q.z) > 0.02 * q.z) {
            ++funnel.depth_disagreement;
            continue;
        }
        const uint8_t* rp = ref.rgba + (y * ref.width + x) * 4;
        const size_t sx = std::min(as_usize(std::round(u)), width - 1);
        const size_t sy = std::min(as_usize(std::round(v)), height - 1);
        const uint8_t* sp = src.rgba + (sy * src.width + sx) * 4;
        const uint32_t err = (uint32_t)std::abs((int)rp[0] - (int)sp[0]) +
                             (uint32_t)std::abs((int)rp[1] - (int)sp[1]) +
                             (uint32_t)std::abs((int)rp[2] - (int)sp[2]);
        if (err > 105) {
            ++funnel.color_disagreement;
            continue;
        }
        ++funnel.accepted;
        Point3 p{(float)world.x, (float)world.y, (float)world.z,
                 (float)(1.0 - std::fabs(other - q.z) / q.z), rp[0], rp[1], rp[2]};
        points.emplace_back(p, GridSite{(uint32_t)x, (uint32_t)y});
    }
    return points;
}

// verified_union (colmap_surface.rs:289-314)
std::vector<VerifiedSample> verified_union(
    const std::vector<std::pair<size_t, std::vector<std::pair<Point3, GridSite>>>>& candidates) {
    std::map<std::pair<uint32_t, uint32_t>, VerifiedSample> u;
    for (const auto& [source, patch] : candidates)
        for (const auto& [point, site] : patch) {
            auto it = u.find({site.y, site.x});
            if (it == u.end()) {
                u.emplace(std::make_pair(site.y, site.x), VerifiedSample{point, site, {source}});
            } else {
                // f32::max: the non-NaN operand when one is NaN
                it->second.point.confidence = std::fmax(it->second.point.confidence, point.confidence);
                it->second.sources.push_back(source);
            }
        }
    std::vector<VerifiedSample> out;
    for (auto& [key, s] : u) {
        std::sort(s.sources.begin(), s.sources.end());
        s.sources.erase(std::unique(s.sources.begin(), s.sources.end()), s.sources.end());
        out.push_back(s);
    }
    return out;
}

// surface_topology (colmap_surface.rs:125-157)
Topology surface_topology(size_t vertex_count, const std::vector<MeshTriangle>& triangles) {
    std::vector<size_t> parent(vertex_count);
    for (size_t i = 0; i < vertex_count; ++i) parent[i] = i;
    auto root = [&](size_t i) {
        while (parent[i] != i) {
            parent[i] = parent[parent[i]];
            i = parent[i];
        }
        return i;
    };
    std::map<std::pair<size_t, size_t>, size_t> edges;
    for (const MeshTriangle& t : triangles)
        for (auto [a, b] : {std::pair<size_t, size_t>{t.a, t.b}, {t.b, t.c}, {t.c, t.a}}) {
            ++edges[{std::min(a, b), std::max(a, b)}];
            const size_t ra = root(a), rb = root(b);
            if (ra != rb) parent[std::max(ra, rb)] = std::min(ra, rb);
        }
    std::map<size_t, size_t> sizes;
    for (const MeshTriangle& t : triangles) ++sizes[root(t.a)];
    Topology top;
    top.islands = sizes.size();
    for (auto& [r, n] : sizes) {
        if (n < 32) {
            ++top.small_islands;
            top.small_island_triangles += n;
        }
        top.largest_island_triangles = std::max(top.largest_island_triangles, n);
    }
    for (auto& [e, n] : edges) top.boundary_edges += n == 1;
    return top;
}

}  // namespace v3do

using namespace v3do;

extern "C" int32_t v3do_verify_depth_grids(const v3d_depth_view* views, uint64_t n_views,
                                           const uint32_t* reference_views, uint64_t n_references,
                                           const int32_t* source_views, uint32_t stride,
                                           uint32_t reference_stride, double focal,
                                           v3d_verified_sample* samples, uint64_t capacity,
                                           uint64_t* sample_offsets, v3d_verification_funnel* funnel) {
    if (!views || !n_views || (n_references && (!reference_views || !source_views)) || !sample_offsets ||
        !funnel || stride == 0 || reference_stride == 0 || reference_stride % stride != 0)
        return V3D_ERR_INVALID_ARGUMENT;
    std::vector<DepthView> dv(n_views);
    for (uint64_t i = 0; i < n_views; ++i) {
        if (views[i].width != views[0].width || views[i].height != views[0].height)
            return V3D_ERR_INVALID_ARGUMENT;
        dv[i].width = views[i].width;
        dv[i].height = views[i].height;
        dv[i].rgba = views[i].rgba;
        dv[i].depth = views[i].depth;
        dv[i].camera.frame_index = views[i].camera.frame_index;
        std::memcpy(dv[i].camera.R, views[i].camera.rotation, sizeof(dv[i].camera.R));
        std::memcpy(dv[i].camera.t, views[i].camera.translation, sizeof(dv[i].camera.t));
    }
    Funnel total;
    std::vector<std::vector<VerifiedSample>> per_ref(n_references);
    uint64_t count = 0;
    for (uint64_t r = 0; r < n_references; ++r) {
        if (reference_views[r] >= n_views) return V3D_ERR_INVALID_ARGUMENT;
        std::vector<std::pair<size_t, std::vector<std::pair<Point3, GridSite>>>> cand;
        for (int j = 0; j < 4; ++j) {
            const int32_t s = source_views[4 * r + j];
            if (s < 0) continue;
            if ((uint64_t)s >= n_views) return V3D_ERR_INVALID_ARGUMENT;
            Funnel f;
            auto patch = verify_patch(dv[reference_views[r]], dv[s], stride, reference_stride, focal, f);
            total.add(f);
            cand.emplace_back((size_t)j, std::move(patch));  // the source's position as its key
        }
        per_ref[r] = verified_union(cand);
        count += per_ref[r].size();
    }
    if (count > capacity) return V3D_ERR_INVALID_ARGUMENT;
    uint64_t k = 0;
    for (uint64_t r = 0; r < n_references; ++r) {
        sample_offsets[r] = k;
        for (const VerifiedSample& s : per_ref[r]) {
            v3d_verified_sample& o = samples[k++];
            o.point = v3d_point{s.point.x, s.point.y, s.point.z, s.point.confidence,
                                s.point.r, s.point.g, s.point.b, 0};
            o.site = v3d_grid_site{s.site.x, s.site.y};
            o.source_mask = 0;
            for (size_t j : s.sources) o.source_mask |= 1u << j;
        }
    }
    sample_offsets[n_references] = k;
    funnel->reference_samples = total.reference_samples;
    funnel->missing_reference_depth = total.missing_reference_depth;
    funnel->insufficient_parallax = total.insufficient_parallax;
    funnel->behind_source = total.behind_source;
    funnel->outside_source = total.outside_source;
    funnel->missing_source_depth = total.missing_source_depth;
    funnel->depth_disagreement = total.depth_disagreement;
    funnel->color_disagreement = total.color_disagreement;
    funnel->accepted = total.accepted;
    return V3D_OK;
}

extern "C" int32_t v3do_surface_topology_of(const v3d_mesh_triangle* triangles, uint64_t n_triangles,
                                            uint64_t vertex_count, v3d_surface_topology* out) {
    if (!out || (n_triangles && !triangles)) return V3D_ERR_INVALID_ARGUMENT;
    std::vector<MeshTriangle> tris(n_triangles);
    for (uint64_t t = 0; t < n_triangles; ++t) {
        if (triangles[t].a >= vertex_count || triangles[t].b >= vertex_count ||
            triangles[t].c >= vertex_count)
            return V3D_ERR_INVALID_ARGUMENT;
        tris[t] = MeshTriangle{(size_t)triangles[t].a, (size_t)triangles[t].b,
                               (size_t)triangles[t].c, triangles[t].confidence};
    }
    const Topology top = surface_topology(vertex_count, tris);
    out->islands = top.islands;
    out->small_islands = top.small_islands;
    out->small_island_triangles = top.small_island_triangles;
    out->largest_island_triangles = top.largest_island_triangles;
    out->boundary_edges = top.boundary_edges;
    return V3D_OK;
}

// The geometric part of the COLMAP export (colmap_surface.rs:380-471): per
// reference, verify every source and unite, mesh the union at the reference
// spacing with the reference-grid gates (mesh.rs:74-220 with no patches, which
// is mesh_legacy.rs:150-358 over all points), append the vertices in the order
// the triangles first use them, record the region; then topology and the
// dominant rejection.  Material baking and the GLB encoding are not part of it.
extern "C" int32_t v3do_mesh_verified_depth_grids(
    const v3d_depth_view* views, uint64_t n_views, const uint32_t* reference_views,
    uint64_t n_references, const int32_t* source_views, uint32_t stride, uint32_t reference_stride,
    double focal, v3d_point* points, v3d_grid_site* sites, uint64_t point_capacity,
    v3d_mesh_triangle* triangles, uint64_t triangle_capacity, v3d_verified_surface_region* regions,
    v3d_verified_surface* out) {
    if (!views || !n_views || !out || (n_references && (!reference_views || !source_views)) ||
        stride == 0 || reference_stride == 0 || reference_stride % stride != 0)
        return V3D_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    std::vector<DepthView> dv(n_views);
    std::vector<Camera> cameras(n_views);
    for (uint64_t i = 0; i < n_views; ++i) {
        if (views[i].width != views[0].width || views[i].height != views[0].height)
            return V3D_ERR_INVALID_ARGUMENT;
        for (uint64_t k = 0; k < i; ++k)
            if (views[k].camera.frame_index == views[i].camera.frame_index) return V3D_ERR_INVALID_ARGUMENT;
        dv[i].width = views[i].width;
        dv[i].height = views[i].height;
        dv[i].rgba = views[i].rgba;
        dv[i].depth = views[i].depth;
        dv[i].camera.frame_index = views[i].camera.frame_index;
        std::memcpy(dv[i].camera.R, views[i].camera.rotation, sizeof(dv[i].camera.R));
        std::memcpy(dv[i].camera.t, views[i].camera.translation, sizeof(dv[i].camera.t));
        cameras[i] = dv[i].camera;
    }
    for (uint64_t r = 0; r < n_references; ++r) {
        if (reference_views[r] >= n_views) return V3D_ERR_INVALID_ARGUMENT;
        for (int j = 0; j < 4; ++j)
            if (source_views[4 * r + j] >= (int64_t)n_views) return V3D_ERR_INVALID_ARGUMENT;
    }
    Funnel total;
    v3d_meshing_funnel m{};
    m.depth_views = n_views;
    std::vector<Point3> P;
    std::vector<GridSite> G;
    std::vector<MeshTriangle> T;
    std::vector<v3d_verified_surface_region> R;
    for (uint64_t r = 0; r < n_references; ++r) {
        const DepthView& ref = dv[reference_views[r]];
        std::vector<std::pair<size_t, std::vector<std::pair<Point3, GridSite>>>> cand;
        for (int j = 0; j < 4; ++j) {
            const int32_t s = source_views[4 * r + j];
            if (s < 0) continue;
            Funnel f;
            auto patch = verify_patch(ref, dv[s], stride, reference_stride, focal, f);
            total.add(f);
            cand.emplace_back((size_t)j, std::move(patch));
        }
        const std::vector<VerifiedSample> uni = verified_union(cand);
        for (const VerifiedSample& v : uni) m.multiply_verified_samples += v.sources.size() > 1;
        const size_t previous = T.size();
        if (!uni.empty()) {
            std::vector<Point3> p;
            std::vector<GridSite> g;
            for (const VerifiedSample& v : uni) {
                p.push_back(v.point);
                g.push_back(v.site);
            }
            MeshDenseInput d;
            d.attempted = true;
            d.reference_frame = ref.camera.frame_index;
            d.grid_stride = reference_stride;
            Control ctl;
            MeshAnalysis mesh = reconstruct_dense_mesh_with_control(p, g, d, cameras, ref.width, ref.height,
                                                                    focal, ctl);
            m.candidate_cells += mesh.stats.candidate_cells;
            m.rejected_discontinuities += mesh.stats.rejected_discontinuities;
            m.rejected_degenerate += mesh.stats.rejected_degenerate;
            const size_t start = P.size();
            std::vector<int64_t> index(p.size(), -1);
            std::vector<uint64_t> frames;
            for (MeshTriangle face : mesh.triangles) {
                for (size_t* corner : {&face.a, &face.b, &face.c}) {
                    const size_t i = *corner;
                    if (index[i] < 0) {
                        index[i] = (int64_t)P.size();
                        P.push_back(p[i]);
                        G.push_back(g[i]);
                        for (size_t j : uni[i].sources) {
                            const uint64_t f = dv[source_views[4 * r + j]].camera.frame_index;
                            if (std::find(frames.begin(), frames.end(), f) == frames.end()) frames.push_back(f);
                        }
                    }
                    *corner = (size_t)index[i];
                }
                T.push_back(face);
            }
            if (P.size() > start) {
                std::sort(frames.begin(), frames.end());
                v3d_verified_surface_region reg{};
                reg.reference_frame = ref.camera.frame_index;
                reg.first_point = start;
                reg.point_count = P.size() - start;
                reg.n_source_frames = (uint32_t)frames.size();
                for (size_t k = 0; k < frames.size(); ++k) reg.source_frames[k] = frames[k];
                R.push_back(reg);
            }
        }
        if (T.size() == previous) continue;
        ++m.meshed_reference_views;
    }
    out->verification = v3d_verification_funnel{
        total.reference_samples, total.missing_reference_depth, total.insufficient_parallax,
        total.behind_source,     total.outside_source,          total.missing_source_depth,
        total.depth_disagreement, total.color_disagreement,     total.accepted};
    m.exported_triangles = T.size();
    out->meshing = m;
    out->n_points = P.size();
    out->n_triangles = T.size();
    out->n_regions = R.size();
    if (T.empty()) return V3D_SKIPPED;  // "COLMAP stereo produced no cross-view verified surface triangles"
    const Topology top = surface_topology(P.size(), T);
    out->topology = v3d_surface_topology{top.islands, top.small_islands, top.small_island_triangles,
                                         top.largest_island_triangles, top.boundary_edges};
    static const char* const names[] = {"missing_reference_depth", "insufficient_parallax", "behind_source",
                                        "outside_source",          "missing_source_depth",  "depth_disagreement",
                                        "color_disagreement"};
    const char* dom = dominant_rejection(total);
    for (int k = 0; k < 7; ++k)
        if (dom && std::strcmp(dom, names[k]) == 0) out->dominant_rejection = k + 1;
    if (P.size() > point_capacity || T.size() > triangle_capacity || !points || !sites || !triangles || !regions)
        return V3D_ERR_INVALID_ARGUMENT;
    for (size_t i = 0; i < P.size(); ++i) {
        points[i] = v3d_point{P[i].x, P[i].y, P[i].z, P[i].confidence, P[i].r, P[i].g, P[i].b, 0};
        sites[i] = v3d_grid_site{G[i].x, G[i].y};
    }
    for (size_t t = 0; t < T.size(); ++t) triangles[t] = v3d_mesh_triangle{T[t].a, T[t].b, T[t].c, T[t].confidence, 0};
    std::copy(R.begin(), R.end(), regions);
    return V3D_OK;
}
