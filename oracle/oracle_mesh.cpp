// TEST INFRASTRUCTURE — CPU oracle, reference-grid triangle gates.
// Restates crates/video-to-3d-core/src/mesh_legacy.rs:150-555 and the
// multi-patch driver of mesh.rs:74-260 in f64.
#include <algorithm>
#include <cmath>
#include <limits>
#include <map>
#include <set>
#include <tuple>

#include "oracle.hpp"

namespace v3do {

namespace {
constexpr double kMaxGridReprojectionOffsetStrides = 0.5;  // mesh_legacy.rs:10
constexpr double kMaxMeshRelativeDepthJump = 0.15;         // :11
constexpr double kMaxBridgeRelativeDepthJump = 0.08;       // :12
constexpr double kMaxMeshEdgeFootprintMultiplier = 3.0;    // :13
constexpr double kMinMeshAreaFootprintRatio = 0.05;        // :14
constexpr double kMinMeshProjectedAreaFootprintRatio = 0.05;  // :15

struct GridVertex {
    size_t point_index;
    Vec3 position;
    double px, py, depth;
    float confidence;
};

enum class Rejection { None, Discontinuity, Degenerate };

MeshAnalysis skipped_mesh(std::optional<size_t> reference_frame, const char* reason) {
    MeshAnalysis m;
    m.stats.reference_frame = reference_frame;
    m.stats.skip_reason = reason;
    return m;
}

bool better_grid_vertex(const GridVertex& c, const GridVertex& cur) {
    return c.confidence > cur.confidence ||
           (c.confidence == cur.confidence && c.point_index < cur.point_index);
}

bool within_original_grid_footprint(double px, double py, GridSite s, size_t stride) {
    if (stride == 0 || !std::isfinite(px) || !std::isfinite(py)) return false;
    double limit = static_cast<double>(stride) * kMaxGridReprojectionOffsetStrides;
    return std::fabs(px - s.x) < limit && std::fabs(py - s.y) < limit;
}

std::optional<int32_t> original_grid_coordinate(uint32_t value, uint32_t limit, uint32_t border,
                                                size_t stride) {
    uint32_t lim = limit > border ? limit - border : 0;
    if (stride == 0 || value < border || value >= lim) return std::nullopt;
    size_t offset = value - border;
    if (offset % stride != 0) return std::nullopt;
    size_t g = offset / stride;
    if (g > static_cast<size_t>(std::numeric_limits<int32_t>::max())) return std::nullopt;
    return static_cast<int32_t>(g);
}

Rejection accepted_triangle(const GridVertex& a, const GridVertex& b, const GridVertex& c,
                            double stride, double focal, double max_jump, MeshTriangle& out) {
    // mesh_legacy.rs:473-537
    double d[3] = {a.depth, b.depth, c.depth};
    for (double v : d)
        if (!std::isfinite(v) || v <= 0.0) return Rejection::Discontinuity;
    double mn = std::numeric_limits<double>::infinity();
    double mx = -std::numeric_limits<double>::infinity();
    for (double v : d) {
        mn = std::fmin(mn, v);
        mx = std::fmax(mx, v);
    }
    if ((mx - mn) / mx > max_jump) return Rejection::Discontinuity;
    double spa = (b.px - a.px) * (c.py - a.py) - (b.py - a.py) * (c.px - a.px);
    double min_spa = stride * stride * kMinMeshProjectedAreaFootprintRatio;
    if (!std::isfinite(spa) || spa <= min_spa) return Rejection::Degenerate;
    double mean_depth = ((0.0 + d[0]) + d[1]) + d[2];
    mean_depth = mean_depth / 3.0;
    double local_step = mean_depth * stride / focal;
    double max_edge = local_step * 1.4142135623730951 * kMaxMeshEdgeFootprintMultiplier;
    double edges[3] = {norm(sub(a.position, b.position)), norm(sub(b.position, c.position)),
                       norm(sub(c.position, a.position))};
    for (double e : edges)
        if (!std::isfinite(e) || e > max_edge) return Rejection::Discontinuity;
    double area = norm(cross(sub(b.position, a.position), sub(c.position, a.position)));
    double min_area = local_step * local_step * kMinMeshAreaFootprintRatio;
    if (!std::isfinite(area) || area <= min_area) return Rejection::Degenerate;
    float conf = std::min(std::min(a.confidence, b.confidence), c.confidence);
    if (conf < 0.0f) conf = 0.0f;
    if (conf > 1.0f) conf = 1.0f;
    out = MeshTriangle{a.point_index, b.point_index, c.point_index, conf};
    return Rejection::None;
}

struct Build {
    std::set<std::tuple<size_t, size_t, size_t>> keys;
    std::vector<MeshTriangle> triangles;
    size_t candidates = 0, discontinuities = 0, degenerate = 0;
    void evaluate(const GridVertex (&t)[3], double stride, double focal, double jump) {
        size_t idx[3] = {t[0].point_index, t[1].point_index, t[2].point_index};
        std::sort(idx, idx + 3);
        if (!keys.insert({idx[0], idx[1], idx[2]}).second) return;
        ++candidates;
        MeshTriangle tri;
        switch (accepted_triangle(t[0], t[1], t[2], stride, focal, jump, tri)) {
            case Rejection::None: triangles.push_back(tri); break;
            case Rejection::Discontinuity: ++discontinuities; break;
            case Rejection::Degenerate: ++degenerate; break;
        }
    }
};
}  // namespace

MeshAnalysis reconstruct_dense_mesh_samples(const std::vector<Point3>& points,
                                            const std::vector<GridSite>& sites,
                                            const MeshDenseInput& dense,
                                            const std::vector<Camera>& cameras, uint32_t width,
                                            uint32_t height, double focal, Control& control) {
    // mesh_legacy.rs:150-358; samples = points.iter().zip(sites)
    size_t count = std::min(points.size(), sites.size());
    if (!dense.attempted)
        return skipped_mesh(dense.reference_frame, "dense reconstruction was not attempted");
    if (count < 3)
        return skipped_mesh(dense.reference_frame,
                            "fewer than three accepted fused dense points are available");
    if (dense.grid_stride == 0)
        return skipped_mesh(dense.reference_frame,
                            "dense reconstruction did not expose a valid reference-grid stride");
    if (width == 0 || height == 0 || !std::isfinite(focal) || focal <= 0.0)
        return skipped_mesh(dense.reference_frame,
                            "the reference camera does not provide finite positive projection "
                            "parameters");
    if (!dense.reference_frame)
        return skipped_mesh(std::nullopt, "dense reconstruction did not select a reference frame");
    size_t rf = *dense.reference_frame;
    const Camera* rc = nullptr;
    for (const Camera& c : cameras)
        if (c.frame_index == rf) {
            rc = &c;
            break;
        }
    if (!rc) return skipped_mesh(rf, "the dense reference frame has no accepted registered camera");
    const double stride = static_cast<double>(dense.grid_stride);
    std::map<std::pair<int32_t, int32_t>, GridVertex> grid;
    for (size_t i = 0; i < count; ++i) {
        if (control.is_canceled()) return skipped_mesh(dense.reference_frame, "mesh reconstruction canceled");
        const Point3& p = points[i];
        Vec3 pos{static_cast<double>(p.x), static_cast<double>(p.y), static_cast<double>(p.z)};
        auto q = project(*rc, pos, width, height, focal);
        if (!q) continue;
        if (!within_original_grid_footprint(q->x, q->y, sites[i], dense.grid_stride)) continue;
        auto gx = original_grid_coordinate(sites[i].x, width, dense.grid_border, dense.grid_stride);
        if (!gx) continue;
        auto gy = original_grid_coordinate(sites[i].y, height, dense.grid_border, dense.grid_stride);
        if (!gy) continue;
        GridVertex v{i, pos, q->x, q->y, q->z, p.confidence};
        auto it = grid.find({*gx, *gy});
        if (it == grid.end())
            grid.emplace(std::make_pair(*gx, *gy), v);
        else if (better_grid_vertex(v, it->second))
            it->second = v;
    }
    MeshAnalysis out;
    out.stats.reference_frame = rf;
    if (grid.size() < 3) {
        out.stats.attempted = true;
        out.stats.skip_reason =
            "fewer than three fused dense points align with the reference sampling grid";
        out.stats.grid_vertices = grid.size();
        out.stats.rejected_grid_vertices = count > grid.size() ? count - grid.size() : 0;
        return out;
    }
    auto get = [&](int32_t x, int32_t y) -> const GridVertex* {
        auto it = grid.find({x, y});
        return it == grid.end() ? nullptr : &it->second;
    };
    std::set<std::pair<int32_t, int32_t>> origins;
    for (auto& kv : grid)
        for (int dx : {-1, 0})
            for (int dy : {-1, 0}) origins.insert({kv.first.first + dx, kv.first.second + dy});
    Build b;
    size_t cells = 0;
    for (auto [gx, gy] : origins) {
        if (control.is_canceled()) return skipped_mesh(dense.reference_frame, "mesh reconstruction canceled");
        const GridVertex* tl = get(gx, gy);
        const GridVertex* tr = get(gx + 1, gy);
        const GridVertex* bl = get(gx, gy + 1);
        const GridVertex* br = get(gx + 1, gy + 1);
        int present = (tl != nullptr) + (tr != nullptr) + (bl != nullptr) + (br != nullptr);
        if (present < 3) continue;
        ++cells;
        // cell_triangles (mesh_legacy.rs:453-471)
        if (tl && tr && bl && br) {
            double d1 = norm_squared(sub(tl->position, br->position));
            double d2 = norm_squared(sub(tr->position, bl->position));
            if (d1 <= d2) {
                GridVertex t1[3] = {*tl, *tr, *br};
                GridVertex t2[3] = {*tl, *br, *bl};
                b.evaluate(t1, stride, focal, kMaxMeshRelativeDepthJump);
                b.evaluate(t2, stride, focal, kMaxMeshRelativeDepthJump);
            } else {
                GridVertex t1[3] = {*tl, *tr, *bl};
                GridVertex t2[3] = {*tr, *br, *bl};
                b.evaluate(t1, stride, focal, kMaxMeshRelativeDepthJump);
                b.evaluate(t2, stride, focal, kMaxMeshRelativeDepthJump);
            }
        } else if (tl && tr && bl) {
            GridVertex t[3] = {*tl, *tr, *bl};
            b.evaluate(t, stride, focal, kMaxMeshRelativeDepthJump);
        } else if (tl && tr && br) {
            GridVertex t[3] = {*tl, *tr, *br};
            b.evaluate(t, stride, focal, kMaxMeshRelativeDepthJump);
        } else if (tl && bl && br) {
            GridVertex t[3] = {*tl, *br, *bl};
            b.evaluate(t, stride, focal, kMaxMeshRelativeDepthJump);
        } else if (tr && bl && br) {
            GridVertex t[3] = {*tr, *br, *bl};
            b.evaluate(t, stride, focal, kMaxMeshRelativeDepthJump);
        }
    }
    int32_t minx = grid.begin()->first.first, maxx = minx;
    int32_t miny = grid.begin()->first.second, maxy = miny;
    for (auto& kv : grid) {
        minx = std::min(minx, kv.first.first);
        maxx = std::max(maxx, kv.first.first);
        miny = std::min(miny, kv.first.second);
        maxy = std::max(maxy, kv.first.second);
    }
    if (maxx - minx >= 2) {
        for (int32_t gx = minx; gx <= maxx - 2; ++gx) {
            if (control.is_canceled()) return skipped_mesh(dense.reference_frame, "mesh reconstruction canceled");
            for (int32_t gy = miny; gy <= maxy; ++gy) {
                // horizontal_gap_bridge (mesh_legacy.rs:370-394)
                const GridVertex* tl = get(gx, gy);
                const GridVertex* tr = get(gx + 2, gy);
                const GridVertex* bl = get(gx, gy + 1);
                const GridVertex* br = get(gx + 2, gy + 1);
                const GridVertex* tm = get(gx + 1, gy);
                const GridVertex* bm = get(gx + 1, gy + 1);
                if (tl && tr && !tm && bm) {
                    GridVertex t[3] = {*tl, *tr, *bm};
                    ++cells;
                    b.evaluate(t, stride, focal, kMaxBridgeRelativeDepthJump);
                } else if (bl && br && tm && !bm) {
                    GridVertex t[3] = {*bl, *tm, *br};
                    ++cells;
                    b.evaluate(t, stride, focal, kMaxBridgeRelativeDepthJump);
                }
            }
        }
    }
    if (maxy - miny >= 2) {
        for (int32_t gx = minx; gx <= maxx; ++gx) {
            if (control.is_canceled()) return skipped_mesh(dense.reference_frame, "mesh reconstruction canceled");
            for (int32_t gy = miny; gy <= maxy - 2; ++gy) {
                // vertical_gap_bridge (mesh_legacy.rs:396-420)
                const GridVertex* tl = get(gx, gy);
                const GridVertex* tr = get(gx + 1, gy);
                const GridVertex* bl = get(gx, gy + 2);
                const GridVertex* br = get(gx + 1, gy + 2);
                const GridVertex* lm = get(gx, gy + 1);
                const GridVertex* rm = get(gx + 1, gy + 1);
                if (tl && bl && !lm && rm) {
                    GridVertex t[3] = {*tl, *rm, *bl};
                    ++cells;
                    b.evaluate(t, stride, focal, kMaxBridgeRelativeDepthJump);
                } else if (tr && br && lm && !rm) {
                    GridVertex t[3] = {*tr, *br, *lm};
                    ++cells;
                    b.evaluate(t, stride, focal, kMaxBridgeRelativeDepthJump);
                }
            }
        }
    }
    out.stats.attempted = true;
    out.stats.grid_vertices = grid.size();
    out.stats.rejected_grid_vertices = count > grid.size() ? count - grid.size() : 0;
    out.stats.candidate_cells = cells;
    out.stats.candidate_triangles = b.candidates;
    out.stats.accepted_triangles = b.triangles.size();
    out.stats.rejected_discontinuities = b.discontinuities;
    out.stats.rejected_degenerate = b.degenerate;
    out.triangles = std::move(b.triangles);
    return out;
}

namespace {
MeshAnalysis mesh_from_legacy(MeshAnalysis r) {
    // mesh.rs:244-281
    if (r.stats.reference_frame) {
        r.reference_frames.push_back(*r.stats.reference_frame);
        MeshStats p = r.stats;
        p.point_count = r.stats.grid_vertices + r.stats.rejected_grid_vertices;
        r.reference_patches.push_back(p);
    }
    return r;
}
}  // namespace

MeshAnalysis reconstruct_dense_mesh_with_control(const std::vector<Point3>& points,
                                                 const std::vector<GridSite>& sites,
                                                 const MeshDenseInput& dense,
                                                 const std::vector<Camera>& cameras,
                                                 uint32_t width, uint32_t height, double focal,
                                                 Control& control) {
    // mesh.rs:74-220
    if (dense.reference_patches.empty()) {
        if (dense.attempted && points.size() >= 3 && points.size() != sites.size())
            return mesh_from_legacy(skipped_mesh(
                dense.reference_frame, "dense point and reference-grid evidence counts disagree"));
        return mesh_from_legacy(reconstruct_dense_mesh_samples(points, sites, dense, cameras,
                                                               width, height, focal, control));
    }
    MeshAnalysis out;
    bool attempted = false;
    for (const PatchStats& patch : dense.reference_patches) {
        if (control.is_canceled()) return MeshAnalysis{};
        // patch_point_indices (mesh.rs:222-240)
        bool ok = points.size() == sites.size();
        size_t pe = patch.primary_start + patch.primary_points;
        size_t ce = patch.completion_start + patch.completed_points;
        if (ok && (pe < patch.primary_start || ce < patch.completion_start)) ok = false;
        if (ok && (pe > points.size() || ce > points.size())) ok = false;
        if (!ok) {
            MeshStats ps;
            ps.reference_frame = patch.reference_frame;
            ps.point_count = patch.accepted_points;
            ps.skip_reason = "dense patch ranges exceed the accepted point evidence";
            out.reference_patches.push_back(ps);
            continue;
        }
        std::vector<size_t> idx;
        for (size_t i = patch.primary_start; i < pe; ++i) idx.push_back(i);
        for (size_t i = patch.completion_start; i < ce; ++i) idx.push_back(i);
        std::vector<Point3> pp;
        std::vector<GridSite> ss;
        for (size_t i : idx) {
            pp.push_back(points[i]);
            ss.push_back(sites[i]);
        }
        MeshDenseInput pd;
        pd.attempted = true;
        pd.reference_frame = patch.reference_frame;
        pd.grid_stride = patch.grid_stride;
        pd.grid_border = patch.grid_border;
        MeshAnalysis r = reconstruct_dense_mesh_samples(pp, ss, pd, cameras, width, height, focal,
                                                        control);
        attempted |= r.stats.attempted;
        out.stats.grid_vertices += r.stats.grid_vertices;
        out.stats.rejected_grid_vertices += r.stats.rejected_grid_vertices;
        out.stats.candidate_cells += r.stats.candidate_cells;
        out.stats.candidate_triangles += r.stats.candidate_triangles;
        out.stats.rejected_discontinuities += r.stats.rejected_discontinuities;
        out.stats.rejected_degenerate += r.stats.rejected_degenerate;
        size_t accepted_here = 0;
        for (const MeshTriangle& t : r.triangles) {
            if (t.a >= idx.size() || t.b >= idx.size() || t.c >= idx.size()) continue;
            out.triangles.push_back({idx[t.a], idx[t.b], idx[t.c], t.confidence});
            ++accepted_here;
        }
        (void)accepted_here;
        MeshStats ps = r.stats;
        ps.reference_frame = patch.reference_frame;
        ps.point_count = idx.size();
        ps.accepted_triangles = r.triangles.size();
        out.reference_patches.push_back(ps);
    }
    for (const MeshStats& p : out.reference_patches)
        out.reference_frames.push_back(p.reference_frame.value_or(0));
    out.stats.attempted = attempted;
    if (out.triangles.empty())
        out.stats.skip_reason = "no reference patch produced an accepted surface triangle";
    if (!out.reference_frames.empty()) out.stats.reference_frame = out.reference_frames.front();
    out.stats.accepted_triangles = out.triangles.size();
    return out;
}

}  // namespace v3do
