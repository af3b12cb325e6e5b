// TEST INFRASTRUCTURE — extern "C" surface of the CPU oracle.
// tests/ use it as the parity checker and bench.py's CPU-baseline leg times
// v3do_reconstruct_reference_patches with OpenMP over references.  The result
// structs are the public ones of include/v3d_dense.h so that the GPU library
// and the oracle can be compared field by field.
#include <omp.h>

#include <cstdlib>
#include <cstring>
#include <memory>
#include <stdexcept>

#include "oracle.hpp"

using namespace v3do;

namespace {

struct Owner {
    std::vector<std::vector<uint64_t>> patch_sources;
};

std::vector<Frame> load_frames(const v3d_frame* frames, uint64_t n) {
    std::vector<Frame> out(n);
    for (uint64_t i = 0; i < n; ++i) {
        Frame& f = out[i];
        f.width = frames[i].width;
        f.height = frames[i].height;
        f.format = frames[i].format;
        size_t bpp = f.format == V3D_PIXEL_RGBA8 ? 4 : f.format == V3D_PIXEL_GRAY_F32 ? 4 : 2;
        size_t bytes = static_cast<size_t>(f.width) * f.height * bpp;
        const uint8_t* p = static_cast<const uint8_t*>(frames[i].data);
        if (p && bytes) f.bytes.assign(p, p + bytes);
    }
    return out;
}

std::vector<Camera> load_cameras(const v3d_camera* cams, uint64_t n) {
    std::vector<Camera> out(n);
    for (uint64_t i = 0; i < n; ++i) {
        out[i].frame_index = cams[i].frame_index;
        std::memcpy(out[i].R, cams[i].rotation, sizeof(out[i].R));
        std::memcpy(out[i].t, cams[i].translation, sizeof(out[i].t));
    }
    return out;
}

std::vector<Vec3> load_sparse(const double* xyz, uint64_t n) {
    std::vector<Vec3> out(n);
    for (uint64_t i = 0; i < n; ++i) out[i] = {xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]};
    return out;
}

Control make_control(v3d_cancel_fn fn, void* user) {
    Control c;
    if (fn) c.poll = [fn, user]() { return fn(user) != 0; };
    return c;
}

void put_reason(char* dst, const std::optional<std::string>& s, int32_t* has) {
    std::memset(dst, 0, V3D_SKIP_REASON_BYTES);
    *has = s.has_value();
    if (s) std::strncpy(dst, s->c_str(), V3D_SKIP_REASON_BYTES - 1);
}

void put_opt(const std::optional<float>& v, int32_t* has, float* dst) {
    *has = v.has_value();
    *dst = v.value_or(0.0f);
}

template <class T>
T* dup(const std::vector<T>& v) {
    if (v.empty()) return nullptr;
    T* p = static_cast<T*>(std::malloc(sizeof(T) * v.size()));
    std::memcpy(p, v.data(), sizeof(T) * v.size());
    return p;
}

void fill_stats(v3d_dense_stats& s, const LegacyStats& l) {
    std::memset(&s, 0, sizeof(s));
    s.attempted = l.attempted;
    s.skip_code = l.skip_reason ? (l.skip_code ? l.skip_code : -1) : 0;
    put_reason(s.skip_reason, l.skip_reason, &s.has_skip_reason);
    s.has_reference_frame = l.reference_frame.has_value();
    s.reference_frame = l.reference_frame.value_or(0);
    s.source_views = l.source_views;
    s.sampled_pixels = l.sampled_pixels;
    s.depth_hypotheses = l.depth_hypotheses;
    s.accepted_points = l.accepted_points;
    s.surface_completion_proposals = l.surface_completion_proposals;
    s.surface_completed_points = l.surface_completed_points;
    s.surface_completion_rejected_texture = l.surface_completion_rejected_texture;
    s.surface_completion_rejected_cross_view = l.surface_completion_rejected_cross_view;
    s.surface_completion_rejected_reciprocal = l.surface_completion_rejected_reciprocal;
    s.surface_completion_rejected_fusion = l.surface_completion_rejected_fusion;
    s.surface_completion_rejected_footprint = l.surface_completion_rejected_footprint;
    s.grid_stride = l.grid_stride;
    s.grid_border = l.grid_border;
    s.reciprocal_checked_points = l.reciprocal_checked_points;
    s.reciprocal_rejected_points = l.reciprocal_rejected_points;
    s.reciprocal_consistent_points = l.reciprocal_consistent_points;
    s.fusion_input_observations = l.fusion_input_observations;
    s.fusion_rejected_observations = l.fusion_rejected_observations;
    s.fusion_rejected_points = l.fusion_rejected_points;
    put_opt(l.median_fusion_observations, &s.has_median_fusion_observations,
            &s.median_fusion_observations);
    put_opt(l.median_supporting_views, &s.has_median_supporting_views, &s.median_supporting_views);
    put_opt(l.median_photometric_error, &s.has_median_photometric_error,
            &s.median_photometric_error);
    put_opt(l.search_min_depth, &s.has_search_min_depth, &s.search_min_depth);
    put_opt(l.search_max_depth, &s.has_search_max_depth, &s.search_max_depth);
}

template <class A>
void fill_arrays(v3d_dense_result* out, const A& a) {
    std::vector<uint64_t> sf(a.stats.source_frames.begin(), a.stats.source_frames.end());
    out->n_source_frames = sf.size();
    out->source_frames = dup(sf);
    out->n_points = a.points.size();
    std::vector<v3d_point> pts(a.points.size());
    for (size_t i = 0; i < a.points.size(); ++i) {
        const Point3& p = a.points[i];
        pts[i] = {p.x, p.y, p.z, p.confidence, p.r, p.g, p.b, 0};
    }
    out->points = dup(pts);
    std::vector<v3d_grid_site> sites(a.grid_sites.size());
    for (size_t i = 0; i < sites.size(); ++i) sites[i] = {a.grid_sites[i].x, a.grid_sites[i].y};
    out->grid_sites = dup(sites);
    std::vector<v3d_point_attributes> attrs(a.point_attributes.size());
    for (size_t i = 0; i < attrs.size(); ++i)
        attrs[i] = {a.point_attributes[i].reciprocal_consistency, a.point_attributes[i].depth_margin};
    out->point_attributes = dup(attrs);
}

void fill_legacy(v3d_dense_result* out, const LegacyAnalysis& a) {
    std::memset(out, 0, sizeof(*out));
    fill_stats(out->stats, a.stats);
    fill_arrays(out, a);
}

void fill_dense(v3d_dense_result* out, const DenseAnalysis& a) {
    std::memset(out, 0, sizeof(*out));
    fill_stats(out->stats, a.stats);
    out->stats.has_reference_view_limit = a.stats.reference_view_limit.has_value();
    out->stats.reference_view_limit = a.stats.reference_view_limit.value_or(0);
    fill_arrays(out, a);
    std::vector<uint64_t> rf(a.stats.reference_frames.begin(), a.stats.reference_frames.end());
    out->n_reference_frames = rf.size();
    out->reference_frames = dup(rf);
    std::vector<v3d_reference_attempt> at(a.stats.reference_attempts.size());
    for (size_t i = 0; i < at.size(); ++i) {
        const AttemptStats& s = a.stats.reference_attempts[i];
        v3d_reference_attempt& d = at[i];
        std::memset(&d, 0, sizeof(d));
        d.reference_frame = s.reference_frame;
        d.attempted = s.attempted;
        d.accepted = s.accepted;
        put_reason(d.skip_reason, s.skip_reason, &d.has_skip_reason);
        d.sampled_pixels = s.sampled_pixels;
        d.accepted_points = s.accepted_points;
        d.reciprocal_checked_points = s.reciprocal_checked_points;
        d.reciprocal_rejected_points = s.reciprocal_rejected_points;
        d.reciprocal_consistent_points = s.reciprocal_consistent_points;
        d.surface_completion_proposals = s.surface_completion_proposals;
        d.surface_completed_points = s.surface_completed_points;
        d.surface_completion_rejected_texture = s.surface_completion_rejected_texture;
        d.surface_completion_rejected_cross_view = s.surface_completion_rejected_cross_view;
        d.surface_completion_rejected_reciprocal = s.surface_completion_rejected_reciprocal;
        d.surface_completion_rejected_fusion = s.surface_completion_rejected_fusion;
        d.surface_completion_rejected_footprint = s.surface_completion_rejected_footprint;
    }
    out->n_attempts = at.size();
    out->attempts = dup(at);
    auto* owner = new Owner;
    std::vector<v3d_reference_patch> ps(a.stats.reference_patches.size());
    for (size_t i = 0; i < ps.size(); ++i) {
        const PatchStats& s = a.stats.reference_patches[i];
        v3d_reference_patch& d = ps[i];
        std::memset(&d, 0, sizeof(d));
        owner->patch_sources.emplace_back(s.source_frames.begin(), s.source_frames.end());
        d.reference_frame = s.reference_frame;
        d.primary_start = s.primary_start;
        d.primary_points = s.primary_points;
        d.completion_start = s.completion_start;
        d.completed_points = s.completed_points;
        d.sampled_pixels = s.sampled_pixels;
        d.accepted_points = s.accepted_points;
        d.reciprocal_consistent_points = s.reciprocal_consistent_points;
        d.grid_stride = s.grid_stride;
        d.grid_border = s.grid_border;
        put_opt(s.search_min_depth, &d.has_search_min_depth, &d.search_min_depth);
        put_opt(s.search_max_depth, &d.has_search_max_depth, &d.search_max_depth);
    }
    for (size_t i = 0; i < ps.size(); ++i) {
        ps[i].n_source_frames = owner->patch_sources[i].size();
        ps[i].source_frames = owner->patch_sources[i].data();
    }
    out->n_patches = ps.size();
    out->patches = dup(ps);
    out->internal = owner;
}

void fill_mesh_stats(v3d_mesh_stats& d, const MeshStats& s) {
    std::memset(&d, 0, sizeof(d));
    d.attempted = s.attempted;
    put_reason(d.skip_reason, s.skip_reason, &d.has_skip_reason);
    d.has_reference_frame = s.reference_frame.has_value();
    d.reference_frame = s.reference_frame.value_or(0);
    d.point_count = s.point_count;
    d.grid_vertices = s.grid_vertices;
    d.rejected_grid_vertices = s.rejected_grid_vertices;
    d.candidate_cells = s.candidate_cells;
    d.candidate_triangles = s.candidate_triangles;
    d.accepted_triangles = s.accepted_triangles;
    d.rejected_discontinuities = s.rejected_discontinuities;
    d.rejected_degenerate = s.rejected_degenerate;
}

}  // namespace

extern "C" {

void v3do_dense_result_free(v3d_dense_result* r) {
    if (!r) return;
    std::free(r->source_frames);
    std::free(r->points);
    std::free(r->grid_sites);
    std::free(r->point_attributes);
    std::free(r->reference_frames);
    std::free(r->attempts);
    std::free(r->patches);
    delete static_cast<Owner*>(r->internal);
    std::memset(r, 0, sizeof(*r));
}

void v3do_mesh_result_free(v3d_mesh_result* r) {
    if (!r) return;
    std::free(r->triangles);
    std::free(r->reference_frames);
    std::free(r->patches);
    std::memset(r, 0, sizeof(*r));
}

int32_t v3do_estimate_depth_points_with_control(const v3d_frame* frames, uint64_t n_frames,
                                                const v3d_camera* cams, uint64_t n_cams,
                                                const double* sparse, uint64_t n_sparse,
                                                double focal, int32_t fine_grid,
                                                const v3d_profile* profile, v3d_cancel_fn cancel,
                                                void* user, v3d_dense_result* out) {
    try {
        auto f = load_frames(frames, n_frames);
        auto c = load_cameras(cams, n_cams);
        auto s = load_sparse(sparse, n_sparse);
        Control ctl = make_control(cancel, user);
        LegacyAnalysis a = estimate_depth_points_with_control(Profile::from_c(*profile), f, c, s,
                                                              focal, fine_grid != 0, ctl);
        fill_legacy(out, a);
        return a.stats.attempted ? V3D_OK : V3D_SKIPPED;
    } catch (const std::invalid_argument&) {
        std::memset(out, 0, sizeof(*out));
        return V3D_ERR_INVALID_ARGUMENT;
    }
}

int32_t v3do_reconstruct_reference_patches(const v3d_frame* frames, uint64_t n_frames,
                                           const v3d_camera* cams, uint64_t n_cams,
                                           const double* sparse, uint64_t n_sparse, double focal,
                                           int32_t fine_grid, const v3d_profile* profile,
                                           const uint64_t* camera_indices, uint64_t n_refs,
                                           int32_t threads, v3d_dense_result* out,
                                           int32_t* present) {
    auto f = load_frames(frames, n_frames);
    auto c = load_cameras(cams, n_cams);
    auto s = load_sparse(sparse, n_sparse);
    Profile prof = Profile::from_c(*profile);
    int32_t status = V3D_OK;
#pragma omp parallel for schedule(dynamic, 1) num_threads(threads > 0 ? threads : 1)
    for (int64_t i = 0; i < static_cast<int64_t>(n_refs); ++i) {
        Control ctl;
        try {
            auto a = reconstruct_reference_patch(prof, f, c, s, focal, camera_indices[i],
                                                 fine_grid != 0, ctl);
            present[i] = a.has_value();
            if (a)
                fill_legacy(&out[i], *a);
            else
                std::memset(&out[i], 0, sizeof(out[i]));
        } catch (const std::invalid_argument&) {
            std::memset(&out[i], 0, sizeof(out[i]));
            present[i] = 0;
#pragma omp atomic write
            status = V3D_ERR_INVALID_ARGUMENT;
        }
    }
    return status;
}

int32_t v3do_estimate_depth_points_limited(const v3d_frame* frames, uint64_t n_frames,
                                           const v3d_camera* cams, uint64_t n_cams,
                                           const double* sparse, uint64_t n_sparse, double focal,
                                           uint64_t reference_views, int32_t fine_grid,
                                           const v3d_profile* profile, v3d_cancel_fn cancel,
                                           void* user, v3d_dense_result* out,
                                           int32_t* omitted) {
    try {
        auto f = load_frames(frames, n_frames);
        auto c = load_cameras(cams, n_cams);
        auto s = load_sparse(sparse, n_sparse);
        Control ctl = make_control(cancel, user);
        auto r = estimate_depth_points_limited(Profile::from_c(*profile), f, c, s, focal,
                                               reference_views, fine_grid != 0, ctl);
        fill_dense(out, r.first);
        *omitted = r.second;
        return r.first.stats.attempted ? V3D_OK : V3D_SKIPPED;
    } catch (const std::invalid_argument&) {
        std::memset(out, 0, sizeof(*out));
        return V3D_ERR_INVALID_ARGUMENT;
    }
}

int32_t v3do_has_distributed_landmarks(const v3d_frame* frames, uint64_t n_frames,
                                       const v3d_camera* cams, uint64_t n_cams,
                                       const double* sparse, uint64_t n_sparse, double focal,
                                       v3d_cancel_fn cancel, void* user) {
    // Only sizes are read; no pixel data is copied.
    std::vector<Frame> f(n_frames);
    for (uint64_t i = 0; i < n_frames; ++i) {
        f[i].width = frames[i].width;
        f[i].height = frames[i].height;
    }
    auto c = load_cameras(cams, n_cams);
    auto s = load_sparse(sparse, n_sparse);
    Control ctl = make_control(cancel, user);
    return has_distributed_landmarks(f, c, s, focal, ctl) ? 1 : 0;
}

int32_t v3do_reference_candidate_order(const v3d_frame* frames, uint64_t n_frames,
                                       const v3d_camera* cams, uint64_t n_cams,
                                       const double* sparse, uint64_t n_sparse, double focal,
                                       uint64_t* order, uint64_t* n_order) {
    std::vector<Frame> f(n_frames);
    for (uint64_t i = 0; i < n_frames; ++i) {
        f[i].width = frames[i].width;
        f[i].height = frames[i].height;
    }
    auto c = load_cameras(cams, n_cams);
    auto s = load_sparse(sparse, n_sparse);
    auto o = reference_candidate_order(f, c, s, focal);
    for (size_t i = 0; i < o.size(); ++i) order[i] = o[i];
    *n_order = o.size();
    return V3D_OK;
}

uint64_t v3do_grid_stride(uint32_t w, uint32_t h, int32_t fine) { return grid_stride(w, h, fine != 0); }

int32_t v3do_reconstruct_dense_mesh_with_control(
    const v3d_point* points, uint64_t n_points, const v3d_grid_site* sites, uint64_t n_sites,
    const v3d_mesh_dense_input* dense, const v3d_camera* cams, uint64_t n_cams, uint32_t width,
    uint32_t height, double focal, v3d_cancel_fn cancel, void* user, v3d_mesh_result* out) {
    std::vector<Point3> p(n_points);
    for (uint64_t i = 0; i < n_points; ++i)
        p[i] = {points[i].x, points[i].y, points[i].z, points[i].confidence,
                points[i].r, points[i].g, points[i].b};
    std::vector<GridSite> s(n_sites);
    for (uint64_t i = 0; i < n_sites; ++i) s[i] = {sites[i].x, sites[i].y};
    MeshDenseInput d;
    d.attempted = dense->attempted != 0;
    if (dense->has_reference_frame) d.reference_frame = dense->reference_frame;
    d.grid_stride = dense->grid_stride;
    d.grid_border = dense->grid_border;
    for (uint64_t i = 0; i < dense->n_patches; ++i) {
        const v3d_reference_patch& q = dense->patches[i];
        PatchStats ps;
        ps.reference_frame = q.reference_frame;
        ps.primary_start = q.primary_start;
        ps.primary_points = q.primary_points;
        ps.completion_start = q.completion_start;
        ps.completed_points = q.completed_points;
        ps.accepted_points = q.accepted_points;
        ps.grid_stride = q.grid_stride;
        ps.grid_border = q.grid_border;
        d.reference_patches.push_back(ps);
    }
    auto c = load_cameras(cams, n_cams);
    Control ctl = make_control(cancel, user);
    MeshAnalysis m = reconstruct_dense_mesh_with_control(p, s, d, c, width, height, focal, ctl);
    std::memset(out, 0, sizeof(*out));
    fill_mesh_stats(out->stats, m.stats);
    std::vector<v3d_mesh_triangle> tris(m.triangles.size());
    for (size_t i = 0; i < tris.size(); ++i)
        tris[i] = {m.triangles[i].a, m.triangles[i].b, m.triangles[i].c, m.triangles[i].confidence, 0};
    out->n_triangles = tris.size();
    out->triangles = dup(tris);
    std::vector<uint64_t> rf(m.reference_frames.begin(), m.reference_frames.end());
    out->n_reference_frames = rf.size();
    out->reference_frames = dup(rf);
    std::vector<v3d_mesh_stats> ps(m.reference_patches.size());
    for (size_t i = 0; i < ps.size(); ++i) fill_mesh_stats(ps[i], m.reference_patches[i]);
    out->n_patches = ps.size();
    out->patches = dup(ps);
    return V3D_OK;
}

// One f64 window cost (dense_legacy.rs:1032-1095 and the ZNCC profile) between
// reference pixel (x, y) at `depth` and a source view; returns 0 and writes
// *cost, or -1 where the reference returns None.  Used to state the cost
// error of the f32 device path against f64.
int32_t v3do_patch_error(const v3d_profile* profile, const v3d_camera* ref_cam,
                         const v3d_camera* src_cam, const v3d_frame* ref_frame,
                         const v3d_frame* src_frame, double x, double y, double depth,
                         double focal, double* cost) {
    auto f = load_frames(ref_frame, 1);
    auto g = load_frames(src_frame, 1);
    auto c = load_cameras(ref_cam, 1);
    auto d = load_cameras(src_cam, 1);
    Plane a = to_luma(f[0]), b = to_luma(g[0]);
    auto e = patch_error(Profile::from_c(*profile), c[0], d[0], a, b, x, y, depth, focal);
    if (!e) return -1;
    *cost = *e;
    return 0;
}

int32_t v3do_max_threads(void) { return omp_get_max_threads(); }

// Bounded CPU-baseline sample: the remapped pass of `camera_index` restricted
// to grid rows [row_begin, row_end), split across `threads` OpenMP threads
// (each sweeps its own rows), completion skipped.  Reports wall seconds and
// the units (sites x hypotheses x source views) swept.
int32_t v3do_time_rows(const v3d_frame* frames, uint64_t n_frames, const v3d_camera* cams,
                       uint64_t n_cams, const double* sparse, uint64_t n_sparse, double focal,
                       const v3d_profile* profile, uint64_t camera_index, uint32_t row_begin,
                       uint32_t row_end, int32_t threads, double* seconds, uint64_t* units) {
    auto f = load_frames(frames, n_frames);
    auto c = load_cameras(cams, n_cams);
    auto s = load_sparse(sparse, n_sparse);
    Profile prof = Profile::from_c(*profile);
    int t = threads > 0 ? threads : 1;
    uint32_t rows = row_end > row_begin ? row_end - row_begin : 0;
    std::vector<RowBand> bands(t);
    for (int i = 0; i < t; ++i) {
        bands[i].begin = row_begin + static_cast<uint32_t>((uint64_t)rows * i / t);
        bands[i].end = row_begin + static_cast<uint32_t>((uint64_t)rows * (i + 1) / t);
    }
    double t0 = omp_get_wtime();
#pragma omp parallel for schedule(static, 1) num_threads(t)
    for (int i = 0; i < t; ++i) {
        Control ctl;
        try {
            reconstruct_reference_patch(prof, f, c, s, focal, camera_index, false, ctl, &bands[i]);
        } catch (const std::invalid_argument&) {
        }
    }
    *seconds = omp_get_wtime() - t0;
    uint64_t u = 0;
    for (auto& b : bands) u += b.units;
    *units = u;
    return V3D_OK;
}

// Per-site sweep outcome of the per-reference pass, the oracle side of v3d_debug_sweep.
int32_t v3do_debug_sweep(const v3d_frame* frames, uint64_t n_frames, const v3d_camera* cams,
                         uint64_t n_cams, const double* sparse, uint64_t n_sparse, double focal,
                         int32_t fine_grid, const v3d_profile* profile, v3d_site_record* out,
                         uint64_t capacity, uint64_t* n_sites) {
    auto f = load_frames(frames, n_frames);
    std::vector<const Frame*> ptrs;
    for (const Frame& x : f) ptrs.push_back(&x);
    auto c = load_cameras(cams, n_cams);
    auto s = load_sparse(sparse, n_sparse);
    Control ctl;
    std::vector<v3d_site_record> rec;
    LegacyAnalysis a;
    try {
        a = estimate_depth_points_ptr(Profile::from_c(*profile), ptrs, c, s, focal, fine_grid != 0,
                                      ctl, &rec);
    } catch (const std::invalid_argument&) {
        return V3D_ERR_INVALID_ARGUMENT;
    }
    *n_sites = rec.size();
    if (!a.stats.attempted && a.stats.skip_reason) return V3D_SKIPPED;
    if (!out || capacity < rec.size()) return V3D_ERR_INVALID_ARGUMENT;
    std::memcpy(out, rec.data(), sizeof(v3d_site_record) * rec.size());
    return V3D_OK;
}

// The remapped pass of one reference camera (as v3do_reconstruct_reference_patches
// runs it), or with camera_index == UINT64_MAX the legacy single call (as
// v3do_estimate_depth_points_with_control runs it), together with its
// ExplainRecords (oracle.hpp): primary sites in raster order, then each
// completion pass's proposals.  row_end > row_begin restricts the pass to
// those grid rows (primaries only, no completion, as the CPU-baseline bands
// run).  *records is malloc'd; free it with v3do_free.  Returns V3D_SKIPPED
// (and no result) where the pass does not run.
int32_t v3do_explain_reference_patch(const v3d_frame* frames, uint64_t n_frames,
                                     const v3d_camera* cams, uint64_t n_cams,
                                     const double* sparse, uint64_t n_sparse, double focal,
                                     int32_t fine_grid, const v3d_profile* profile,
                                     uint64_t camera_index, uint32_t row_begin,
                                     uint32_t row_end, v3d_dense_result* out,
                                     ExplainRecord** records, uint64_t* n_records) {
    static_assert(sizeof(ExplainRecord) == 56, "ExplainRecord layout");
    *records = nullptr;
    *n_records = 0;
    std::memset(out, 0, sizeof(*out));
    auto f = load_frames(frames, n_frames);
    auto c = load_cameras(cams, n_cams);
    auto s = load_sparse(sparse, n_sparse);
    Control ctl;
    std::vector<ExplainRecord> rec;
    RowBand band;
    band.begin = row_begin;
    band.end = row_end;
    const RowBand* bp = row_end > row_begin ? &band : nullptr;
    try {
        std::optional<LegacyAnalysis> a;
        if (camera_index == UINT64_MAX) {
            std::vector<const Frame*> ptrs;
            for (const Frame& x : f) ptrs.push_back(&x);
            a = estimate_depth_points_ptr(Profile::from_c(*profile), ptrs, c, s, focal,
                                          fine_grid != 0, ctl, nullptr, bp, &rec);
            if (!bp && !a->stats.attempted) return V3D_SKIPPED;
        } else {
            a = reconstruct_reference_patch(Profile::from_c(*profile), f, c, s, focal,
                                            camera_index, fine_grid != 0, ctl, bp, &rec);
        }
        if (!a) return V3D_SKIPPED;
        fill_legacy(out, *a);
    } catch (const std::invalid_argument&) {
        return V3D_ERR_INVALID_ARGUMENT;
    }
    *records = dup(rec);
    *n_records = rec.size();
    return V3D_OK;
}

void v3do_free(void* p) { std::free(p); }

// estimate_working_set (dense.rs:423-605), twelve u64 fields in
// DenseWorkingSetEstimate order.
int32_t v3do_estimate_working_set(const v3d_frame* frames, uint64_t n_frames,
                                  uint64_t max_features, uint32_t descriptor_radius,
                                  uint64_t reference_views, int32_t fine_grid, uint64_t* out) {
    auto f = load_frames(frames, n_frames);
    WorkingSet w = estimate_working_set(f, max_features, descriptor_radius, reference_views,
                                        fine_grid != 0);
    const uint64_t v[12] = {w.frame_bytes, w.retry_frame_bytes, w.remapped_frame_bytes,
                            w.luminance_bytes, w.sparse_pipeline_bytes, w.dense_sample_bytes,
                            w.topology_bytes, w.mesh_builder_bytes, w.surface_fusion_bytes,
                            w.retained_candidate_bytes, w.packed_output_bytes, w.total_bytes};
    std::memcpy(out, v, sizeof(v));
    return V3D_OK;
}

// estimate_depth_points_with_budget_and_control (dense.rs:355-420): the result,
// and in plan[0..16) the estimate (12 fields), the budget, the full plan's
// bytes, the fine-grid flag and the plan's reference views (0: budget skip).
int32_t v3do_estimate_depth_points_with_budget(const v3d_frame* frames, uint64_t n_frames,
                                               const v3d_camera* cams, uint64_t n_cams,
                                               const double* sparse, uint64_t n_sparse,
                                               double focal, uint64_t budget,
                                               uint64_t max_features, uint32_t descriptor_radius,
                                               const v3d_profile* profile, v3d_cancel_fn cancel,
                                               void* user, v3d_dense_result* out,
                                               uint64_t* plan) {
    try {
        auto f = load_frames(frames, n_frames);
        auto c = load_cameras(cams, n_cams);
        auto s = load_sparse(sparse, n_sparse);
        Control ctl = make_control(cancel, user);
        BudgetedAnalysis b = estimate_depth_points_with_budget(
            Profile::from_c(*profile), f, c, s, focal, budget, max_features, descriptor_radius,
            ctl);
        const WorkingSet& w = b.estimate;
        const uint64_t v[16] = {w.frame_bytes, w.retry_frame_bytes, w.remapped_frame_bytes,
                                w.luminance_bytes, w.sparse_pipeline_bytes, w.dense_sample_bytes,
                                w.topology_bytes, w.mesh_builder_bytes, w.surface_fusion_bytes,
                                w.retained_candidate_bytes, w.packed_output_bytes, w.total_bytes,
                                b.budget_bytes, b.full_bytes, b.fine_grid ? 1u : 0u,
                                b.reference_views};
        std::memcpy(plan, v, sizeof(v));
        fill_dense(out, b.analysis);
        if (b.reference_views == 0) out->stats.skip_code = V3D_SKIP_WORKING_SET_BUDGET;
        return b.analysis.stats.attempted ? V3D_OK : V3D_SKIPPED;
    } catch (const std::invalid_argument&) {
        std::memset(out, 0, sizeof(*out));
        return V3D_ERR_INVALID_ARGUMENT;
    }
}

}  // extern "C"
