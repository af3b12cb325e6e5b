// C ABI of the reference-grid triangle gates: mesh.rs:74-260 over the device
// pass of mesh_legacy.rs:150-358 (mesh_kernels.cu).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdlib>
#include <cstring>
#include <string>

#include "host.hpp"

using namespace v3d;

namespace {

template <class T>
T* dup(const std::vector<T>& v) {
    if (v.empty()) return nullptr;
    T* p = static_cast<T*>(std::malloc(sizeof(T) * v.size()));
    if (p) std::memcpy(p, v.data(), sizeof(T) * v.size());
    return p;
}

void mesh_skip(v3d_mesh_stats& s, bool has_ref, uint64_t ref, const char* reason) {
    std::memset(&s, 0, sizeof(s));
    s.has_reference_frame = has_ref;
    s.reference_frame = ref;
    s.has_skip_reason = 1;
    std::strncpy(s.skip_reason, reason, V3D_SKIP_REASON_BYTES - 1);
}

// legacy::reconstruct_dense_mesh_samples (mesh_legacy.rs:150-358)
int32_t legacy_mesh(v3d_context* ctx, const v3d_point* pts, const v3d_grid_site* sites,
                    const std::vector<uint32_t>& map, size_t n_src, size_t count, bool attempted,
                    bool has_ref, uint64_t ref, uint64_t stride, uint32_t border,
                    const v3d_camera* cams, uint64_t n_cams, uint32_t width, uint32_t height,
                    double focal, CancelPoll& cancel, v3d_mesh_stats& stats,
                    std::vector<v3d_mesh_triangle>& tris) {
    tris.clear();
    if (!attempted) {
        mesh_skip(stats, has_ref, ref, "dense reconstruction was not attempted");
        return V3D_OK;
    }
    if (count < 3) {
        mesh_skip(stats, has_ref, ref, "fewer than three accepted fused dense points are available");
        return V3D_OK;
    }
    if (stride == 0) {
        mesh_skip(stats, has_ref, ref, "dense reconstruction did not expose a valid reference-grid stride");
        return V3D_OK;
    }
    if (width == 0 || height == 0 || !std::isfinite(focal) || focal <= 0.0) {
        mesh_skip(stats, has_ref, ref,
                  "the reference camera does not provide finite positive projection parameters");
        return V3D_OK;
    }
    if (!has_ref) {
        mesh_skip(stats, false, 0, "dense reconstruction did not select a reference frame");
        return V3D_OK;
    }
    const v3d_camera* cam = nullptr;
    for (uint64_t i = 0; i < n_cams; ++i)
        if (cams[i].frame_index == ref) {
            cam = &cams[i];
            break;
        }
    if (!cam) {
        mesh_skip(stats, true, ref, "the dense reference frame has no accepted registered camera");
        return V3D_OK;
    }
    HCamera hc;
    hc.frame_index = cam->frame_index;
    std::memcpy(hc.R, cam->rotation, sizeof(hc.R));
    std::memcpy(hc.t, cam->translation, sizeof(hc.t));
    std::vector<uint32_t> m = map;
    if (m.empty() && count != n_src) {
        m.resize(count);
        for (size_t i = 0; i < count; ++i) m[i] = static_cast<uint32_t>(i);
    }
    bool canceled = false;
    int32_t st = run_mesh_patch(ctx, pts, sites, m, n_src, hc, width, height, border,
                                static_cast<uint32_t>(stride), focal, cancel, stats, tris, canceled);
    if (st < 0) return st;
    if (canceled) {
        tris.clear();
        mesh_skip(stats, true, ref, "mesh reconstruction canceled");
        return V3D_OK;
    }
    stats.has_reference_frame = 1;
    stats.reference_frame = ref;
    return V3D_OK;
}

}  // namespace

extern "C" {

void v3d_mesh_result_free(v3d_mesh_result* r) {
    if (!r) return;
    // a batch's triangles live in its pinned block, which `internal` holds
    if (r->internal)
        delete static_cast<v3d::HostBlock*>(r->internal);
    else
        std::free(r->triangles);
    std::free(r->reference_frames);
    std::free(r->patches);
    std::memset(r, 0, sizeof(*r));
}

int32_t v3d_reconstruct_dense_mesh_with_control(v3d_context* ctx, const v3d_point* points,
                                                uint64_t n_points, const v3d_grid_site* grid_sites,
                                                uint64_t n_grid_sites,
                                                const v3d_mesh_dense_input* dense,
                                                const v3d_camera* cameras, uint64_t n_cameras,
                                                uint32_t width, uint32_t height, double focal,
                                                v3d_cancel_fn cancel, void* cancel_user,
                                                v3d_mesh_result* out) {
    if (!out || !dense) return V3D_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    if (!ctx || !ctx->stream) return V3D_ERR_NO_DEVICE;
    if ((n_points && !points) || (n_grid_sites && !grid_sites) || (n_cameras && !cameras) ||
        (dense->n_patches && !dense->patches))
        return V3D_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    CancelPoll cp{cancel, cancel_user};
    std::vector<v3d_mesh_triangle> tris;
    std::vector<v3d_mesh_stats> patches;
    std::vector<uint64_t> rfs;
    if (dense->n_patches == 0) {
        // mesh.rs:84-99
        v3d_mesh_stats s;
        if (dense->attempted && n_points >= 3 && n_points != n_grid_sites) {
            mesh_skip(s, dense->has_reference_frame, dense->reference_frame,
                      "dense point and reference-grid evidence counts disagree");
        } else {
            size_t count = std::min(n_points, n_grid_sites);
            int32_t st = legacy_mesh(ctx, points, grid_sites, {}, count, count, dense->attempted,
                                     dense->has_reference_frame, dense->reference_frame,
                                     dense->grid_stride, dense->grid_border, cameras, n_cameras,
                                     width, height, focal, cp, s, tris);
            if (st < 0) return st;
        }
        out->stats = s;
        if (s.has_reference_frame) {
            v3d_mesh_stats p = s;
            p.point_count = s.grid_vertices + s.rejected_grid_vertices;
            patches.push_back(p);
            rfs.push_back(s.reference_frame);
        }
    } else {
        bool attempted = false;
        v3d_mesh_stats& s = out->stats;
        for (uint64_t pi = 0; pi < dense->n_patches; ++pi) {
            if (cp.poll()) {
                std::memset(out, 0, sizeof(*out));
                return V3D_OK;
            }
            const v3d_reference_patch& pa = dense->patches[pi];
            uint64_t pe = pa.primary_start + pa.primary_points;
            uint64_t ce = pa.completion_start + pa.completed_points;
            bool ok = n_points == n_grid_sites && pe >= pa.primary_start && ce >= pa.completion_start &&
                      pe <= n_points && ce <= n_points;
            if (!ok) {
                v3d_mesh_stats ps;
                mesh_skip(ps, true, pa.reference_frame,
                          "dense patch ranges exceed the accepted point evidence");
                ps.attempted = 0;
                ps.point_count = pa.accepted_points;
                patches.push_back(ps);
                continue;
            }
            std::vector<uint32_t> idx;
            for (uint64_t i = pa.primary_start; i < pe; ++i) idx.push_back(static_cast<uint32_t>(i));
            for (uint64_t i = pa.completion_start; i < ce; ++i) idx.push_back(static_cast<uint32_t>(i));
            v3d_mesh_stats ps;
            std::vector<v3d_mesh_triangle> pt;
            int32_t st = legacy_mesh(ctx, points, grid_sites, idx, n_points, idx.size(), true, true,
                                     pa.reference_frame, pa.grid_stride, pa.grid_border, cameras,
                                     n_cameras, width, height, focal, cp, ps, pt);
            if (st < 0) return st;
            attempted = attempted || ps.attempted;
            s.grid_vertices += ps.grid_vertices;
            s.rejected_grid_vertices += ps.rejected_grid_vertices;
            s.candidate_cells += ps.candidate_cells;
            s.candidate_triangles += ps.candidate_triangles;
            s.rejected_discontinuities += ps.rejected_discontinuities;
            s.rejected_degenerate += ps.rejected_degenerate;
            for (const v3d_mesh_triangle& t : pt) {
                if (t.a >= idx.size() || t.b >= idx.size() || t.c >= idx.size()) continue;
                tris.push_back({idx[t.a], idx[t.b], idx[t.c], t.confidence, 0});
            }
            ps.point_count = idx.size();
            ps.accepted_triangles = pt.size();
            patches.push_back(ps);
        }
        for (const v3d_mesh_stats& p : patches) rfs.push_back(p.reference_frame);
        s.attempted = attempted;
        if (tris.empty()) {
            s.has_skip_reason = 1;
            std::strncpy(s.skip_reason, "no reference patch produced an accepted surface triangle",
                         V3D_SKIP_REASON_BYTES - 1);
        }
        if (!rfs.empty()) {
            s.has_reference_frame = 1;
            s.reference_frame = rfs[0];
        }
        s.accepted_triangles = tris.size();
    }
    out->n_triangles = tris.size();
    out->triangles = dup(tris);
    out->n_reference_frames = rfs.size();
    out->reference_frames = dup(rfs);
    out->n_patches = patches.size();
    out->patches = dup(patches);
    return V3D_OK;
}

}  // extern "C"
