// C ABI of the dense plane-sweep library (include/v3d_dense.h).
//
// The per-reference pass and the multi-reference driver are host
// orchestration around one device batch; no entry point computes anything on
// the CPU that the reference computes per grid site.  Without a CUDA device
// every compute entry point fails with V3D_ERR_NO_DEVICE.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <set>
#include <string>

#include "host.hpp"

using namespace v3d;

namespace {

// What a C result holds besides its malloc'd arrays: the source-frame lists
// of its patches and, when its points live in a batch's pinned block, a
// reference to that block (the point arrays are then not freed one by one).
struct ResultOwner {
    std::vector<std::vector<uint64_t>> patch_sources;
    HostBlock block;
};

ResultOwner* owner_of(v3d_dense_result* out) {
    if (!out->internal) out->internal = new ResultOwner;
    return static_cast<ResultOwner*>(out->internal);
}

template <class T>
T* dup(const std::vector<T>& v) {
    if (v.empty()) return nullptr;
    T* p = static_cast<T*>(std::malloc(sizeof(T) * v.size()));
    if (p) std::memcpy(p, v.data(), sizeof(T) * v.size());
    return p;
}

void set_reason(char* dst, int32_t* has, const std::string& s) {
    std::memset(dst, 0, V3D_SKIP_REASON_BYTES);
    *has = 1;
    std::strncpy(dst, s.c_str(), V3D_SKIP_REASON_BYTES - 1);
}

bool valid_profile(const v3d_profile* p) {
    return p && (p->cost == V3D_COST_ZSAD || p->cost == V3D_COST_ZNCC) && p->patch_radius >= 1 &&
           p->patch_radius <= V3D_MAX_PATCH_RADIUS && p->depth_hypotheses >= 2 &&
           p->depth_hypotheses <= V3D_MAX_DEPTH_HYPOTHESES && p->max_source_views >= 1 &&
           p->max_source_views <= V3D_MAX_SOURCE_VIEWS && p->grid_stride >= 0 &&
           (p->precision == V3D_PRECISION_EXACT64 || p->precision == V3D_PRECISION_FAST32 ||
            p->precision == V3D_PRECISION_FAST32_SUMS32) &&
           p->error_confidence_scale > 0 && p->depth_margin_saturation > 0;
}

bool valid_frames(const v3d_frame* frames, uint64_t n) {
    if (n && !frames) return false;
    for (uint64_t i = 0; i < n; ++i) {
        if (frames[i].format < V3D_PIXEL_RGBA8 || frames[i].format > V3D_PIXEL_GRAY_BF16)
            return false;
        // the kernels address pixels with 32-bit offsets
        if (static_cast<uint64_t>(frames[i].width) * frames[i].height >= (uint64_t{1} << 32))
            return false;
    }
    return true;
}

void fill_pass(v3d_dense_result* out, const PassResult& r) {
    std::memset(out, 0, sizeof(*out));
    out->stats = r.stats;
    std::vector<uint64_t> sf(r.plan.source_frames.begin(), r.plan.source_frames.end());
    if (r.stats.attempted) {
        out->n_source_frames = sf.size();
        out->source_frames = dup(sf);
        out->stats.source_views = sf.size();
    }
    out->n_points = r.points.size();
    if (!r.points.empty()) {
        out->points = r.points.begin();
        out->grid_sites = r.sites.begin();
        out->point_attributes = r.attrs.begin();
        owner_of(out)->block = r.block;
    }
}

int32_t status_of(const PassResult& r) { return r.stats.attempted ? V3D_OK : V3D_SKIPPED; }

bool ensure_device(v3d_context* ctx) {
    return ctx && ctx->stream != nullptr;
}

// Emulates the reference's per-row cancellation polls of the grid sweep
// (dense_legacy.rs:273): one poll per grid row, canceled -> skipped.
bool sweep_canceled(const RefPlan& p, CancelPoll& cancel) {
    if (!cancel.fn) return cancel.canceled;
    for (uint32_t row = 0; row < p.ny; ++row)
        if (cancel.poll()) return true;
    return false;
}

void canceled_result(PassResult& r) {
    skip_result(r, V3D_SKIP_CANCELED, "dense reconstruction canceled");
}

// DenseReferenceAttemptStats (dense.rs:749-785)
v3d_reference_attempt attempt_of(uint64_t reference_frame, const v3d_dense_stats& s,
                                 uint64_t accepted_points, bool accepted) {
    v3d_reference_attempt a;
    std::memset(&a, 0, sizeof(a));
    if (!accepted) {
        std::string reason;
        if (s.has_skip_reason)
            reason = s.skip_reason;
        else if (!s.attempted)
            reason = "dense estimation did not run for this reference";
        else
            reason = "reference produced " + std::to_string(accepted_points) +
                     " accepted dense points; at least 3 are required for a surface patch";
        set_reason(a.skip_reason, &a.has_skip_reason, reason);
    }
    a.reference_frame = reference_frame;
    a.attempted = s.attempted;
    a.accepted = accepted;
    a.sampled_pixels = s.sampled_pixels;
    a.accepted_points = accepted_points;
    a.reciprocal_checked_points = s.reciprocal_checked_points;
    a.reciprocal_rejected_points = s.reciprocal_rejected_points;
    a.reciprocal_consistent_points = s.reciprocal_consistent_points;
    a.surface_completion_proposals = s.surface_completion_proposals;
    a.surface_completed_points = s.surface_completed_points;
    a.surface_completion_rejected_texture = s.surface_completion_rejected_texture;
    a.surface_completion_rejected_cross_view = s.surface_completion_rejected_cross_view;
    a.surface_completion_rejected_reciprocal = s.surface_completion_rejected_reciprocal;
    a.surface_completion_rejected_fusion = s.surface_completion_rejected_fusion;
    a.surface_completion_rejected_footprint = s.surface_completion_rejected_footprint;
    return a;
}

v3d_reference_patch patch_of(const PassResult& r, uint64_t primary_start, uint64_t primary_points,
                             uint64_t completion_start, uint64_t completed_points) {
    v3d_reference_patch p;
    std::memset(&p, 0, sizeof(p));
    p.reference_frame = r.stats.reference_frame;
    p.primary_start = primary_start;
    p.primary_points = primary_points;
    p.completion_start = completion_start;
    p.completed_points = completed_points;
    p.sampled_pixels = r.stats.sampled_pixels;
    p.accepted_points = primary_points + completed_points;
    p.reciprocal_consistent_points = r.stats.reciprocal_consistent_points;
    p.grid_stride = r.stats.grid_stride;
    p.grid_border = r.stats.grid_border;
    p.has_search_min_depth = r.stats.has_search_min_depth;
    p.search_min_depth = r.stats.search_min_depth;
    p.has_search_max_depth = r.stats.has_search_max_depth;
    p.search_max_depth = r.stats.search_max_depth;
    return p;
}

// from_legacy (dense.rs:997-1082)
void fill_from_legacy(v3d_dense_result* out, const PassResult& r) {
    fill_pass(out, r);
    const v3d_dense_stats& s = r.stats;
    if (!s.has_reference_frame) return;
    uint64_t n = r.points.size();
    uint64_t completion = std::min<uint64_t>(s.surface_completed_points, n);
    uint64_t primary = n - completion;
    std::vector<uint64_t> rf{s.reference_frame};
    out->n_reference_frames = 1;
    out->reference_frames = dup(rf);
    std::vector<v3d_reference_attempt> at{attempt_of(s.reference_frame, s, n, s.attempted && n >= 3)};
    out->n_attempts = 1;
    out->attempts = dup(at);
    if (s.attempted) {
        ResultOwner* owner = owner_of(out);
        owner->patch_sources.emplace_back(r.plan.source_frames.begin(), r.plan.source_frames.end());
        std::vector<v3d_reference_patch> ps{patch_of(r, 0, primary, primary, completion)};
        ps[0].n_source_frames = owner->patch_sources[0].size();
        ps[0].source_frames = owner->patch_sources[0].data();
        out->n_patches = 1;
        out->patches = dup(ps);
    }
}

}  // namespace

extern "C" {

int32_t v3d_abi_version(void) { return V3D_ABI_VERSION; }

const char* v3d_status_text(int32_t status) {
    switch (status) {
        case V3D_OK: return "ok";
        case V3D_SKIPPED: return "skipped";
        case V3D_ERR_INVALID_ARGUMENT: return "invalid argument";
        case V3D_ERR_CUDA: return "CUDA error";
        case V3D_ERR_OUT_OF_MEMORY: return "out of device memory";
        case V3D_ERR_NO_DEVICE: return "no CUDA device";
        case V3D_ERR_INTERNAL: return "internal error";
        case V3D_ERR_TIMEOUT: return "request not done within the timeout";
        case V3D_ERR_SHUTDOWN: return "server stopped before the request ran";
    }
    return "unknown status";
}

const char* v3d_skip_reason_text(int32_t code) {
    switch (code) {
        case V3D_SKIP_NONE: return "";
        case V3D_SKIP_NO_FRAMES: return "no sampled frames are available";
        case V3D_SKIP_FEWER_THAN_TWO_CAMERAS:
            return "fewer than two accepted registered cameras are available";
        case V3D_SKIP_FEW_SPARSE_LANDMARKS: return "fewer than 8 accepted sparse landmarks are available";
        case V3D_SKIP_FRAMES_TOO_SMALL: return "sampled frames are too small for coarse depth estimation";
        case V3D_SKIP_NO_REFERENCE_CAMERA:
            return "no registered camera sees at least 8 accepted sparse landmarks inside its image";
        case V3D_SKIP_NO_DEPTH_ENVELOPE:
            return "visible sparse landmarks do not provide a finite positive depth-search envelope";
        case V3D_SKIP_REFERENCE_FRAME_MISSING: return "the selected reference camera has no sampled frame";
        case V3D_SKIP_NO_SOURCE_VIEW:
            return "no second registered camera has sufficient baseline, overlap, and at least 8 "
                   "visible sparse landmarks for reciprocal depth consistency";
        case V3D_SKIP_CANCELED: return "dense reconstruction canceled";
    }
    return "";
}

const char* v3d_last_error(const v3d_context* ctx) { return ctx ? ctx->last_error.c_str() : ""; }

int32_t v3d_last_run_info(const v3d_context* ctx, v3d_run_info* out) {
    if (!ctx || !out) return V3D_ERR_INVALID_ARGUMENT;
    out->device_ms = ctx->last_ms;
    out->kernel_launches = ctx->last_launches;
    out->grid_sites = ctx->last_sites;
    out->plane_view_units = ctx->last_units;
    out->sweep_ms = ctx->last_sweep_ms;
    out->reciprocal_ms = ctx->last_recip_ms;
    out->completion_ms = ctx->last_completion_ms;
    out->reciprocal_plane_evaluations = ctx->last_recip_evals;
    out->candidates = ctx->last_candidates;
    out->host_plan_ms = ctx->last_plan_ms;
    out->host_enqueue_ms = ctx->last_enqueue_ms;
    out->host_wait_ms = ctx->last_wait_ms;
    out->host_assemble_ms = ctx->last_assemble_ms;
    out->mesh_ms = ctx->last_mesh_ms;
    out->triangles = ctx->last_triangles;
    out->host_block_ms = ctx->last_block_ms;
    out->host_readback_ms = ctx->last_readback_ms;
    out->result_bytes = ctx->last_result_bytes;
    out->sweep_chunks = ctx->last_chunks;
    out->sweep_tile_x = ctx->last_tile_x;
    for (int i = 0; i < 12; ++i) out->merge_stage_ms[i] = ctx->last_merge_stage_ms[i];
    out->recip_sweep_ms = ctx->last_recip_sweep_ms;
    out->recip_prepare_ms = ctx->last_recip_prepare_ms;
    return V3D_OK;
}

int32_t v3d_context_create(int32_t device, v3d_context** out) {
    if (!out) return V3D_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int count = 0;
    if (cudaGetDeviceCount(&count) != cudaSuccess || count <= 0 || device < 0 || device >= count) {
        cudaGetLastError();
        return V3D_ERR_NO_DEVICE;
    }
    if (cudaSetDevice(device) != cudaSuccess) return V3D_ERR_CUDA;
    auto* ctx = new v3d_context;
    ctx->device = device;
    cudaStream_t s;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        return V3D_ERR_CUDA;
    }
    ctx->stream = s;
    *out = ctx;
    return V3D_OK;
}

void v3d_context_destroy(v3d_context* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) {
        cudaStreamSynchronize(static_cast<cudaStream_t>(ctx->stream));
        cudaStreamDestroy(static_cast<cudaStream_t>(ctx->stream));
    }
    if (ctx->arena) cudaFree(ctx->arena);
    if (ctx->pinned) cudaFreeHost(ctx->pinned);
    delete ctx;
}

void v3d_profile_reference(v3d_profile* p) {
    // dense_legacy.rs:6-21
    std::memset(p, 0, sizeof(*p));
    p->cost = V3D_COST_ZSAD;
    p->patch_radius = 1;
    p->depth_hypotheses = 24;
    p->max_source_views = 4;
    p->grid_stride = 0;
    p->precision = V3D_PRECISION_EXACT64;
    p->min_reference_contrast = 14.0;
    p->max_photometric_error = 18.0;
    p->min_ambiguity_margin = 1.0;
    p->depth_margin_saturation = 6.0;
    p->error_confidence_scale = 8.0;
    p->min_window_variance = 0.0;
}

void v3d_profile_zncc(v3d_profile* p, int32_t radius, int32_t planes, int32_t sources,
                      int32_t stride) {
    // Project-defined ZNCC profile on [0, 1] images; cost = 1 - ZNCC.
    std::memset(p, 0, sizeof(*p));
    p->cost = V3D_COST_ZNCC;
    p->patch_radius = radius;
    p->depth_hypotheses = planes;
    p->max_source_views = sources;
    p->grid_stride = stride;
    p->precision = V3D_PRECISION_FAST32;
    p->min_reference_contrast = 14.0 / 255.0;
    p->max_photometric_error = 0.5;
    p->min_ambiguity_margin = 0.002;
    p->depth_margin_saturation = 0.05;
    p->error_confidence_scale = 0.2;
    p->min_window_variance = 1.0e-5;
}

uint64_t v3d_grid_stride(uint32_t width, uint32_t height, int32_t fine_grid) {
    return reference_grid_stride(width, height, fine_grid != 0);
}

void v3d_dense_result_free(v3d_dense_result* r) {
    if (!r) return;
    auto* owner = static_cast<ResultOwner*>(r->internal);
    std::free(r->source_frames);
    if (!owner || !owner->block) {
        std::free(r->points);
        std::free(r->grid_sites);
        std::free(r->point_attributes);
    }
    std::free(r->reference_frames);
    std::free(r->attempts);
    std::free(r->patches);
    delete owner;
    std::memset(r, 0, sizeof(*r));
}

int32_t v3d_estimate_depth_points_with_control(v3d_context* ctx, const v3d_frame* frames,
                                               uint64_t n_frames, const v3d_camera* cameras,
                                               uint64_t n_cameras, const double* sparse_xyz,
                                               uint64_t n_sparse, double focal, int32_t fine_grid,
                                               const v3d_profile* profile, v3d_cancel_fn cancel,
                                               void* cancel_user, v3d_dense_result* out) {
    if (!out) return V3D_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    if (!ensure_device(ctx)) return V3D_ERR_NO_DEVICE;
    if (!valid_profile(profile) || !valid_frames(frames, n_frames) ||
        (n_cameras && !cameras) || (n_sparse && !sparse_xyz))
        return V3D_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    Inputs in = load_inputs(frames, n_frames, cameras, n_cameras, sparse_xyz, n_sparse, focal);
    std::vector<RefPlan> plans{plan_legacy(*profile, frames, n_frames, in.cameras, in.sparse, focal,
                                           fine_grid != 0, nullptr)};
    if (plans[0].skip_code == -2) {
        ctx->last_error = plans[0].skip_reason;
        return V3D_ERR_INVALID_ARGUMENT;
    }
    CancelPoll cp{cancel, cancel_user};
    std::vector<PassResult> res;
    if (!plans[0].skipped && sweep_canceled(plans[0], cp)) {
        res.assign(1, PassResult{});
        canceled_result(res[0]);
    } else {
        int32_t st = run_batch(ctx, *profile, frames, n_frames, focal, plans, res);
        if (st < 0) return st;
    }
    fill_pass(out, res[0]);
    return status_of(res[0]);
}

}  // extern "C"

namespace {

// mesh.rs from_legacy (mesh.rs:244-281) of one patch's legacy mesh.
void fill_mesh(v3d_mesh_result* out, const MeshOut& m) {
    std::memset(out, 0, sizeof(*out));
    out->stats = m.stats;
    out->n_triangles = m.tris.size();
    if (!m.tris.empty()) {
        // the triangles stay in the batch's pinned block; `internal` holds it
        out->triangles = m.tris.begin();
        out->internal = new HostBlock(m.block);
    }
    if (m.stats.has_reference_frame) {
        std::vector<uint64_t> rf{m.stats.reference_frame};
        out->n_reference_frames = 1;
        out->reference_frames = dup(rf);
        v3d_mesh_stats p = m.stats;
        p.point_count = m.stats.grid_vertices + m.stats.rejected_grid_vertices;
        std::vector<v3d_mesh_stats> ps{p};
        out->n_patches = 1;
        out->patches = dup(ps);
    }
}

}  // namespace

Inputs v3d::load_inputs(const v3d_frame* frames, uint64_t n_frames, const v3d_camera* cams,
                   uint64_t n_cams, const double* sparse, uint64_t n_sparse, double focal) {
    Inputs in;
    in.frames = frames;
    in.n_frames = n_frames;
    in.cameras.resize(n_cams);
    for (uint64_t i = 0; i < n_cams; ++i) {
        in.cameras[i].frame_index = cams[i].frame_index;
        std::memcpy(in.cameras[i].R, cams[i].rotation, sizeof(in.cameras[i].R));
        std::memcpy(in.cameras[i].t, cams[i].translation, sizeof(in.cameras[i].t));
    }
    in.sparse.resize(n_sparse);
    for (uint64_t i = 0; i < n_sparse; ++i)
        in.sparse[i] = {sparse[3 * i], sparse[3 * i + 1], sparse[3 * i + 2]};
    in.focal = focal;
    return in;
}

int32_t v3d::clip_batch(v3d_context* ctx, const std::vector<ClipJob>& jobs, int32_t fine_grid,
                        const v3d_profile& batch_prof, v3d_cancel_fn cancel, void* cancel_user,
                        v3d_dense_result* out, v3d_mesh_result* mesh_out, int32_t* present,
                        std::vector<uint64_t>* units) {
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    const auto t_plan = std::chrono::steady_clock::now();
    std::vector<size_t> job_of, first_of(jobs.size() + 1, 0), frame_base(jobs.size() + 1, 0);
    for (size_t j = 0; j < jobs.size(); ++j) {
        first_of[j + 1] = first_of[j] + jobs[j].n_refs;
        frame_base[j + 1] = frame_base[j] + jobs[j].in.n_frames;
        for (uint64_t i = 0; i < jobs[j].n_refs; ++i) job_of.push_back(j);
    }
    const size_t n_refs = first_of.back();
    std::vector<RefPlan> plans(n_refs);
    std::vector<uint8_t> pres8(n_refs, 0), canceled(n_refs, 0);
    parallel_for(n_refs, [&](size_t i) {
        const ClipJob& J = jobs[job_of[i]];
        bool p = false;
        plans[i] = plan_reference_patch(J.prof, J.in, J.camera_indices[i - first_of[job_of[i]]],
                                        fine_grid != 0, p);
        pres8[i] = p;
    });
    CancelPoll cp{cancel, cancel_user};
    for (size_t i = 0; i < n_refs; ++i) {
        if (!pres8[i]) {
            plans[i].skipped = true;
            continue;
        }
        if (plans[i].skip_code == -2) {
            ctx->last_error = plans[i].skip_reason;
            return V3D_ERR_INVALID_ARGUMENT;
        }
        if (!plans[i].skipped && cp.fn && sweep_canceled(plans[i], cp)) {
            canceled[i] = 1;
            plans[i].skipped = true;
        }
        // frame slots into the batch's concatenated frame list
        const size_t fb = frame_base[job_of[i]];
        plans[i].ref_slot += fb;
        for (size_t& s : plans[i].src_slots) s += fb;
    }
    const v3d_frame* frames = jobs.empty() ? nullptr : jobs[0].in.frames;
    std::vector<v3d_frame> all_frames;
    if (jobs.size() > 1) {
        all_frames.reserve(frame_base.back());
        for (const ClipJob& J : jobs) all_frames.insert(all_frames.end(), J.in.frames, J.in.frames + J.in.n_frames);
        frames = all_frames.data();
    }
    // device-resident frames (a server's clips), when the jobs carry them
    std::vector<ResidentFrame> resident;
    const bool on_device = !jobs.empty() && jobs[0].resident != nullptr;
    if (on_device) {
        resident.reserve(frame_base.back());
        for (const ClipJob& J : jobs) {
            if (!J.resident) {
                ctx->last_error = "jobs of one batch must all carry resident frames or none";
                return V3D_ERR_INVALID_ARGUMENT;
            }
            resident.insert(resident.end(), J.resident, J.resident + J.in.n_frames);
        }
    }
    if (units) {
        units->assign(n_refs, 0);
        for (size_t i = 0; i < n_refs; ++i)
            if (!plans[i].skipped)
                (*units)[i] = static_cast<uint64_t>(plans[i].nx) * plans[i].ny * plans[i].planes *
                              plans[i].src_slots.size();
    }
    const double plan_ms = std::chrono::duration<double, std::milli>(
                               std::chrono::steady_clock::now() - t_plan).count();
    std::vector<PassResult> res;
    std::vector<MeshOut> meshes;
    const double focal = jobs.empty() ? 0.0 : jobs[0].in.focal;  // each plan carries its own
    int32_t st = run_batch(ctx, batch_prof, frames, frame_base.back(), focal, plans, res,
                           mesh_out ? &meshes : nullptr, on_device ? &resident : nullptr);
    ctx->last_plan_ms = plan_ms;
    if (st < 0) return st;
    if (mesh_out && meshes.size() != n_refs) {
        meshes.assign(n_refs, MeshOut{});
        for (size_t i = 0; i < n_refs; ++i) {
            v3d_mesh_stats& s = meshes[i].stats;
            s.has_reference_frame = plans[i].have_reference;
            s.reference_frame = plans[i].reference_frame;
            s.has_skip_reason = 1;
            std::strncpy(s.skip_reason, "dense reconstruction was not attempted",
                         V3D_SKIP_REASON_BYTES - 1);
        }
    }
    for (size_t i = 0; i < n_refs; ++i) {
        present[i] = pres8[i] ? 1 : 0;
        if (!pres8[i]) continue;
        if (canceled[i]) canceled_result(res[i]);
        const ClipJob& J = jobs[job_of[i]];
        // dense.rs:734: the patch reports its reference frame even when skipped
        res[i].stats.has_reference_frame = 1;
        res[i].stats.reference_frame =
            J.in.cameras[J.camera_indices[i - first_of[job_of[i]]]].frame_index;
        fill_pass(&out[i], res[i]);
        if (mesh_out) {
            if (canceled[i] || !res[i].stats.attempted) {
                v3d_mesh_stats& s = meshes[i].stats;
                std::memset(&s, 0, sizeof(s));
                meshes[i].tris = {};
                meshes[i].block.reset();
                s.has_reference_frame = 1;
                s.reference_frame = res[i].stats.reference_frame;
                s.has_skip_reason = 1;
                std::strncpy(s.skip_reason, "dense reconstruction was not attempted",
                             V3D_SKIP_REASON_BYTES - 1);
            }
            fill_mesh(&mesh_out[i], meshes[i]);
        }
    }
    return V3D_OK;
}

namespace {

void clear_outputs(uint64_t n, v3d_dense_result* out, v3d_mesh_result* mesh_out, int32_t* present) {
    for (uint64_t i = 0; i < n; ++i) {
        std::memset(&out[i], 0, sizeof(out[i]));
        if (mesh_out) std::memset(&mesh_out[i], 0, sizeof(mesh_out[i]));
        present[i] = 0;
    }
}

int32_t reference_patches(v3d_context* ctx, const v3d_frame* frames, uint64_t n_frames,
                          const v3d_camera* cameras, uint64_t n_cameras, const double* sparse_xyz,
                          uint64_t n_sparse, double focal, int32_t fine_grid,
                          const v3d_profile* profile, const uint64_t* camera_indices,
                          uint64_t n_refs, v3d_cancel_fn cancel, void* cancel_user,
                          v3d_dense_result* out, v3d_mesh_result* mesh_out, int32_t* present) {
    if (!out || !present || (n_refs && !camera_indices)) return V3D_ERR_INVALID_ARGUMENT;
    clear_outputs(n_refs, out, mesh_out, present);
    if (!ensure_device(ctx)) return V3D_ERR_NO_DEVICE;
    if (!valid_profile(profile) || !valid_frames(frames, n_frames) ||
        (n_cameras && !cameras) || (n_sparse && !sparse_xyz))
        return V3D_ERR_INVALID_ARGUMENT;
    std::vector<ClipJob> jobs(1);
    jobs[0].in = load_inputs(frames, n_frames, cameras, n_cameras, sparse_xyz, n_sparse, focal);
    jobs[0].prof = *profile;
    jobs[0].camera_indices = camera_indices;
    jobs[0].n_refs = n_refs;
    return clip_batch(ctx, jobs, fine_grid, *profile, cancel, cancel_user, out, mesh_out, present);
}

}  // namespace

extern "C" {

int32_t v3d_reconstruct_clips(v3d_context* ctx, const v3d_clip* clips, uint64_t n_clips,
                              int32_t fine_grid, const v3d_profile* profile, v3d_cancel_fn cancel,
                              void* cancel_user, v3d_dense_result* out,
                              v3d_mesh_result* mesh_out, int32_t* present) {
    if (!out || !present || (n_clips && !clips)) return V3D_ERR_INVALID_ARGUMENT;
    uint64_t n_refs = 0;
    for (uint64_t c = 0; c < n_clips; ++c) {
        if (clips[c].n_references && !clips[c].camera_indices) return V3D_ERR_INVALID_ARGUMENT;
        n_refs += clips[c].n_references;
    }
    clear_outputs(n_refs, out, mesh_out, present);
    if (!ensure_device(ctx)) return V3D_ERR_NO_DEVICE;
    if (!valid_profile(profile)) return V3D_ERR_INVALID_ARGUMENT;
    std::vector<ClipJob> jobs(n_clips);
    for (uint64_t c = 0; c < n_clips; ++c) {
        const v3d_clip& k = clips[c];
        if (!valid_frames(k.frames, k.n_frames) || (k.n_cameras && !k.cameras) ||
            (k.n_sparse && !k.sparse_xyz))
            return V3D_ERR_INVALID_ARGUMENT;
        ClipJob& J = jobs[c];
        J.prof = *profile;
        if (k.depth_hypotheses > 0) J.prof.depth_hypotheses = k.depth_hypotheses;
        if (k.max_source_views > 0) J.prof.max_source_views = k.max_source_views;
        if (!valid_profile(&J.prof)) return V3D_ERR_INVALID_ARGUMENT;
        J.in = load_inputs(k.frames, k.n_frames, k.cameras, k.n_cameras, k.sparse_xyz, k.n_sparse,
                           k.focal);
        J.camera_indices = k.camera_indices;
        J.n_refs = k.n_references;
    }
    return clip_batch(ctx, jobs, fine_grid, *profile, cancel, cancel_user, out, mesh_out, present);
}

int32_t v3d_reconstruct_reference_patches(v3d_context* ctx, const v3d_frame* frames,
                                          uint64_t n_frames, const v3d_camera* cameras,
                                          uint64_t n_cameras, const double* sparse_xyz,
                                          uint64_t n_sparse, double focal, int32_t fine_grid,
                                          const v3d_profile* profile,
                                          const uint64_t* camera_indices, uint64_t n_refs,
                                          v3d_cancel_fn cancel, void* cancel_user,
                                          v3d_dense_result* out, int32_t* present) {
    return reference_patches(ctx, frames, n_frames, cameras, n_cameras, sparse_xyz, n_sparse,
                             focal, fine_grid, profile, camera_indices, n_refs, cancel,
                             cancel_user, out, nullptr, present);
}

int32_t v3d_reconstruct_reference_patches_meshed(
    v3d_context* ctx, const v3d_frame* frames, uint64_t n_frames, const v3d_camera* cameras,
    uint64_t n_cameras, const double* sparse_xyz, uint64_t n_sparse, double focal,
    int32_t fine_grid, const v3d_profile* profile, const uint64_t* camera_indices,
    uint64_t n_refs, v3d_cancel_fn cancel, void* cancel_user, v3d_dense_result* out,
    v3d_mesh_result* mesh_out, int32_t* present) {
    if (!mesh_out) return V3D_ERR_INVALID_ARGUMENT;
    return reference_patches(ctx, frames, n_frames, cameras, n_cameras, sparse_xyz, n_sparse,
                             focal, fine_grid, profile, camera_indices, n_refs, cancel,
                             cancel_user, out, mesh_out, present);
}

int32_t v3d_has_distributed_landmarks(const v3d_frame* frames, uint64_t n_frames,
                                      const v3d_camera* cameras, uint64_t n_cameras,
                                      const double* sparse_xyz, uint64_t n_sparse, double focal,
                                      v3d_cancel_fn cancel, void* cancel_user) {
    if ((n_frames && !frames) || (n_cameras && !cameras) || (n_sparse && !sparse_xyz)) return 0;
    Inputs in = load_inputs(frames, n_frames, cameras, n_cameras, sparse_xyz, n_sparse, focal);
    CancelPoll cp{cancel, cancel_user};
    return has_distributed_landmarks(in, cp) ? 1 : 0;
}

int32_t v3d_estimate_depth_points_limited(v3d_context* ctx, const v3d_frame* frames,
                                          uint64_t n_frames, const v3d_camera* cameras,
                                          uint64_t n_cameras, const double* sparse_xyz,
                                          uint64_t n_sparse, double focal,
                                          uint64_t reference_views, int32_t fine_grid,
                                          const v3d_profile* profile, v3d_cancel_fn cancel,
                                          void* cancel_user, v3d_dense_result* out,
                                          int32_t* omitted_references) {
    // dense.rs:250-330
    if (!out || !omitted_references) return V3D_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    *omitted_references = 0;
    if (!ensure_device(ctx)) return V3D_ERR_NO_DEVICE;
    if (!valid_profile(profile) || !valid_frames(frames, n_frames) ||
        (n_cameras && !cameras) || (n_sparse && !sparse_xyz))
        return V3D_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    Inputs in = load_inputs(frames, n_frames, cameras, n_cameras, sparse_xyz, n_sparse, focal);
    CancelPoll cp{cancel, cancel_user};
    const bool fine = fine_grid != 0;

    auto run_legacy = [&](PassResult& r) -> int32_t {
        std::vector<RefPlan> plans{
            plan_legacy(*profile, frames, n_frames, in.cameras, in.sparse, focal, fine, nullptr)};
        if (plans[0].skip_code == -2) {
            ctx->last_error = plans[0].skip_reason;
            return V3D_ERR_INVALID_ARGUMENT;
        }
        std::vector<PassResult> res;
        if (!plans[0].skipped && sweep_canceled(plans[0], cp)) {
            res.assign(1, PassResult{});
            res[0].plan = plans[0];
            canceled_result(res[0]);
        } else {
            int32_t st = run_batch(ctx, *profile, frames, n_frames, focal, plans, res);
            if (st < 0) return st;
        }
        r = res[0];
        if (!r.stats.attempted) r.stats.has_reference_frame = 0;
        return V3D_OK;
    };

    std::vector<size_t> order = reference_candidate_order(in);
    if (order.empty()) {
        PassResult r;
        int32_t st = run_legacy(r);
        if (st < 0) return st;
        fill_from_legacy(out, r);
        return status_of(r);
    }
    const size_t n_try = std::min<size_t>(order.size(), 6);
    // Each reference pass depends only on its own inputs, so without a cancel
    // callback every attempt runs as one speculative device batch and the
    // sequential acceptance below reads the results in order.
    std::vector<PassResult> tried;
    std::vector<bool> pres(n_try, false);
    if (!cancel) {
        std::vector<RefPlan> plans(n_try);
        for (size_t i = 0; i < n_try; ++i) {
            bool p = false;
            plans[i] = plan_reference_patch(*profile, in, order[i], fine, p);
            pres[i] = p;
            if (!p) plans[i].skipped = true;
            if (plans[i].skip_code == -2) {
                ctx->last_error = plans[i].skip_reason;
                return V3D_ERR_INVALID_ARGUMENT;
            }
        }
        int32_t st = run_batch(ctx, *profile, frames, n_frames, focal, plans, tried);
        if (st < 0) return st;
    }
    struct Patch {
        PassResult r;
        size_t primary, completion;
    };
    std::vector<Patch> patches;
    std::vector<v3d_reference_attempt> attempts;
    bool omitted = false;
    for (size_t i = 0; i < n_try; ++i) {
        if (cp.poll()) {
            // dense.rs:280-282: a canceled run returns the default analysis
            return V3D_SKIPPED;
        }
        PassResult r;
        bool p = false;
        if (!cancel) {
            p = pres[i];
            r = tried[i];
        } else {
            std::vector<RefPlan> one{plan_reference_patch(*profile, in, order[i], fine, p)};
            if (p) {
                if (one[0].skip_code == -2) {
                    ctx->last_error = one[0].skip_reason;
                    return V3D_ERR_INVALID_ARGUMENT;
                }
                std::vector<PassResult> res;
                if (!one[0].skipped && sweep_canceled(one[0], cp)) {
                    res.assign(1, PassResult{});
                    res[0].plan = one[0];
                    canceled_result(res[0]);
                } else {
                    int32_t st = run_batch(ctx, *profile, frames, n_frames, focal, one, res);
                    if (st < 0) return st;
                }
                r = res[0];
            }
        }
        if (!p) continue;
        const uint64_t rf = in.cameras[order[i]].frame_index;
        r.stats.has_reference_frame = 1;
        r.stats.reference_frame = rf;
        const uint64_t n = r.points.size();
        const bool accepted = r.stats.attempted && n >= 3;
        attempts.push_back(attempt_of(rf, r.stats, n, accepted));
        if (!accepted) continue;
        uint64_t completion = std::min<uint64_t>(r.stats.surface_completed_points, n);
        patches.push_back({r, n - completion, completion});
        if (patches.size() >= reference_views) {
            omitted = i + 1 < n_try;
            break;
        }
    }
    if (patches.empty()) {
        PassResult r;
        int32_t st = run_legacy(r);
        if (st < 0) return st;
        fill_from_legacy(out, r);
        // merge_fallback_attempts (dense.rs:787-804)
        std::vector<v3d_reference_attempt> merged = attempts;
        for (uint64_t k = 0; k < out->n_attempts; ++k) {
            const v3d_reference_attempt& f = out->attempts[k];
            auto it = std::find_if(merged.begin(), merged.end(), [&](const v3d_reference_attempt& a) {
                return a.reference_frame == f.reference_frame;
            });
            if (it != merged.end()) {
                if (f.accepted && !it->accepted) *it = f;
            } else {
                merged.push_back(f);
            }
        }
        std::free(out->attempts);
        out->n_attempts = merged.size();
        out->attempts = dup(merged);
        return status_of(r);
    }
    // combine_patches (dense.rs:842-995)
    std::vector<v3d_point> pts;
    std::vector<v3d_grid_site> sites;
    std::vector<v3d_point_attributes> attrs;
    std::vector<uint64_t> pstart, cstart;
    for (const Patch& p : patches) {
        pstart.push_back(pts.size());
        pts.insert(pts.end(), p.r.points.begin(), p.r.points.begin() + p.primary);
        sites.insert(sites.end(), p.r.sites.begin(), p.r.sites.begin() + p.primary);
        attrs.insert(attrs.end(), p.r.attrs.begin(), p.r.attrs.begin() + p.primary);
    }
    uint64_t total_completion = 0;
    for (const Patch& p : patches) {
        cstart.push_back(pts.size());
        total_completion += p.completion;
        pts.insert(pts.end(), p.r.points.begin() + p.primary, p.r.points.end());
        sites.insert(sites.end(), p.r.sites.begin() + p.primary, p.r.sites.end());
        attrs.insert(attrs.end(), p.r.attrs.begin() + p.primary, p.r.attrs.end());
    }
    const uint64_t primary_reference = patches[0].r.stats.reference_frame;
    std::set<uint64_t> participating;
    for (const Patch& p : patches) {
        participating.insert(p.r.stats.reference_frame);
        participating.insert(p.r.plan.source_frames.begin(), p.r.plan.source_frames.end());
    }
    participating.erase(primary_reference);
    std::vector<uint64_t> sf(participating.begin(), participating.end());
    v3d_dense_stats& s = out->stats;
    const v3d_dense_stats& first = patches[0].r.stats;
    const bool single = patches.size() == 1;
    s.attempted = 1;
    s.has_reference_frame = 1;
    s.reference_frame = primary_reference;
    s.source_views = sf.size();
    for (const Patch& p : patches) {
        const v3d_dense_stats& q = p.r.stats;
        s.sampled_pixels += q.sampled_pixels;
        s.depth_hypotheses = std::max(s.depth_hypotheses, q.depth_hypotheses);
        s.surface_completion_proposals += q.surface_completion_proposals;
        s.surface_completion_rejected_texture += q.surface_completion_rejected_texture;
        s.surface_completion_rejected_cross_view += q.surface_completion_rejected_cross_view;
        s.surface_completion_rejected_reciprocal += q.surface_completion_rejected_reciprocal;
        s.surface_completion_rejected_fusion += q.surface_completion_rejected_fusion;
        s.surface_completion_rejected_footprint += q.surface_completion_rejected_footprint;
        s.reciprocal_checked_points += q.reciprocal_checked_points;
        s.reciprocal_rejected_points += q.reciprocal_rejected_points;
        s.reciprocal_consistent_points += q.reciprocal_consistent_points;
        s.fusion_input_observations += q.fusion_input_observations;
        s.fusion_rejected_observations += q.fusion_rejected_observations;
        s.fusion_rejected_points += q.fusion_rejected_points;
    }
    s.accepted_points = pts.size();
    s.surface_completed_points = total_completion;
    s.grid_stride = first.grid_stride;
    s.grid_border = first.grid_border;
    if (single) {
        s.has_median_fusion_observations = first.has_median_fusion_observations;
        s.median_fusion_observations = first.median_fusion_observations;
        s.has_median_supporting_views = first.has_median_supporting_views;
        s.median_supporting_views = first.median_supporting_views;
        s.has_median_photometric_error = first.has_median_photometric_error;
        s.median_photometric_error = first.median_photometric_error;
        s.has_search_min_depth = first.has_search_min_depth;
        s.search_min_depth = first.search_min_depth;
        s.has_search_max_depth = first.has_search_max_depth;
        s.search_max_depth = first.search_max_depth;
    }
    out->n_source_frames = sf.size();
    out->source_frames = dup(sf);
    out->n_points = pts.size();
    out->points = dup(pts);
    out->grid_sites = dup(sites);
    out->point_attributes = dup(attrs);
    std::vector<uint64_t> rfs;
    ResultOwner* owner = owner_of(out);
    std::vector<v3d_reference_patch> ps;
    for (size_t i = 0; i < patches.size(); ++i) {
        const Patch& p = patches[i];
        rfs.push_back(p.r.stats.reference_frame);
        owner->patch_sources.emplace_back(p.r.plan.source_frames.begin(), p.r.plan.source_frames.end());
        ps.push_back(patch_of(p.r, pstart[i], p.primary, cstart[i], p.completion));
    }
    for (size_t i = 0; i < ps.size(); ++i) {
        ps[i].n_source_frames = owner->patch_sources[i].size();
        ps[i].source_frames = owner->patch_sources[i].data();
    }
    out->n_reference_frames = rfs.size();
    out->reference_frames = dup(rfs);
    out->n_attempts = attempts.size();
    out->attempts = dup(attempts);
    out->n_patches = ps.size();
    out->patches = dup(ps);
    *omitted_references = omitted ? 1 : 0;
    return V3D_OK;
}

int32_t v3d_debug_sweep(v3d_context* ctx, const v3d_frame* frames, uint64_t n_frames,
                        const v3d_camera* cameras, uint64_t n_cameras, const double* sparse_xyz,
                        uint64_t n_sparse, double focal, int32_t fine_grid,
                        const v3d_profile* profile, v3d_site_record* out, uint64_t capacity,
                        uint64_t* n_sites) {
    if (!n_sites) return V3D_ERR_INVALID_ARGUMENT;
    *n_sites = 0;
    if (!ensure_device(ctx)) return V3D_ERR_NO_DEVICE;
    if (!valid_profile(profile) || !valid_frames(frames, n_frames) ||
        (n_cameras && !cameras) || (n_sparse && !sparse_xyz))
        return V3D_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    Inputs in = load_inputs(frames, n_frames, cameras, n_cameras, sparse_xyz, n_sparse, focal);
    RefPlan plan = plan_legacy(*profile, frames, n_frames, in.cameras, in.sparse, focal,
                               fine_grid != 0, nullptr);
    if (plan.skip_code == -2) return V3D_ERR_INVALID_ARGUMENT;
    if (plan.skipped) return V3D_SKIPPED;
    std::vector<v3d_site_record> rec;
    int32_t st = run_sweep_records(ctx, *profile, frames, n_frames, focal, plan, rec);
    if (st < 0) return st;
    *n_sites = rec.size();
    if (!out) return V3D_OK;  // size query
    if (capacity < rec.size()) return V3D_ERR_INVALID_ARGUMENT;
    if (!rec.empty()) std::memcpy(out, rec.data(), sizeof(v3d_site_record) * rec.size());
    return V3D_OK;
}

}  // extern "C"
