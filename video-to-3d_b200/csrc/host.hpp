// Host-side planning and batch execution of the dense pass.
#pragma once

#include <cstddef>
#include <cstdint>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/v3d_dense.h"

namespace v3d {

struct HVec3 {
    double x, y, z;
};

struct HCamera {
    size_t frame_index;
    double R[9];  // row-major world->camera
    double t[3];
};

// Planned inputs of one per-reference pass (dense_legacy.rs:157-256).
struct RefPlan {
    bool skipped = false;
    int skip_code = 0;
    std::string skip_reason;
    bool have_reference = false;
    size_t reference_frame = 0;           // caller-visible frame index
    std::vector<size_t> source_frames;    // caller-visible frame indices
    size_t ref_slot = 0;                  // index into the call's frame array
    std::vector<size_t> src_slots;
    HCamera ref_cam{};
    std::vector<HCamera> src_cams;
    std::vector<double> src_min, src_max;
    double search_min = 0, search_max = 0;
    uint32_t width = 0, height = 0, stride = 0, border = 0, nx = 0, ny = 0;
    int planes = 0;    // depth hypotheses (the profile's, per clip in a multi-clip batch)
    double focal = 0;  // the clip's focal length
};

// surface_topology (colmap_surface.rs:125-157) of host triangles whose indices
// are already checked, with ctx->mu held and the device current
// (surface_topology.cu).  Uses the arena from its start.
int32_t surface_topology_locked(v3d_context* ctx, const v3d_mesh_triangle* triangles, uint64_t nt,
                                uint64_t n, v3d_surface_topology* out, float* device_ms,
                                uint64_t* launches);

// Offsets of device buffers carved one after another from the context's
// arena, each 256-byte aligned (at least one element each).
struct Carve {
    size_t off = 0;
    template <class T>
    size_t take(uint64_t count) {
        const size_t at = (off + 255) & ~size_t(255);
        off = at + sizeof(T) * (count > 1 ? count : 1);
        return at;
    }
};

// Blocks of 256 threads for a grid-stride loop over n items: at most 16 per
// SM of a 148-SM B200, at least one.
inline unsigned grid_of(uint64_t n) {
    uint64_t b = (n + 255) / 256;
    if (b > 148ull * 16) b = 148ull * 16;
    return (unsigned)(b ? b : 1);
}

// Incremental SHA-256 on the host (sha256.cpp).
struct Sha256 {
    uint32_t h[8];
    uint8_t buf[64];
    uint64_t length = 0;
    size_t fill = 0;
    Sha256();
    void update(const void* data, size_t n);
    void finish(uint8_t digest[32]);
};

// Page-locked host memory shared by the results of one batch
// (host_block.cpp); the deleter returns it to a process-wide cache.
using HostBlock = std::shared_ptr<uint8_t>;
HostBlock host_block(size_t bytes);  // empty on allocation failure
size_t host_block_bytes(const HostBlock& b);  // capacity of a block from host_block

// A view of `size()` elements inside a HostBlock.
template <class T>
struct Span {
    T* ptr = nullptr;
    size_t len = 0;
    size_t size() const { return len; }
    bool empty() const { return len == 0; }
    T* begin() const { return ptr; }
    T* end() const { return ptr + len; }
    T& operator[](size_t i) const { return ptr[i]; }
};

// A frame already in device memory (a server's clip store): the frame as
// handed in and, for RGBA8, its u8 luma plane (else `luma` is the frame).
struct ResidentFrame {
    const void* raw = nullptr;
    const uint8_t* luma = nullptr;
};

// One patch's reference-grid triangles (mesh_legacy.rs:40-43).
struct MeshOut {
    v3d_mesh_stats stats{};
    Span<v3d_mesh_triangle> tris;
    HostBlock block;  // holds `tris`
};

// One pass's output (dense_legacy.rs:62-68 DenseAnalysis with DenseStats).
struct PassResult {
    RefPlan plan;
    Span<v3d_point> points;
    Span<v3d_grid_site> sites;
    Span<v3d_point_attributes> attrs;
    HostBlock block;  // holds the three arrays
    v3d_dense_stats stats{};
};

struct Inputs {
    const v3d_frame* frames = nullptr;
    size_t n_frames = 0;
    std::vector<HCamera> cameras;
    std::vector<HVec3> sparse;
    double focal = 0;
};

struct CancelPoll {
    v3d_cancel_fn fn = nullptr;
    void* user = nullptr;
    bool canceled = false;
    bool poll() {
        if (!canceled && fn && fn(user)) canceled = true;
        return canceled;
    }
};

// One clip of a device batch: its inputs, its profile and the cameras to use
// as references; `resident` (one entry per frame, or null) when its frames
// already live in device memory.
struct ClipJob {
    Inputs in;
    v3d_profile prof{};
    const uint64_t* camera_indices = nullptr;
    uint64_t n_refs = 0;
    const ResidentFrame* resident = nullptr;
};

// The caller's cameras and landmarks as planning inputs (api.cpp); `frames`
// is referenced, not copied.
Inputs load_inputs(const v3d_frame* frames, uint64_t n_frames, const v3d_camera* cams,
                   uint64_t n_cams, const double* sparse, uint64_t n_sparse, double focal);

// ---- launch-shape tuning of the tiled sweep (sweep_tuner.cpp) ----
struct SweepShapeKey {
    int device, radius, stride, tiles, planes, sources;  // the last three as log2 buckets
};
SweepShapeKey sweep_shape_key(int device, int radius, int stride, uint64_t tiles, int planes,
                              int sources);
// How the tiled sweep runs: the tile (32x8 or 16x16 sites) and its plane chunks.
struct SweepPlan {
    int tile_x = 32;
    int chunks = 1;
};
// The plan for a batch of this shape: a candidate while the shape is being
// measured, then the fastest one.  heuristic32 / heuristic16 are the
// occupancy heuristic's chunk counts for the two tiles.
SweepPlan sweep_plan_pick(const SweepShapeKey& key, int heuristic32, int heuristic16,
                          int max_chunks);
// Sweep device time of a batch run with `plan`, over `units` window costs.
void sweep_plan_record(const SweepShapeKey& key, SweepPlan plan, double sweep_ms, uint64_t units);

// ---- planning (host_plan.cpp) ----
uint32_t reference_grid_stride(uint32_t w, uint32_t h, bool fine);
HVec3 camera_center(const HCamera& c);
bool project_h(const HCamera& c, HVec3 p, uint32_t w, uint32_t h, double focal, HVec3& out);
HVec3 unproject_h(const HCamera& c, double x, double y, double depth, uint32_t w, uint32_t h,
                  double focal);
bool in_image_bounds_h(double x, double y, uint32_t w, uint32_t h);

// dense_legacy.rs:157-256 on an explicit view list: `cams[i]` with frame slots
// `slot_of_frame_index(cams[i].frame_index)`.
// `first_camera_sees_all`: the caller guarantees every landmark is visible in
// cams[0] at frame 0's size (the remapped per-reference call), which lets the
// reference selection skip scanning the other cameras.
RefPlan plan_legacy(const v3d_profile& prof, const v3d_frame* frames, size_t n_frames,
                    const std::vector<HCamera>& cams, const std::vector<HVec3>& sparse,
                    double focal, bool fine_grid, const std::vector<size_t>* slot_map,
                    bool first_camera_sees_all = false);

// Runs fn(i) for i in [0, n) on the host's hardware threads.
void parallel_for(size_t n, const std::function<void(size_t)>& fn);

// dense.rs:674-747: remap so the reference comes first; `present` is false
// where the reference returns None.
RefPlan plan_reference_patch(const v3d_profile& prof, const Inputs& in, size_t camera_index,
                             bool fine_grid, bool& present);

// The context's device arena grown to at least `need` bytes (its contents are
// not kept); false when the allocation fails.
bool ensure_arena(v3d_context* ctx, size_t need);

// Returns from an entry point that holds `ctx` when a CUDA call fails, with
// the failing call and CUDA's text in ctx->last_error.
#define V3D_CTX_CK(call)                                                             \
    do {                                                                             \
        cudaError_t e_ = (call);                                                     \
        if (e_ != cudaSuccess) {                                                     \
            ctx->last_error = std::string(#call) + ": " + cudaGetErrorString(e_);    \
            return e_ == cudaErrorMemoryAllocation ? V3D_ERR_OUT_OF_MEMORY : V3D_ERR_CUDA; \
        }                                                                            \
    } while (0)

std::vector<size_t> reference_candidate_order(const Inputs& in);
// dense.rs:627-671 given each camera's visible landmark count (-1 where the
// camera's frame is missing); shared with the device scan of v3d_plan_clips.
std::vector<size_t> order_from_visible(const std::vector<HCamera>& cameras,
                                       const std::vector<int64_t>& visible);
bool has_distributed_landmarks(const Inputs& in, CancelPoll& cancel);

void skip_result(PassResult& r, int code, const std::string& reason);

}  // namespace v3d

struct v3d_context {
    int device = 0;
    int sm_count = 0;        // multiprocessors of `device`, read on first use
    void* stream = nullptr;  // cudaStream_t
    std::mutex mu;
    std::string last_error;
    // growable device arena
    void* arena = nullptr;
    size_t arena_bytes = 0;
    // pinned host staging for results
    void* pinned = nullptr;
    size_t pinned_bytes = 0;
    // account of the last run_batch (v3d_last_run_info)
    float last_ms = 0.f;
    uint64_t last_launches = 0;
    uint64_t last_sites = 0;
    uint64_t last_units = 0;
    float last_sweep_ms = 0.f, last_recip_ms = 0.f, last_completion_ms = 0.f;
    float last_recip_sweep_ms = 0.f, last_recip_prepare_ms = 0.f;
    uint64_t last_recip_evals = 0, last_candidates = 0;
    double last_plan_ms = 0, last_enqueue_ms = 0, last_wait_ms = 0, last_assemble_ms = 0;
    float last_mesh_ms = 0.f;
    uint64_t last_triangles = 0;
    double last_block_ms = 0, last_readback_ms = 0;
    uint64_t last_result_bytes = 0;
    uint64_t last_chunks = 1;
    uint64_t last_tile_x = 32;
    double last_merge_stage_ms[12] = {};
};

namespace v3d {
// ---- execution (pipeline.cpp) ----
// Runs every non-skipped plan of `plans` as one device batch and fills
// `results` (same order).  Returns a v3d_status.
// With `mesh` set, the reference-grid triangle gates of every patch run on
// the device after completion and (*mesh)[i] receives plan i's mesh.
// With `resident` (one entry per frame slot) the frames are read where they
// lie in device memory and nothing is uploaded; `frames` then supplies sizes
// and the pixel format only.
int32_t run_batch(v3d_context* ctx, const v3d_profile& prof, const v3d_frame* frames,
                  size_t n_frames, double focal, const std::vector<RefPlan>& plans,
                  std::vector<PassResult>& results, std::vector<MeshOut>* mesh = nullptr,
                  const std::vector<ResidentFrame>* resident = nullptr);

// dense.rs:674-747 for every (clip, reference camera) of `jobs`, run as one
// device batch (api.cpp); out, mesh_out and present hold the references clip
// by clip, `units` (optional) each reference's sites x hypotheses x sources.
int32_t clip_batch(v3d_context* ctx, const std::vector<ClipJob>& jobs, int32_t fine_grid,
                   const v3d_profile& batch_prof, v3d_cancel_fn cancel, void* cancel_user,
                   v3d_dense_result* out, v3d_mesh_result* mesh_out, int32_t* present,
                   std::vector<uint64_t>* units = nullptr);

// The sweep of one planned pass alone, as per-site records (v3d_debug_sweep).
int32_t run_sweep_records(v3d_context* ctx, const v3d_profile& prof, const v3d_frame* frames,
                          size_t n_frames, double focal, const RefPlan& plan,
                          std::vector<v3d_site_record>& out);

// One legacy mesh pass (mesh_legacy.rs:200-358) over points[map[i]] (every
// point when `map` is empty); triangle indices refer to the mapped list.
int32_t run_mesh_patch(v3d_context* ctx, const v3d_point* points, const v3d_grid_site* sites,
                       const std::vector<uint32_t>& map, size_t n_points, const HCamera& cam,
                       uint32_t width, uint32_t height, uint32_t border, uint32_t stride,
                       double focal, CancelPoll& cancel, v3d_mesh_stats& stats,
                       std::vector<v3d_mesh_triangle>& tris, bool& canceled);
}  // namespace v3d
