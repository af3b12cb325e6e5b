// Batched execution of planned reference passes on one CUDA stream.
//
// HBM layout of a batch (one arena, 256-byte aligned sub-buffers):
//   frames      the caller's frames as handed in (RGBA8 or gray f32/f16/bf16),
//               plus a u8 luma plane per RGBA8 frame; every source of every
//               reference reads these shared copies
//   refs        DevReference per reference (cameras, envelopes, homography parts)
//   per site    SiteRank, status, occupancy and proposal records, flat over
//               all references (site_off gives each reference's range)
//   per cand    candidates, 16 reciprocal slots, fused output, status
//   pool        accepted points: primaries, then completion pass 1, then pass 2,
//               each segment in (reference, raster) order
#include <cuda_runtime.h>

#include <cub/block/block_scan.cuh>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <future>
#include <stdexcept>

#include "host.hpp"
#include "mesh_batch.cuh"
#include "pass_kernels.cuh"

namespace v3d {

namespace {

struct Carver {
    size_t off = 0;
    template <class T>
    size_t take(size_t count) {
        off = (off + 255) & ~size_t(255);
        size_t at = off;
        off += count * sizeof(T);
        return at;
    }
};

int storage_of(int format) {
    switch (format) {
        case V3D_PIXEL_RGBA8: return kU8;
        case V3D_PIXEL_GRAY_F32: return kF32;
        case V3D_PIXEL_GRAY_F16: return kF16;
        case V3D_PIXEL_GRAY_BF16: return kBF16;
    }
    return -1;
}

size_t bytes_per_pixel(int format) {
    return format == V3D_PIXEL_RGBA8 || format == V3D_PIXEL_GRAY_F32 ? 4 : 2;
}

// 3x3 products in f64 for the fast policy's homography parts.
void mat_mul(const double* a, const double* b, double* out) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += a[i * 3 + k] * b[k * 3 + j];
            out[i * 3 + j] = s;
        }
}

// Parts of the homography that maps pixel p of camera `from` at depth d along
// `from`'s optical axis to camera `to`:  A p + (1/d) b  (homogeneous pixel).
void homography_parts(const HCamera& from, uint32_t fw, uint32_t fh, const HCamera& to,
                      uint32_t tw, uint32_t th, double f, float* A_out, float* b_out) {
    double Rt[9];  // from.R^T
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) Rt[i * 3 + j] = from.R[j * 3 + i];
    double M[9];
    mat_mul(to.R, Rt, M);
    double c[3];
    for (int i = 0; i < 3; ++i)
        c[i] = to.t[i] - (M[i * 3] * from.t[0] + M[i * 3 + 1] * from.t[1] + M[i * 3 + 2] * from.t[2]);
    const double Kinv[9] = {1.0 / f, 0, -(fw * 0.5) / f, 0, 1.0 / f, -(fh * 0.5) / f, 0, 0, 1};
    const double K[9] = {f, 0, tw * 0.5, 0, f, th * 0.5, 0, 0, 1};
    double MK[9], A[9];
    mat_mul(M, Kinv, MK);
    mat_mul(K, MK, A);
    for (int i = 0; i < 9; ++i) A_out[i] = static_cast<float>(A[i]);
    for (int i = 0; i < 3; ++i)
        b_out[i] = static_cast<float>(K[i * 3] * c[0] + K[i * 3 + 1] * c[1] + K[i * 3 + 2] * c[2]);
}

void set_cam(DevCamera& d, const HCamera& h) {
    std::memcpy(d.R, h.R, sizeof(d.R));
    std::memcpy(d.t, h.t, sizeof(d.t));
}

bool grow(void** ptr, size_t* have, size_t need, bool pinned) {
    if (*have >= need) return true;
    size_t cap = std::max(need, *have + *have / 2);
    if (*ptr) {
        if (pinned)
            cudaFreeHost(*ptr);
        else
            cudaFree(*ptr);
        *ptr = nullptr;
        *have = 0;
    }
    cudaError_t e = pinned ? cudaMallocHost(ptr, cap) : cudaMalloc(ptr, cap);
    if (e != cudaSuccess) {
        *ptr = nullptr;
        cudaGetLastError();
        return false;
    }
    *have = cap;
    return true;
}

struct Seg {
    uint32_t begin, end;
};

}  // namespace

bool ensure_arena(v3d_context* ctx, size_t need) {
    return grow(&ctx->arena, &ctx->arena_bytes, need, false);
}

#define V3D_CK(call)                                              \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) {                                  \
            ctx->last_error = std::string(#call) + ": " + cudaGetErrorString(e_); \
            return e_ == cudaErrorMemoryAllocation ? V3D_ERR_OUT_OF_MEMORY : V3D_ERR_CUDA; \
        }                                                         \
    } while (0)

namespace {

// Device state of one batch after upload: the arena carve-out, the
// DevReference array and the kernel-facing BatchDev.
struct Prepared {
    std::vector<size_t> active;
    size_t n_active = 0;
    uint64_t total = 0, cap = 1;
    uint32_t max_nx = 0, max_ny = 0, stride0 = 0;
    bool tiled = false;
    int chunks = 1;             // plane chunks of the tiled sweep
    int tile_x = 32;            // its tile: 32x8 or 16x16 sites
    SweepShapeKey shape{};      // its launch-shape key for the tuner
    Rank* d_partial = nullptr;  // [chunks][sites] when chunks > 1
    BatchDev b{};
    uint32_t* d_siteref = nullptr;
    SiteRank* d_rank = nullptr;
    uint8_t* d_status = nullptr;
    RefCounters* d_ctr = nullptr;
    void* d_scratch = nullptr;
    uint32_t* d_idx = nullptr;
    Cand* d_cands = nullptr;
    uint8_t* d_cstat = nullptr;
    RecipObs* d_obs = nullptr;
    OutPoint* d_fused = nullptr;
    OutPoint* d_pool = nullptr;
    int32_t* d_occ = nullptr;
    uint8_t* d_pstat = nullptr;
    Cand* d_prop = nullptr;
    uint32_t* d_counts = nullptr;
    RecipQueue queue{};         // the reciprocal sweep's work queue
    // output: the pool in per-reference order (primaries, then completions)
    v3d_point* o_pts = nullptr;
    v3d_grid_site* o_sites = nullptr;
    v3d_point_attributes* o_attrs = nullptr;
    MedianKey* o_med = nullptr;
    uint32_t* o_patch = nullptr;  // reference of each output point (mesh input)
    uint32_t* o_local = nullptr;  // index inside its reference (mesh input)
    uint32_t* o_base = nullptr;   // [n_active + 1] first output index per reference
    uint32_t* m_range = nullptr;  // [2][3][n_active] per-(segment, reference) pool ranges
    // mesh stage
    uint64_t total_slots = 0;
    v3d_mesh_triangle* m_tris = nullptr;
    uint32_t* m_tpatch = nullptr;
    MeshScratch mesh{};
};

int32_t prepare(v3d_context* ctx, const v3d_profile& prof, const v3d_frame* frames,
                size_t n_frames, double focal, const std::vector<RefPlan>& plans,
                const std::vector<size_t>& active, bool sweep_only, Prepared& P,
                bool with_mesh = false, const std::vector<ResidentFrame>* resident = nullptr) {
    cudaStream_t stream = static_cast<cudaStream_t>(ctx->stream);
    P.active = active;

    // frames touched by the batch, all in one storage format
    std::vector<int64_t> dev_of(n_frames, -1);
    std::vector<size_t> used;
    int format = -1;
    auto use = [&](size_t slot) -> bool {
        if (slot >= n_frames) return false;
        if (dev_of[slot] < 0) {
            dev_of[slot] = static_cast<int64_t>(used.size());
            used.push_back(slot);
        }
        if (format < 0) format = frames[slot].format;
        const bool has_data = resident ? (*resident)[slot].raw != nullptr && (*resident)[slot].luma
                                       : frames[slot].data != nullptr;
        return frames[slot].format == format && has_data;
    };
    for (size_t a : active) {
        if (!use(plans[a].ref_slot)) {
            ctx->last_error = "frames of one call must share a pixel format and carry data";
            return V3D_ERR_INVALID_ARGUMENT;
        }
        for (size_t s : plans[a].src_slots)
            if (!use(s)) {
                ctx->last_error = "frames of one call must share a pixel format and carry data";
                return V3D_ERR_INVALID_ARGUMENT;
            }
    }
    const int storage = storage_of(format);
    if (storage < 0) {
        ctx->last_error = "unknown pixel format";
        return V3D_ERR_INVALID_ARGUMENT;
    }
    const bool rgba = format == V3D_PIXEL_RGBA8;
    const size_t n_active = active.size();
    std::vector<uint64_t> site_off(n_active + 1, 0);
    uint32_t max_nx = 0, max_ny = 0;
    bool uniform_stride = true;
    for (size_t k = 0; k < n_active; ++k) {
        const RefPlan& p = plans[active[k]];
        site_off[k + 1] = site_off[k] + static_cast<uint64_t>(p.nx) * p.ny;
        max_nx = std::max(max_nx, p.nx);
        max_ny = std::max(max_ny, p.ny);
        uniform_stride = uniform_stride && p.stride == plans[active[0]].stride;
    }
    const uint64_t total = site_off[n_active];
    const uint64_t cap = std::max<uint64_t>(total, 1);
    // the box-filter sweep and, for batches of few tiles, its plane chunks:
    // enough CTAs for two waves of four per SM, at least 4 hypotheses a chunk
    {
        const uint32_t s0 = plans[active[0]].stride;
        const int w = 2 * prof.patch_radius + 1;
        P.tiled = prof.precision != V3D_PRECISION_EXACT64 && prof.cost == V3D_COST_ZNCC &&
                  uniform_stride && s0 >= 1 && s0 <= 4 && static_cast<int>(s0) < w;
        P.chunks = 1;
        P.tile_x = 32;
        if (P.tiled) {
            uint64_t tiles = 0, tiles16 = 0;
            int min_planes = kMaxPlanes;
            for (size_t k = 0; k < n_active; ++k) {
                const RefPlan& p = plans[active[k]];
                tiles += static_cast<uint64_t>((p.nx + 31) / 32) * ((p.ny + 7) / 8);
                tiles16 += static_cast<uint64_t>((p.nx + 15) / 16) * ((p.ny + 15) / 16);
                min_planes = std::min(min_planes, p.planes);
            }
            if (!ctx->sm_count &&
                cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount,
                                       ctx->device) != cudaSuccess) {
                cudaGetLastError();
                ctx->sm_count = 148;
            }
            const uint64_t target = static_cast<uint64_t>(ctx->sm_count) * 8;
            const int max_chunks = std::max(1, std::min(16, min_planes / 4));
            auto heuristic = [&](uint64_t n) {
                return n && n < target
                           ? static_cast<int>(std::min<uint64_t>((target + n - 1) / n, max_chunks))
                           : 1;
            };
            int max_src = 1;
            for (size_t k = 0; k < n_active; ++k)
                max_src = std::max<int>(max_src, static_cast<int>(plans[active[k]].src_slots.size()));
            P.shape = sweep_shape_key(ctx->device, prof.patch_radius, static_cast<int>(s0), tiles,
                                      min_planes, max_src);
            const SweepPlan plan =
                sweep_plan_pick(P.shape, heuristic(tiles), heuristic(tiles16), max_chunks);
            P.chunks = plan.chunks;
            P.tile_x = plan.tile_x;
        }
    }
    P.n_active = n_active;
    P.total = total;
    P.cap = cap;
    P.max_nx = max_nx;
    P.max_ny = max_ny;

    // ---- arena layout ----
    Carver cv;
    std::vector<size_t> raw_off(used.size()), luma_off(used.size());
    for (size_t u = 0; !resident && u < used.size(); ++u) {
        const v3d_frame& f = frames[used[u]];
        size_t px = static_cast<size_t>(f.width) * f.height;
        raw_off[u] = cv.take<uint8_t>(px * bytes_per_pixel(format));
        luma_off[u] = rgba ? cv.take<uint8_t>(px) : raw_off[u];
    }
    const size_t o_refs = cv.take<DevReference>(n_active);
    // per reference a [kMaxSources][planes] table of source inverse depths
    std::vector<uint64_t> inv_off(n_active + 1, 0);
    for (size_t k = 0; k < n_active; ++k)
        inv_off[k + 1] = inv_off[k] + kMaxSources * static_cast<uint64_t>(plans[active[k]].planes);
    const size_t inv_count = inv_off[n_active];
    const size_t o_srcinv = cv.take<float>(inv_count);
    const size_t o_siteoff = cv.take<uint64_t>(n_active + 1);
    const size_t o_siteref = cv.take<uint32_t>(cap);
    const size_t o_rank = cv.take<SiteRank>(cap);
    const size_t o_status = cv.take<uint8_t>(cap);
    const size_t o_partial = cv.take<Rank>(P.chunks > 1 ? static_cast<uint64_t>(P.chunks) * cap : 1);
    const size_t o_ctr = cv.take<RefCounters>(n_active);
    const uint64_t pc = sweep_only ? 1 : cap;  // pass buffers are not needed for the sweep alone
    // the reciprocal sweep's work queue: a flag and a list entry per (candidate, source)
    size_t queue_src = 1;
    for (size_t k = 0; k < n_active; ++k)
        queue_src = std::max(queue_src, plans[active[k]].src_slots.size());
    const uint64_t pq = pc * queue_src;
    if (pq >= (1ull << 32)) {
        ctx->last_error = "batch too large: 2^32 or more (grid site, source) pairs";
        return V3D_ERR_INVALID_ARGUMENT;
    }
    const size_t o_scratch = cv.take<uint8_t>(compaction_scratch_bytes(pq));
    const size_t o_qflags = cv.take<uint8_t>(pq);
    const size_t o_qitems = cv.take<uint32_t>(pq);
    const size_t o_qfall = cv.take<uint32_t>(pq);
    const size_t o_idx = cv.take<uint32_t>(pc);
    const size_t o_cands = cv.take<Cand>(pc);
    const size_t o_cstat = cv.take<uint8_t>(pc);
    const size_t o_obs = cv.take<RecipObs>(pc * kMaxSources);
    const size_t o_fused = cv.take<OutPoint>(pc);
    const size_t o_pool = cv.take<OutPoint>(pc);
    const size_t o_occ = cv.take<int32_t>(pc);
    const size_t o_pstat = cv.take<uint8_t>(pc);
    const size_t o_prop = cv.take<Cand>(pc);
    const size_t o_counts = cv.take<uint32_t>(16);
    // mesh stage: pool as mesh input, per-(segment, reference) ranges, scratch, triangles
    uint64_t total_slots = 0;
    for (size_t k = 0; k < n_active; ++k)
        total_slots += mesh_slots(plans[active[k]].nx, plans[active[k]].ny);
    P.total_slots = with_mesh ? total_slots : 0;
    const uint64_t mc = with_mesh ? cap : 1;
    const size_t o_opts = cv.take<v3d_point>(pc);
    const size_t o_osites = cv.take<v3d_grid_site>(pc);
    const size_t o_oattrs = cv.take<v3d_point_attributes>(pc);
    const size_t o_omed = cv.take<MedianKey>(pc);
    const size_t o_opatch = cv.take<uint32_t>(mc);
    const size_t o_olocal = cv.take<uint32_t>(mc);
    const size_t o_obase = cv.take<uint32_t>(n_active + 1);
    const size_t o_mrange = cv.take<uint32_t>(6 * n_active);
    const size_t mesh_bytes =
        with_mesh ? mesh_scratch_layout(nullptr, static_cast<uint32_t>(n_active), cap, total,
                                        total_slots, nullptr)
                  : 0;
    const size_t o_mscratch = cv.take<uint8_t>(mesh_bytes + 256);
    const size_t o_mtris = cv.take<v3d_mesh_triangle>(with_mesh ? std::max<uint64_t>(total_slots, 1) : 1);
    const size_t o_mtpatch = cv.take<uint32_t>(with_mesh ? std::max<uint64_t>(total_slots, 1) : 1);
    const size_t arena_need = cv.off + 256;
    if (!grow(&ctx->arena, &ctx->arena_bytes, arena_need, false)) {
        ctx->last_error = "device arena allocation failed";
        return V3D_ERR_OUT_OF_MEMORY;
    }
    char* base = static_cast<char*>(ctx->arena);
    auto at = [&](size_t off) { return base + off; };

    // ---- uploads (none for resident frames) ----
    std::vector<const void*> raw_ptr(used.size()), luma_ptr(used.size());
    for (size_t u = 0; u < used.size(); ++u) {
        if (resident) {
            raw_ptr[u] = (*resident)[used[u]].raw;
            luma_ptr[u] = (*resident)[used[u]].luma;
            continue;
        }
        const v3d_frame& f = frames[used[u]];
        size_t px = static_cast<size_t>(f.width) * f.height;
        V3D_CK(cudaMemcpyAsync(at(raw_off[u]), f.data, px * bytes_per_pixel(format),
                               cudaMemcpyHostToDevice, stream));
        if (rgba)
            V3D_CK(launch_luma(reinterpret_cast<const uint8_t*>(at(raw_off[u])),
                               reinterpret_cast<uint8_t*>(at(luma_off[u])), px, stream));
        raw_ptr[u] = at(raw_off[u]);
        luma_ptr[u] = at(luma_off[u]);
    }
    const size_t staging = sizeof(DevReference) * n_active + sizeof(uint64_t) * (n_active + 1) +
                           sizeof(float) * inv_count;
    if (!grow(&ctx->pinned, &ctx->pinned_bytes, staging, true)) {
        ctx->last_error = "pinned staging allocation failed";
        return V3D_ERR_OUT_OF_MEMORY;
    }
    DevReference* hrefs = static_cast<DevReference*>(ctx->pinned);
    std::memset(hrefs, 0, sizeof(DevReference) * n_active);
    for (size_t k = 0; k < n_active; ++k) {
        const RefPlan& p = plans[active[k]];
        DevReference& d = hrefs[k];
        set_cam(d.cam, p.ref_cam);
        size_t ru = static_cast<size_t>(dev_of[p.ref_slot]);
        d.img = DevImage{luma_ptr[ru], frames[p.ref_slot].width, frames[p.ref_slot].height};
        d.rgba = rgba ? static_cast<const uint8_t*>(raw_ptr[ru]) : nullptr;
        d.focal = p.focal;
        d.planes = p.planes;
        d.inv_off = inv_off[k];
        d.search_min = p.search_min;
        d.search_max = p.search_max;
        d.border = p.border;
        d.stride = p.stride;
        d.nx = p.nx;
        d.ny = p.ny;
        d.n_src = static_cast<int32_t>(p.src_slots.size());
        for (size_t j = 0; j < p.src_slots.size(); ++j) {
            DevSource& s = d.src[j];
            size_t su = static_cast<size_t>(dev_of[p.src_slots[j]]);
            const v3d_frame& sf = frames[p.src_slots[j]];
            set_cam(s.cam, p.src_cams[j]);
            s.img = DevImage{luma_ptr[su], sf.width, sf.height};
            s.search_min = p.src_min[j];
            s.search_max = p.src_max[j];
            homography_parts(p.ref_cam, d.img.width, d.img.height, p.src_cams[j], sf.width,
                             sf.height, p.focal, s.fwd_A, s.fwd_b);
            homography_parts(p.src_cams[j], sf.width, sf.height, p.ref_cam, d.img.width,
                             d.img.height, p.focal, s.bwd_A, s.bwd_b);
        }
    }
    uint64_t* hoff = reinterpret_cast<uint64_t*>(hrefs + n_active);
    std::memcpy(hoff, site_off.data(), sizeof(uint64_t) * (n_active + 1));
    // 1/depth of every source hypothesis, from the f64 hypothesis formula
    // (dense_legacy.rs:286-293, 908-916) rounded once to f32
    float* hinv = reinterpret_cast<float*>(hoff + n_active + 1);
    std::memset(hinv, 0, sizeof(float) * inv_count);
    for (size_t k = 0; k < n_active; ++k) {
        const RefPlan& pl = plans[active[k]];
        const int n_hyp = pl.planes;
        for (size_t j = 0; j < pl.src_slots.size(); ++j)
            for (int q = 0; q < n_hyp; ++q) {
                double t = n_hyp == 1 ? 0.0 : static_cast<double>(q) / static_cast<double>(n_hyp - 1);
                double inv = (1.0 / pl.src_min[j]) * (1.0 - t) + (1.0 / pl.src_max[j]) * t;
                double depth = 1.0 / inv;
                hinv[inv_off[k] + j * n_hyp + q] = static_cast<float>(1.0 / depth);
            }
    }
    V3D_CK(cudaMemcpyAsync(at(o_refs), hrefs, sizeof(DevReference) * n_active,
                           cudaMemcpyHostToDevice, stream));
    V3D_CK(cudaMemcpyAsync(at(o_siteoff), hoff, sizeof(uint64_t) * (n_active + 1),
                           cudaMemcpyHostToDevice, stream));
    V3D_CK(cudaMemcpyAsync(at(o_srcinv), hinv, sizeof(float) * inv_count, cudaMemcpyHostToDevice,
                           stream));

    P.d_partial = P.chunks > 1 ? reinterpret_cast<Rank*>(at(o_partial)) : nullptr;
    auto* d_siteref = P.d_siteref = reinterpret_cast<uint32_t*>(at(o_siteref));
    P.d_rank = reinterpret_cast<SiteRank*>(at(o_rank));
    auto* d_status = P.d_status = reinterpret_cast<uint8_t*>(at(o_status));
    auto* d_ctr = P.d_ctr = reinterpret_cast<RefCounters*>(at(o_ctr));
    P.d_scratch = at(o_scratch);
    P.d_idx = reinterpret_cast<uint32_t*>(at(o_idx));
    P.d_cands = reinterpret_cast<Cand*>(at(o_cands));
    P.d_cstat = reinterpret_cast<uint8_t*>(at(o_cstat));
    P.d_obs = reinterpret_cast<RecipObs*>(at(o_obs));
    P.queue = RecipQueue{reinterpret_cast<uint8_t*>(at(o_qflags)),
                         reinterpret_cast<uint32_t*>(at(o_qitems)), nullptr, P.d_scratch, pq};
    P.d_fused = reinterpret_cast<OutPoint*>(at(o_fused));
    P.d_pool = reinterpret_cast<OutPoint*>(at(o_pool));
    P.d_occ = reinterpret_cast<int32_t*>(at(o_occ));
    P.d_pstat = reinterpret_cast<uint8_t*>(at(o_pstat));
    P.d_prop = reinterpret_cast<Cand*>(at(o_prop));
    auto* d_counts = P.d_counts = reinterpret_cast<uint32_t*>(at(o_counts));
    P.queue.n_items = P.d_counts + 9;  // [8] completion seeds, [9] reciprocal items
    P.queue.fallback = reinterpret_cast<uint32_t*>(at(o_qfall));
    P.queue.n_fallback = P.d_counts + 10;  // [10] pairs for the per-hypothesis sweep
    P.o_pts = reinterpret_cast<v3d_point*>(at(o_opts));
    P.o_sites = reinterpret_cast<v3d_grid_site*>(at(o_osites));
    P.o_attrs = reinterpret_cast<v3d_point_attributes*>(at(o_oattrs));
    P.o_med = reinterpret_cast<MedianKey*>(at(o_omed));
    P.o_patch = with_mesh ? reinterpret_cast<uint32_t*>(at(o_opatch)) : nullptr;
    P.o_local = with_mesh ? reinterpret_cast<uint32_t*>(at(o_olocal)) : nullptr;
    P.o_base = reinterpret_cast<uint32_t*>(at(o_obase));
    P.m_range = reinterpret_cast<uint32_t*>(at(o_mrange));
    P.m_tris = reinterpret_cast<v3d_mesh_triangle*>(at(o_mtris));
    P.m_tpatch = reinterpret_cast<uint32_t*>(at(o_mtpatch));
    if (with_mesh)
        mesh_scratch_layout(at(o_mscratch), static_cast<uint32_t>(n_active), cap, total,
                            total_slots, &P.mesh);

    V3D_CK(cudaMemsetAsync(d_status, 0, cap, stream));
    V3D_CK(cudaMemsetAsync(d_ctr, 0, sizeof(RefCounters) * n_active, stream));
    V3D_CK(cudaMemsetAsync(d_counts, 0, sizeof(uint32_t) * 16, stream));
    V3D_CK(launch_site_ref(reinterpret_cast<const uint64_t*>(at(o_siteoff)),
                           static_cast<int32_t>(n_active), total, d_siteref, stream));

    BatchDev& b = P.b;
    b.refs = reinterpret_cast<const DevReference*>(at(o_refs));
    b.site_off = reinterpret_cast<const uint64_t*>(at(o_siteoff));
    b.src_inv = reinterpret_cast<const float*>(at(o_srcinv));
    b.n_refs = static_cast<int32_t>(n_active);
    b.max_src = 1;
    for (size_t k = 0; k < n_active; ++k)
        b.max_src = std::max<int32_t>(b.max_src, static_cast<int32_t>(plans[active[k]].src_slots.size()));
    b.storage = storage;
    b.prof.cost = prof.cost;
    b.prof.radius = prof.patch_radius;
    b.prof.planes = 1;
    for (size_t k = 0; k < n_active; ++k) b.prof.planes = std::max(b.prof.planes, plans[active[k]].planes);
    b.prof.pad = 0;
    b.prof.min_contrast = prof.min_reference_contrast;
    b.prof.max_error = prof.max_photometric_error;
    b.prof.min_margin = prof.min_ambiguity_margin;
    b.prof.margin_saturation = prof.depth_margin_saturation;
    b.prof.error_scale = prof.error_confidence_scale;
    b.prof.min_variance = prof.min_window_variance;
    b.exact = prof.precision == V3D_PRECISION_EXACT64;
    b.sums32 = prof.precision == V3D_PRECISION_FAST32_SUMS32;

    P.stride0 = plans[active[0]].stride;
    return V3D_OK;
}

}  // namespace

namespace {

// Per-(segment, reference) ranges of the point pool: every segment is ordered
// by reference.  range[s][k] = first pool index of reference k in segment s,
// range_end likewise; empty ranges stay [0, 0).
__global__ void k_pool_ranges(const OutPoint* __restrict__ pool, const uint32_t* __restrict__ seg,
                              uint32_t n_refs, uint32_t* __restrict__ start,
                              uint32_t* __restrict__ end) {
    const uint32_t n = seg[2];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t s = i < seg[0] ? 0 : (i < seg[1] ? 1 : 2);
        const uint32_t b = s == 0 ? 0 : seg[s - 1], e = seg[s];
        const uint32_t k = pool[i].ref;
        if (i == b || pool[i - 1].ref != k) start[s * n_refs + k] = i;
        if (i + 1 == e || pool[i + 1].ref != k) end[s * n_refs + k] = i + 1;
    }
}

// Exclusive prefix of the references' output sizes (their three segment
// ranges): base[k] is reference k's first output index, base[n_refs] the total.
__global__ void __launch_bounds__(1024) k_ref_bases(const uint32_t* __restrict__ start,
                                                    const uint32_t* __restrict__ end,
                                                    uint32_t n_refs, uint32_t* __restrict__ base) {
    using Scan = cub::BlockScan<uint32_t, 1024>;
    __shared__ typename Scan::TempStorage tmp;
    uint32_t carry = 0;
    for (uint32_t k0 = 0; k0 < n_refs; k0 += 1024) {
        const uint32_t k = k0 + threadIdx.x;
        uint32_t c = 0;
        if (k < n_refs)
            for (int s = 0; s < 3; ++s) c += end[s * n_refs + k] - start[s * n_refs + k];
        uint32_t x, agg;
        Scan(tmp).ExclusiveSum(c, x, agg);
        if (k < n_refs) base[k] = carry + x;
        carry += agg;
        __syncthreads();
    }
    if (threadIdx.x == 0) base[n_refs] = carry;
}

// The pool in output order: reference by reference, each reference's
// primaries then its completions of pass 1 and pass 2 (the order in which
// dense_legacy.rs:397-412 and 727-733 push them), as the arrays the caller receives,
// the median keys and, for the mesh stage, each point's reference and index
// inside it.
__global__ void k_pool_output(const OutPoint* __restrict__ pool, const uint32_t* __restrict__ seg,
                              uint32_t n_refs, const uint32_t* __restrict__ start,
                              const uint32_t* __restrict__ end, const uint32_t* __restrict__ base,
                              v3d_point* __restrict__ pts, v3d_grid_site* __restrict__ sites,
                              v3d_point_attributes* __restrict__ attrs,
                              MedianKey* __restrict__ med, uint32_t* __restrict__ patch,
                              uint32_t* __restrict__ local) {
    const uint32_t n = seg[2];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t s = i < seg[0] ? 0 : (i < seg[1] ? 1 : 2);
        const OutPoint& q = pool[i];
        const uint32_t k = q.ref;
        uint32_t l = i - start[s * n_refs + k];
        for (uint32_t t = 0; t < s; ++t) l += end[t * n_refs + k] - start[t * n_refs + k];
        const uint32_t o = base[k] + l;
        pts[o] = q.p;
        sites[o] = q.s;
        attrs[o] = q.a;
        MedianKey m;
        m.error = (float)q.error;
        m.support = (uint8_t)fmin(fmax(q.support, 0.0), 255.0);
        m.observations = (uint8_t)fmin(fmax(q.observations, 0.0), 255.0);
        m.primary = s == 0;
        m.pad = 0;
        med[o] = m;
        if (patch) {
            patch[o] = k;
            local[o] = l;
        }
    }
}

}  // namespace

int32_t run_batch(v3d_context* ctx, const v3d_profile& prof, const v3d_frame* frames,
                  size_t n_frames, double focal, const std::vector<RefPlan>& plans,
                  std::vector<PassResult>& results, std::vector<MeshOut>* mesh,
                  const std::vector<ResidentFrame>* resident) {
    cudaStream_t stream = static_cast<cudaStream_t>(ctx->stream);
    results.assign(plans.size(), PassResult{});
    std::vector<size_t> active;
    for (size_t i = 0; i < plans.size(); ++i) {
        results[i].plan = plans[i];
        if (plans[i].skipped)
            skip_result(results[i], plans[i].skip_code, plans[i].skip_reason);
        else
            active.push_back(i);
    }
    if (active.empty()) return V3D_OK;
    using clk = std::chrono::steady_clock;
    auto ms_since = [](clk::time_point t) {
        return std::chrono::duration<double, std::milli>(clk::now() - t).count();
    };
    const clk::time_point t_upload = clk::now();
    const uint64_t launches0 = g_kernel_launches;
    Prepared P;
    int32_t pst = prepare(ctx, prof, frames, n_frames, focal, plans, active, false, P,
                          mesh != nullptr, resident);
    if (pst != V3D_OK) return pst;
    const size_t n_active = P.n_active;
    const uint64_t total = P.total, cap = P.cap;
    const BatchDev& b = P.b;
    uint32_t* d_siteref = P.d_siteref;
    SiteRank* d_rank = P.d_rank;
    uint8_t* d_status = P.d_status;
    RefCounters* d_ctr = P.d_ctr;
    void* d_scratch = P.d_scratch;
    uint32_t* d_idx = P.d_idx;
    Cand* d_cands = P.d_cands;
    uint8_t* d_cstat = P.d_cstat;
    RecipObs* d_obs = P.d_obs;
    OutPoint* d_fused = P.d_fused;
    OutPoint* d_pool = P.d_pool;
    int32_t* d_occ = P.d_occ;
    uint8_t* d_pstat = P.d_pstat;
    Cand* d_prop = P.d_prop;
    uint32_t* c_cand = P.d_counts + 0;
    uint32_t* c_acc = P.d_counts + 1;
    uint32_t* c_pool = P.d_counts + 2;
    uint32_t* c_seg = P.d_counts + 3;  // [3] segment ends
    const uint32_t max_nx = P.max_nx, max_ny = P.max_ny, stride0 = P.stride0;
    const bool tiled = P.tiled;

    cudaEvent_t ev0, ev1;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    cudaEventRecord(ev0, stream);
    ctx->last_chunks = static_cast<uint64_t>(P.chunks);
    ctx->last_tile_x = static_cast<uint64_t>(P.tiled ? P.tile_x : 0);
    ctx->last_sites = total;
    ctx->last_units = 0;
    for (size_t k = 0; k < n_active; ++k) {
        const RefPlan& pl = plans[active[k]];
        ctx->last_units += static_cast<uint64_t>(pl.nx) * pl.ny * pl.planes *
                           pl.src_slots.size();
    }

    // stage events: sweep | primary reciprocal | completion passes
    cudaEvent_t es[8];
    for (auto& e : es) cudaEventCreate(&e);
    // the reciprocal check's kernels, per launch (primary, completion 1, 2)
    cudaEvent_t er[3][3];
    for (auto& row : er)
        for (auto& e : row) cudaEventCreate(&e);
    auto timed_queue = [&](int i) {
        RecipQueue q = P.queue;
        q.t_prepare = er[i][0];
        q.t_sweep = er[i][1];
        q.t_end = er[i][2];
        return q;
    };
    // primary sweep, reciprocal check and fusion
    cudaEventRecord(es[0], stream);
    V3D_CK(launch_sweep_dispatch(b, d_siteref, total, max_nx, max_ny, stride0, tiled, d_rank,
                                 d_status, d_ctr, stream,
                                 SweepChunks{P.chunks, P.d_partial, P.tile_x}));
    cudaEventRecord(es[1], stream);
    V3D_CK(launch_compact(d_status, kSiteAccepted, total, d_idx, c_cand, d_scratch, stream));
    V3D_CK(launch_make_primary_cands(b, d_idx, c_cand, cap, d_siteref, d_rank, d_cands, stream));
    cudaEventRecord(es[2], stream);
    V3D_CK(launch_reciprocal(b, d_cands, c_cand, cap, d_obs, d_ctr, timed_queue(0), stream));
    cudaEventRecord(es[3], stream);
    V3D_CK(cudaMemsetAsync(d_cstat, 0, cap, stream));
    V3D_CK(launch_fuse(b, d_cands, c_cand, cap, d_obs, false, 0, d_fused, d_cstat, d_ctr, stream));
    V3D_CK(launch_compact(d_cstat, kCandAccepted, cap, d_idx, c_acc, d_scratch, stream));
    V3D_CK(launch_append(d_idx, c_acc, cap, d_fused, d_pool, c_pool, c_seg + 0, stream));
    V3D_CK(launch_occupancy_clear(d_occ, total, stream));
    V3D_CK(launch_occupy(b, d_pool, nullptr, c_seg + 0, cap, d_occ, stream));

    // two surface-completion passes (dense_legacy.rs:542-734)
    cudaEventRecord(es[4], stream);
    for (int pass = 0; pass < 2; ++pass) {
        V3D_CK(launch_propose(b, pass, total, d_siteref, d_occ, d_pool, d_pstat, d_prop, d_ctr,
                              d_idx, P.d_counts + 8, d_scratch, stream));
        V3D_CK(launch_compact(d_pstat, kPropCandidate, total, d_idx, c_cand, d_scratch, stream));
        V3D_CK(launch_gather_cands(d_idx, c_cand, cap, d_prop, d_cands, stream));
        V3D_CK(launch_reciprocal(b, d_cands, c_cand, cap, d_obs, d_ctr, timed_queue(pass + 1),
                                 stream));
        V3D_CK(cudaMemsetAsync(d_cstat, 0, cap, stream));
        V3D_CK(launch_fuse(b, d_cands, c_cand, cap, d_obs, true, pass, d_fused, d_cstat, d_ctr,
                           stream));
        V3D_CK(launch_compact(d_cstat, kCandAccepted, cap, d_idx, c_acc, d_scratch, stream));
        V3D_CK(launch_append(d_idx, c_acc, cap, d_fused, d_pool, c_pool, c_seg + pass + 1, stream));
        V3D_CK(launch_occupy(b, d_pool, c_seg + pass, c_seg + pass + 1, cap, d_occ, stream));
    }
    cudaEventRecord(es[5], stream);
    // the pool in output order
    {
        const unsigned gb = static_cast<unsigned>(std::min<uint64_t>((cap + 255) / 256, 148 * 16));
        V3D_CK(cudaMemsetAsync(P.m_range, 0, sizeof(uint32_t) * 6 * n_active, stream));
        V3D_COUNTED k_pool_ranges<<<gb, 256, 0, stream>>>(d_pool, c_seg, static_cast<uint32_t>(n_active),
                                              P.m_range, P.m_range + 3 * n_active);
        V3D_COUNTED k_ref_bases<<<1, 1024, 0, stream>>>(P.m_range, P.m_range + 3 * n_active,
                                           static_cast<uint32_t>(n_active), P.o_base);
        V3D_COUNTED k_pool_output<<<gb, 256, 0, stream>>>(d_pool, c_seg, static_cast<uint32_t>(n_active),
                                              P.m_range, P.m_range + 3 * n_active, P.o_base,
                                              P.o_pts, P.o_sites, P.o_attrs, P.o_med, P.o_patch,
                                              P.o_local);
        V3D_CK(cudaGetLastError());
    }
    // The result block, acquired on a helper thread while the device works,
    // sized like the last call's results: a caller that still holds those
    // needs a second block, and pinning one takes longer than the copies.
    // Started only now, once every kernel before the read-back is enqueued:
    // pinning can hold up this thread's CUDA calls while it runs.
    std::future<HostBlock> early;
    if (ctx->last_result_bytes)
        early = std::async(std::launch::async, [dev = ctx->device, bytes = ctx->last_result_bytes] {
            cudaSetDevice(dev);  // a new thread starts on device 0
            return host_block(bytes);
        });
    std::vector<MeshPatchDev> mp;
    if (mesh) {
        // patch descriptors need the per-reference point counts: one read of the counters
        std::vector<RefCounters> c0(n_active);
        V3D_CK(cudaMemcpyAsync(c0.data(), d_ctr, sizeof(RefCounters) * n_active,
                               cudaMemcpyDeviceToHost, stream));
        V3D_CK(cudaStreamSynchronize(stream));
        mp.resize(n_active);
        uint64_t slot_off = 0;
        for (size_t k = 0; k < n_active; ++k) {
            const RefPlan& pl = plans[active[k]];
            MeshPatchDev& m = mp[k];
            std::memset(&m, 0, sizeof(m));
            set_cam(m.cam, pl.ref_cam);
            m.focal = pl.focal;
            m.width = frames[pl.ref_slot].width;
            m.height = frames[pl.ref_slot].height;
            m.border = pl.border;
            m.stride = pl.stride;
            m.gw = pl.nx;
            m.gh = pl.ny;
            m.slot_off = slot_off;
            m.n_points = c0[k].primary_points + c0[k].completed;
            slot_off += mesh_slots(pl.nx, pl.ny);
        }
        uint64_t go = 0;
        for (size_t k = 0; k < n_active; ++k) {
            mp[k].grid_off = go;
            go += static_cast<uint64_t>(mp[k].gw) * mp[k].gh;
        }
        V3D_CK(cudaMemcpyAsync(P.mesh.patches, mp.data(), sizeof(MeshPatchDev) * n_active,
                               cudaMemcpyHostToDevice, stream));
        cudaEventRecord(es[6], stream);
        // the output arrays bound the loops; every point beyond their size is unused
        uint64_t n_points = 0;
        for (size_t k = 0; k < n_active; ++k) n_points += mp[k].n_points;
        V3D_CK(mesh_batch_enqueue(P.mesh, static_cast<uint32_t>(n_active), total, P.total_slots,
                                  P.o_pts, P.o_sites, P.o_patch, P.o_local, n_points, P.m_tris,
                                  P.m_tpatch, stream));
    }
    cudaEventRecord(es[7], stream);
    cudaEventRecord(ev1, stream);
    ctx->last_launches = g_kernel_launches - launches0;

    // ---- read back ----
    ctx->last_enqueue_ms = ms_since(t_upload);
    const clk::time_point t_wait = clk::now();
    std::vector<RefCounters> ctr(n_active);
    std::vector<uint32_t> base(n_active + 1);
    std::vector<MeshCounters> mcount(mesh ? n_active : 0);
    uint32_t n_tris = 0;
    V3D_CK(cudaMemcpyAsync(ctr.data(), d_ctr, sizeof(RefCounters) * n_active,
                           cudaMemcpyDeviceToHost, stream));
    V3D_CK(cudaMemcpyAsync(base.data(), P.o_base, sizeof(uint32_t) * (n_active + 1),
                           cudaMemcpyDeviceToHost, stream));
    if (mesh) {
        V3D_CK(cudaMemcpyAsync(&n_tris, P.mesh.count, sizeof(uint32_t), cudaMemcpyDeviceToHost,
                               stream));
        V3D_CK(cudaMemcpyAsync(mcount.data(), P.mesh.counters, sizeof(MeshCounters) * n_active,
                               cudaMemcpyDeviceToHost, stream));
    }
    V3D_CK(cudaStreamSynchronize(stream));
    cudaEventElapsedTime(&ctx->last_ms, ev0, ev1);
    cudaEventElapsedTime(&ctx->last_sweep_ms, es[0], es[1]);
    if (P.tiled)
        sweep_plan_record(P.shape, SweepPlan{P.tile_x, P.chunks}, ctx->last_sweep_ms,
                          ctx->last_units);
    cudaEventElapsedTime(&ctx->last_recip_ms, es[2], es[3]);
    ctx->last_recip_sweep_ms = ctx->last_recip_prepare_ms = 0.f;
    for (auto& row : er) {
        float a = 0.f, c = 0.f;
        cudaEventElapsedTime(&a, row[0], row[1]);
        cudaEventElapsedTime(&c, row[1], row[2]);
        ctx->last_recip_prepare_ms += a;
        ctx->last_recip_sweep_ms += c;
    }
    cudaEventElapsedTime(&ctx->last_completion_ms, es[4], es[5]);
    ctx->last_mesh_ms = 0.f;
    if (mesh) cudaEventElapsedTime(&ctx->last_mesh_ms, es[6], es[7]);
    cudaEventDestroy(ev0);
    cudaEventDestroy(ev1);
    for (auto& e : es) cudaEventDestroy(e);
    for (auto& row : er)
        for (auto& e : row) cudaEventDestroy(e);
    ctx->last_recip_evals = 0;
    ctx->last_candidates = 0;
    for (const RefCounters& c : ctr) {
        ctx->last_recip_evals += c.recip_evals;
        ctx->last_candidates += c.candidates;
    }
    ctx->last_triangles = n_tris;
    const size_t n_out = base[n_active];
    if (mesh) {
        uint64_t acc = 0;
        for (const MeshCounters& c : mcount) acc += c.accepted;
        if (acc != n_tris) {
            ctx->last_error = "mesh triangle counts disagree";
            return V3D_ERR_INTERNAL;
        }
    }
    // one pinned block receives every array of the batch; the results point into it
    Carver hl;
    const size_t h_pts = hl.take<v3d_point>(n_out);
    const size_t h_sites = hl.take<v3d_grid_site>(n_out);
    const size_t h_attrs = hl.take<v3d_point_attributes>(n_out);
    const size_t h_med = hl.take<MedianKey>(n_out);
    const size_t h_tris = hl.take<v3d_mesh_triangle>(n_tris);
    HostBlock block;
    ctx->last_block_ms = ctx->last_readback_ms = 0;
    ctx->last_result_bytes = n_out || n_tris ? hl.off : 0;
    if (n_out || n_tris) {
        const clk::time_point t_block = clk::now();
        if (early.valid()) block = early.get();
        if (host_block_bytes(block) < hl.off) block = host_block(hl.off);
        if (!block) {
            ctx->last_error = "pinned result block allocation failed";
            return V3D_ERR_OUT_OF_MEMORY;
        }
        ctx->last_block_ms = ms_since(t_block);
        const clk::time_point t_copy = clk::now();
        uint8_t* hb = block.get();
        if (n_out) {
            V3D_CK(cudaMemcpyAsync(hb + h_pts, P.o_pts, sizeof(v3d_point) * n_out,
                                   cudaMemcpyDeviceToHost, stream));
            V3D_CK(cudaMemcpyAsync(hb + h_sites, P.o_sites, sizeof(v3d_grid_site) * n_out,
                                   cudaMemcpyDeviceToHost, stream));
            V3D_CK(cudaMemcpyAsync(hb + h_attrs, P.o_attrs, sizeof(v3d_point_attributes) * n_out,
                                   cudaMemcpyDeviceToHost, stream));
            V3D_CK(cudaMemcpyAsync(hb + h_med, P.o_med, sizeof(MedianKey) * n_out,
                                   cudaMemcpyDeviceToHost, stream));
        }
        if (n_tris)
            V3D_CK(cudaMemcpyAsync(hb + h_tris, P.m_tris, sizeof(v3d_mesh_triangle) * n_tris,
                                   cudaMemcpyDeviceToHost, stream));
        V3D_CK(cudaStreamSynchronize(stream));
        ctx->last_readback_ms = ms_since(t_copy);
    }
    ctx->last_wait_ms = ms_since(t_wait);
    const clk::time_point t_assemble = clk::now();
    uint8_t* hb = block.get();
    v3d_point* o_pts = reinterpret_cast<v3d_point*>(hb + h_pts);
    v3d_grid_site* o_sites = reinterpret_cast<v3d_grid_site*>(hb + h_sites);
    v3d_point_attributes* o_attrs = reinterpret_cast<v3d_point_attributes*>(hb + h_attrs);
    const MedianKey* o_med = reinterpret_cast<const MedianKey*>(hb + h_med);
    v3d_mesh_triangle* o_tris = reinterpret_cast<v3d_mesh_triangle*>(hb + h_tris);
    if (mesh) {
        // triangles are in patch order; accepted counts give each patch's range
        mesh->assign(plans.size(), MeshOut{});
        size_t t0 = 0;
        for (size_t k = 0; k < n_active; ++k) {
            MeshOut& m = (*mesh)[active[k]];
            const MeshCounters& c = mcount[k];
            const uint64_t npts = mp[k].n_points;
            v3d_mesh_stats& s = m.stats;
            std::memset(&s, 0, sizeof(s));
            s.has_reference_frame = 1;
            s.reference_frame = plans[active[k]].reference_frame;
            auto reason = [&](const char* r) {
                s.has_skip_reason = 1;
                std::strncpy(s.skip_reason, r, V3D_SKIP_REASON_BYTES - 1);
            };
            const size_t first = t0;
            t0 += c.accepted;
            if (npts < 3) {
                reason("fewer than three accepted fused dense points are available");
                continue;
            }
            s.attempted = 1;
            s.grid_vertices = c.vertices;
            s.rejected_grid_vertices = npts > c.vertices ? npts - c.vertices : 0;
            if (c.vertices < 3) {
                reason("fewer than three fused dense points align with the reference sampling grid");
                continue;
            }
            s.candidate_cells = c.candidate_cells;
            s.candidate_triangles = c.candidate_triangles;
            s.accepted_triangles = c.accepted;
            s.rejected_discontinuities = c.discontinuities;
            s.rejected_degenerate = c.degenerate;
            if (c.accepted) {
                m.tris = Span<v3d_mesh_triangle>{o_tris + first, c.accepted};
                m.block = block;
            }
        }
        for (size_t i = 0; i < plans.size(); ++i) {
            if (!plans[i].skipped) continue;
            MeshOut& m = (*mesh)[i];
            std::memset(&m.stats, 0, sizeof(m.stats));
            m.stats.has_reference_frame = plans[i].have_reference;
            m.stats.reference_frame = plans[i].reference_frame;
            m.stats.has_skip_reason = 1;
            std::strncpy(m.stats.skip_reason, "dense reconstruction was not attempted",
                         V3D_SKIP_REASON_BYTES - 1);
        }
    }
    // ---- assemble per reference ----
    parallel_for(n_active, [&](size_t k) {
        PassResult& r = results[active[k]];
        const RefPlan& p = plans[active[k]];
        const RefCounters& c = ctr[k];
        const size_t b0 = base[k], n = base[k + 1] - base[k];
        if (n) {
            r.points = Span<v3d_point>{o_pts + b0, n};
            r.sites = Span<v3d_grid_site>{o_sites + b0, n};
            r.attrs = Span<v3d_point_attributes>{o_attrs + b0, n};
            r.block = block;
        }
        // medians: round((n - 1) * 0.5) = n / 2-th order statistic (dense_legacy.rs:1168-1182)
        std::vector<float> errors(n);
        uint64_t sup_hist[256] = {0}, obs_hist[256] = {0};
        uint64_t n_obs = 0;
        for (size_t i = 0; i < n; ++i) {
            const MedianKey& m = o_med[b0 + i];
            errors[i] = m.error;
            ++sup_hist[m.support];
            if (m.primary) {
                ++obs_hist[m.observations];
                ++n_obs;
            }
        }
        auto hist_kth = [](const uint64_t* h, uint64_t kth) {
            uint64_t acc = 0;
            for (int v = 0; v < 256; ++v) {
                acc += h[v];
                if (acc > kth) return static_cast<double>(v);
            }
            return 255.0;
        };
        v3d_dense_stats& s = r.stats;
        std::memset(&s, 0, sizeof(s));
        s.attempted = 1;
        s.has_reference_frame = p.have_reference;
        s.reference_frame = p.reference_frame;
        s.source_views = p.src_slots.size();
        s.sampled_pixels = c.sampled;
        s.depth_hypotheses = static_cast<uint64_t>(p.planes);
        s.accepted_points = n;
        s.surface_completion_proposals = c.proposals;
        s.surface_completed_points = c.completed;
        s.surface_completion_rejected_texture = c.rej_texture;
        s.surface_completion_rejected_cross_view = c.rej_cross;
        s.surface_completion_rejected_reciprocal = c.rej_recip;
        s.surface_completion_rejected_fusion = c.rej_fusion;
        s.surface_completion_rejected_footprint = c.rej_footprint;
        s.grid_stride = p.stride;
        s.grid_border = p.border;
        s.reciprocal_checked_points = c.checked;
        s.reciprocal_rejected_points = c.recip_rejected;
        s.reciprocal_consistent_points = c.consistent;
        s.fusion_input_observations = c.fusion_input;
        s.fusion_rejected_observations = c.fusion_rejected_obs;
        s.fusion_rejected_points = c.fusion_rejected_pts;
        if (n_obs) {
            s.has_median_fusion_observations = 1;
            s.median_fusion_observations = static_cast<float>(hist_kth(obs_hist, n_obs / 2));
        }
        if (n) {
            s.has_median_supporting_views = 1;
            s.median_supporting_views = static_cast<float>(hist_kth(sup_hist, n / 2));
            std::nth_element(errors.begin(), errors.begin() + n / 2, errors.end());
            s.has_median_photometric_error = 1;
            s.median_photometric_error = errors[n / 2];
        }
        s.has_search_min_depth = 1;
        s.search_min_depth = static_cast<float>(p.search_min);
        s.has_search_max_depth = 1;
        s.search_max_depth = static_cast<float>(p.search_max);
    });
    ctx->last_assemble_ms = ms_since(t_assemble);
    return V3D_OK;
}

int32_t run_sweep_records(v3d_context* ctx, const v3d_profile& prof, const v3d_frame* frames,
                          size_t n_frames, double focal, const RefPlan& plan,
                          std::vector<v3d_site_record>& out) {
    out.clear();
    if (plan.skipped) return V3D_OK;
    cudaStream_t stream = static_cast<cudaStream_t>(ctx->stream);
    std::vector<RefPlan> plans{plan};
    Prepared P;
    int32_t pst = prepare(ctx, prof, frames, n_frames, focal, plans, {0}, true, P);
    if (pst != V3D_OK) return pst;
    V3D_CK(launch_sweep_dispatch(P.b, P.d_siteref, P.total, P.max_nx, P.max_ny, P.stride0, P.tiled,
                                 P.d_rank, P.d_status, P.d_ctr, stream,
                                 SweepChunks{P.chunks, P.d_partial, P.tile_x}));
    std::vector<SiteRank> rank(P.total);
    std::vector<uint8_t> status(P.total);
    if (P.total) {
        V3D_CK(cudaMemcpyAsync(rank.data(), P.d_rank, sizeof(SiteRank) * P.total,
                               cudaMemcpyDeviceToHost, stream));
        V3D_CK(cudaMemcpyAsync(status.data(), P.d_status, P.total, cudaMemcpyDeviceToHost, stream));
    }
    V3D_CK(cudaStreamSynchronize(stream));
    out.resize(P.total);
    for (uint64_t i = 0; i < P.total; ++i) {
        v3d_site_record& r = out[i];
        std::memset(&r, 0, sizeof(r));
        uint32_t gy = static_cast<uint32_t>(i / plan.nx), gx = static_cast<uint32_t>(i % plan.nx);
        r.x = plan.border + gx * plan.stride;
        r.y = plan.border + gy * plan.stride;
        r.status = status[i];
        if (status[i] >= kSiteGateRejected) {
            r.plane = rank[i].plane;
            r.support = rank[i].support;
            r.error = rank[i].error;
            r.margin = rank[i].margin;
        } else {
            r.plane = -1;
        }
    }
    return V3D_OK;
}

}  // namespace v3d
