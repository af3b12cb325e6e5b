// The multi-reference planner's landmark scans for many clips in one device
// pass, behind v3d_plan_clips: reference_candidate_order (dense.rs:620-672)
// needs every camera's count of visible landmarks, has_distributed_landmarks
// (dense.rs:165-213) every camera's landmarks per 4x4 image tile.  A block
// owns one camera of one clip and projects all of that clip's landmarks
// (project, dense_legacy.rs:1013-1029, in exact f64), counting in shared
// memory; the host then sorts each clip's order with the reference's rules
// (order_from_visible) and applies the majority rule.  Counts are integers, so
// orders and flags equal the reference's.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/v3d_dense.h"
#include "host.hpp"
#include "pass_kernels.cuh"

namespace v3d {
namespace {

struct PlanCamera {
    DevCamera cam;
    double focal;
    uint64_t first, last;  // the clip's landmarks [first, last); empty for a camera without frame
    uint32_t width, height;
};

__global__ void k_landmark_coverage(const PlanCamera* __restrict__ cams, uint64_t n_cams,
                                    const D3* __restrict__ pts, uint32_t* __restrict__ visible,
                                    uint32_t* __restrict__ tiles) {
    __shared__ uint32_t s_visible, s_tiles[16];
    for (uint64_t c = blockIdx.x; c < n_cams; c += gridDim.x) {
        if (threadIdx.x == 0) s_visible = 0;
        if (threadIdx.x < 16) s_tiles[threadIdx.x] = 0;
        __syncthreads();
        const PlanCamera pc = cams[c];
        const double w = (double)pc.width, h = (double)pc.height;
        for (uint64_t i = pc.first + threadIdx.x; i < pc.last; i += blockDim.x) {
            D3 q;
            if (!project_exact(pc.cam, pts[i], pc.width, pc.height, pc.focal, q)) continue;
            // in_image_bounds (dense_legacy.rs:1129-1131); the tile test of
            // dense.rs:187-190 is the same range
            if (!(isfinite(q.x) && isfinite(q.y) && q.x >= 0.0 && q.y >= 0.0 && q.x < w && q.y < h))
                continue;
            atomicAdd(&s_visible, 1u);
            const uint32_t col = (uint32_t)ddiv(dmul(4.0, q.x), w);
            const uint32_t row = (uint32_t)ddiv(dmul(4.0, q.y), h);
            atomicAdd(&s_tiles[row * 4 + col], 1u);
        }
        __syncthreads();
        if (threadIdx.x == 0) visible[c] = s_visible;
        if (threadIdx.x < 16) tiles[c * 16 + threadIdx.x] = s_tiles[threadIdx.x];
        __syncthreads();
    }
}

}  // namespace
}  // namespace v3d

using namespace v3d;


extern "C" int32_t v3d_plan_clips(v3d_context* ctx, const v3d_clip* clips, uint64_t n_clips,
                                  uint64_t* orders, uint64_t* order_counts, int32_t* distributed) {
    if (!ctx || (n_clips && (!clips || !order_counts || !distributed))) return V3D_ERR_INVALID_ARGUMENT;
    std::vector<PlanCamera> cams;
    std::vector<D3> pts;
    std::vector<uint64_t> cam_base(n_clips + 1, 0);
    std::vector<Inputs> inputs(n_clips);
    for (uint64_t k = 0; k < n_clips; ++k) {
        const v3d_clip& c = clips[k];
        if ((c.n_cameras && !c.cameras) || (c.n_sparse && !c.sparse_xyz) || (c.n_frames && !c.frames))
            return V3D_ERR_INVALID_ARGUMENT;
        inputs[k] = load_inputs(c.frames, c.n_frames, c.cameras, c.n_cameras, c.sparse_xyz, c.n_sparse,
                                c.focal);
        const uint64_t first = pts.size();
        for (uint64_t i = 0; i < c.n_sparse; ++i)
            pts.push_back(D3{c.sparse_xyz[3 * i], c.sparse_xyz[3 * i + 1], c.sparse_xyz[3 * i + 2]});
        for (uint64_t j = 0; j < c.n_cameras; ++j) {
            PlanCamera pc{};
            std::memcpy(pc.cam.R, c.cameras[j].rotation, sizeof(pc.cam.R));
            std::memcpy(pc.cam.t, c.cameras[j].translation, sizeof(pc.cam.t));
            pc.focal = c.focal;
            const bool has_frame = c.cameras[j].frame_index < c.n_frames;
            pc.first = first;
            pc.last = has_frame ? pts.size() : first;
            pc.width = has_frame ? c.frames[c.cameras[j].frame_index].width : 0;
            pc.height = has_frame ? c.frames[c.cameras[j].frame_index].height : 0;
            cams.push_back(pc);
        }
        cam_base[k + 1] = cams.size();
    }
    if (cam_base[n_clips] && !orders) return V3D_ERR_INVALID_ARGUMENT;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(ctx->stream);
    const uint64_t nc = cams.size();
    std::vector<uint32_t> visible(std::max<uint64_t>(nc, 1)), tiles(16 * std::max<uint64_t>(nc, 1));
    if (nc) {
        auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
        const size_t o_cams = 0, o_pts = up(sizeof(PlanCamera) * nc),
                     o_vis = up(o_pts + sizeof(D3) * std::max<size_t>(pts.size(), 1)),
                     o_tiles = up(o_vis + sizeof(uint32_t) * nc), need = o_tiles + sizeof(uint32_t) * 16 * nc;
        if (!ensure_arena(ctx, need)) {
            ctx->last_error = "device arena allocation failed";
            return V3D_ERR_OUT_OF_MEMORY;
        }
        char* base = static_cast<char*>(ctx->arena);
        auto* d_cams = reinterpret_cast<PlanCamera*>(base + o_cams);
        auto* d_pts = reinterpret_cast<D3*>(base + o_pts);
        auto* d_vis = reinterpret_cast<uint32_t*>(base + o_vis);
        auto* d_tiles = reinterpret_cast<uint32_t*>(base + o_tiles);
        V3D_CTX_CK(cudaMemcpyAsync(d_cams, cams.data(), sizeof(PlanCamera) * nc, cudaMemcpyHostToDevice, st));
        if (!pts.empty())
            V3D_CTX_CK(cudaMemcpyAsync(d_pts, pts.data(), sizeof(D3) * pts.size(), cudaMemcpyHostToDevice, st));
        const uint64_t launches0 = g_kernel_launches;
        const unsigned blocks = (unsigned)std::min<uint64_t>(nc, 148ull * 32);
        V3D_COUNTED k_landmark_coverage<<<blocks, 256, 0, st>>>(d_cams, nc, d_pts, d_vis, d_tiles);
        V3D_CTX_CK(cudaGetLastError());
        V3D_CTX_CK(cudaMemcpyAsync(visible.data(), d_vis, sizeof(uint32_t) * nc, cudaMemcpyDeviceToHost, st));
        V3D_CTX_CK(cudaMemcpyAsync(tiles.data(), d_tiles, sizeof(uint32_t) * 16 * nc, cudaMemcpyDeviceToHost, st));
        V3D_CTX_CK(cudaStreamSynchronize(st));
        ctx->last_launches = g_kernel_launches - launches0;
    }
    for (uint64_t k = 0; k < n_clips; ++k) {
        const Inputs& in = inputs[k];
        const uint64_t b = cam_base[k], n = cam_base[k + 1] - b;
        std::vector<int64_t> vis(n, -1);
        size_t covered = 0;
        for (uint64_t j = 0; j < n; ++j) {
            if (in.cameras[j].frame_index >= in.n_frames) continue;
            vis[j] = visible[b + j];
            size_t supported = 0;  // tiles that reached 2 landmarks (dense.rs:191-196)
            for (int t = 0; t < 16; ++t) supported += tiles[16 * (b + j) + t] >= 2;
            if (supported >= 8) ++covered;
        }
        const std::vector<size_t> order = order_from_visible(in.cameras, vis);
        for (size_t i = 0; i < order.size(); ++i) orders[b + i] = order[i];
        order_counts[k] = order.size();
        distributed[k] = covered >= n / 2 + 1 ? 1 : 0;
    }
    return V3D_OK;
}
