// v3d_mesh_patch_device_noalloc: the device mesh gates of one patch with all
// working memory in a file-scope device array, for callers that cannot
// allocate GPU memory (see include/v3d_dense.h).
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>

#include "mesh_batch.cuh"

namespace v3d {
namespace {

constexpr size_t kScratchBytes = V3D_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

// Working memory of every call; each GPU that loads the library holds it
// until exit.  Host code must not use the symbol itself as an address.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

std::mutex g_setup_mu;
void* g_scratch_addr[kMaxDevices] = {};

// Device address of the array on the current device, looked up once per device.
cudaError_t scratch_address(void** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_addr[dev]) {
        void* ptr = nullptr;
        e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_addr[dev] = ptr;
    }
    *out = g_scratch_addr[dev];
    return cudaSuccess;
}

__global__ void k_put_patch(MeshPatchDev* dst, MeshPatchDev patch) { *dst = patch; }

}  // namespace
}  // namespace v3d

using namespace v3d;

extern "C" int32_t v3d_mesh_patch_device_noalloc(
    const v3d_point* points_dev, const v3d_grid_site* sites_dev, uint64_t n_points,
    const v3d_camera* reference_camera, uint32_t width, uint32_t height, uint32_t grid_border,
    uint64_t grid_stride, double focal, v3d_mesh_triangle* triangles_dev,
    uint64_t triangle_capacity, v3d_mesh_counts* counts_dev, void* stream) {
    if (!reference_camera || !counts_dev || (n_points && (!points_dev || !sites_dev)) ||
        grid_stride == 0 || grid_stride > 0xFFFFFFFFull || width == 0 || height == 0 ||
        !std::isfinite(focal) || focal <= 0.0 || n_points > 0xFFFFFFFFull)
        return V3D_ERR_INVALID_ARGUMENT;
    const uint32_t stride = static_cast<uint32_t>(grid_stride);
    // the border arithmetic in 64 bits: 2 * grid_border does not wrap
    const uint64_t border2 = 2ull * grid_border;
    const uint32_t gw = width > border2 ? (uint32_t)((width - border2 + stride - 1) / stride) : 0;
    const uint32_t gh = height > border2 ? (uint32_t)((height - border2 + stride - 1) / stride) : 0;
    const uint64_t cells = static_cast<uint64_t>(gw) * gh;
    const uint64_t slots = mesh_slots(gw, gh);
    if (triangle_capacity < slots || (slots && !triangles_dev)) return V3D_ERR_INVALID_ARGUMENT;
    // sizes beyond the array are rejected before anything is enqueued
    if (mesh_scratch_layout(nullptr, 1, n_points, cells, slots, nullptr) > kScratchBytes)
        return V3D_ERR_INVALID_ARGUMENT;
    void* base = nullptr;
    if (scratch_address(&base) != cudaSuccess) return V3D_ERR_CUDA;
    MeshScratch s{};
    mesh_scratch_layout(base, 1, n_points, cells, slots, &s);
    MeshPatchDev patch;
    std::memset(&patch, 0, sizeof(patch));
    std::memcpy(patch.cam.R, reference_camera->rotation, sizeof(patch.cam.R));
    std::memcpy(patch.cam.t, reference_camera->translation, sizeof(patch.cam.t));
    patch.focal = focal;
    patch.width = width;
    patch.height = height;
    patch.border = grid_border;
    patch.stride = stride;
    patch.gw = gw;
    patch.gh = gh;
    patch.grid_off = 0;
    patch.slot_off = 0;
    patch.n_points = n_points;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the descriptor travels as a kernel argument (copied at launch), not as a
    // copy from this stack frame
    k_put_patch<<<1, 1, 0, st>>>(s.patches, patch);
    if (cudaGetLastError() != cudaSuccess) return V3D_ERR_CUDA;
    if (mesh_batch_enqueue(s, 1, cells, slots, points_dev, sites_dev, nullptr, nullptr, n_points,
                           triangles_dev, nullptr, st) != cudaSuccess)
        return V3D_ERR_CUDA;
    static_assert(sizeof(MeshCounters) == sizeof(v3d_mesh_counts), "counter layouts differ");
    if (cudaMemcpyAsync(counts_dev, s.counters, sizeof(v3d_mesh_counts), cudaMemcpyDeviceToDevice,
                        st) != cudaSuccess)
        return V3D_ERR_CUDA;
    return V3D_OK;
}
