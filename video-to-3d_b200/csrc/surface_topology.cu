// Mesh topology diagnostics on the device: the reference's surface_topology
// (colmap_surface.rs:125-157) behind v3d_surface_topology_of.
//
// Islands are the connected components of the vertices under the triangle
// edges, found with a lock-free union-find (a root hooks under the smaller
// root by compare-and-swap, so every component ends with its smallest vertex
// as root, whatever the order of the unions), counted over the triangles as
// the reference counts them; boundary edges are the edge keys that occur once
// after a radix sort.  Every figure is an integer count, so the result equals
// the reference's exactly.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/v3d_dense.h"
#include "host.hpp"
#include "pass_kernels.cuh"

namespace v3d {
namespace {

constexpr uint64_t kSmallIsland = 32;  // SMALL_ISLAND_TRIANGLES, colmap_surface.rs:123

// Parent links always point to smaller vertices (a root only ever hooks
// under a smaller root), so every walk to a root ends.  Links are read through
// L2 (ld.global.cg): other SMs change them while the kernels run, and L1 is not
// coherent with their writes.
__device__ __forceinline__ uint32_t find_root(const uint32_t* parent, uint32_t x) {
    uint32_t p = __ldcg(parent + x);
    while (p != x) {
        x = p;
        p = __ldcg(parent + x);
    }
    return x;
}

// The root of v, shortening the walked path: each visited
// link is pointed at its grandparent, an ancestor, so every path stays a path
// to the same root.  Only roots are ever swapped by unite, and a visited link
// is never a root's, so the plain stores and the swaps touch different links.
__device__ __forceinline__ uint32_t find_shortening(uint32_t* parent, uint32_t v) {
    uint32_t curr = __ldcg(parent + v);
    if (curr != v) {
        uint32_t prev = v, next;
        while (curr > (next = __ldcg(parent + curr))) {
            parent[prev] = next;
            prev = curr;
            curr = next;
        }
    }
    return curr;
}

// Joins the components of a and b: the larger root hooks under the smaller.
// A failed swap means another thread hooked that root meanwhile; retry from
// the new roots.  Every retry follows a successful hook elsewhere, so the loop
// ends; the bound on retries only guards that argument, recording a failure
// in *err instead of spinning on.
__device__ __forceinline__ void unite(uint32_t* parent, uint32_t a, uint32_t b, uint32_t* err) {
    for (uint32_t tries = 0; tries < (1u << 24); ++tries) {
        a = find_shortening(parent, a);
        b = find_shortening(parent, b);
        if (a == b) return;
        if (a < b) {
            const uint32_t t = a;
            a = b;
            b = t;
        }
        if (atomicCAS(&parent[a], a, b) == a) return;
    }
    atomicExch(err, 1u);
}

__global__ void k_init_parent(uint32_t* parent, uint64_t n) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x)
        parent[v] = (uint32_t)v;
}

// Unions over two edges of every triangle and the keys of all three (min << bits | max, with
// `bits` enough for any vertex index, so the sort needs only 2 * bits).
__global__ void k_unite_edges(const v3d_mesh_triangle* __restrict__ tris, uint64_t nt,
                              uint32_t* parent, unsigned long long* __restrict__ keys,
                              uint32_t* err, int bits) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nt;
         t += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v[3] = {(uint32_t)tris[t].a, (uint32_t)tris[t].b, (uint32_t)tris[t].c};
        for (int e = 0; e < 3; ++e) {
            const uint32_t a = v[e], b = v[(e + 1) % 3];
            const uint32_t lo = min(a, b), hi = max(a, b);
            keys[3 * t + e] = ((unsigned long long)lo << bits) | hi;
            if (e < 2) unite(parent, a, b, err);  // two edges already join all three corners
        }
    }
}

// Every vertex linked straight to its root, once the unions are done.  Only
// the vertex's own thread writes its link, so each link ends at the root; a
// walk that meets an updated link just arrives sooner.
__global__ void k_flatten(uint32_t* parent, uint64_t n) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x)
        parent[v] = find_root(parent, (uint32_t)v);
}

// Triangles per island root (the root of each triangle's first vertex).  The
// lanes of a warp that share a root add once (neighbouring triangles mostly
// share one), so a large island does not serialise on one address.
__global__ void k_island_sizes(const v3d_mesh_triangle* __restrict__ tris, uint64_t nt,
                               const uint32_t* __restrict__ root, unsigned long long* __restrict__ size) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const uint64_t first = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    // every lane of a warp takes the same number of turns, so the warp stays whole
    const uint64_t warp_first = first - (threadIdx.x & 31);
    for (uint64_t t0 = warp_first; t0 < nt; t0 += stride) {
        const uint64_t t = t0 + (threadIdx.x & 31);
        const uint32_t r = t < nt ? root[tris[t].a] : 0xFFFFFFFFu;
        const unsigned same = __match_any_sync(0xFFFFFFFFu, r);
        if (r != 0xFFFFFFFFu && (threadIdx.x & 31) == __ffs(same) - 1)
            atomicAdd(&size[r], (unsigned long long)__popc(same));
    }
}

// The island figures over the roots, and the edges that occur once.
__global__ void k_topology_counts(const unsigned long long* __restrict__ size, uint64_t n,
                                  const unsigned long long* __restrict__ sorted, uint64_t n_keys,
                                  unsigned long long* __restrict__ out) {
    unsigned long long islands = 0, small = 0, small_tris = 0, largest = 0, boundary = 0;
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long s = size[v];
        if (!s) continue;
        ++islands;
        if (s < kSmallIsland) {
            ++small;
            small_tris += s;
        }
        largest = max(largest, s);
    }
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_keys;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const unsigned long long k = sorted[i];
        if ((i == 0 || sorted[i - 1] != k) && (i + 1 == n_keys || sorted[i + 1] != k)) ++boundary;
    }
    // one atomic per block and figure: the warps reduce by shuffles, the
    // block through shared memory
    unsigned long long v[5] = {islands, small, small_tris, largest, boundary};
#pragma unroll
    for (int k = 0; k < 5; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            const unsigned long long w = __shfl_down_sync(0xFFFFFFFFu, v[k], o);
            v[k] = k == 3 ? max(v[k], w) : v[k] + w;
        }
    __shared__ unsigned long long part[5][32];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, warps = (blockDim.x + 31) >> 5;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < 5; ++k) part[k][warp] = v[k];
    __syncthreads();
    if (threadIdx.x < 5) {
        const int k = threadIdx.x;
        unsigned long long a = 0;
        for (int w = 0; w < warps; ++w) a = k == 3 ? max(a, part[k][w]) : a + part[k][w];
        if (a) {
            if (k == 3) atomicMax(&out[3], a);
            else atomicAdd(&out[k], a);
        }
    }
}

}  // namespace
}  // namespace v3d

using namespace v3d;


extern "C" int32_t v3d_surface_topology_of(v3d_context* ctx, const v3d_mesh_triangle* triangles,
                                           uint64_t nt, uint64_t n, v3d_surface_topology* out) {
    if (!ctx || !out || (nt && !triangles)) return V3D_ERR_INVALID_ARGUMENT;
    std::memset(out, 0, sizeof(*out));
    if (n >= 0xFFFFFFFFull || nt >= 0x40000000ull) {
        ctx->last_error = "surface topology takes fewer than 2^32 vertices and 2^30 triangles";
        return V3D_ERR_INVALID_ARGUMENT;
    }
    for (uint64_t t = 0; t < nt; ++t)
        if (triangles[t].a >= n || triangles[t].b >= n || triangles[t].c >= n) {
            ctx->last_error = "a triangle index is not below the vertex count";
            return V3D_ERR_INVALID_ARGUMENT;
        }
    if (nt == 0) return V3D_OK;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    float ms = 0.f;
    uint64_t launches = 0;
    const int32_t status = v3d::surface_topology_locked(ctx, triangles, nt, n, out, &ms, &launches);
    if (status == V3D_OK) {
        ctx->last_ms = ms;
        ctx->last_launches = launches;
    }
    return status;
}

namespace v3d {

int32_t surface_topology_locked(v3d_context* ctx, const v3d_mesh_triangle* triangles, uint64_t nt,
                                uint64_t n, v3d_surface_topology* out, float* device_ms,
                                uint64_t* launches) {
    cudaStream_t st = static_cast<cudaStream_t>(ctx->stream);
    const uint64_t nk = 3 * nt;
    size_t t_sort = 0;
    int bits = 1;  // bits of the largest vertex index
    while (bits < 32 && (n - 1) >> bits) ++bits;
    cub::DeviceRadixSort::SortKeys(nullptr, t_sort, (unsigned long long*)nullptr,
                                   (unsigned long long*)nullptr, (int)nk, 0, 2 * bits, st);
    auto up = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t o_tris = 0, o_parent = up(o_tris + sizeof(v3d_mesh_triangle) * nt),
                 o_size = up(o_parent + sizeof(uint32_t) * n),
                 o_keys = up(o_size + sizeof(unsigned long long) * n),
                 o_keys2 = up(o_keys + sizeof(unsigned long long) * nk),
                 o_out = up(o_keys2 + sizeof(unsigned long long) * nk), o_tmp = up(o_out + 64 + 16),
                 need = o_tmp + t_sort + 256;
    if (!ensure_arena(ctx, need)) {
        ctx->last_error = "device arena allocation failed";
        return V3D_ERR_OUT_OF_MEMORY;
    }
    char* base = static_cast<char*>(ctx->arena);
    auto* d_tris = reinterpret_cast<v3d_mesh_triangle*>(base + o_tris);
    auto* d_parent = reinterpret_cast<uint32_t*>(base + o_parent);
    auto* d_size = reinterpret_cast<unsigned long long*>(base + o_size);
    auto* d_keys = reinterpret_cast<unsigned long long*>(base + o_keys);
    auto* d_keys2 = reinterpret_cast<unsigned long long*>(base + o_keys2);
    auto* d_out = reinterpret_cast<unsigned long long*>(base + o_out);
    const uint64_t launches0 = g_kernel_launches;
    V3D_CTX_CK(cudaMemcpyAsync(d_tris, triangles, sizeof(v3d_mesh_triangle) * nt, cudaMemcpyHostToDevice, st));
    V3D_CTX_CK(cudaMemsetAsync(d_size, 0, sizeof(unsigned long long) * std::max<uint64_t>(n, 1), st));
    uint32_t* d_err = reinterpret_cast<uint32_t*>(base + o_out + 64);
    V3D_CTX_CK(cudaMemsetAsync(d_out, 0, 64 + 16, st));
    cudaEvent_t ev0, ev1;
    cudaEventCreate(&ev0);
    cudaEventCreate(&ev1);
    struct Events {
        cudaEvent_t a, b;
        ~Events() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } events{ev0, ev1};
    cudaEventRecord(ev0, st);
    V3D_COUNTED k_init_parent<<<grid_of(n), 256, 0, st>>>(d_parent, n);
    V3D_COUNTED k_unite_edges<<<grid_of(nt), 256, 0, st>>>(d_tris, nt, d_parent, d_keys, d_err, bits);
    V3D_COUNTED k_flatten<<<grid_of(n), 256, 0, st>>>(d_parent, n);
    V3D_COUNTED k_island_sizes<<<grid_of(nt), 256, 0, st>>>(d_tris, nt, d_parent, d_size);
    V3D_CTX_CK(cudaGetLastError());
    size_t bytes = t_sort;
    V3D_CTX_CK(cub::DeviceRadixSort::SortKeys(base + o_tmp, bytes, d_keys, d_keys2, (int)nk, 0, 2 * bits, st));
    V3D_COUNTED k_topology_counts<<<grid_of(std::max(n, nk)), 256, 0, st>>>(d_size, n, d_keys2, nk, d_out);
    V3D_CTX_CK(cudaGetLastError());
    cudaEventRecord(ev1, st);
    unsigned long long h[5];
    uint32_t err = 0;
    V3D_CTX_CK(cudaMemcpyAsync(h, d_out, sizeof(h), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaMemcpyAsync(&err, d_err, sizeof(err), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaStreamSynchronize(st));
    if (err) {
        ctx->last_error = "surface topology: a union did not settle within its retry bound";
        return V3D_ERR_CUDA;
    }
    out->islands = h[0];
    out->small_islands = h[1];
    out->small_island_triangles = h[2];
    out->largest_island_triangles = h[3];
    out->boundary_edges = h[4];
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess) *device_ms = ms;
    *launches = g_kernel_launches - launches0;
    return V3D_OK;
}

}  // namespace v3d
