// Reference-grid triangle gates (mesh_legacy.rs:150-555) on the device.
//
// The reference keys grid vertices in a BTreeMap, walks cell origins in
// BTreeSet order and deduplicates triangles by their sorted point-index
// triple.  Three corners of a unit cell identify that cell, and a gap bridge
// spans two cells in one direction, so no two candidates ever share a triple
// and the dedup never fires: every cell and every bridge is an independent
// work item.  Output order is restored by compacting the per-item slots in
// the reference's iteration order (cells x-major, then horizontal bridges,
// then vertical bridges).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "host.hpp"
#include "v3d_device.cuh"

namespace v3d {
namespace {

constexpr double kMaxGridReprojectionOffsetStrides = 0.5;  // mesh_legacy.rs:10
constexpr double kMaxMeshRelativeDepthJump = 0.15;         // :11
constexpr double kMaxBridgeRelativeDepthJump = 0.08;       // :12
constexpr double kMaxMeshEdgeFootprintMultiplier = 3.0;    // :13
constexpr double kMinMeshAreaFootprintRatio = 0.05;        // :14
constexpr double kMinMeshProjectedAreaFootprintRatio = 0.05;  // :15
constexpr unsigned long long kEmpty = 0ull;

struct MeshParams {
    DevCamera cam;
    uint32_t width, height, border, stride;
    double focal;
    uint32_t gw, gh;  // lattice size
    uint32_t n;       // points
};

struct Vtx {
    double x, y, z;     // position
    double px, py, d;   // projection into the reference
    float conf;
    uint32_t index;
};

// Orderable key: larger confidence first, then the smaller point index.
__device__ __forceinline__ unsigned long long vertex_key(float conf, uint32_t index) {
    uint32_t b = __float_as_uint(conf);
    b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
    return ((unsigned long long)b << 32) | (unsigned long long)(0xFFFFFFFFu - index);
}

__global__ void k_mesh_vertices(MeshParams mp, const v3d_point* __restrict__ pts,
                                const v3d_grid_site* __restrict__ sites,
                                const uint32_t* __restrict__ map,
                                unsigned long long* __restrict__ grid, Vtx* __restrict__ vtx) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < mp.n; i += gridDim.x * blockDim.x) {
        uint32_t pi = map ? map[i] : i;
        const v3d_point p = pts[pi];
        const v3d_grid_site s = sites[pi];
        D3 pos{(double)p.x, (double)p.y, (double)p.z};
        D3 q;
        vtx[i].index = 0xFFFFFFFFu;
        if (!project_exact(mp.cam, pos, mp.width, mp.height, mp.focal, q)) continue;
        // within_original_grid_footprint (mesh_legacy.rs:428-440)
        double limit = dmul((double)mp.stride, kMaxGridReprojectionOffsetStrides);
        if (!isfinite(q.x) || !isfinite(q.y)) continue;
        if (!(fabs(dsub(q.x, (double)s.x)) < limit && fabs(dsub(q.y, (double)s.y)) < limit)) continue;
        // original_grid_coordinate (mesh_legacy.rs:442-451)
        uint32_t limx = mp.width > mp.border ? mp.width - mp.border : 0;
        uint32_t limy = mp.height > mp.border ? mp.height - mp.border : 0;
        if (s.x < mp.border || s.x >= limx || s.y < mp.border || s.y >= limy) continue;
        uint32_t ox = s.x - mp.border, oy = s.y - mp.border;
        if (ox % mp.stride || oy % mp.stride) continue;
        uint32_t gx = ox / mp.stride, gy = oy / mp.stride;
        if (gx >= mp.gw || gy >= mp.gh) continue;
        Vtx v;
        v.x = pos.x;
        v.y = pos.y;
        v.z = pos.z;
        v.px = q.x;
        v.py = q.y;
        v.d = q.z;
        v.conf = p.confidence;
        v.index = i;
        vtx[i] = v;
        atomicMax(&grid[(size_t)gy * mp.gw + gx], vertex_key(p.confidence, i));
    }
}

struct Extent {
    int minx, maxx, miny, maxy;
    unsigned long long vertices;
};

__global__ void k_mesh_extent(MeshParams mp, const unsigned long long* __restrict__ grid,
                              int* __restrict__ ext, unsigned long long* __restrict__ count) {
    size_t total = (size_t)mp.gw * mp.gh;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < total;
         i += (size_t)gridDim.x * blockDim.x) {
        if (grid[i] == kEmpty) continue;
        int gy = (int)(i / mp.gw), gx = (int)(i - (size_t)gy * mp.gw);
        atomicMin(&ext[0], gx);
        atomicMax(&ext[1], gx);
        atomicMin(&ext[2], gy);
        atomicMax(&ext[3], gy);
        atomicAdd(count, 1ull);
    }
}

__device__ __forceinline__ const Vtx* vertex_at(const MeshParams& mp,
                                                const unsigned long long* grid, const Vtx* vtx,
                                                int gx, int gy) {
    if (gx < 0 || gy < 0 || gx >= (int)mp.gw || gy >= (int)mp.gh) return nullptr;
    unsigned long long k = grid[(size_t)gy * mp.gw + gx];
    if (k == kEmpty) return nullptr;
    uint32_t i = 0xFFFFFFFFu - (uint32_t)(k & 0xFFFFFFFFull);
    return vtx + i;
}

__device__ __forceinline__ double dnorm(double x, double y, double z) {
    return __dsqrt_rn(dadd(dadd(dmul(x, x), dmul(y, y)), dmul(z, z)));
}

// accepted_triangle (mesh_legacy.rs:473-537): 1 accepted, 2 discontinuity, 3 degenerate.
__device__ uint8_t gate(const MeshParams& mp, const Vtx& a, const Vtx& b, const Vtx& c,
                        double max_jump, v3d_mesh_triangle& out) {
    const double d0 = a.d, d1 = b.d, d2 = c.d;
    if (!isfinite(d0) || d0 <= 0.0 || !isfinite(d1) || d1 <= 0.0 || !isfinite(d2) || d2 <= 0.0)
        return 2;
    double mn = fmin(fmin(fmin(__longlong_as_double(0x7ff0000000000000LL), d0), d1), d2);
    double mx = fmax(fmax(fmax(-__longlong_as_double(0x7ff0000000000000LL), d0), d1), d2);
    if (ddiv(dsub(mx, mn), mx) > max_jump) return 2;
    const double stride = (double)mp.stride;
    double spa = dsub(dmul(dsub(b.px, a.px), dsub(c.py, a.py)), dmul(dsub(b.py, a.py), dsub(c.px, a.px)));
    double min_spa = dmul(dmul(stride, stride), kMinMeshProjectedAreaFootprintRatio);
    if (!isfinite(spa) || spa <= min_spa) return 3;
    double mean = ddiv(dadd(dadd(d0, d1), d2), 3.0);
    double step = ddiv(dmul(mean, stride), mp.focal);
    double max_edge = dmul(dmul(step, 1.4142135623730951), kMaxMeshEdgeFootprintMultiplier);
    double e0 = dnorm(dsub(a.x, b.x), dsub(a.y, b.y), dsub(a.z, b.z));
    double e1 = dnorm(dsub(b.x, c.x), dsub(b.y, c.y), dsub(b.z, c.z));
    double e2 = dnorm(dsub(c.x, a.x), dsub(c.y, a.y), dsub(c.z, a.z));
    if (!isfinite(e0) || e0 > max_edge || !isfinite(e1) || e1 > max_edge || !isfinite(e2) ||
        e2 > max_edge)
        return 2;
    double ux = dsub(b.x, a.x), uy = dsub(b.y, a.y), uz = dsub(b.z, a.z);
    double vx = dsub(c.x, a.x), vy = dsub(c.y, a.y), vz = dsub(c.z, a.z);
    double area = dnorm(dsub(dmul(uy, vz), dmul(uz, vy)), dsub(dmul(uz, vx), dmul(ux, vz)),
                        dsub(dmul(ux, vy), dmul(uy, vx)));
    double min_area = dmul(dmul(step, step), kMinMeshAreaFootprintRatio);
    if (!isfinite(area) || area <= min_area) return 3;
    float conf = fminf(fminf(a.conf, b.conf), c.conf);
    conf = fminf(fmaxf(conf, 0.0f), 1.0f);
    out.a = a.index;
    out.b = b.index;
    out.c = c.index;
    out.confidence = conf;
    out.pad = 0;
    return 1;
}

// Slots: [cells x 2][horizontal bridges][vertical bridges]
struct Layout {
    int ox0, oy0, cw, ch;   // cell origins: ox in [ox0, ox0+cw), oy in [oy0, oy0+ch)
    int hx0, hy0, hw, hh;   // horizontal bridges
    int vx0, vy0, vw, vh;   // vertical bridges
    size_t cells, hb, vb;
};

__global__ void k_mesh_triangles(MeshParams mp, Layout L, const unsigned long long* __restrict__ grid,
                                 const Vtx* __restrict__ vtx, uint8_t* __restrict__ slot_status,
                                 v3d_mesh_triangle* __restrict__ tris,
                                 unsigned long long* __restrict__ tallies) {
    // tallies: [0] origins in the BTreeSet, [1] candidate cells
    const size_t total = L.cells + L.hb + L.vb;
    for (size_t it = blockIdx.x * (size_t)blockDim.x + threadIdx.x; it < total;
         it += (size_t)gridDim.x * blockDim.x) {
        if (it < L.cells) {
            int oxi = (int)(it / L.ch), oyi = (int)(it - (size_t)oxi * L.ch);
            int ox = L.ox0 + oxi, oy = L.oy0 + oyi;
            const Vtx* tl = vertex_at(mp, grid, vtx, ox, oy);
            const Vtx* tr = vertex_at(mp, grid, vtx, ox + 1, oy);
            const Vtx* bl = vertex_at(mp, grid, vtx, ox, oy + 1);
            const Vtx* br = vertex_at(mp, grid, vtx, ox + 1, oy + 1);
            int present = (tl != nullptr) + (tr != nullptr) + (bl != nullptr) + (br != nullptr);
            slot_status[2 * it] = 0;
            slot_status[2 * it + 1] = 0;
            if (present > 0) atomicAdd(&tallies[0], 1ull);
            if (present < 3) continue;
            atomicAdd(&tallies[1], 1ull);
            const Vtx *t0[3], *t1[3];
            int n = 1;
            if (tl && tr && bl && br) {
                double a = dadd(dadd(dmul(dsub(tl->x, br->x), dsub(tl->x, br->x)),
                                     dmul(dsub(tl->y, br->y), dsub(tl->y, br->y))),
                                dmul(dsub(tl->z, br->z), dsub(tl->z, br->z)));
                double b = dadd(dadd(dmul(dsub(tr->x, bl->x), dsub(tr->x, bl->x)),
                                     dmul(dsub(tr->y, bl->y), dsub(tr->y, bl->y))),
                                dmul(dsub(tr->z, bl->z), dsub(tr->z, bl->z)));
                n = 2;
                if (a <= b) {
                    t0[0] = tl; t0[1] = tr; t0[2] = br;
                    t1[0] = tl; t1[1] = br; t1[2] = bl;
                } else {
                    t0[0] = tl; t0[1] = tr; t0[2] = bl;
                    t1[0] = tr; t1[1] = br; t1[2] = bl;
                }
            } else if (tl && tr && bl) {
                t0[0] = tl; t0[1] = tr; t0[2] = bl;
            } else if (tl && tr && br) {
                t0[0] = tl; t0[1] = tr; t0[2] = br;
            } else if (tl && bl && br) {
                t0[0] = tl; t0[1] = br; t0[2] = bl;
            } else {
                t0[0] = tr; t0[1] = br; t0[2] = bl;
            }
            slot_status[2 * it] = gate(mp, *t0[0], *t0[1], *t0[2], kMaxMeshRelativeDepthJump, tris[2 * it]);
            if (n == 2)
                slot_status[2 * it + 1] =
                    gate(mp, *t1[0], *t1[1], *t1[2], kMaxMeshRelativeDepthJump, tris[2 * it + 1]);
        } else if (it < L.cells + L.hb) {
            size_t k = it - L.cells;
            int gxi = (int)(k / L.hh), gyi = (int)(k - (size_t)gxi * L.hh);
            int gx = L.hx0 + gxi, gy = L.hy0 + gyi;
            size_t slot = 2 * L.cells + k;
            slot_status[slot] = 0;
            // horizontal_gap_bridge (mesh_legacy.rs:370-394)
            const Vtx* tl = vertex_at(mp, grid, vtx, gx, gy);
            const Vtx* tr = vertex_at(mp, grid, vtx, gx + 2, gy);
            const Vtx* bl = vertex_at(mp, grid, vtx, gx, gy + 1);
            const Vtx* br = vertex_at(mp, grid, vtx, gx + 2, gy + 1);
            const Vtx* tm = vertex_at(mp, grid, vtx, gx + 1, gy);
            const Vtx* bm = vertex_at(mp, grid, vtx, gx + 1, gy + 1);
            if (tl && tr && !tm && bm) {
                atomicAdd(&tallies[1], 1ull);
                slot_status[slot] = gate(mp, *tl, *tr, *bm, kMaxBridgeRelativeDepthJump, tris[slot]);
            } else if (bl && br && tm && !bm) {
                atomicAdd(&tallies[1], 1ull);
                slot_status[slot] = gate(mp, *bl, *tm, *br, kMaxBridgeRelativeDepthJump, tris[slot]);
            }
        } else {
            size_t k = it - L.cells - L.hb;
            int gxi = (int)(k / L.vh), gyi = (int)(k - (size_t)gxi * L.vh);
            int gx = L.vx0 + gxi, gy = L.vy0 + gyi;
            size_t slot = 2 * L.cells + L.hb + k;
            slot_status[slot] = 0;
            // vertical_gap_bridge (mesh_legacy.rs:396-420)
            const Vtx* tl = vertex_at(mp, grid, vtx, gx, gy);
            const Vtx* tr = vertex_at(mp, grid, vtx, gx + 1, gy);
            const Vtx* bl = vertex_at(mp, grid, vtx, gx, gy + 2);
            const Vtx* br = vertex_at(mp, grid, vtx, gx + 1, gy + 2);
            const Vtx* lm = vertex_at(mp, grid, vtx, gx, gy + 1);
            const Vtx* rm = vertex_at(mp, grid, vtx, gx + 1, gy + 1);
            if (tl && bl && !lm && rm) {
                atomicAdd(&tallies[1], 1ull);
                slot_status[slot] = gate(mp, *tl, *rm, *bl, kMaxBridgeRelativeDepthJump, tris[slot]);
            } else if (tr && br && lm && !rm) {
                atomicAdd(&tallies[1], 1ull);
                slot_status[slot] = gate(mp, *tr, *br, *lm, kMaxBridgeRelativeDepthJump, tris[slot]);
            }
        }
    }
}

bool grow_dev(void** p, size_t* have, size_t need) {
    if (*have >= need) return true;
    if (*p) cudaFree(*p);
    *p = nullptr;
    *have = 0;
    size_t cap = std::max(need, (size_t)1 << 20);
    if (cudaMalloc(p, cap) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    *have = cap;
    return true;
}

}  // namespace

// One legacy mesh pass over points[map[i]] (all points when map is empty).
// Fills `stats` and `tris` (indices into the mapped list).  Returns a status.
int32_t run_mesh_patch(v3d_context* ctx, const v3d_point* points, const v3d_grid_site* sites,
                       const std::vector<uint32_t>& map, size_t n_points, const HCamera& cam,
                       uint32_t width, uint32_t height, uint32_t border, uint32_t stride,
                       double focal, CancelPoll& cancel, v3d_mesh_stats& stats,
                       std::vector<v3d_mesh_triangle>& tris, bool& canceled) {
    cudaStream_t st = static_cast<cudaStream_t>(ctx->stream);
    canceled = false;
    tris.clear();
    const uint32_t gw = width > 2 * border ? (width - 2 * border + stride - 1) / stride : 0;
    const uint32_t gh = height > 2 * border ? (height - 2 * border + stride - 1) / stride : 0;
    const size_t n = map.empty() ? n_points : map.size();
    const size_t src_points = n_points;
    // device buffers: points, sites, map, grid, vertices, tallies, slots, triangles
    size_t off = 0;
    auto take = [&](size_t bytes) {
        off = (off + 255) & ~size_t(255);
        size_t a = off;
        off += bytes;
        return a;
    };
    const size_t o_pts = take(sizeof(v3d_point) * std::max<size_t>(src_points, 1));
    const size_t o_sites = take(sizeof(v3d_grid_site) * std::max<size_t>(src_points, 1));
    const size_t o_map = take(sizeof(uint32_t) * std::max<size_t>(map.size(), 1));
    const size_t o_grid = take(sizeof(unsigned long long) * std::max<size_t>((size_t)gw * gh, 1));
    const size_t o_vtx = take(sizeof(Vtx) * std::max<size_t>(n, 1));
    const size_t o_ext = take(sizeof(int) * 4 + sizeof(unsigned long long) * 4);
    const size_t base_need = off;
    if (!grow_dev(&ctx->arena, &ctx->arena_bytes, base_need + (1 << 20))) return V3D_ERR_OUT_OF_MEMORY;
    char* base = static_cast<char*>(ctx->arena);
    MeshParams mp;
    std::memcpy(mp.cam.R, cam.R, sizeof(mp.cam.R));
    std::memcpy(mp.cam.t, cam.t, sizeof(mp.cam.t));
    mp.width = width;
    mp.height = height;
    mp.border = border;
    mp.stride = stride;
    mp.focal = focal;
    mp.gw = gw;
    mp.gh = gh;
    mp.n = static_cast<uint32_t>(n);
    auto* d_pts = reinterpret_cast<v3d_point*>(base + o_pts);
    auto* d_sites = reinterpret_cast<v3d_grid_site*>(base + o_sites);
    auto* d_map = reinterpret_cast<uint32_t*>(base + o_map);
    auto* d_grid = reinterpret_cast<unsigned long long*>(base + o_grid);
    auto* d_vtx = reinterpret_cast<Vtx*>(base + o_vtx);
    auto* d_ext = reinterpret_cast<int*>(base + o_ext);
    auto* d_cnt = reinterpret_cast<unsigned long long*>(base + o_ext + 16);
    if (src_points) {
        cudaMemcpyAsync(d_pts, points, sizeof(v3d_point) * src_points, cudaMemcpyHostToDevice, st);
        cudaMemcpyAsync(d_sites, sites, sizeof(v3d_grid_site) * src_points, cudaMemcpyHostToDevice, st);
    }
    if (!map.empty())
        cudaMemcpyAsync(d_map, map.data(), sizeof(uint32_t) * map.size(), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(d_grid, 0, sizeof(unsigned long long) * std::max<size_t>((size_t)gw * gh, 1), st);
    int ext_init[4] = {0x7fffffff, -1, 0x7fffffff, -1};
    cudaMemcpyAsync(d_ext, ext_init, sizeof(ext_init), cudaMemcpyHostToDevice, st);
    cudaMemsetAsync(d_cnt, 0, sizeof(unsigned long long) * 4, st);
    if (n) {
        unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16);
        V3D_COUNTED k_mesh_vertices<<<blocks, 256, 0, st>>>(mp, d_pts, d_sites, map.empty() ? nullptr : d_map,
                                                d_grid, d_vtx);
    }
    size_t cells = (size_t)gw * gh;
    if (cells) {
        unsigned blocks = (unsigned)std::min<size_t>((cells + 255) / 256, 148 * 16);
        V3D_COUNTED k_mesh_extent<<<blocks, 256, 0, st>>>(mp, d_grid, d_ext, d_cnt);
    }
    int ext[4];
    unsigned long long vertices = 0;
    cudaMemcpyAsync(ext, d_ext, sizeof(ext), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(&vertices, d_cnt, sizeof(vertices), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        ctx->last_error = cudaGetErrorString(cudaGetLastError());
        return V3D_ERR_CUDA;
    }
    // the reference polls once per point while building the grid (mesh_legacy.rs:204-207)
    for (size_t i = 0; i < n; ++i)
        if (cancel.poll()) {
            canceled = true;
            return V3D_OK;
        }
    std::memset(&stats, 0, sizeof(stats));
    stats.attempted = 1;
    stats.grid_vertices = vertices;
    stats.rejected_grid_vertices = n > vertices ? n - vertices : 0;
    if (vertices < 3) {
        std::string r = "fewer than three fused dense points align with the reference sampling grid";
        stats.has_skip_reason = 1;
        std::strncpy(stats.skip_reason, r.c_str(), V3D_SKIP_REASON_BYTES - 1);
        return V3D_OK;
    }
    Layout L;
    L.ox0 = ext[0] - 1;
    L.oy0 = ext[2] - 1;
    L.cw = ext[1] - ext[0] + 2;
    L.ch = ext[3] - ext[2] + 2;
    L.cells = (size_t)L.cw * L.ch;
    L.hx0 = ext[0];
    L.hy0 = ext[2];
    L.hw = ext[1] - ext[0] >= 2 ? ext[1] - ext[0] - 1 : 0;
    L.hh = ext[3] - ext[2] + 1;
    L.hb = (size_t)L.hw * L.hh;
    L.vx0 = ext[0];
    L.vy0 = ext[2];
    L.vw = ext[1] - ext[0] + 1;
    L.vh = ext[3] - ext[2] >= 2 ? ext[3] - ext[2] - 1 : 0;
    L.vb = (size_t)L.vw * L.vh;
    const size_t slots = 2 * L.cells + L.hb + L.vb;
    size_t off2 = (base_need + 255) & ~size_t(255);
    const size_t o_slot = off2;
    off2 += slots;
    off2 = (off2 + 255) & ~size_t(255);
    const size_t o_tri = off2;
    off2 += slots * sizeof(v3d_mesh_triangle);
    if (off2 > ctx->arena_bytes) {
        // keep the vertex data: grow into a fresh buffer and copy the prefix over
        void* fresh = nullptr;
        if (cudaMalloc(&fresh, off2 + (1 << 20)) != cudaSuccess) {
            cudaGetLastError();
            return V3D_ERR_OUT_OF_MEMORY;
        }
        cudaMemcpyAsync(fresh, ctx->arena, base_need, cudaMemcpyDeviceToDevice, st);
        cudaStreamSynchronize(st);
        cudaFree(ctx->arena);
        ctx->arena = fresh;
        ctx->arena_bytes = off2 + (1 << 20);
        base = static_cast<char*>(ctx->arena);
        d_grid = reinterpret_cast<unsigned long long*>(base + o_grid);
        d_vtx = reinterpret_cast<Vtx*>(base + o_vtx);
        d_cnt = reinterpret_cast<unsigned long long*>(base + o_ext + 16);
    }
    auto* d_slot = reinterpret_cast<uint8_t*>(base + o_slot);
    auto* d_tri = reinterpret_cast<v3d_mesh_triangle*>(base + o_tri);
    {
        size_t items = L.cells + L.hb + L.vb;
        unsigned blocks = (unsigned)std::max<size_t>(1, std::min<size_t>((items + 255) / 256, 148 * 16));
        V3D_COUNTED k_mesh_triangles<<<blocks, 256, 0, st>>>(mp, L, d_grid, d_vtx, d_slot, d_tri, d_cnt + 1);
    }
    std::vector<uint8_t> hs(slots);
    std::vector<v3d_mesh_triangle> ht(slots);
    unsigned long long tallies[2];
    cudaMemcpyAsync(hs.data(), d_slot, slots, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(ht.data(), d_tri, slots * sizeof(v3d_mesh_triangle), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(tallies, d_cnt + 1, sizeof(tallies), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) {
        ctx->last_error = cudaGetErrorString(cudaGetLastError());
        return V3D_ERR_CUDA;
    }
    // polls: one per cell origin, then one per bridge column (mesh_legacy.rs:274-307, 321-328)
    size_t polls = tallies[0] + static_cast<size_t>(L.hw) + (L.vh > 0 ? static_cast<size_t>(L.vw) : 0);
    for (size_t i = 0; i < polls; ++i)
        if (cancel.poll()) {
            canceled = true;
            return V3D_OK;
        }
    stats.candidate_cells = tallies[1];
    for (size_t i = 0; i < slots; ++i) {
        if (hs[i] == 0) continue;
        ++stats.candidate_triangles;
        if (hs[i] == 1)
            tris.push_back(ht[i]);
        else if (hs[i] == 2)
            ++stats.rejected_discontinuities;
        else
            ++stats.rejected_degenerate;
    }
    stats.accepted_triangles = tris.size();
    return V3D_OK;
}

}  // namespace v3d
