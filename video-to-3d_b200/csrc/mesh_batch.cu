// Device-only reference-grid triangle gates over many patches
// (mesh_legacy.rs:150-555); see mesh_batch.cuh for the candidate layout.
#include <cuda_runtime.h>

#include "mesh_batch.cuh"
#include "pass_kernels.cuh"

namespace v3d {
namespace {

constexpr double kMaxGridReprojectionOffsetStrides = 0.5;     // mesh_legacy.rs:10
constexpr double kMaxMeshRelativeDepthJump = 0.15;            // :11
constexpr double kMaxBridgeRelativeDepthJump = 0.08;          // :12
constexpr double kMaxMeshEdgeFootprintMultiplier = 3.0;       // :13
constexpr double kMinMeshAreaFootprintRatio = 0.05;           // :14
constexpr double kMinMeshProjectedAreaFootprintRatio = 0.05;  // :15
constexpr uint32_t kNone = 0xFFFFFFFFu;

struct MVtx {
    double x, y, z;    // position (the f32 point widened)
    double px, py, d;  // projection into the reference camera
    float conf;
    uint32_t local;    // patch-local point index; kNone when off the grid
};

// Larger confidence first, then the smaller local index (better_grid_vertex,
// mesh_legacy.rs:422-426); 0 is never a key.
__device__ __forceinline__ unsigned long long vkey(float conf, uint32_t local) {
    uint32_t b = __float_as_uint(conf);
    b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);
    return ((unsigned long long)b << 32) | (unsigned long long)(0xFFFFFFFFu - local);
}

__device__ __forceinline__ uint32_t patch_of_slot(const MeshPatchDev* P, uint32_t n, uint64_t g) {
    uint32_t lo = 0, hi = n - 1;
    while (lo < hi) {
        uint32_t mid = (lo + hi + 1) >> 1;
        if (P[mid].slot_off <= g)
            lo = mid;
        else
            hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ const MVtx* vertex(const MeshScratch& s, const MeshPatchDev& P, int gx,
                                              int gy) {
    if (gx < 0 || gy < 0 || gx >= (int)P.gw || gy >= (int)P.gh) return nullptr;
    uint32_t w = s.winners[P.grid_off + (uint64_t)gy * P.gw + gx];
    return w == kNone ? nullptr : static_cast<const MVtx*>(s.vtx) + w;
}

__device__ __forceinline__ double dnorm3(double x, double y, double z) {
    return __dsqrt_rn(dadd(dadd(dmul(x, x), dmul(y, y)), dmul(z, z)));
}

// accepted_triangle (mesh_legacy.rs:473-537): 1 accepted, 2 discontinuity, 3 degenerate.
__device__ uint8_t gate(const MeshPatchDev& P, const MVtx& a, const MVtx& b, const MVtx& c,
                        double max_jump) {
    const double d0 = a.d, d1 = b.d, d2 = c.d;
    if (!isfinite(d0) || d0 <= 0.0 || !isfinite(d1) || d1 <= 0.0 || !isfinite(d2) || d2 <= 0.0)
        return 2;
    const double inf = __longlong_as_double(0x7ff0000000000000LL);
    double mn = fmin(fmin(fmin(inf, d0), d1), d2);
    double mx = fmax(fmax(fmax(-inf, d0), d1), d2);
    if (ddiv(dsub(mx, mn), mx) > max_jump) return 2;
    const double stride = (double)P.stride;
    double spa = dsub(dmul(dsub(b.px, a.px), dsub(c.py, a.py)), dmul(dsub(b.py, a.py), dsub(c.px, a.px)));
    if (!isfinite(spa) || spa <= dmul(dmul(stride, stride), kMinMeshProjectedAreaFootprintRatio))
        return 3;
    double step = ddiv(dmul(ddiv(dadd(dadd(d0, d1), d2), 3.0), stride), P.focal);
    double max_edge = dmul(dmul(step, 1.4142135623730951), kMaxMeshEdgeFootprintMultiplier);
    double e0 = dnorm3(dsub(a.x, b.x), dsub(a.y, b.y), dsub(a.z, b.z));
    double e1 = dnorm3(dsub(b.x, c.x), dsub(b.y, c.y), dsub(b.z, c.z));
    double e2 = dnorm3(dsub(c.x, a.x), dsub(c.y, a.y), dsub(c.z, a.z));
    if (!isfinite(e0) || e0 > max_edge || !isfinite(e1) || e1 > max_edge || !isfinite(e2) ||
        e2 > max_edge)
        return 2;
    double ux = dsub(b.x, a.x), uy = dsub(b.y, a.y), uz = dsub(b.z, a.z);
    double vx = dsub(c.x, a.x), vy = dsub(c.y, a.y), vz = dsub(c.z, a.z);
    double area = dnorm3(dsub(dmul(uy, vz), dmul(uz, vy)), dsub(dmul(uz, vx), dmul(ux, vz)),
                         dsub(dmul(ux, vy), dmul(uy, vx)));
    if (!isfinite(area) || area <= dmul(dmul(step, step), kMinMeshAreaFootprintRatio)) return 3;
    return 1;
}

// The candidate triangle of patch-local slot j, if any (cell_triangles,
// horizontal_gap_bridge, vertical_gap_bridge of mesh_legacy.rs:370-471).
// `first_of_cell` is set for the first slot of a cell with >= 3 corners.
__device__ bool slot_triangle(const MeshScratch& s, const MeshPatchDev& P, uint64_t j,
                              const MVtx*& a, const MVtx*& b, const MVtx*& c, double& jump,
                              bool& counts_cell) {
    counts_cell = false;
    const uint64_t cells = (uint64_t)(P.gw + 1) * (P.gh + 1);
    if (j < 2 * cells) {
        const uint64_t cell = j >> 1;
        const int which = (int)(j & 1);
        const int ox = (int)(cell / (P.gh + 1)) - 1, oy = (int)(cell % (P.gh + 1)) - 1;
        const MVtx* tl = vertex(s, P, ox, oy);
        const MVtx* tr = vertex(s, P, ox + 1, oy);
        const MVtx* bl = vertex(s, P, ox, oy + 1);
        const MVtx* br = vertex(s, P, ox + 1, oy + 1);
        const int present = (tl != nullptr) + (tr != nullptr) + (bl != nullptr) + (br != nullptr);
        if (present < 3) return false;
        counts_cell = which == 0;
        jump = kMaxMeshRelativeDepthJump;
        if (present == 4) {
            double d1 = dadd(dadd(dmul(dsub(tl->x, br->x), dsub(tl->x, br->x)),
                                  dmul(dsub(tl->y, br->y), dsub(tl->y, br->y))),
                             dmul(dsub(tl->z, br->z), dsub(tl->z, br->z)));
            double d2 = dadd(dadd(dmul(dsub(tr->x, bl->x), dsub(tr->x, bl->x)),
                                  dmul(dsub(tr->y, bl->y), dsub(tr->y, bl->y))),
                             dmul(dsub(tr->z, bl->z), dsub(tr->z, bl->z)));
            if (d1 <= d2) {
                if (which == 0) { a = tl; b = tr; c = br; } else { a = tl; b = br; c = bl; }
            } else {
                if (which == 0) { a = tl; b = tr; c = bl; } else { a = tr; b = br; c = bl; }
            }
            return true;
        }
        if (which == 1) return false;
        if (tl && tr && bl) { a = tl; b = tr; c = bl; }
        else if (tl && tr && br) { a = tl; b = tr; c = br; }
        else if (tl && bl && br) { a = tl; b = br; c = bl; }
        else { a = tr; b = br; c = bl; }
        return true;
    }
    uint64_t k = j - 2 * cells;
    const uint64_t hb = P.gw >= 3 ? (uint64_t)(P.gw - 2) * P.gh : 0;
    jump = kMaxBridgeRelativeDepthJump;
    if (k < hb) {
        const int gx = (int)(k / P.gh), gy = (int)(k % P.gh);
        const MVtx* tl = vertex(s, P, gx, gy);
        const MVtx* tr = vertex(s, P, gx + 2, gy);
        const MVtx* bl = vertex(s, P, gx, gy + 1);
        const MVtx* br = vertex(s, P, gx + 2, gy + 1);
        const MVtx* tm = vertex(s, P, gx + 1, gy);
        const MVtx* bm = vertex(s, P, gx + 1, gy + 1);
        if (tl && tr && !tm && bm) { a = tl; b = tr; c = bm; counts_cell = true; return true; }
        if (bl && br && tm && !bm) { a = bl; b = tm; c = br; counts_cell = true; return true; }
        return false;
    }
    k -= hb;
    const uint32_t vh = P.gh - 2;
    const int gx = (int)(k / vh), gy = (int)(k % vh);
    const MVtx* tl = vertex(s, P, gx, gy);
    const MVtx* tr = vertex(s, P, gx + 1, gy);
    const MVtx* bl = vertex(s, P, gx, gy + 2);
    const MVtx* br = vertex(s, P, gx + 1, gy + 2);
    const MVtx* lm = vertex(s, P, gx, gy + 1);
    const MVtx* rm = vertex(s, P, gx + 1, gy + 1);
    if (tl && bl && !lm && rm) { a = tl; b = rm; c = bl; counts_cell = true; return true; }
    if (tr && br && lm && !rm) { a = tr; b = br; c = lm; counts_cell = true; return true; }
    return false;
}

__global__ void k_mb_vertices(MeshScratch s, const v3d_point* __restrict__ pts,
                              const v3d_grid_site* __restrict__ sites,
                              const uint32_t* __restrict__ patch_of,
                              const uint32_t* __restrict__ local_of, uint64_t n) {
    MVtx* vtx = static_cast<MVtx*>(s.vtx);
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t pi = patch_of ? patch_of[i] : 0u;
        const MeshPatchDev& P = s.patches[pi];
        const uint32_t local = local_of ? local_of[i] : (uint32_t)i;
        vtx[i].local = kNone;
        const v3d_point p = pts[i];
        const v3d_grid_site st = sites[i];
        D3 pos{(double)p.x, (double)p.y, (double)p.z};
        D3 q;
        if (!project_exact(P.cam, pos, P.width, P.height, P.focal, q)) continue;
        // within_original_grid_footprint (mesh_legacy.rs:428-440)
        const double limit = dmul((double)P.stride, kMaxGridReprojectionOffsetStrides);
        if (!(fabs(dsub(q.x, (double)st.x)) < limit && fabs(dsub(q.y, (double)st.y)) < limit))
            continue;
        // original_grid_coordinate (mesh_legacy.rs:442-451)
        const uint32_t limx = P.width > P.border ? P.width - P.border : 0;
        const uint32_t limy = P.height > P.border ? P.height - P.border : 0;
        if (st.x < P.border || st.x >= limx || st.y < P.border || st.y >= limy) continue;
        const uint32_t ox = st.x - P.border, oy = st.y - P.border;
        if (ox % P.stride || oy % P.stride) continue;
        const uint32_t gx = ox / P.stride, gy = oy / P.stride;
        if (gx >= P.gw || gy >= P.gh) continue;
        MVtx v;
        v.x = pos.x;
        v.y = pos.y;
        v.z = pos.z;
        v.px = q.x;
        v.py = q.y;
        v.d = q.z;
        v.conf = p.confidence;
        v.local = local;
        vtx[i] = v;
        atomicMax(&s.grid_keys[P.grid_off + (uint64_t)gy * P.gw + gx], vkey(p.confidence, local));
    }
}

// Adds one lane's outcome counts to its patch's counters.  Consecutive
// lanes nearly always share a patch: the warp then reduces its counts and
// adds once per counter instead of every lane hitting the same addresses.
// Every lane of the warp must call this.
__device__ __forceinline__ void add_patch_counts(MeshCounters* counters, uint32_t pi, bool valid,
                                                 unsigned vertices, unsigned cells, unsigned cands,
                                                 unsigned acc, unsigned disc, unsigned degen) {
    const unsigned full = 0xFFFFFFFFu;
    const uint32_t pi0 = __shfl_sync(full, pi, 0);
    if (__all_sync(full, !valid || pi == pi0)) {
        vertices = __reduce_add_sync(full, vertices);
        cells = __reduce_add_sync(full, cells);
        cands = __reduce_add_sync(full, cands);
        acc = __reduce_add_sync(full, acc);
        disc = __reduce_add_sync(full, disc);
        degen = __reduce_add_sync(full, degen);
        if ((threadIdx.x & 31) != 0) return;
        pi = pi0;
    } else if (!valid) {
        return;
    }
    MeshCounters& c = counters[pi];
    if (vertices) atomicAdd(&c.vertices, (unsigned long long)vertices);
    if (cells) atomicAdd(&c.candidate_cells, (unsigned long long)cells);
    if (cands) atomicAdd(&c.candidate_triangles, (unsigned long long)cands);
    if (acc) atomicAdd(&c.accepted, (unsigned long long)acc);
    if (disc) atomicAdd(&c.discontinuities, (unsigned long long)disc);
    if (degen) atomicAdd(&c.degenerate, (unsigned long long)degen);
}

__global__ void k_mb_winners(MeshScratch s, const v3d_grid_site* __restrict__ sites,
                             const uint32_t* __restrict__ patch_of, uint64_t n) {
    const MVtx* vtx = static_cast<const MVtx*>(s.vtx);
    const unsigned lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    // warp-aligned turns, so every lane reaches the counter reduction
    for (uint64_t i0 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x - lane; i0 < n; i0 += stride) {
        const uint64_t i = i0 + lane;
        uint32_t pi = 0;
        unsigned won = 0;
        if (i < n) {
            const MVtx v = vtx[i];
            pi = patch_of ? patch_of[i] : 0u;
            if (v.local != kNone) {
                const MeshPatchDev& P = s.patches[pi];
                const v3d_grid_site st = sites[i];
                const uint64_t cell = P.grid_off + (uint64_t)((st.y - P.border) / P.stride) * P.gw +
                                      (st.x - P.border) / P.stride;
                if (s.grid_keys[cell] == vkey(v.conf, v.local)) {
                    s.winners[cell] = (uint32_t)i;
                    won = 1;
                }
            }
        }
        add_patch_counts(s.counters, pi, i < n, won, 0, 0, 0, 0, 0);
    }
}

__global__ void k_mb_slots(MeshScratch s, uint32_t n_patches, uint64_t total_slots) {
    const unsigned lane = threadIdx.x & 31;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t g0 = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x - lane; g0 < total_slots; g0 += stride) {
        const uint64_t g = g0 + lane;
        uint32_t pi = 0;
        unsigned cells = 0, cands = 0, acc = 0, disc = 0, degen = 0;
        if (g < total_slots) {
            s.slot_status[g] = 0;
            pi = patch_of_slot(s.patches, n_patches, g);
            const MeshPatchDev& P = s.patches[pi];
            const MVtx *a, *b, *cc;
            double jump;
            bool counts_cell;
            if (P.n_points >= 3 && s.counters[pi].vertices >= 3 &&
                slot_triangle(s, P, g - P.slot_off, a, b, cc, jump, counts_cell)) {
                cells = counts_cell ? 1u : 0u;
                cands = 1;
                const uint8_t st = gate(P, *a, *b, *cc, jump);
                s.slot_status[g] = st;
                acc = st == 1;
                disc = st == 2;
                degen = st != 1 && st != 2;
            }
        }
        add_patch_counts(s.counters, pi, g < total_slots, 0, cells, cands, acc, disc, degen);
    }
}

__global__ void k_mb_emit(MeshScratch s, uint32_t n_patches, v3d_mesh_triangle* __restrict__ tris,
                          uint32_t* __restrict__ tri_patch) {
    const uint32_t n = *s.count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint64_t g = s.slot_idx[i];
        const uint32_t pi = patch_of_slot(s.patches, n_patches, g);
        const MeshPatchDev& P = s.patches[pi];
        const MVtx *a, *b, *c;
        double jump;
        bool counts_cell;
        slot_triangle(s, P, g - P.slot_off, a, b, c, jump, counts_cell);
        v3d_mesh_triangle t;
        t.a = a->local;
        t.b = b->local;
        t.c = c->local;
        t.confidence = fminf(fmaxf(fminf(fminf(a->conf, b->conf), c->conf), 0.0f), 1.0f);
        t.pad = 0;
        tris[i] = t;
        if (tri_patch) tri_patch[i] = pi;
    }
}

unsigned blocks_for(uint64_t n) {
    uint64_t b = (n + 255) / 256;
    if (b > 148 * 32) b = 148 * 32;
    return (unsigned)(b ? b : 1);
}

}  // namespace

size_t mesh_scratch_layout(void* base, uint32_t n_patches, uint64_t n_points,
                           uint64_t total_cells, uint64_t total_slots, MeshScratch* s) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        off = (off + 255) & ~size_t(255);
        size_t at = off;
        off += bytes;
        return at;
    };
    const size_t o_p = take(sizeof(MeshPatchDev) * n_patches);
    const size_t o_c = take(sizeof(MeshCounters) * n_patches);
    const size_t o_k = take(sizeof(unsigned long long) * total_cells);
    const size_t o_w = take(sizeof(uint32_t) * total_cells);
    const size_t o_v = take(sizeof(MVtx) * n_points);
    const size_t o_s = take(total_slots);
    const size_t o_i = take(sizeof(uint32_t) * total_slots);
    const size_t o_n = take(sizeof(uint32_t));
    const size_t o_x = take(compaction_scratch_bytes(total_slots > 0 ? total_slots : 1));
    if (base && s) {
        char* b = static_cast<char*>(base);
        s->patches = reinterpret_cast<MeshPatchDev*>(b + o_p);
        s->counters = reinterpret_cast<MeshCounters*>(b + o_c);
        s->grid_keys = reinterpret_cast<unsigned long long*>(b + o_k);
        s->winners = reinterpret_cast<uint32_t*>(b + o_w);
        s->vtx = b + o_v;
        s->slot_status = reinterpret_cast<uint8_t*>(b + o_s);
        s->slot_idx = reinterpret_cast<uint32_t*>(b + o_i);
        s->count = reinterpret_cast<uint32_t*>(b + o_n);
        s->compact_scratch = b + o_x;
    }
    return off;
}

cudaError_t mesh_batch_enqueue(const MeshScratch& s, uint32_t n_patches, uint64_t total_cells,
                               uint64_t total_slots, const v3d_point* points,
                               const v3d_grid_site* sites, const uint32_t* patch_of,
                               const uint32_t* local_of, uint64_t n_points,
                               v3d_mesh_triangle* tris, uint32_t* tri_patch,
                               cudaStream_t stream) {
    cudaError_t e;
    if ((e = cudaMemsetAsync(s.counters, 0, sizeof(MeshCounters) * n_patches, stream))) return e;
    if ((e = cudaMemsetAsync(s.grid_keys, 0, sizeof(unsigned long long) * total_cells, stream)))
        return e;
    if ((e = cudaMemsetAsync(s.winners, 0xFF, sizeof(uint32_t) * total_cells, stream))) return e;
    if (n_points) {
        V3D_COUNTED k_mb_vertices<<<blocks_for(n_points), 256, 0, stream>>>(s, points, sites, patch_of, local_of,
                                                                n_points);
        V3D_COUNTED k_mb_winners<<<blocks_for(n_points), 256, 0, stream>>>(s, sites, patch_of, n_points);
    }
    if (total_slots) {
        V3D_COUNTED k_mb_slots<<<blocks_for(total_slots), 256, 0, stream>>>(s, n_patches, total_slots);
    }
    if ((e = cudaGetLastError())) return e;
    if ((e = launch_compact(s.slot_status, 1, total_slots, s.slot_idx, s.count, s.compact_scratch,
                            stream)))
        return e;
    V3D_COUNTED k_mb_emit<<<blocks_for(total_slots), 256, 0, stream>>>(s, n_patches, tris, tri_patch);
    return cudaGetLastError();
}

}  // namespace v3d
