// Cross-reference surface fusion on the device: the reference's
// fuse_mutually_supported_vertices_with_control (surface_fusion.rs:369-549)
// with its vertex evidence (surface_fusion.rs:723-814) and topology gate
// (surface_fusion.rs:566-696), behind v3d_fuse_mutually_supported_vertices.
//
// Every f64 operation is written with explicitly rounded intrinsics in the
// reference's order (nalgebra's left-to-right dot and norm, component-wise
// vector arithmetic, no fused multiply-add), and every order the reference's
// result depends on is kept: per-vertex normal and edge sums run over the
// vertex's triangles in index order (a stable radix sort of the incidence
// entries by vertex), the global edge scale is the median of the sorted
// lengths, and each vertex scans its 27 neighbour cells dz-dy-dx from -1 to 1
// with every cell's vertices in index order (cells found through a hash table,
// the eligible vertices sorted stably by their cell's representative), so the
// nearest-neighbour tie rule sees the candidates in the reference's order.  Moves, pairs and moved indices come out of
// order-preserving compactions.  The outcome is the reference's bit for bit.
//
// The work is HBM- and latency-bound integer/f64 bookkeeping: per triangle
// and per vertex kernels, CUB sorts and scans, and a handful of host reads
// (the global edge scale, and one flag per topology round).
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "../../include/v3d_dense.h"
#include "host.hpp"
#include "pass_kernels.cuh"

namespace v3d {
namespace {

constexpr double kGeometricEpsilon = 1.0e-9;           // surface_fusion.rs:6
constexpr double kMaxLocalEdgeFraction = 0.28;         // :7
constexpr double kMaxGlobalEdgeFraction = 0.35;        // :8
constexpr double kMinNormalAlignment = 0.94;           // :9
constexpr double kMinIncidentNormalAlignment = 0.985;  // :10
constexpr double kMinIncidentAreaRatio = 0.75;         // :11
constexpr double kMinConfidenceWeight = 0.05;          // :12
constexpr uint32_t kNone = 0xFFFFFFFFu;

__device__ __forceinline__ D3 vsub(D3 a, D3 b) { return D3{dsub(a.x, b.x), dsub(a.y, b.y), dsub(a.z, b.z)}; }
__device__ __forceinline__ double vdot(D3 a, D3 b) {
    return dadd(dadd(dmul(a.x, b.x), dmul(a.y, b.y)), dmul(a.z, b.z));
}
__device__ __forceinline__ double vnorm(D3 v) { return __dsqrt_rn(vdot(v, v)); }
__device__ __forceinline__ D3 vcross(D3 a, D3 b) {
    return D3{dsub(dmul(a.y, b.z), dmul(a.z, b.y)), dsub(dmul(a.z, b.x), dmul(a.x, b.z)),
              dsub(dmul(a.x, b.y), dmul(a.y, b.x))};
}
// point_position (surface_fusion.rs:824-830)
__device__ __forceinline__ bool position_of(const v3d_point& p, D3& v) {
    v = D3{(double)p.x, (double)p.y, (double)p.z};
    return isfinite(v.x) && isfinite(v.y) && isfinite(v.z);
}
// Rust's `f64 as i64`: saturating, NaN to 0
__device__ __forceinline__ int64_t as_i64(double v) {
    if (isnan(v)) return 0;
    if (v >= 9223372036854775807.0) return INT64_MAX;
    if (v <= -9223372036854775808.0) return INT64_MIN;
    return (int64_t)v;
}

struct Cell {
    int64_t x, y, z;
};
__device__ __forceinline__ bool cell_eq(const Cell& a, const Cell& b) {
    return a.x == b.x && a.y == b.y && a.z == b.z;
}
__device__ __forceinline__ uint32_t cell_hash(const Cell& c) {
    uint64_t h = (uint64_t)c.x * 0x9E3779B97F4A7C15ull ^ (uint64_t)c.y * 0xC2B2AE3D27D4EB4Full ^
                 (uint64_t)c.z * 0x165667B19E3779F9ull;
    h ^= h >> 29;
    h *= 0xBF58476D1CE4E5B9ull;
    h ^= h >> 32;
    return (uint32_t)h;
}

// An eligible vertex as the neighbour scan reads it, in cell order.
struct Member {
    float x, y, z;
    uint32_t index;
    int64_t group;
    double scale;
    D3 normal;
    uint32_t rep;  // eligible position of its cell's representative
    uint32_t pad;  // 64 bytes
};

struct Move {
    uint32_t first, second;
    D3 position;
};

// vertex_surface_evidence, per triangle (surface_fusion.rs:736-783): the
// validity gates, the three edge lengths and the confidence-weighted unit
// normal.
__global__ void k_tri_evidence(const v3d_point* __restrict__ pts, uint64_t n,
                               const v3d_mesh_triangle* __restrict__ tris, uint64_t nt,
                               uint32_t* __restrict__ valid, double* __restrict__ len,
                               D3* __restrict__ wn) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nt;
         t += (uint64_t)gridDim.x * blockDim.x) {
        valid[t] = 0;
        const v3d_mesh_triangle tr = tris[t];
        if (tr.a == tr.b || tr.b == tr.c || tr.c == tr.a || tr.a >= n || tr.b >= n || tr.c >= n)
            continue;
        D3 a, b, c;
        if (!position_of(pts[tr.a], a) || !position_of(pts[tr.b], b) || !position_of(pts[tr.c], c))
            continue;
        const D3 ab = vsub(b, a), ac = vsub(c, a), bc = vsub(c, b);
        const double lab = vnorm(ab), lac = vnorm(ac), lbc = vnorm(bc);
        if (!isfinite(lab) || lab <= kGeometricEpsilon || !isfinite(lac) ||
            lac <= kGeometricEpsilon || !isfinite(lbc) || lbc <= kGeometricEpsilon)
            continue;
        const D3 nrm = vcross(ab, ac);
        const double nl = vnorm(nrm);
        if (!isfinite(nl) || nl <= kGeometricEpsilon) continue;
        double conf = (double)tr.confidence;  // clamp(0.05, 1.0), NaN stays NaN
        if (conf < kMinConfidenceWeight) conf = kMinConfidenceWeight;
        if (conf > 1.0) conf = 1.0;
        wn[t] = D3{dmul(ddiv(nrm.x, nl), conf), dmul(ddiv(nrm.y, nl), conf),
                   dmul(ddiv(nrm.z, nl), conf)};
        len[3 * t] = lab;
        len[3 * t + 1] = lac;
        len[3 * t + 2] = lbc;
        valid[t] = 1;
    }
}

// Incidence entries of the valid triangles in triangle order: vertex keys,
// triangle values, and each valid triangle's edge lengths for the median.
__global__ void k_incidence(const v3d_mesh_triangle* __restrict__ tris, uint64_t nt,
                            const uint32_t* __restrict__ valid, const uint32_t* __restrict__ pos,
                            const double* __restrict__ len, uint32_t* __restrict__ keys,
                            uint32_t* __restrict__ vals, double* __restrict__ lengths,
                            uint32_t* __restrict__ vcount) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nt;
         t += (uint64_t)gridDim.x * blockDim.x) {
        if (!valid[t]) continue;
        const uint64_t e = 3ull * pos[t];
        const uint32_t v[3] = {(uint32_t)tris[t].a, (uint32_t)tris[t].b, (uint32_t)tris[t].c};
        for (int k = 0; k < 3; ++k) {
            keys[e + k] = v[k];
            vals[e + k] = (uint32_t)t;
            lengths[e + k] = len[3 * t + k];
            atomicAdd(&vcount[v[k]], 1u);
        }
    }
}

// vertex_surface_evidence, per vertex (surface_fusion.rs:760-813): the normal
// and edge sums over the vertex's triangles in index order, the unit normal
// and the local edge scale.
__global__ void k_vertex_evidence(uint64_t n, const v3d_mesh_triangle* __restrict__ tris,
                                  const uint32_t* __restrict__ off, const uint32_t* __restrict__ tri_of,
                                  const double* __restrict__ len, const D3* __restrict__ wn,
                                  D3* __restrict__ normal, double* __restrict__ scale,
                                  uint8_t* __restrict__ has) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x) {
        D3 s{0.0, 0.0, 0.0};
        double es = 0.0;
        uint64_t cnt = 0;
        for (uint32_t i = off[v]; i < off[v + 1]; ++i) {
            const uint32_t t = tri_of[i];
            const D3 w = wn[t];
            s = D3{dadd(s.x, w.x), dadd(s.y, w.y), dadd(s.z, w.z)};
            const double lab = len[3 * t], lac = len[3 * t + 1], lbc = len[3 * t + 2];
            const v3d_mesh_triangle tr = tris[t];
            const double e = tr.a == v ? dadd(lab, lac) : tr.b == v ? dadd(lab, lbc) : dadd(lac, lbc);
            es = dadd(es, e);
            cnt += 2;
        }
        uint8_t h = 0;
        const double l = vnorm(s);
        if (isfinite(l) && l > kGeometricEpsilon) {
            normal[v] = D3{ddiv(s.x, l), ddiv(s.y, l), ddiv(s.z, l)};
            h |= 1;
        }
        if (cnt > 0 && isfinite(es)) {
            scale[v] = ddiv(es, (double)cnt);
            h |= 2;
        }
        has[v] = h;
    }
}

// Eligible vertices (surface_fusion.rs:400-416) and their cells.
__global__ void k_eligible(const v3d_point* __restrict__ pts, uint64_t n,
                           const int64_t* __restrict__ membership, const uint8_t* __restrict__ has,
                           double cell_size, uint8_t* __restrict__ eligible, Cell* __restrict__ cell) {
    for (uint64_t v = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; v < n;
         v += (uint64_t)gridDim.x * blockDim.x) {
        D3 p;
        const bool ok = membership[v] >= 0 && has[v] == 3 && position_of(pts[v], p);
        eligible[v] = ok ? 1 : 0;
        if (ok)
            cell[v] = Cell{as_i64(floor(ddiv(p.x, cell_size))), as_i64(floor(ddiv(p.y, cell_size))),
                           as_i64(floor(ddiv(p.z, cell_size)))};
    }
}

__global__ void k_gather_cells(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ count,
                               const Cell* __restrict__ cell, Cell* __restrict__ out) {
    const uint32_t m = *count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
        out[k] = cell[idx[k]];
}

// The cell table: open addressing over `mask + 1` slots, each holding the
// eligible position k of the first vertex that claimed its cell; every
// eligible vertex learns its cell's representative, which keys the sort.
__global__ void k_cell_insert(const Cell* __restrict__ el_cell, const uint32_t* __restrict__ count,
                              uint32_t* __restrict__ table, uint32_t mask, uint32_t* __restrict__ rep) {
    const uint32_t m = *count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const Cell c = el_cell[k];
        uint32_t h = cell_hash(c) & mask, r = k;
        for (uint32_t probe = 0; probe <= mask; ++probe, h = (h + 1) & mask) {
            const uint32_t prev = atomicCAS(&table[h], kNone, k);
            if (prev == kNone) break;
            if (cell_eq(el_cell[prev], c)) {
                r = prev;
                break;
            }
        }
        rep[k] = r;
    }
}

// Cell-ordered member records and each cell's [begin, end) range, by
// representative.
__global__ void k_members(const uint32_t* __restrict__ sorted_rep, const uint32_t* __restrict__ sorted_v,
                          const uint32_t* __restrict__ count, const v3d_point* __restrict__ pts,
                          const int64_t* __restrict__ membership, const D3* __restrict__ normal,
                          const double* __restrict__ scale, Member* __restrict__ members,
                          uint32_t* __restrict__ begin, uint32_t* __restrict__ end) {
    const uint32_t m = *count;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < m; j += gridDim.x * blockDim.x) {
        const uint32_t v = sorted_v[j], r = sorted_rep[j];
        const v3d_point p = pts[v];
        members[j] = Member{p.x, p.y, p.z, v, membership[v], scale[v], normal[v], r, 0u};
        if (j == 0 || sorted_rep[j - 1] != r) begin[r] = j;
        if (j + 1 == m || sorted_rep[j + 1] != r) end[r] = j + 1;
    }
}

// The mutually-nearest search (surface_fusion.rs:418-481), a thread per
// eligible vertex in cell order: its 27 neighbour cells in the reference's
// order (dz, dy, dx from -1 to 1), each cell's vertices in index order, the
// reference's replace rule.  The scan waits on L2 reads (cell table, member
// records), so the kernel trades registers for resident warps: six blocks of
// 256 threads per SM.
__global__ void __launch_bounds__(256, 6) k_nearest(const Member* __restrict__ members, const Cell* __restrict__ el_cell,
                          const uint32_t* __restrict__ n_el_dev, const uint32_t* __restrict__ table,
                          uint32_t mask, const uint32_t* __restrict__ begin,
                          const uint32_t* __restrict__ end, double global,
                          uint32_t* __restrict__ nearest, double* __restrict__ nearest_d,
                          unsigned long long* __restrict__ counters) {
    const uint32_t n_el = *n_el_dev;
    const double gmax = dmul(global, kMaxGlobalEdgeFraction);
    unsigned long long cand = 0, rejn = 0;
    for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n_el; j += gridDim.x * blockDim.x) {
        const Member me = members[j];
        const uint32_t i = me.index;
        const Cell c = el_cell[me.rep];
        const D3 p{(double)me.x, (double)me.y, (double)me.z};
        uint32_t best = kNone;
        double best_d = 0.0;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    const Cell q{(int64_t)((uint64_t)c.x + (uint64_t)(int64_t)dx),
                                 (int64_t)((uint64_t)c.y + (uint64_t)(int64_t)dy),
                                 (int64_t)((uint64_t)c.z + (uint64_t)(int64_t)dz)};
                    uint32_t r = kNone, h = cell_hash(q) & mask;
                    for (uint32_t probe = 0; probe <= mask; ++probe, h = (h + 1) & mask) {
                        const uint32_t s = table[h];
                        if (s == kNone) break;
                        if (cell_eq(el_cell[s], q)) {
                            r = s;
                            break;
                        }
                    }
                    if (r == kNone) continue;
                    for (uint32_t k = begin[r]; k < end[r]; ++k) {
                        const Member o = members[k];
                        if (o.index == i || o.group == me.group) continue;
                        const D3 op{(double)o.x, (double)o.y, (double)o.z};
                        const double maxd =
                            fmin(dmul(fmin(me.scale, o.scale), kMaxLocalEdgeFraction), gmax);
                        const double d = vnorm(vsub(op, p));
                        if (!isfinite(d) || d > maxd) continue;
                        if (i < o.index) ++cand;
                        const double align = fabs(vdot(me.normal, o.normal));
                        if (align < kMinNormalAlignment) {
                            if (i < o.index) ++rejn;
                            continue;
                        }
                        bool replace = best == kNone;
                        if (!replace)
                            replace = d < dsub(best_d, kGeometricEpsilon) ||
                                      (fabs(dsub(d, best_d)) <= kGeometricEpsilon && o.index < best);
                        if (replace) {
                            best = o.index;
                            best_d = d;
                        }
                    }
                }
        nearest[i] = best;
        nearest_d[i] = best_d;
    }
    // one atomic per block and counter (per-thread atomics on two addresses
    // serialise in L2)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        cand += __shfl_down_sync(0xFFFFFFFFu, cand, o);
        rejn += __shfl_down_sync(0xFFFFFFFFu, rejn, o);
    }
    __shared__ unsigned long long part[2][8];
    if ((threadIdx.x & 31) == 0) {
        part[0][threadIdx.x >> 5] = cand;
        part[1][threadIdx.x >> 5] = rejn;
    }
    __syncthreads();
    if (threadIdx.x < 2) {
        unsigned long long a = 0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) a += part[threadIdx.x][w];
        if (a) atomicAdd(&counters[threadIdx.x], a);
    }
}

// Mutually nearest pairs and their confidence-weighted positions
// (surface_fusion.rs:483-510), flagged at the pair's first vertex.
__global__ void k_mutual(const v3d_point* __restrict__ pts, uint64_t n,
                         const uint32_t* __restrict__ nearest, uint8_t* __restrict__ flag,
                         D3* __restrict__ fused) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        flag[i] = 0;
        const uint32_t o = nearest[i];
        if (o == kNone || i >= o || nearest[o] != (uint32_t)i) continue;
        D3 p, q;
        if (!position_of(pts[i], p) || !position_of(pts[o], q)) continue;
        const double w = fmax((double)pts[i].confidence, kMinConfidenceWeight);
        const double ow = fmax((double)pts[o].confidence, kMinConfidenceWeight);
        const double ws = dadd(w, ow);
        fused[i] = D3{ddiv(dadd(dmul(p.x, w), dmul(q.x, ow)), ws),
                      ddiv(dadd(dmul(p.y, w), dmul(q.y, ow)), ws),
                      ddiv(dadd(dmul(p.z, w), dmul(q.z, ow)), ws)};
        flag[i] = 1;
    }
}

__global__ void k_make_moves(const uint32_t* __restrict__ first, const uint32_t* __restrict__ count,
                             const uint32_t* __restrict__ nearest, const D3* __restrict__ fused,
                             Move* __restrict__ moves, int32_t* __restrict__ move_of,
                             uint8_t* __restrict__ active) {
    const uint32_t m = *count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const uint32_t i = first[k], o = nearest[i];
        moves[k] = Move{i, o, fused[i]};
        move_of[i] = (int32_t)k;
        move_of[o] = (int32_t)k;
        active[k] = 1;
    }
}

__device__ __forceinline__ bool proposed_of(uint64_t v, const v3d_point* pts, const Move* moves,
                                            const uint8_t* active, const int32_t* move_of, D3& out) {
    const int32_t m = move_of[v];
    if (m >= 0 && active[m]) {
        out = moves[m].position;
        return true;
    }
    return position_of(pts[v], out);
}

// One round of topology_safe_moves (surface_fusion.rs:594-637): every valid
// triangle with a vertex in an active move is checked against the complete
// active move set (triangle_preserved_with_moves, surface_fusion.rs:652-696);
// a triangle that fails rejects every active move on its vertices.
__global__ void k_topology_round(const v3d_point* __restrict__ pts,
                                 const v3d_mesh_triangle* __restrict__ tris, uint64_t nt,
                                 const uint32_t* __restrict__ valid, const Move* __restrict__ moves,
                                 const uint8_t* __restrict__ active,
                                 const int32_t* __restrict__ move_of, uint8_t* __restrict__ reject,
                                 uint32_t* __restrict__ any) {
    for (uint64_t t = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; t < nt;
         t += (uint64_t)gridDim.x * blockDim.x) {
        if (!valid[t]) continue;
        const v3d_mesh_triangle tr = tris[t];
        const uint64_t v3[3] = {tr.a, tr.b, tr.c};
        bool touched = false;
        for (int k = 0; k < 3; ++k) {
            const int32_t m = move_of[v3[k]];
            touched = touched || (m >= 0 && active[m]);
        }
        if (!touched) continue;
        bool keep = false;
        D3 a, b, c;
        if (position_of(pts[tr.a], a) && position_of(pts[tr.b], b) && position_of(pts[tr.c], c)) {
            const D3 on = vcross(vsub(b, a), vsub(c, a));
            const double oa = vnorm(on);
            D3 pa, pb, pc;
            if (isfinite(oa) && oa > kGeometricEpsilon &&
                proposed_of(tr.a, pts, moves, active, move_of, pa) &&
                proposed_of(tr.b, pts, moves, active, move_of, pb) &&
                proposed_of(tr.c, pts, moves, active, move_of, pc)) {
                const D3 pn = vcross(vsub(pb, pa), vsub(pc, pa));
                const double ps = vnorm(pn);
                keep = isfinite(ps) && !(ps < dmul(oa, kMinIncidentAreaRatio)) &&
                       ddiv(vdot(on, pn), dmul(oa, ps)) >= kMinIncidentNormalAlignment;
            }
        }
        if (keep) continue;
        for (int k = 0; k < 3; ++k) {
            const int32_t m = move_of[v3[k]];
            if (m >= 0 && active[m]) reject[m] = 1;
        }
        *any = 1;
    }
}

__global__ void k_apply_rejects(uint8_t* __restrict__ active, const uint8_t* __restrict__ reject,
                                const uint32_t* __restrict__ count) {
    const uint32_t m = *count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x)
        if (reject[k]) active[k] = 0;
}

// The accepted moves applied (surface_fusion.rs:522-531): both vertices take
// the f32 position; a vertex counts as moved when its point changed.
__global__ void k_apply_moves(v3d_point* __restrict__ pts, const Move* __restrict__ moves,
                              const uint8_t* __restrict__ active, const uint32_t* __restrict__ count,
                              uint8_t* __restrict__ moved) {
    const uint32_t m = *count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        if (!active[k]) continue;
        const Move mv = moves[k];
        for (uint32_t idx : {mv.first, mv.second}) {
            const v3d_point orig = pts[idx];
            v3d_point now = orig;
            now.x = (float)mv.position.x;
            now.y = (float)mv.position.y;
            now.z = (float)mv.position.z;
            const bool same = now.x == orig.x && now.y == orig.y && now.z == orig.z &&
                              now.confidence == orig.confidence;  // colours unchanged
            pts[idx] = now;
            moved[idx] = same ? 0 : 1;
        }
    }
}

__global__ void k_pairs_out(const Move* __restrict__ moves, const uint32_t* __restrict__ acc,
                            const uint32_t* __restrict__ count, const v3d_point* __restrict__ pts,
                            v3d_fusion_pair* __restrict__ pairs, v3d_point* __restrict__ pair_pts) {
    const uint32_t m = *count;
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < m; k += gridDim.x * blockDim.x) {
        const Move mv = moves[acc[k]];
        pairs[k] = v3d_fusion_pair{mv.first, mv.second};
        pair_pts[2 * k] = pts[mv.first];
        pair_pts[2 * k + 1] = pts[mv.second];
    }
}

// A bump allocator over the context's arena, regrown (and the carve redone)
// when a call needs more than it holds.
}  // namespace
}  // namespace v3d

using namespace v3d;


extern "C" int32_t v3d_fuse_mutually_supported_vertices(
    v3d_context* ctx, v3d_point* points, uint64_t n, const v3d_mesh_triangle* triangles,
    uint64_t nt, const int64_t* membership, v3d_cancel_fn cancel, void* cancel_user,
    v3d_fusion_stats* stats, v3d_fusion_pair* pairs, uint64_t* n_pairs, uint64_t* moved,
    uint64_t* n_moved) {
    if (!ctx || !stats || !n_pairs || !n_moved || (n && (!points || !membership || !pairs || !moved)) ||
        (nt && !triangles))
        return V3D_ERR_INVALID_ARGUMENT;
    std::memset(stats, 0, sizeof(*stats));
    *n_pairs = 0;
    *n_moved = 0;
    // the sorts take int item counts, and a triangle has three incidence entries
    if (n >= 0x40000000ull || nt > 0x7FFFFFFFull / 3) {
        ctx->last_error = "surface fusion takes fewer than 2^30 points and 715,827,882 triangles";
        return V3D_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(ctx->stream);
    // the reference's FusionOutcome::default() on cancellation: nothing changes
    auto canceled = [&] { return cancel && cancel(cancel_user) != 0; };
    if (canceled()) return V3D_OK;
    if (n == 0 || nt == 0) return V3D_OK;  // no triangles: no global edge scale
    const uint64_t ne = 3 * nt;           // incidence entries at most
    int vbits = 1;
    while (vbits < 32 && (1ull << vbits) <= n) ++vbits;

    // ---- CUB temporary storage sizes ----
    size_t t_scan = 0, t_pairs = 0, t_keys = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, t_scan, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                  (int)std::max<uint64_t>(nt, n + 1), st);
    cub::DeviceRadixSort::SortPairs(nullptr, t_pairs, (uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (uint32_t*)nullptr, (uint32_t*)nullptr,
                                    (int)std::max<uint64_t>(ne, n), 0, vbits, st);
    cub::DeviceRadixSort::SortKeys(nullptr, t_keys, (double*)nullptr, (double*)nullptr, (int)ne, 0,
                                   64, st);
    const size_t t_cub = std::max(std::max(t_scan, t_pairs), t_keys);
    uint32_t table_slots = 2;  // a power of two above twice the eligible vertices
    while (table_slots < 2 * n + 2) table_slots <<= 1;

    // ---- arena ----
    Carve cv;
    const size_t o_pts = cv.take<v3d_point>(n), o_tris = cv.take<v3d_mesh_triangle>(nt),
                 o_mem = cv.take<int64_t>(n), o_valid = cv.take<uint32_t>(nt),
                 o_pos = cv.take<uint32_t>(nt), o_len = cv.take<double>(ne),
                 o_wn = cv.take<D3>(nt), o_keys = cv.take<uint32_t>(ne),
                 o_vals = cv.take<uint32_t>(ne), o_keys2 = cv.take<uint32_t>(ne),
                 o_vals2 = cv.take<uint32_t>(ne), o_lens = cv.take<double>(ne),
                 o_lens2 = cv.take<double>(ne), o_vcnt = cv.take<uint32_t>(n + 1),
                 o_voff = cv.take<uint32_t>(n + 1), o_nrm = cv.take<D3>(n),
                 o_scale = cv.take<double>(n), o_has = cv.take<uint8_t>(n),
                 o_elig = cv.take<uint8_t>(n), o_cell = cv.take<Cell>(n),
                 o_elv = cv.take<uint32_t>(n), o_elc = cv.take<Cell>(n),
                 o_table = cv.take<uint32_t>(table_slots), o_rep = cv.take<uint32_t>(n),
                 o_rep2 = cv.take<uint32_t>(n), o_elv2 = cv.take<uint32_t>(n),
                 o_mem_rec = cv.take<Member>(n), o_cbeg = cv.take<uint32_t>(n),
                 o_cend = cv.take<uint32_t>(n),
                 o_near = cv.take<uint32_t>(n), o_neard = cv.take<double>(n),
                 o_flag = cv.take<uint8_t>(n), o_fused = cv.take<D3>(n),
                 o_first = cv.take<uint32_t>(n), o_moves = cv.take<Move>(n / 2 + 1),
                 o_moveof = cv.take<int32_t>(n), o_active = cv.take<uint8_t>(n / 2 + 1),
                 o_reject = cv.take<uint8_t>(n / 2 + 1), o_acc = cv.take<uint32_t>(n / 2 + 1),
                 o_moved = cv.take<uint8_t>(n), o_movedi = cv.take<uint32_t>(n),
                 o_pairs = cv.take<v3d_fusion_pair>(n / 2 + 1),
                 o_ppts = cv.take<v3d_point>(n + 2), o_counts = cv.take<uint32_t>(16),
                 o_ctr = cv.take<unsigned long long>(4),
                 o_scratch = cv.take<uint8_t>(compaction_scratch_bytes(std::max(n, nt))),
                 o_cub = cv.take<uint8_t>(t_cub);
    if (!ensure_arena(ctx, cv.off + 256)) {
        ctx->last_error = "device arena allocation failed";
        return V3D_ERR_OUT_OF_MEMORY;
    }
    char* base = static_cast<char*>(ctx->arena);
    auto at = [&](size_t o) { return base + o; };
    auto* d_pts = reinterpret_cast<v3d_point*>(at(o_pts));
    auto* d_tris = reinterpret_cast<v3d_mesh_triangle*>(at(o_tris));
    auto* d_mem = reinterpret_cast<int64_t*>(at(o_mem));
    auto* d_valid = reinterpret_cast<uint32_t*>(at(o_valid));
    auto* d_pos = reinterpret_cast<uint32_t*>(at(o_pos));
    auto* d_len = reinterpret_cast<double*>(at(o_len));
    auto* d_wn = reinterpret_cast<D3*>(at(o_wn));
    auto* d_keys = reinterpret_cast<uint32_t*>(at(o_keys));
    auto* d_vals = reinterpret_cast<uint32_t*>(at(o_vals));
    auto* d_keys2 = reinterpret_cast<uint32_t*>(at(o_keys2));
    auto* d_vals2 = reinterpret_cast<uint32_t*>(at(o_vals2));
    auto* d_lens = reinterpret_cast<double*>(at(o_lens));
    auto* d_lens2 = reinterpret_cast<double*>(at(o_lens2));
    auto* d_vcnt = reinterpret_cast<uint32_t*>(at(o_vcnt));
    auto* d_voff = reinterpret_cast<uint32_t*>(at(o_voff));
    auto* d_nrm = reinterpret_cast<D3*>(at(o_nrm));
    auto* d_scale = reinterpret_cast<double*>(at(o_scale));
    auto* d_has = reinterpret_cast<uint8_t*>(at(o_has));
    auto* d_elig = reinterpret_cast<uint8_t*>(at(o_elig));
    auto* d_cell = reinterpret_cast<Cell*>(at(o_cell));
    auto* d_elv = reinterpret_cast<uint32_t*>(at(o_elv));
    auto* d_elc = reinterpret_cast<Cell*>(at(o_elc));
    auto* d_table = reinterpret_cast<uint32_t*>(at(o_table));
    auto* d_rep = reinterpret_cast<uint32_t*>(at(o_rep));
    auto* d_rep2 = reinterpret_cast<uint32_t*>(at(o_rep2));
    auto* d_elv2 = reinterpret_cast<uint32_t*>(at(o_elv2));
    auto* d_members = reinterpret_cast<Member*>(at(o_mem_rec));
    auto* d_cbeg = reinterpret_cast<uint32_t*>(at(o_cbeg));
    auto* d_cend = reinterpret_cast<uint32_t*>(at(o_cend));
    auto* d_near = reinterpret_cast<uint32_t*>(at(o_near));
    auto* d_neard = reinterpret_cast<double*>(at(o_neard));
    auto* d_flag = reinterpret_cast<uint8_t*>(at(o_flag));
    auto* d_fused = reinterpret_cast<D3*>(at(o_fused));
    auto* d_first = reinterpret_cast<uint32_t*>(at(o_first));
    auto* d_moves = reinterpret_cast<Move*>(at(o_moves));
    auto* d_moveof = reinterpret_cast<int32_t*>(at(o_moveof));
    auto* d_active = reinterpret_cast<uint8_t*>(at(o_active));
    auto* d_reject = reinterpret_cast<uint8_t*>(at(o_reject));
    auto* d_acc = reinterpret_cast<uint32_t*>(at(o_acc));
    auto* d_moved = reinterpret_cast<uint8_t*>(at(o_moved));
    auto* d_movedi = reinterpret_cast<uint32_t*>(at(o_movedi));
    auto* d_pairs = reinterpret_cast<v3d_fusion_pair*>(at(o_pairs));
    auto* d_ppts = reinterpret_cast<v3d_point*>(at(o_ppts));
    auto* d_counts = reinterpret_cast<uint32_t*>(at(o_counts));
    auto* d_ctr = reinterpret_cast<unsigned long long*>(at(o_ctr));
    void* d_scratch = at(o_scratch);
    void* d_cub = at(o_cub);
    size_t cub_bytes = t_cub;
    // counts: [0] eligible, [1] cells, [2] moves, [3] accepted, [4] moved, [5] round flag
    uint32_t* c_el = d_counts + 0;
    uint32_t* c_moves = d_counts + 2;
    uint32_t* c_acc = d_counts + 3;
    uint32_t* c_moved = d_counts + 4;
    uint32_t* c_any = d_counts + 5;
    const uint64_t launches0 = g_kernel_launches;

    // ---- upload ----
    V3D_CTX_CK(cudaMemcpyAsync(d_pts, points, sizeof(v3d_point) * n, cudaMemcpyHostToDevice, st));
    V3D_CTX_CK(cudaMemcpyAsync(d_tris, triangles, sizeof(v3d_mesh_triangle) * nt,
                            cudaMemcpyHostToDevice, st));
    V3D_CTX_CK(cudaMemcpyAsync(d_mem, membership, sizeof(int64_t) * n, cudaMemcpyHostToDevice, st));
    V3D_CTX_CK(cudaMemsetAsync(d_counts, 0, sizeof(uint32_t) * 16, st));
    V3D_CTX_CK(cudaMemsetAsync(d_ctr, 0, sizeof(unsigned long long) * 4, st));
    V3D_CTX_CK(cudaMemsetAsync(d_vcnt, 0, sizeof(uint32_t) * (n + 1), st));

    // the device span from the first kernel to the last (with the host reads
    // between the stages) for the run info's device_ms
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

    // ---- vertex evidence ----
    V3D_COUNTED k_tri_evidence<<<grid_of(nt), 256, 0, st>>>(d_pts, n, d_tris, nt, d_valid, d_len, d_wn);
    V3D_CTX_CK(cudaGetLastError());
    V3D_CTX_CK(cub::DeviceScan::ExclusiveSum(d_cub, cub_bytes, d_valid, d_pos, (int)nt, st));
    V3D_COUNTED k_incidence<<<grid_of(nt), 256, 0, st>>>(d_tris, nt, d_valid, d_pos, d_len, d_keys,
                                                          d_vals, d_lens, d_vcnt);
    V3D_CTX_CK(cudaGetLastError());
    uint32_t nv_last[2] = {0, 0};
    V3D_CTX_CK(cudaMemcpyAsync(&nv_last[0], d_pos + (nt - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaMemcpyAsync(&nv_last[1], d_valid + (nt - 1), sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaStreamSynchronize(st));
    const uint64_t n_valid = (uint64_t)nv_last[0] + nv_last[1];
    const uint64_t n_ent = 3 * n_valid;
    if (canceled()) return V3D_OK;
    if (n_valid == 0) return V3D_OK;  // no edge lengths: no global edge scale
    cub_bytes = t_cub;
    V3D_CTX_CK(cub::DeviceRadixSort::SortPairs(d_cub, cub_bytes, d_keys, d_keys2, d_vals, d_vals2,
                                            (int)n_ent, 0, vbits, st));
    cub_bytes = t_cub;
    V3D_CTX_CK(cub::DeviceScan::ExclusiveSum(d_cub, cub_bytes, d_vcnt, d_voff, (int)(n + 1), st));
    V3D_COUNTED k_vertex_evidence<<<grid_of(n), 256, 0, st>>>(n, d_tris, d_voff, d_vals2, d_len, d_wn,
                                                               d_nrm, d_scale, d_has);
    V3D_CTX_CK(cudaGetLastError());
    cub_bytes = t_cub;
    V3D_CTX_CK(cub::DeviceRadixSort::SortKeys(d_cub, cub_bytes, d_lens, d_lens2, (int)n_ent, 0, 64, st));
    double mid[2] = {0, 0};
    const uint64_t half = n_ent / 2;
    V3D_CTX_CK(cudaMemcpyAsync(&mid[1], d_lens2 + half, sizeof(double), cudaMemcpyDeviceToHost, st));
    if (n_ent % 2 == 0)
        V3D_CTX_CK(cudaMemcpyAsync(&mid[0], d_lens2 + half - 1, sizeof(double), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaStreamSynchronize(st));
    // median (surface_fusion.rs:838-849)
    const double global = n_ent % 2 == 0 ? (mid[0] + mid[1]) * 0.5 : mid[1];
    const double cell_size = std::max(global * kMaxGlobalEdgeFraction, kGeometricEpsilon);
    if (canceled()) return V3D_OK;

    // ---- eligible vertices, sorted by cell ----
    V3D_COUNTED k_eligible<<<grid_of(n), 256, 0, st>>>(d_pts, n, d_mem, d_has, cell_size, d_elig, d_cell);
    V3D_CTX_CK(cudaGetLastError());
    V3D_CTX_CK(launch_compact(d_elig, 1, n, d_elv, c_el, d_scratch, st));
    V3D_COUNTED k_gather_cells<<<grid_of(n), 256, 0, st>>>(d_elv, c_el, d_cell, d_elc);
    V3D_CTX_CK(cudaGetLastError());
    uint32_t n_el = 0;
    V3D_CTX_CK(cudaMemcpyAsync(&n_el, c_el, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaStreamSynchronize(st));
    stats->eligible_vertices = n_el;
    // cells: a hash table of representatives, the eligible vertices sorted by
    // representative (stable, so each cell keeps index order), member records
    V3D_CTX_CK(cudaMemsetAsync(d_table, 0xFF, sizeof(uint32_t) * table_slots, st));
    V3D_COUNTED k_cell_insert<<<grid_of(n), 256, 0, st>>>(d_elc, c_el, d_table, table_slots - 1, d_rep);
    V3D_CTX_CK(cudaGetLastError());
    if (n_el) {
        cub_bytes = t_cub;
        V3D_CTX_CK(cub::DeviceRadixSort::SortPairs(d_cub, cub_bytes, d_rep, d_rep2, d_elv, d_elv2,
                                                (int)n_el, 0, vbits, st));
    }
    V3D_COUNTED k_members<<<grid_of(n), 256, 0, st>>>(d_rep2, d_elv2, c_el, d_pts, d_mem, d_nrm, d_scale,
                                                       d_members, d_cbeg, d_cend);
    V3D_CTX_CK(cudaGetLastError());

    // ---- nearest cross-group neighbours, mutual pairs ----
    V3D_CTX_CK(cudaMemsetAsync(d_near, 0xFF, sizeof(uint32_t) * n, st));
    V3D_COUNTED k_nearest<<<grid_of(n), 256, 0, st>>>(d_members, d_elc, c_el, d_table, table_slots - 1,
                                                       d_cbeg, d_cend, global, d_near, d_neard, d_ctr);
    V3D_CTX_CK(cudaGetLastError());
    V3D_COUNTED k_mutual<<<grid_of(n), 256, 0, st>>>(d_pts, n, d_near, d_flag, d_fused);
    V3D_CTX_CK(cudaGetLastError());
    V3D_CTX_CK(launch_compact(d_flag, 1, n, d_first, c_moves, d_scratch, st));
    V3D_CTX_CK(cudaMemsetAsync(d_moveof, 0xFF, sizeof(int32_t) * n, st));
    V3D_COUNTED k_make_moves<<<grid_of(n / 2 + 1), 256, 0, st>>>(d_first, c_moves, d_near, d_fused,
                                                                  d_moves, d_moveof, d_active);
    V3D_CTX_CK(cudaGetLastError());
    uint32_t n_moves = 0;
    unsigned long long ctr[2] = {0, 0};
    V3D_CTX_CK(cudaMemcpyAsync(&n_moves, c_moves, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaMemcpyAsync(ctr, d_ctr, sizeof(ctr), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaStreamSynchronize(st));
    if (canceled()) {
        std::memset(stats, 0, sizeof(*stats));
        return V3D_OK;
    }

    // ---- topology gate: rounds until no active move is rejected ----
    for (uint32_t round = 0; n_moves > 0; ++round) {
        V3D_CTX_CK(cudaMemsetAsync(d_reject, 0, n_moves, st));
        V3D_CTX_CK(cudaMemsetAsync(c_any, 0, sizeof(uint32_t), st));
        V3D_COUNTED k_topology_round<<<grid_of(nt), 256, 0, st>>>(d_pts, d_tris, nt, d_valid, d_moves,
                                                                   d_active, d_moveof, d_reject, c_any);
        V3D_CTX_CK(cudaGetLastError());
        uint32_t any = 0;
        V3D_CTX_CK(cudaMemcpyAsync(&any, c_any, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        V3D_CTX_CK(cudaStreamSynchronize(st));
        if (canceled()) {
            std::memset(stats, 0, sizeof(*stats));
            return V3D_OK;
        }
        if (!any) break;
        V3D_COUNTED k_apply_rejects<<<grid_of(n_moves), 256, 0, st>>>(d_active, d_reject, c_moves);
        V3D_CTX_CK(cudaGetLastError());
    }

    // ---- apply, pairs, moved indices ----
    V3D_CTX_CK(cudaMemsetAsync(d_moved, 0, n, st));
    V3D_COUNTED k_apply_moves<<<grid_of(n_moves), 256, 0, st>>>(d_pts, d_moves, d_active, c_moves, d_moved);
    V3D_CTX_CK(cudaGetLastError());
    V3D_CTX_CK(launch_compact(d_active, 1, n_moves, d_acc, c_acc, d_scratch, st));
    V3D_CTX_CK(launch_compact(d_moved, 1, n, d_movedi, c_moved, d_scratch, st));
    V3D_COUNTED k_pairs_out<<<grid_of(n_moves), 256, 0, st>>>(d_moves, d_acc, c_acc, d_pts, d_pairs, d_ppts);
    V3D_CTX_CK(cudaGetLastError());
    cudaEventRecord(ev1, st);
    uint32_t cnt[2] = {0, 0};
    V3D_CTX_CK(cudaMemcpyAsync(cnt, c_acc, sizeof(cnt), cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaStreamSynchronize(st));
    const uint32_t n_acc = cnt[0], n_mv = cnt[1];
    std::vector<uint32_t> mv(n_mv);
    std::vector<v3d_point> ppts(2ull * n_acc);
    if (n_acc) {
        V3D_CTX_CK(cudaMemcpyAsync(pairs, d_pairs, sizeof(v3d_fusion_pair) * n_acc,
                                cudaMemcpyDeviceToHost, st));
        V3D_CTX_CK(cudaMemcpyAsync(ppts.data(), d_ppts, sizeof(v3d_point) * 2 * n_acc,
                                cudaMemcpyDeviceToHost, st));
    }
    if (n_mv)
        V3D_CTX_CK(cudaMemcpyAsync(mv.data(), d_movedi, sizeof(uint32_t) * n_mv,
                                cudaMemcpyDeviceToHost, st));
    V3D_CTX_CK(cudaStreamSynchronize(st));
    for (uint32_t k = 0; k < n_acc; ++k) {
        points[pairs[k].first] = ppts[2ull * k];
        points[pairs[k].second] = ppts[2ull * k + 1];
    }
    for (uint32_t k = 0; k < n_mv; ++k) moved[k] = mv[k];
    stats->candidate_pairs = ctr[0];
    stats->rejected_normal_pairs = ctr[1];
    stats->rejected_topology_pairs = n_moves - n_acc;
    stats->fused_pairs = n_acc;
    *n_pairs = n_acc;
    *n_moved = n_mv;
    ctx->last_launches = g_kernel_launches - launches0;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, ev0, ev1) == cudaSuccess) ctx->last_ms = ms;
    return V3D_OK;
}
