// The connected-surface merge (surface_merge.rs:312-1078 with
// surface_merge_clip.rs and surface_merge_stitch.rs) behind
// v3d_merge_fused_patches_owned.
//
// Patches are processed in priority order (more triangles first), and each
// patch's decisions read the footprints of the patches before it, so the
// patch loop is sequential; inside a patch every candidate triangle is judged
// independently.  That per-candidate work -- projecting the candidate into
// each linked owner's reference image, the bounded grid lookup of owner
// triangles, the convex clip against each of them, the depth agreement at
// every overlap corner and the owned image and surface areas -- runs on the
// device, one thread per (candidate, owner), as do the relative depth-scale
// samples of each (owner, patch) pair.  The host keeps what is inherently
// ordered: the fold over owners and the decisions in triangle order, the 3D
// coverage fallback for the few candidates no image could judge, the greedy
// seam stitching, the clips (which share derived vertices in job order), the
// edge-conforming split and the final assembly.  Footprints (a patch's kept
// triangles projected into its own reference image, with a frozen grid) are
// built once on the host, read there by stitching and clipping, and copied to
// the device for the candidate lookups.
//
// Every f64 expression is evaluated in the reference's order with separately
// rounded operations (merge_geom.cuh), so the result equals the reference's
// bit for bit: the same triangles, points, lineage and statistics.
#include <algorithm>
#include <array>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <map>
#include <memory>
#include <optional>
#include <set>
#include <string>
#include <atomic>
#include <thread>
#include <unordered_map>
#include <unordered_set>
#include <vector>

#include <cuda_runtime.h>

#include "host.hpp"
#include "merge_geom.cuh"

namespace v3d {
extern thread_local uint64_t g_kernel_launches;  // pass_kernels.cu
}

namespace v3d {
namespace merge {

using mg::Cam;
using mg::Poly;
using mg::PT;
using mg::V2;
using mg::V3;

constexpr double kMaxOverlapDistanceFraction = 0.9;     // surface_merge.rs:60
constexpr size_t kMaxGridCells = 1728;                  // :63
constexpr size_t kMaxUncoveredPieces = 128;             // :65
constexpr uint32_t kMaxPostings = 512;                  // :73 MAX_POSTINGS_PER_QUERY
constexpr double kMinNormalAlignment = 0.94;            // :76
constexpr double kMinImageOwnershipShare = 0.8;         // :81
constexpr double kMaxRelativeDepthDisagreement = 0.035; // :89
constexpr double kMaxRelativeScaleSample = 0.1;         // :93
constexpr size_t kMinScaleSamples = 5;                  // :95
constexpr uint32_t kMaxScaleSamples = 4096;             // :99
constexpr double kOwnershipEpsilon = 1.0e-9;            // :1304
constexpr uint64_t kMaxImageGridCells = 4096;           // :1307

// lookup outcomes (QueryLimit, Unjudged)
enum : uint8_t { kJudged = 0, kUnprojectable = 1, kTooManyCells = 2, kPostingBound = 3 };

// ---- device side ------------------------------------------------------------------

// One footprint as the device reads it.
struct DevFootprint {
    Cam cam;
    double cell;
    int32_t levels;
    uint32_t tri_off;      // into the projected-triangle, component and vertex arrays
    uint32_t n_tri;
    uint32_t bucket_off;   // into the bucket array
    uint32_t n_buckets;
    uint32_t item_off;     // into the item array: bucketed items, then unindexed ones
    uint32_t n_bucketed;
    uint32_t n_unindexed;
    uint32_t omit_off;     // into the omitted-component array
    uint32_t n_omit;
};

struct DevStore {
    const double* corners;          // 9 per mesh triangle (world corners, f64)
    const DevFootprint* fps;
    const double* fp_tri;           // 9 per footprint triangle: x0 x1 x2 y0 y1 y2 z0 z1 z2
    const uint32_t* fp_comp;        // original mesh component of each footprint triangle
    const uint32_t* fp_vert;        // 3 per footprint triangle
    const mg::GridBucket* buckets;
    const uint32_t* items;
    const int32_t* cluster;         // per component (vertex index): linked cluster or -1
    const uint32_t* omitted;        // components of each footprint's unprojectable kept triangles
};

// A patch's candidates and its linked owners (one lookup per pair).
struct Cand {
    uint32_t triangle, own_comp;
};
struct OwnerRef {
    uint32_t slot;
    uint32_t pad_;
    double scale;
};
struct PairOut {
    double share, surface;
    uint32_t used;
    uint32_t status;
};
// A candidate's fold over its owners (surface_merge.rs:654-706).
struct CandOut {
    double share, surface, scale;  // the best-owning judged owner (share 0: none)
    uint32_t slot;                 // its footprint, or 0xffffffff
    uint32_t max_used;             // most postings of the lookups the fold recorded
    uint32_t bound_hits;           // lookups of those cut off at the posting bound
    uint32_t flags;                // 1: cut off (kept unjudged); 2: judged by every owner
};

// One lookup: a candidate triangle against one owner footprint.
struct Job {
    uint32_t triangle;    // mesh index of the candidate
    uint32_t footprint;   // owner
    uint32_t own_comp;    // the candidate's original component
    uint32_t anchors_off; // ratio jobs: this owner pair's sorted anchor vertices
    uint32_t n_anchors;
    uint32_t out_off;     // ratio jobs: first output slot; limit = out_limit - out_off
    uint32_t out_limit;
    double scale;
};

struct JobOut {
    double share, surface;  // ownership: image share and owned surface area
    uint32_t used;          // postings the lookup took
    uint32_t count;         // ratio jobs: agreeing samples
    uint8_t status;
};

__device__ __forceinline__ PT load_pt(const double* p) {
    PT t;
    for (int i = 0; i < 3; ++i) {
        t.x[i] = p[i];
        t.y[i] = p[3 + i];
        t.z[i] = p[6 + i];
    }
    return t;
}

// A warp's lookup scratch: the postings of one query, then per posting (in
// ascending order) its sample and whether the query's loop takes it.
constexpr int kLookupWarps = 4;  // warps per block of the warp-per-lookup kernel
struct WarpPostings {
    uint32_t idx[kMaxPostings];
    double a[kMaxPostings];
    uint8_t ok[kMaxPostings];
    uint32_t n;
};

// The candidate's postings on one footprint grid (LevelGrid::query_bounded), by
// the warp's lanes: w.idx[0, n) ascending (the reference's BTreeSet order), or a
// QueryLimit status.  Every lane returns the same status, n and used.  The
// reference takes postings cell by cell until one does not fit the budget; the
// counts only grow, so that happens exactly when the query's total exceeds it,
// and the order the lanes gather them in does not matter before the sort.
__device__ uint8_t warp_grid_lookup(const DevStore& s, const DevFootprint& f, const PT& c,
                                    WarpPostings& w, uint32_t lane, uint32_t& n, uint32_t& used) {
    double lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
    for (int i = 0; i < 3; ++i) {
        lo[0] = fmin(lo[0], c.x[i]);
        hi[0] = fmax(hi[0], c.x[i]);
        lo[1] = fmin(lo[1], c.y[i]);
        hi[1] = fmax(hi[1], c.y[i]);
    }
    n = 0;
    used = 0;
    for (int level = 0; level < f.levels; ++level) {
        uint64_t count = 1;
        for (int a = 0; a < 2; ++a) {
            int64_t first, last;
            if (!mg::axis_range(f.cell, level, lo[a], hi[a], first, last)) return kTooManyCells;
            first = mg::sat_sub(first, mg::kMaxAnchorCellSpan);
            if (last < first) return kTooManyCells;
            const uint64_t span = (uint64_t)last - (uint64_t)first;
            if (span == UINT64_MAX) return kTooManyCells;
            const uint64_t cells = span + 1;
            count = (count != 0 && cells > UINT64_MAX / count) ? UINT64_MAX : count * cells;
        }
        if (count > kMaxImageGridCells) return kTooManyCells;
    }
    const mg::GridBucket* b = s.buckets + f.bucket_off;
    // the bucket of cell (level, x, y): its first item and count
    auto bucket = [&](int level, int64_t x, int64_t y, uint32_t& start) -> uint32_t {
        uint32_t l = 0, h = f.n_buckets;
        while (l < h) {
            const uint32_t mid = (l + h) >> 1;
            if (mg::bucket_less(b[mid], level, x, y)) l = mid + 1;
            else h = mid;
        }
        if (l < f.n_buckets && b[l].level == level && b[l].x == x && b[l].y == y) {
            start = b[l].start;
            return (l + 1 < f.n_buckets ? b[l + 1].start : f.n_bucketed) - b[l].start;
        }
        return 0;
    };
    // each cell of each level's (first..last)^2 range, lanes over cells; pass 0
    // counts, pass 1 gathers
    for (int pass = 0; pass < 2; ++pass) {
        uint32_t mine = 0;
        for (int level = 0; level < f.levels; ++level) {
            int64_t x0, x1, y0, y1;
            mg::axis_range(f.cell, level, lo[0], hi[0], x0, x1);
            mg::axis_range(f.cell, level, lo[1], hi[1], y0, y1);
            x0 = mg::sat_sub(x0, mg::kMaxAnchorCellSpan);
            y0 = mg::sat_sub(y0, mg::kMaxAnchorCellSpan);
            const uint32_t nx = (uint32_t)(x1 - x0 + 1), ncell = nx * (uint32_t)(y1 - y0 + 1);
            for (uint32_t q = lane; q < ncell; q += 32) {
                uint32_t start = 0;
                const uint32_t k = bucket(level, x0 + (int64_t)(q % nx), y0 + (int64_t)(q / nx), start);
                if (!k) continue;
                if (pass == 0) {
                    mine += k;
                } else {
                    const uint32_t at = atomicAdd(&w.n, k);
                    for (uint32_t i = 0; i < k; ++i) w.idx[at + i] = s.items[f.item_off + start + i];
                }
            }
        }
        if (pass == 1) break;
        for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(0xffffffffu, mine, o);
        const uint64_t total = (uint64_t)mine + f.n_unindexed;
        if (total > kMaxPostings) {
            used = kMaxPostings;
            return kPostingBound;
        }
        n = used = (uint32_t)total;
        for (uint32_t i = lane; i < f.n_unindexed; i += 32)
            w.idx[i] = s.items[f.item_off + f.n_bucketed + i];
        if (lane == 0) w.n = f.n_unindexed;
        __syncwarp();
    }
    __syncwarp();
    // ascending: a bitonic sort over the next power of two, padded with the largest key
    uint32_t N = 1;
    while (N < n) N <<= 1;
    for (uint32_t i = n + lane; i < N; i += 32) w.idx[i] = 0xffffffffu;
    __syncwarp();
    for (uint32_t k = 2; k <= N; k <<= 1)
        for (uint32_t j = k >> 1; j > 0; j >>= 1) {
            for (uint32_t i = lane; i < N; i += 32) {
                const uint32_t l = i ^ j;
                if (l > i) {
                    const uint32_t x = w.idx[i], y = w.idx[l];
                    if ((x > y) == ((i & k) == 0)) {
                        w.idx[i] = y;
                        w.idx[l] = x;
                    }
                }
            }
            __syncwarp();
        }
    return kJudged;
}

// The candidate's postings on one footprint grid, ascending (the reference's
// BTreeSet), or a QueryLimit status (LevelGrid::query_bounded).
__device__ uint8_t grid_lookup(const DevStore& s, const DevFootprint& f, const PT& c,
                               uint32_t* found, uint32_t& n, uint32_t& used) {
    double lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
    for (int i = 0; i < 3; ++i) {
        lo[0] = fmin(lo[0], c.x[i]);
        hi[0] = fmax(hi[0], c.x[i]);
        lo[1] = fmin(lo[1], c.y[i]);
        hi[1] = fmax(hi[1], c.y[i]);
    }
    n = 0;
    used = 0;
    for (int level = 0; level < f.levels; ++level) {
        uint64_t count = 1;
        for (int a = 0; a < 2; ++a) {
            int64_t first, last;
            if (!mg::axis_range(f.cell, level, lo[a], hi[a], first, last)) return kTooManyCells;
            first = mg::sat_sub(first, mg::kMaxAnchorCellSpan);
            if (last < first) return kTooManyCells;
            const uint64_t span = (uint64_t)last - (uint64_t)first;
            if (span == UINT64_MAX) return kTooManyCells;
            const uint64_t cells = span + 1;
            count = (count != 0 && cells > UINT64_MAX / count) ? UINT64_MAX : count * cells;
        }
        if (count > kMaxImageGridCells) return kTooManyCells;
    }
    auto take = [&](uint32_t from, uint32_t k) -> bool {
        if (k > kMaxPostings - used) {
            used = kMaxPostings;
            return false;
        }
        for (uint32_t i = 0; i < k; ++i) found[n++] = s.items[f.item_off + from + i];
        used += k;
        return true;
    };
    if (!take(f.n_bucketed, f.n_unindexed)) return kPostingBound;
    const mg::GridBucket* b = s.buckets + f.bucket_off;
    for (int level = 0; level < f.levels; ++level) {
        int64_t x0, x1, y0, y1;
        mg::axis_range(f.cell, level, lo[0], hi[0], x0, x1);
        mg::axis_range(f.cell, level, lo[1], hi[1], y0, y1);
        x0 = mg::sat_sub(x0, mg::kMaxAnchorCellSpan);
        y0 = mg::sat_sub(y0, mg::kMaxAnchorCellSpan);
        for (int64_t y = y0;; ++y) {
            for (int64_t x = x0;; ++x) {
                // buckets sorted by (level, x, y): one binary search per cell
                uint32_t l = 0, h = f.n_buckets;
                while (l < h) {
                    uint32_t mid = (l + h) >> 1;
                    if (mg::bucket_less(b[mid], level, x, y)) l = mid + 1;
                    else h = mid;
                }
                if (l < f.n_buckets && b[l].level == level && b[l].x == x && b[l].y == y) {
                    const uint32_t end = l + 1 < f.n_buckets ? b[l + 1].start : f.n_bucketed;
                    if (!take(b[l].start, end - b[l].start)) return kPostingBound;
                }
                if (x == x1) break;
            }
            if (y == y1) break;
        }
    }
    // ascending, as the reference's BTreeSet iterates
    for (uint32_t i = 1; i < n; ++i) {
        uint32_t v = found[i];
        uint32_t j = i;
        while (j > 0 && found[j - 1] > v) {
            found[j] = found[j - 1];
            --j;
        }
        found[j] = v;
    }
    return kJudged;
}

__device__ __forceinline__ bool linked(const DevStore& s, uint32_t own, uint32_t comp) {
    if (own == comp) return false;
    const int32_t c = s.cluster[own];
    return c >= 0 && s.cluster[comp] == c;
}

__device__ __forceinline__ bool anchored(const uint32_t* anchors, uint32_t n, const uint32_t* v) {
    for (int k = 0; k < 3; ++k) {
        uint32_t l = 0, h = n;
        while (l < h) {
            uint32_t mid = (l + h) >> 1;
            if (anchors[mid] < v[k]) l = mid + 1;
            else h = mid;
        }
        if (l < n && anchors[l] == v[k]) return true;
    }
    return false;
}

__device__ bool project_candidate(const DevFootprint& f, const double* w, PT& c) {
    V3 corners[3] = {V3{w[0], w[1], w[2]}, V3{w[3], w[4], w[5]}, V3{w[6], w[7], w[8]}};
    if (!mg::project_triangle(f.cam, corners, c)) return false;
    return mg::image_area(c) > mg::mul(mg::kGeomEps, mg::kGeomEps);
}

// Footprint::ownership_tallied (surface_merge.rs:1520-1578) for one
// (candidate, owner) pair: thread per pair, pair j = candidate j / n_owners,
// owner j % n_owners.
__global__ void __launch_bounds__(128) k_ownership(DevStore s, const Cand* cands, uint32_t n_cand,
                                                    const OwnerRef* owners, uint32_t n_owners,
                                                    PairOut* out) {
    const uint64_t j = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= (uint64_t)n_cand * n_owners) return;
    const Cand cd = cands[j / n_owners];
    const OwnerRef ow = owners[j % n_owners];
    const DevFootprint f = s.fps[ow.slot];
    PairOut o{0.0, 0.0, 0u, kJudged};
    const double* w = s.corners + (size_t)cd.triangle * 9;
    PT cand;
    if (!project_candidate(f, w, cand)) {
        o.status = kUnprojectable;
        out[j] = o;
        return;
    }
    uint32_t found[kMaxPostings];
    uint32_t n, used;
    o.status = grid_lookup(s, f, cand, found, n, used);
    o.used = used;
    if (o.status != kJudged) {
        out[j] = o;
        return;
    }
    const double total = mg::image_area(cand);
    V3 corners[3] = {V3{w[0], w[1], w[2]}, V3{w[3], w[4], w[5]}, V3{w[6], w[7], w[8]}};
    V3 normal;
    double offset;
    const bool has_plane = mg::camera_plane(f.cam, corners, normal, offset);
    double image = 0.0, surface = 0.0;
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t idx = found[k];
        if (!linked(s, cd.own_comp, s.fp_comp[f.tri_off + idx])) continue;
        const PT kept = load_pt(s.fp_tri + (size_t)(f.tri_off + idx) * 9);
        Poly<8> poly;
        if (!mg::clip_to_triangle(cand, kept, poly)) continue;
        if (!(mg::poly_area(poly) > 0.0)) continue;
        bool agrees = true;
        for (int v = 0; v < poly.n && agrees; ++v) {
            double ic, ik;
            if (!mg::inverse_depth(cand, poly.v[v], ic) || !mg::inverse_depth(kept, poly.v[v], ik)) {
                agrees = false;
                break;
            }
            const double cdd = mg::dvd(1.0, ic), kd = mg::dvd(ow.scale, ik);
            agrees = fabs(mg::sub(cdd, kd)) <= mg::mul(kMaxRelativeDepthDisagreement, kd);
        }
        if (agrees) {
            image = mg::add(image, mg::poly_area(poly));
            surface = mg::add(surface, has_plane ? mg::back_projected_area(poly, normal, offset) : 0.0);
        }
    }
    o.share = fmin(mg::dvd(image, total), 1.0);
    o.surface = surface;
    out[j] = o;
}

// The fold over a candidate's owners in owner order (surface_merge.rs:654-706):
// the lookups it records (up to and including a cut-off one), the best share
// by strict improvement, and whether every owner judged it (a judged owner
// below the removal share leaves it unjudged when a kept triangle it could not
// project belongs to a linked component).
__global__ void __launch_bounds__(128) k_fold(DevStore s, const Cand* cands, uint32_t n_cand,
                                               const OwnerRef* owners, uint32_t n_owners,
                                               const PairOut* pairs, CandOut* out) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n_cand) return;
    const Cand cd = cands[c];
    CandOut o{0.0, 0.0, 1.0, 0xffffffffu, 0u, 0u, 0u};
    uint32_t judged = 0;
    for (uint32_t k = 0; k < n_owners; ++k) {
        const PairOut p = pairs[(size_t)c * n_owners + k];
        if (p.status == kUnprojectable) continue;
        o.max_used = max(o.max_used, p.used);
        if (p.status == kPostingBound) {
            o.bound_hits += 1;
            o.flags |= 1u;
            break;
        }
        if (p.status == kTooManyCells) continue;
        const DevFootprint f = s.fps[owners[k].slot];
        bool unjudged = false;
        if (p.share < kMinImageOwnershipShare)
            for (uint32_t q = 0; q < f.n_omit && !unjudged; ++q)
                unjudged = linked(s, cd.own_comp, s.omitted[f.omit_off + q]);
        if (!unjudged) judged += 1;
        if (p.share > o.share) {
            o.share = p.share;
            o.surface = p.surface;
            o.scale = owners[k].scale;
            o.slot = owners[k].slot;
        }
    }
    if (judged == n_owners) o.flags |= 2u;
    out[c] = o;
}

// Footprint::depth_ratios_tallied (surface_merge.rs:1475-1510): the anchored
// overlaps' candidate-to-owner depth ratios that agree within 10 %.  WRITE
// false counts them; WRITE true stores the first (out_limit - out_off) of them
// at ratios[out_off...].
template <bool WRITE>
__global__ void __launch_bounds__(32 * kLookupWarps) k_ratios(DevStore s, const Job* jobs, uint32_t n_jobs,
                                                               const uint32_t* anchors, JobOut* out,
                                                               double* ratios) {
    __shared__ WarpPostings scratch[kLookupWarps];
    const uint32_t lane = threadIdx.x & 31u;
    WarpPostings& w = scratch[threadIdx.x >> 5];
    const uint32_t j = blockIdx.x * kLookupWarps + (threadIdx.x >> 5);
    if (j >= n_jobs) return;
    const Job job = jobs[j];
    if (WRITE && job.out_off >= job.out_limit) return;
    const DevFootprint f = s.fps[job.footprint];
    const double* wc = s.corners + (size_t)job.triangle * 9;
    PT cand;
    JobOut o{0.0, 0.0, 0u, 0u, kJudged};
    if (!project_candidate(f, wc, cand)) {
        o.status = kUnprojectable;
        if (!WRITE && lane == 0) out[j] = o;
        return;
    }
    uint32_t n, used;
    o.status = warp_grid_lookup(s, f, cand, w, lane, n, used);
    o.used = used;
    if (o.status != kJudged) {
        if (!WRITE && lane == 0) out[j] = o;
        return;
    }
    // each posting's sample in parallel, then the first `limit` in ascending order
    for (uint32_t k = lane; k < n; k += 32) {
        const uint32_t t = f.tri_off + w.idx[k];
        bool ok = false;
        double ratio = 0.0;
        if (linked(s, job.own_comp, s.fp_comp[t]) &&
            anchored(anchors + job.anchors_off, job.n_anchors, s.fp_vert + (size_t)t * 3)) {
            const PT kept = load_pt(s.fp_tri + (size_t)t * 9);
            Poly<8> poly;
            if (mg::clip_to_triangle(cand, kept, poly) && mg::poly_area(poly) > 0.0) {
                V2 sum{0.0, 0.0};
                for (int v = 0; v < poly.n; ++v) sum = sum + poly.v[v];
                const V2 centroid = sum / (double)poly.n;
                double owner, own;
                if (mg::inverse_depth(kept, centroid, owner) && mg::inverse_depth(cand, centroid, own)) {
                    ratio = mg::dvd(owner, own);
                    ok = fabs(mg::sub(ratio, 1.0)) <= kMaxRelativeScaleSample;
                }
            }
        }
        w.ok[k] = ok ? 1 : 0;
        w.a[k] = ratio;
    }
    __syncwarp();
    if (lane == 0) {
        const uint32_t limit = WRITE ? job.out_limit - job.out_off : 0xffffffffu;
        uint32_t count = 0;
        for (uint32_t k = 0; k < n && count < limit; ++k)
            if (w.ok[k]) {
                if (WRITE) ratios[job.out_off + count] = w.a[k];
                ++count;
            }
        o.count = count;
        if (!WRITE) out[j] = o;
    }
}

}  // namespace merge
}  // namespace v3d

// ---- host side ------------------------------------------------------------------------
namespace v3d {
namespace merge {
namespace {

using Clock = std::chrono::steady_clock;
double ms_since(Clock::time_point t0) {
    return std::chrono::duration<double, std::milli>(Clock::now() - t0).count();
}

bool total_less(double a, double b) {
    int64_t l, r;
    std::memcpy(&l, &a, 8);
    std::memcpy(&r, &b, 8);
    l ^= (int64_t)(((uint64_t)(l >> 63)) >> 1);
    r ^= (int64_t)(((uint64_t)(r >> 63)) >> 1);
    return l < r;
}

using Poly2 = std::vector<V2>;

double poly_area(const Poly2& p) {
    if (p.size() < 3) return 0.0;
    double s = -0.0;
    for (size_t i = 0; i < p.size(); ++i) s += mg::cross2(p[i], p[(i + 1) % p.size()]);
    return std::fabs(s) * 0.5;
}

double poly_signed_area(const Poly2& p) {
    double s = -0.0;
    for (size_t i = 0; i < p.size(); ++i) s += mg::cross2(p[i], p[(i + 1) % p.size()]);
    return s * 0.5;
}

// split_polygon (surface_merge.rs:1886-1917): (included, excluded)
void split_polygon(const Poly2& polygon, V2 a, V2 b, double orientation, Poly2& in, Poly2* ex) {
    in.clear();
    if (ex) ex->clear();
    if (polygon.empty()) return;
    const V2 ba = b - a;
    const size_t n = polygon.size();
    for (size_t i = 0; i < n; ++i) {
        const V2 prev = polygon[(i + n - 1) % n], cur = polygon[i];
        const double before = orientation * mg::cross2(ba, prev - a);
        const double after = orientation * mg::cross2(ba, cur - a);
        if ((before < 0.0 && after > 0.0) || (before > 0.0 && after < 0.0)) {
            const V2 x = prev + (cur - prev) * (before / (before - after));
            in.push_back(x);
            if (ex) ex->push_back(x);
        }
        if (after >= 0.0) in.push_back(cur);
        if (after <= 0.0 && ex) ex->push_back(cur);
    }
}

// TriangleGeometry (surface_merge.rs:1137-1191)
struct Geometry {
    V3 c[3];
    V3 normal;
    double e[3];
    double area() const { return mg::norm3(mg::cross3(c[1] - c[0], c[2] - c[0])) * 0.5; }
    void aabb(double pad, double lo[3], double hi[3]) const {
        for (int a = 0; a < 3; ++a) {
            double l = INFINITY, h = -INFINITY;
            for (int i = 0; i < 3; ++i) {
                const double v = a == 0 ? c[i].x : a == 1 ? c[i].y : c[i].z;
                l = std::fmin(l, v);
                h = std::fmax(h, v);
            }
            lo[a] = l - pad;
            hi[a] = h + pad;
        }
    }
};

bool make_geometry(const V3 c[3], Geometry& g) {
    for (int i = 0; i < 3; ++i)
        if (!std::isfinite(c[i].x) || !std::isfinite(c[i].y) || !std::isfinite(c[i].z)) return false;
    const V3 n = mg::cross3(c[1] - c[0], c[2] - c[0]);
    const double length = mg::norm3(n);
    if (!std::isfinite(length) || length <= mg::kGeomEps) return false;
    for (int i = 0; i < 3; ++i) g.c[i] = c[i];
    g.normal = V3{n.x / length, n.y / length, n.z / length};
    g.e[0] = mg::norm3(c[1] - c[0]);
    g.e[1] = mg::norm3(c[2] - c[1]);
    g.e[2] = mg::norm3(c[0] - c[2]);
    return true;
}

enum class Limit { None, Cells, Postings };

// PostingBudget / PostingTally (surface_merge.rs:1825-1869)
struct Budget {
    size_t limit = kMaxPostings, used = 0;
    // take `items` into `out` (the caller sorts), or the prefix that fits
    Limit take(const uint32_t* items, size_t n, std::vector<uint32_t>& out) {
        const size_t room = limit - used;
        if (n <= room) {
            used += n;
            out.insert(out.end(), items, items + n);
            return Limit::None;
        }
        used = limit;
        out.insert(out.end(), items, items + room);
        return Limit::Postings;
    }
};
struct Tally {
    size_t max_postings = 0, bound_hits = 0;
    void record(size_t used, Limit l) {
        max_postings = std::max(max_postings, used);
        if (l == Limit::Postings) bound_hits += 1;
    }
};

// LevelGrid<3> (surface_merge.rs:1685-1815), mutable: the kept triangles of
// processed patches and the stitches.
struct Grid3 {
    struct Key {
        int32_t level;
        int64_t k[3];
        bool operator==(const Key& o) const {
            return level == o.level && k[0] == o.k[0] && k[1] == o.k[1] && k[2] == o.k[2];
        }
    };
    struct KeyHash {
        size_t operator()(const Key& key) const {
            uint64_t h = (uint64_t)key.level * 0x9E3779B97F4A7C15ull;
            for (int a = 0; a < 3; ++a) {
                h ^= (uint64_t)key.k[a] + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
            }
            return (size_t)h;
        }
    };
    double cell;
    int32_t levels = 0;
    std::unordered_map<Key, std::vector<uint32_t>, KeyHash> cells;
    std::vector<uint32_t> unindexed;
    explicit Grid3(double c) : cell(c) {}

    void insert(uint32_t item, const double lo[3], const double hi[3]) {
        for (int level = 0; level < mg::kMaxGridLevels; ++level) {
            int64_t f[3], l[3];
            bool ok = true;
            for (int a = 0; a < 3 && ok; ++a) ok = mg::axis_range(cell, level, lo[a], hi[a], f[a], l[a]);
            if (!ok) break;
            bool fits = true;
            for (int a = 0; a < 3; ++a)
                if (mg::sat_sub(l[a], f[a]) > mg::kMaxAnchorCellSpan) fits = false;
            if (fits) {
                cells[Key{level, {f[0], f[1], f[2]}}].push_back(item);
                levels = std::max(levels, level + 1);
                return;
            }
        }
        unindexed.push_back(item);
    }

    // LevelGrid::query_bounded: postings appended to `out` unsorted
    Limit query(const double lo[3], const double hi[3], size_t max_cells, Budget& budget,
                std::vector<uint32_t>& out) const {
        struct R {
            int64_t f[3], l[3];
        };
        std::vector<R> ranges(levels);
        for (int level = 0; level < levels; ++level) {
            R& r = ranges[level];
            size_t count = 1;
            for (int a = 0; a < 3; ++a) {
                if (!mg::axis_range(cell, level, lo[a], hi[a], r.f[a], r.l[a])) return Limit::Cells;
                r.f[a] = mg::sat_sub(r.f[a], mg::kMaxAnchorCellSpan);
                if (r.l[a] < r.f[a]) return Limit::Cells;
                const uint64_t span = (uint64_t)r.l[a] - (uint64_t)r.f[a];
                if (span == UINT64_MAX) return Limit::Cells;
                const uint64_t cells_a = span + 1;
                count = (count != 0 && cells_a > SIZE_MAX / count) ? SIZE_MAX : count * cells_a;
            }
            if (count > max_cells) return Limit::Cells;
        }
        Limit q = budget.take(unindexed.data(), unindexed.size(), out);
        if (q != Limit::None) return q;
        for (int level = 0; level < levels; ++level) {
            const R& r = ranges[level];
            for (int64_t z = r.f[2];; ++z) {
                for (int64_t y = r.f[1];; ++y) {
                    for (int64_t x = r.f[0];; ++x) {
                        auto it = cells.find(Key{level, {x, y, z}});
                        if (it != cells.end()) {
                            q = budget.take(it->second.data(), it->second.size(), out);
                            if (q != Limit::None) return q;
                        }
                        if (x == r.l[0]) break;
                    }
                    if (y == r.l[1]) break;
                }
                if (z == r.l[2]) break;
            }
        }
        return Limit::None;
    }
};

// Footprint (surface_merge.rs:1320-1592): a processed patch's kept triangles in
// its own reference image, with a frozen grid of one posting per triangle.
struct Footprint {
    size_t patch;
    Cam cam;
    std::vector<PT> tri;
    std::vector<uint32_t> comp;
    std::vector<std::array<uint32_t, 3>> vert;
    std::vector<uint32_t> mesh;
    std::vector<std::pair<uint32_t, uint32_t>> omitted;  // (component, mesh index)
    double cell = 1.0;
    int32_t levels = 0;
    std::vector<mg::GridBucket> buckets;
    std::vector<uint32_t> items;  // bucketed (by bucket), then unindexed
    uint32_t n_bucketed = 0;

    bool project_candidate(const Geometry& g, PT& c) const {
        if (!mg::project_triangle(cam, g.c, c)) return false;
        return mg::image_area(c) > mg::kGeomEps * mg::kGeomEps;
    }

    // LevelGrid<2>::query_bounded with MAX_IMAGE_GRID_CELLS; sorted postings
    Limit lookup(const PT& c, std::vector<uint32_t>& found, size_t& used) const {
        double lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
        for (int i = 0; i < 3; ++i) {
            lo[0] = std::fmin(lo[0], c.x[i]);
            hi[0] = std::fmax(hi[0], c.x[i]);
            lo[1] = std::fmin(lo[1], c.y[i]);
            hi[1] = std::fmax(hi[1], c.y[i]);
        }
        found.clear();
        used = 0;
        struct R {
            int64_t f[2], l[2];
        };
        R ranges[mg::kMaxGridLevels];
        for (int level = 0; level < levels; ++level) {
            R& r = ranges[level];
            uint64_t count = 1;
            for (int a = 0; a < 2; ++a) {
                if (!mg::axis_range(cell, level, lo[a], hi[a], r.f[a], r.l[a])) return Limit::Cells;
                r.f[a] = mg::sat_sub(r.f[a], mg::kMaxAnchorCellSpan);
                if (r.l[a] < r.f[a]) return Limit::Cells;
                const uint64_t span = (uint64_t)r.l[a] - (uint64_t)r.f[a];
                if (span == UINT64_MAX) return Limit::Cells;
                const uint64_t cells_a = span + 1;
                count = (count != 0 && cells_a > UINT64_MAX / count) ? UINT64_MAX : count * cells_a;
            }
            if (count > kMaxImageGridCells) return Limit::Cells;
        }
        Budget budget;
        Limit q = budget.take(items.data() + n_bucketed, items.size() - n_bucketed, found);
        if (q != Limit::None) {
            used = budget.used;
            return q;
        }
        for (int level = 0; level < levels; ++level) {
            const R& r = ranges[level];
            for (int64_t y = r.f[1];; ++y) {
                for (int64_t x = r.f[0];; ++x) {
                    auto it = std::lower_bound(buckets.begin(), buckets.end(), 0,
                                               [&](const mg::GridBucket& b, int) {
                                                   return mg::bucket_less(b, level, x, y);
                                               });
                    if (it != buckets.end() && it->level == level && it->x == x && it->y == y) {
                        const uint32_t end = it + 1 != buckets.end() ? (it + 1)->start : n_bucketed;
                        q = budget.take(items.data() + it->start, end - it->start, found);
                        if (q != Limit::None) {
                            used = budget.used;
                            return q;
                        }
                    }
                    if (x == r.l[0]) break;
                }
                if (y == r.l[1]) break;
            }
        }
        used = budget.used;
        std::sort(found.begin(), found.end());
        return Limit::None;
    }
};

void build_footprint_grid(Footprint& f) {
    std::vector<double> edges;
    edges.reserve(f.tri.size() * 3);
    for (const PT& t : f.tri)
        for (int i = 0; i < 3; ++i) edges.push_back(mg::norm2(t.p((i + 1) % 3) - t.p(i)));
    const size_t mid = edges.size() / 2;
    std::nth_element(edges.begin(), edges.begin() + mid, edges.end(), total_less);
    f.cell = std::fmax(edges[mid] * 2.0, mg::kGeomEps);
    struct Entry {
        int32_t level;
        int64_t x, y;
        uint32_t item;
    };
    std::vector<Entry> entries;
    std::vector<uint32_t> unindexed;
    entries.reserve(f.tri.size());
    for (uint32_t i = 0; i < f.tri.size(); ++i) {
        const PT& t = f.tri[i];
        double lo[2] = {INFINITY, INFINITY}, hi[2] = {-INFINITY, -INFINITY};
        for (int k = 0; k < 3; ++k) {
            lo[0] = std::fmin(lo[0], t.x[k]);
            hi[0] = std::fmax(hi[0], t.x[k]);
            lo[1] = std::fmin(lo[1], t.y[k]);
            hi[1] = std::fmax(hi[1], t.y[k]);
        }
        bool placed = false;
        for (int level = 0; level < mg::kMaxGridLevels; ++level) {
            int64_t fx, lx, fy, ly;
            if (!mg::axis_range(f.cell, level, lo[0], hi[0], fx, lx) ||
                !mg::axis_range(f.cell, level, lo[1], hi[1], fy, ly))
                break;
            if (mg::sat_sub(lx, fx) <= mg::kMaxAnchorCellSpan &&
                mg::sat_sub(ly, fy) <= mg::kMaxAnchorCellSpan) {
                entries.push_back({level, fx, fy, i});
                f.levels = std::max(f.levels, level + 1);
                placed = true;
                break;
            }
        }
        if (!placed) unindexed.push_back(i);
    }
    std::sort(entries.begin(), entries.end(), [](const Entry& a, const Entry& b) {
        if (a.level != b.level) return a.level < b.level;
        if (a.x != b.x) return a.x < b.x;
        if (a.y != b.y) return a.y < b.y;
        return a.item < b.item;
    });
    f.items.clear();
    f.buckets.clear();
    for (size_t i = 0; i < entries.size(); ++i) {
        if (i == 0 || entries[i].level != entries[i - 1].level || entries[i].x != entries[i - 1].x ||
            entries[i].y != entries[i - 1].y)
            f.buckets.push_back({entries[i].x, entries[i].y, entries[i].level, (uint32_t)i});
        f.items.push_back(entries[i].item);
    }
    f.n_bucketed = (uint32_t)f.items.size();
    f.items.insert(f.items.end(), unindexed.begin(), unindexed.end());
}

}  // namespace
}  // namespace merge
}  // namespace v3d

namespace v3d {
namespace merge {
namespace {

enum class Cover { Full, Partial, Uncovered, Exhausted };

// TriangleGeometry::coverage (surface_merge.rs:1213-1290)
Cover coverage(const Geometry& self, const std::vector<const Geometry*>& surfaces, double tolerance) {
    const V3 origin = self.c[0];
    const V3 d = self.c[1] - origin;
    const double dn = mg::norm3(d);
    const V3 u{d.x / dn, d.y / dn, d.z / dn};
    const V3 v = mg::cross3(self.normal, u);
    auto project = [&](V3 p) {
        const V3 rel = p - origin;
        return V2{mg::dot3(rel, u), mg::dot3(rel, v)};
    };
    double m = 1.0e-12;
    for (double e : self.e) m = std::fmax(m, e);
    const double area_epsilon = m * m * 1.0e-10;
    std::vector<Poly2> remaining{Poly2{project(self.c[0]), project(self.c[1]), project(self.c[2])}};
    bool partially = false;
    Poly2 inside, included, excluded;
    for (const Geometry* s : surfaces) {
        if (std::fabs(mg::dot3(self.normal, s->normal)) < kMinNormalAlignment) continue;
        const V2 pr[3] = {project(s->c[0]), project(s->c[1]), project(s->c[2])};
        const double winding = mg::cross2(pr[1] - pr[0], pr[2] - pr[0]);
        if (std::fabs(winding) <= area_epsilon) continue;
        const double orientation = mg::signum(winding);
        std::vector<Poly2> next;
        for (Poly2& polygon : remaining) {
            inside = std::move(polygon);
            std::vector<Poly2> outside;
            for (int e = 0; e < 3; ++e) {
                split_polygon(inside, pr[e], pr[(e + 1) % 3], orientation, included, &excluded);
                if (poly_area(excluded) > area_epsilon) outside.push_back(excluded);
                inside.swap(included);
                if (inside.empty()) break;
            }
            if (poly_area(inside) > area_epsilon) {
                bool supported = true;
                for (const V2& p : inside) {
                    const V3 point = (origin + u * p.x) + v * p.y;
                    if (!(std::fabs(mg::dot3(point - s->c[0], s->normal)) <= tolerance)) {
                        supported = false;
                        break;
                    }
                }
                if (supported) partially = true;
                else outside.push_back(inside);
            }
            for (auto& o : outside) next.push_back(std::move(o));
            if (next.size() > kMaxUncoveredPieces) return Cover::Exhausted;
        }
        remaining = std::move(next);
        if (remaining.empty()) return Cover::Full;
    }
    return partially ? Cover::Partial : Cover::Uncovered;
}

double distance_to_line(V2 a, V2 b, V2 p) {
    const V2 dir = b - a;
    const double length = mg::norm2(dir);
    if (length <= 0.0) return mg::norm2(p - a);
    return mg::cross2(dir, p - a) / length;
}

// ear_clip (surface_merge_clip.rs:220-257)
bool ear_clip(const Poly2& polygon, double tolerance, std::vector<std::array<uint32_t, 3>>& tris) {
    std::vector<uint32_t> rem(polygon.size());
    for (uint32_t i = 0; i < rem.size(); ++i) rem[i] = i;
    tris.clear();
    const double floor_ = tolerance * tolerance;
    while (rem.size() > 3) {
        const size_t count = rem.size();
        size_t found = SIZE_MAX;
        for (size_t slot = 0; slot < count && found == SIZE_MAX; ++slot) {
            const uint32_t pv = rem[(slot + count - 1) % count], cu = rem[slot], nx = rem[(slot + 1) % count];
            const V2 a = polygon[pv], b = polygon[cu], c = polygon[nx];
            if (mg::cross2(b - a, c - a) <= floor_) continue;
            const V2 ear[3] = {a, b, c};
            bool blocked = false;
            for (uint32_t other : rem) {
                if (other == pv || other == cu || other == nx) continue;
                const V2 p = polygon[other];
                if (mg::norm2(p - a) <= tolerance || mg::norm2(p - b) <= tolerance ||
                    mg::norm2(p - c) <= tolerance)
                    continue;
                bool in = true;
                for (int e = 0; e < 3 && in; ++e)
                    in = distance_to_line(ear[e], ear[(e + 1) % 3], p) >= -tolerance;
                if (in) {
                    blocked = true;
                    break;
                }
            }
            if (!blocked) found = slot;
        }
        if (found == SIZE_MAX) return false;
        const size_t cnt = rem.size();
        tris.push_back({rem[(found + cnt - 1) % cnt], rem[found], rem[(found + 1) % cnt]});
        rem.erase(rem.begin() + (ptrdiff_t)found);
    }
    if (rem.size() < 3) return false;
    if (mg::cross2(polygon[rem[1]] - polygon[rem[0]], polygon[rem[2]] - polygon[rem[0]]) <= floor_)
        return false;
    tris.push_back({rem[0], rem[1], rem[2]});
    return true;
}

using EdgeKey = std::pair<uint64_t, uint64_t>;
EdgeKey ekey(uint64_t a, uint64_t b) { return {std::min(a, b), std::max(a, b)}; }
struct PairHash {
    size_t operator()(const EdgeKey& k) const {
        return (size_t)(k.first * 0x9E3779B97F4A7C15ull ^ (k.second + 0x7F4A7C159E3779B9ull));
    }
};
struct CrossHash {
    size_t operator()(const std::pair<EdgeKey, EdgeKey>& k) const {
        PairHash h;
        return h(k.first) * 31 + h(k.second);
    }
};

struct Derived {
    v3d_point point;
    int64_t group;
    v3d_derived_vertex_source source;
};

// ClipState (surface_merge_clip.rs:96-155)
struct ClipState {
    uint64_t base;
    std::vector<Derived> derived;
    std::unordered_map<std::pair<EdgeKey, EdgeKey>, uint64_t, CrossHash> crossings;
    std::unordered_map<EdgeKey, std::vector<std::pair<double, uint64_t>>, PairHash> carriers;
    std::unordered_map<uint64_t, std::vector<EdgeKey>> vertex_carriers;
    void record(EdgeKey edge, double parameter, uint64_t vertex) {
        if (edge.first == vertex || edge.second == vertex) return;
        auto& entries = carriers[edge];
        for (const auto& e : entries)
            if (e.second == vertex) return;
        entries.push_back({parameter, vertex});
        auto& list = vertex_carriers[vertex];
        if (std::find(list.begin(), list.end(), edge) == list.end()) list.push_back(edge);
    }
};

}  // namespace
}  // namespace merge
}  // namespace v3d

namespace v3d {
namespace merge {
namespace {

constexpr size_t kMaxClipOwnerTriangles = 48;   // surface_merge_clip.rs:48
constexpr size_t kMaxClipNodes = 160;           // :50
constexpr double kMaxClipDepthDisagreement = 0.014;  // :60
constexpr double kRelativeTolerance = 1.0e-5;   // :65
constexpr double kAreaTolerance = 1.0e-4;       // :67

struct ClipJob {
    uint32_t triangle, footprint;
    double scale;
};

// Everything the host stages read.
struct Inputs {
    const v3d_point* points;
    uint64_t n_points;
    const int64_t* membership;
    const int32_t* origins;
    uint64_t n_origins;
    std::vector<v3d_mesh_triangle>* triangles;   // re-indexed in place
    const std::vector<uint8_t>* has_geometry;
    const std::vector<Geometry>* geometry;
    const std::vector<Footprint>* footprints;
    const std::vector<uint32_t>* component_by_triangle;
    const std::vector<int32_t>* cluster;         // per component root
    const std::vector<std::pair<uint64_t, std::array<uint64_t, 3>>>* reindexed;

    int64_t group(uint64_t v) const { return v < n_points ? membership[v] : -1; }
    // point_origins.get(v).copied().flatten()
    int32_t origin(uint64_t v) const { return v < n_origins ? origins[v] : V3D_ORIGIN_NONE; }
    bool linked(uint32_t triangle, uint32_t comp) const {
        const uint32_t own = (*component_by_triangle)[triangle];
        if (own == comp) return false;
        const int32_t c = (*cluster)[own];
        return c >= 0 && (*cluster)[comp] == c;
    }
    V3 position(uint64_t v) const {
        return V3{(double)points[v].x, (double)points[v].y, (double)points[v].z};
    }
    std::array<uint64_t, 3> source_corners(uint64_t mesh_index) const {
        auto it = std::lower_bound(reindexed->begin(), reindexed->end(), mesh_index,
                                   [](const auto& e, uint64_t v) { return e.first < v; });
        if (it != reindexed->end() && it->first == mesh_index) return it->second;
        const v3d_mesh_triangle& t = (*triangles)[mesh_index];
        return {t.a, t.b, t.c};
    }
};

// The candidate's overlaps with linked owner triangles (Footprint::visit_overlaps)
// as (polygon, footprint index); false when the lookup was cut off.
template <class Include, class Visit>
bool visit_overlaps(const Footprint& f, const PT& cand, Include include, Visit visit, Tally& tally) {
    std::vector<uint32_t> found;
    size_t used;
    const Limit q = f.lookup(cand, found, used);
    tally.record(used, q);
    if (q != Limit::None) return false;
    Poly<8> poly;
    for (uint32_t idx : found) {
        if (!include(idx)) continue;
        if (!mg::clip_to_triangle(cand, f.tri[idx], poly)) continue;
        if (mg::poly_area(poly) > 0.0) {
            Poly2 p(poly.v, poly.v + poly.n);
            if (!visit(p, idx)) break;
        }
    }
    return true;
}

double world_parameter(double t, const double depths[2]) {
    const double numerator = t * depths[0];
    const double denominator = numerator + (1.0 - t) * depths[1];
    if (std::fabs(denominator) <= mg::kF64MinPositive) return t;
    double r = numerator / denominator;
    if (r < 0.0) r = 0.0;
    if (r > 1.0) r = 1.0;
    return r;
}

double parameter(V2 a, V2 b, V2 p) {
    const V2 dir = b - a;
    return mg::dot2(p - a, dir) / (dir.x * dir.x + dir.y * dir.y);
}

bool strictly_inside(const V2 tri[3], V2 p, double tolerance) {
    const double o = mg::signum(mg::cross2(tri[1] - tri[0], tri[2] - tri[0]));
    for (int e = 0; e < 3; ++e)
        if (!(o * distance_to_line(tri[e], tri[(e + 1) % 3], p) > tolerance)) return false;
    return true;
}

struct ClipNode {
    V2 pos;
    bool vertex;
    uint64_t id;
    EdgeKey subject, owner;  // crossing: the ids as on each segment (not sorted)
    double owner_t;
    uint32_t owner_triangle;
};
struct ClipSeg {
    size_t nodes[2];
    uint64_t ids[2];
    double depths[2];
    std::vector<std::pair<double, size_t>> inside;
};
// The geometric half of one clip: its arrangement, faces and kept pieces,
// which read the inputs only, so clips are planned concurrently.
struct ClipPlan {
    uint32_t footprint;
    bool flipped;
    std::vector<ClipNode> nodes;
    std::vector<ClipSeg> segs;
    std::vector<std::array<size_t, 3>> kept;
    std::unordered_map<uint64_t, double> owner_depth;
};

// clip_overlap (surface_merge_clip.rs:294-694) up to the area balance; false:
// kept whole
bool plan_clip(const Inputs& in, const ClipJob& job, Tally& tally, ClipPlan& plan) {
    plan.footprint = job.footprint;
    const Footprint& f = (*in.footprints)[job.footprint];
    const v3d_mesh_triangle tri = (*in.triangles)[job.triangle];
    if (!(*in.has_geometry)[job.triangle]) return false;
    PT cand;
    if (!f.project_candidate((*in.geometry)[job.triangle], cand)) return false;
    std::vector<std::pair<uint32_t, double>> owned;
    bool overflow = false;
    if (!visit_overlaps(
            f, cand, [&](uint32_t idx) { return in.linked(job.triangle, f.comp[idx]); },
            [&](const Poly2& poly, uint32_t idx) {
                const PT& kept = f.tri[idx];
                bool agrees = true;
                for (const V2& pt : poly) {
                    double own, owner;
                    if (!mg::inverse_depth(cand, pt, own) || !mg::inverse_depth(kept, pt, owner)) {
                        agrees = false;
                        break;
                    }
                    const double o = 1.0 / own, w = job.scale / owner;
                    if (!(std::fabs(o - w) <= kMaxClipDepthDisagreement * w)) {
                        agrees = false;
                        break;
                    }
                }
                if (agrees) {
                    owned.push_back({idx, poly_area(poly)});
                    if (owned.size() > kMaxClipOwnerTriangles) {
                        overflow = true;
                        return false;
                    }
                }
                return true;
            },
            tally))
        return false;
    if (overflow || owned.empty()) return false;
    double owned_area = -0.0;
    for (const auto& o : owned) owned_area += o.second;

    const uint64_t ids3[3] = {tri.a, tri.b, tri.c};
    const double signed_ = mg::cross2(cand.p(1) - cand.p(0), cand.p(2) - cand.p(0));
    const bool flipped = signed_ < 0.0;
    const int order[3] = {0, flipped ? 2 : 1, flipped ? 1 : 2};
    V2 spos[3];
    double sdepth[3];
    uint64_t sid[3];
    for (int i = 0; i < 3; ++i) {
        spos[i] = cand.p(order[i]);
        sdepth[i] = cand.z[order[i]];
        sid[i] = ids3[order[i]];
    }
    double extent = 0.0;
    for (int e = 0; e < 3; ++e) extent = std::fmax(extent, mg::norm2(spos[(e + 1) % 3] - spos[e]));
    const double tolerance = extent * kRelativeTolerance;
    const double subject_area = std::fabs(signed_) * 0.5;

    auto& nodes = plan.nodes;
    nodes.clear();
    std::unordered_map<uint64_t, size_t> by_id;
    for (int i = 0; i < 3; ++i) {
        by_id[sid[i]] = nodes.size();
        nodes.push_back(ClipNode{spos[i], true, sid[i], {}, {}, 0.0, 0});
    }
    auto& owner_depth = plan.owner_depth;
    owner_depth.clear();
    for (const auto& o : owned)
        for (int k = 0; k < 3; ++k) {
            const uint64_t id = f.vert[o.first][k];
            const V2 pos = f.tri[o.first].p(k);
            owner_depth[id] = f.tri[o.first].z[k];
            if (by_id.count(id)) continue;
            size_t node = SIZE_MAX;
            for (int s = 0; s < 3; ++s)
                if (mg::norm2(spos[s] - pos) <= tolerance) {
                    node = (size_t)s;
                    break;
                }
            if (node == SIZE_MAX) {
                nodes.push_back(ClipNode{pos, true, id, {}, {}, 0.0, 0});
                node = nodes.size() - 1;
            }
            by_id[id] = node;
        }
    auto& segs = plan.segs;
    segs.clear();
    for (int e = 0; e < 3; ++e) {
        const int n = (e + 1) % 3;
        segs.push_back(ClipSeg{{(size_t)e, (size_t)n}, {sid[e], sid[n]}, {sdepth[e], sdepth[n]}, {}});
    }
    struct OE {
        uint64_t a, b;
        uint32_t index;
    };
    std::map<EdgeKey, OE> owner_edges;
    for (const auto& o : owned)
        for (int k = 0; k < 3; ++k) {
            const uint64_t a = f.vert[o.first][k], b = f.vert[o.first][(k + 1) % 3];
            owner_edges.emplace(ekey(a, b), OE{a, b, o.first});
        }
    const size_t owner_first = segs.size();
    std::vector<uint32_t> owner_triangle_of;
    for (const auto& kv : owner_edges) {
        const size_t na = by_id.at(kv.second.a), nb = by_id.at(kv.second.b);
        if (na == nb) continue;
        segs.push_back(ClipSeg{{na, nb}, {kv.second.a, kv.second.b},
                           {owner_depth.at(kv.second.a), owner_depth.at(kv.second.b)}, {}});
        owner_triangle_of.push_back(kv.second.index);
    }
    std::set<size_t> owner_nodes;
    for (const auto& kv : by_id)
        if (kv.second > 2) owner_nodes.insert(kv.second);
    auto on_segment = [&](ClipSeg& sg, size_t node) {
        const V2 a = nodes[sg.nodes[0]].pos, b = nodes[sg.nodes[1]].pos;
        const double length = mg::norm2(b - a);
        const V2 p = nodes[node].pos;
        const double t = parameter(a, b, p);
        if (std::fabs(distance_to_line(a, b, p)) <= tolerance && t * length > tolerance &&
            (1.0 - t) * length > tolerance)
            sg.inside.push_back({t, node});
    };
    for (int e = 0; e < 3; ++e)
        for (size_t node : owner_nodes) on_segment(segs[e], node);
    for (size_t sg = owner_first; sg < segs.size(); ++sg)
        for (size_t node = 0; node < 3; ++node)
            if (node != segs[sg].nodes[0] && node != segs[sg].nodes[1]) on_segment(segs[sg], node);
    for (int e = 0; e < 3; ++e)
        for (size_t sg = owner_first; sg < segs.size(); ++sg) {
            const size_t p = segs[e].nodes[0], q = segs[e].nodes[1];
            const size_t a = segs[sg].nodes[0], b = segs[sg].nodes[1];
            if (p == a || p == b || q == a || q == b) continue;
            const V2 pp = nodes[p].pos, qp = nodes[q].pos, ap = nodes[a].pos, bp = nodes[b].pos;
            const double da = distance_to_line(pp, qp, ap), db = distance_to_line(pp, qp, bp);
            const double dp = distance_to_line(ap, bp, pp), dq = distance_to_line(ap, bp, qp);
            if (std::fabs(da) <= tolerance || std::fabs(db) <= tolerance ||
                std::fabs(dp) <= tolerance || std::fabs(dq) <= tolerance)
                continue;
            if (mg::signum(da) == mg::signum(db) || mg::signum(dp) == mg::signum(dq)) continue;
            const double st = dp / (dp - dq), ot = da / (da - db);
            if (nodes.size() >= kMaxClipNodes) return false;
            const size_t node = nodes.size();
            nodes.push_back(ClipNode{pp + (qp - pp) * st, false, 0, {segs[e].ids[0], segs[e].ids[1]},
                                 {segs[sg].ids[0], segs[sg].ids[1]}, ot,
                                 owner_triangle_of[sg - owner_first]});
            segs[e].inside.push_back({st, node});
            segs[sg].inside.push_back({ot, node});
        }
    if (nodes.size() > kMaxClipNodes) return false;

    std::set<std::pair<size_t, size_t>> edges;
    for (size_t index = 0; index < segs.size(); ++index) {
        ClipSeg& sg = segs[index];
        std::stable_sort(sg.inside.begin(), sg.inside.end(),
                         [](const auto& x, const auto& y) { return total_less(x.first, y.first); });
        std::vector<size_t> chain{sg.nodes[0]};
        for (const auto& e : sg.inside) chain.push_back(e.second);
        chain.push_back(sg.nodes[1]);
        chain.erase(std::unique(chain.begin(), chain.end()), chain.end());
        for (size_t i = 0; i + 1 < chain.size(); ++i) {
            const size_t from = chain[i], to = chain[i + 1];
            if (from == to) continue;
            if (index >= owner_first) {
                const V2 middle = (nodes[from].pos + nodes[to].pos) * 0.5;
                if (!strictly_inside(spos, middle, tolerance)) continue;
            }
            edges.insert({std::min(from, to), std::max(from, to)});
        }
    }
    std::vector<std::vector<size_t>> nb(nodes.size());
    for (const auto& e : edges) {
        nb[e.first].push_back(e.second);
        nb[e.second].push_back(e.first);
    }
    std::vector<size_t> parent(nodes.size());
    for (size_t i = 0; i < parent.size(); ++i) parent[i] = i;
    auto find = [&](size_t i) {
        size_t r = i;
        while (parent[r] != r) r = parent[r];
        while (parent[i] != r) {
            const size_t n = parent[i];
            parent[i] = r;
            i = n;
        }
        return r;
    };
    for (const auto& e : edges) {
        const size_t a = find(e.first), b = find(e.second);
        parent[a] = b;
    }
    size_t first_used = SIZE_MAX;
    for (size_t node = 0; node < nodes.size(); ++node)
        if (!nb[node].empty()) {
            first_used = node;
            break;
        }
    if (first_used == SIZE_MAX) return false;
    const size_t root = find(first_used);
    for (size_t node = 0; node < nodes.size(); ++node)
        if (!nb[node].empty() && (find(node) != root || nb[node].size() < 2)) return false;
    for (size_t node = 0; node < nodes.size(); ++node) {
        const V2 o = nodes[node].pos;
        std::stable_sort(nb[node].begin(), nb[node].end(), [&](size_t a, size_t b) {
            const V2 da = nodes[a].pos - o, db = nodes[b].pos - o;
            return total_less(std::atan2(da.y, da.x), std::atan2(db.y, db.x));
        });
    }
    std::set<std::pair<size_t, size_t>> visited;
    std::vector<std::vector<size_t>> faces;
    size_t outer = 0;
    const size_t limit = 2 * edges.size() + 2;
    for (const auto& e : edges) {
        const std::pair<size_t, size_t> starts[2] = {{e.first, e.second}, {e.second, e.first}};
        for (const auto& st : starts) {
            if (visited.count(st)) continue;
            std::vector<size_t> face;
            size_t from = st.first, to = st.second;
            for (;;) {
                if (!visited.insert({from, to}).second || face.size() > limit) return false;
                face.push_back(from);
                const auto& around = nb[to];
                size_t back = SIZE_MAX;
                for (size_t i = 0; i < around.size(); ++i)
                    if (around[i] == from) {
                        back = i;
                        break;
                    }
                if (back == SIZE_MAX) return false;
                const size_t following = around[(back + around.size() - 1) % around.size()];
                from = to;
                to = following;
                if (from == st.first && to == st.second) break;
            }
            Poly2 poly;
            for (size_t node : face) poly.push_back(nodes[node].pos);
            if (poly_signed_area(poly) > 0.0) faces.push_back(std::move(face));
            else outer += 1;
        }
    }
    if (outer != 1) return false;
    auto& kept = plan.kept;
    kept.clear();
    double kept_area = 0.0, removed_area = 0.0;
    std::vector<std::array<uint32_t, 3>> ears;
    for (const auto& face : faces) {
        Poly2 poly;
        for (size_t node : face) poly.push_back(nodes[node].pos);
        if (!ear_clip(poly, tolerance, ears)) return false;
        V2 largest{0.0, 0.0};
        double best = -INFINITY;
        for (const auto& ear : ears) {
            const V2 a = poly[ear[0]], b = poly[ear[1]], c = poly[ear[2]];
            const double area = mg::cross2(b - a, c - a);
            if (area > best) {
                best = area;
                largest = ((a + b) + c) / 3.0;
            }
        }
        const double area = poly_signed_area(poly);
        bool removed = false;
        for (const auto& o : owned) {
            const V2 ot[3] = {f.tri[o.first].p(0), f.tri[o.first].p(1), f.tri[o.first].p(2)};
            if (strictly_inside(ot, largest, 0.0)) {
                removed = true;
                break;
            }
        }
        if (removed) {
            removed_area += area;
            continue;
        }
        kept_area += area;
        for (const auto& ear : ears) kept.push_back({face[ear[0]], face[ear[1]], face[ear[2]]});
    }
    const double balance = kAreaTolerance * subject_area;
    if (std::fabs((kept_area + removed_area) - subject_area) > balance ||
        std::fabs(removed_area - owned_area) > balance)
        return false;
    plan.flipped = flipped;
    return true;
}

// clip_overlap (surface_merge_clip.rs:696-759): the planned clip's vertex ids,
// its derived vertices and edge records committed to `state`; false (state
// unchanged) when a new crossing would join corners of different origins
bool commit_clip(const Inputs& in, ClipState& state, const ClipPlan& plan,
                 std::vector<std::array<uint64_t, 3>>& out) {
    const Footprint& f = (*in.footprints)[plan.footprint];
    const auto& nodes = plan.nodes;
    const auto& segs = plan.segs;
    const auto& kept = plan.kept;
    const auto& owner_depth = plan.owner_depth;
    const bool flipped = plan.flipped;
    std::set<size_t> used_nodes;
    for (const auto& k : kept) used_nodes.insert(k.begin(), k.end());
    std::unordered_map<size_t, uint64_t> ids;
    struct Fresh {
        uint64_t id;
        Derived point;
        std::pair<EdgeKey, EdgeKey> crossing;
    };
    std::vector<Fresh> fresh;
    uint64_t next_index = state.base + state.derived.size();
    for (size_t node : used_nodes) {
        const ClipNode& nd = nodes[node];
        uint64_t id;
        if (nd.vertex) {
            id = nd.id;
        } else {
            const uint64_t a = nd.owner.first, b = nd.owner.second;
            const auto crossing = std::make_pair(ekey(nd.subject.first, nd.subject.second), ekey(a, b));
            auto it = state.crossings.find(crossing);
            if (it != state.crossings.end()) {
                id = it->second;
            } else {
                if (in.origin(a) != in.origin(b)) return false;
                const double depths[2] = {owner_depth.at(a), owner_depth.at(b)};
                const double s = world_parameter(nd.owner_t, depths);
                const uint32_t mesh_index = f.mesh[nd.owner_triangle];
                const auto& cur = f.vert[nd.owner_triangle];
                Derived d{};
                d.source.point_index = next_index;
                d.source.source_triangle = mesh_index;
                const auto sc = in.source_corners(mesh_index);
                for (int k = 0; k < 3; ++k) {
                    d.source.source_corners[k] = sc[k];
                    d.source.barycentric[k] = cur[k] == a ? 1.0 - s : cur[k] == b ? s : 0.0;
                }
                const v3d_point pa = in.points[a], pb = in.points[b];
                auto lerp = [&](float x, float y) { return (float)((double)x * (1.0 - s) + (double)y * s); };
                auto lerp8 = [&](uint8_t x, uint8_t y) {
                    double v = std::round((double)x * (1.0 - s) + (double)y * s);
                    if (v < 0.0) v = 0.0;
                    if (v > 255.0) v = 255.0;
                    return std::isnan(v) ? (uint8_t)0 : (uint8_t)v;
                };
                d.point = v3d_point{lerp(pa.x, pb.x), lerp(pa.y, pb.y), lerp(pa.z, pb.z),
                                    lerp(pa.confidence, pb.confidence), lerp8(pa.r, pb.r),
                                    lerp8(pa.g, pb.g), lerp8(pa.b, pb.b), 0};
                d.group = in.group(a);
                id = next_index++;
                fresh.push_back({id, d, crossing});
            }
        }
        ids[node] = id;
    }
    for (auto& fr : fresh) {
        state.crossings[fr.crossing] = fr.id;
        state.derived.push_back(fr.point);
    }
    for (const ClipSeg& sg : segs) {
        const EdgeKey edge = ekey(sg.ids[0], sg.ids[1]);
        const bool forward = edge.first == sg.ids[0];
        for (const auto& e : sg.inside) {
            auto it = ids.find(e.second);
            if (it == ids.end()) continue;
            const double s = world_parameter(e.first, sg.depths);
            state.record(edge, forward ? s : 1.0 - s, it->second);
        }
    }
    out.clear();
    for (const auto& k : kept) {
        const std::array<uint64_t, 3> c{ids.at(k[0]), ids.at(k[1]), ids.at(k[2])};
        out.push_back(flipped ? std::array<uint64_t, 3>{c[0], c[2], c[1]} : c);
    }
    return true;
}

}  // namespace
}  // namespace merge
}  // namespace v3d

namespace v3d {
namespace merge {
namespace {

// conform_edges (surface_merge_clip.rs:775-879); false when canceled.  Every
// triangle's split reads the edge records only, so slots are split
// concurrently and the extra pieces appended in slot order afterwards.
template <class Pos, class Cancel>
bool conform_edges(const ClipState& state, std::vector<v3d_mesh_triangle>& tris, Pos position,
                   Cancel canceled, std::vector<uint64_t>& split, uint64_t& failures) {
    const size_t n = tris.size();
    // the reference polls once every 256 slots; none of them may cancel
    for (size_t slot = 0; slot < n; slot += 256)
        if (canceled()) return false;
    auto parameter_on = [&](const EdgeKey& edge, uint64_t v, double& t) -> bool {
        if (v == edge.first) {
            t = 0.0;
            return true;
        }
        if (v == edge.second) {
            t = 1.0;
            return true;
        }
        auto it = state.carriers.find(edge);
        if (it == state.carriers.end()) return false;
        for (const auto& e : it->second)
            if (e.second == v) {
                t = e.first;
                return true;
            }
        return false;
    };
    // vertices an edge record can involve: carrier edge endpoints and recorded vertices
    std::unordered_set<uint64_t> touched;
    for (const auto& kv : state.carriers) {
        touched.insert(kv.first.first);
        touched.insert(kv.first.second);
    }
    for (const auto& kv : state.vertex_carriers) touched.insert(kv.first);
    const V2 frame[3] = {V2{0.0, 0.0}, V2{1.0, 0.0}, V2{0.0, 1.0}};
    struct Part {
        std::vector<std::pair<uint64_t, std::vector<v3d_mesh_triangle>>> pieces;  // (slot, pieces)
        uint64_t failures = 0;
    };
    const size_t n_threads = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), 16));
    const size_t chunk = (n + n_threads - 1) / n_threads;
    std::vector<Part> parts(n_threads);
    auto work = [&](size_t k) {
        Part& part = parts[k];
        std::vector<std::pair<uint64_t, V2>> boundary;
        std::vector<EdgeKey> carriers;
        std::vector<std::pair<double, uint64_t>> between;
        std::vector<std::array<uint32_t, 3>> ears;
        const size_t lo = k * chunk, hi = std::min(n, lo + chunk);
        for (size_t slot = lo; slot < hi; ++slot) {
            const v3d_mesh_triangle t = tris[slot];
            const uint64_t corners[3] = {t.a, t.b, t.c};
            // no record can apply to an edge none of whose endpoints is touched
            if (!touched.count(t.a) && !touched.count(t.b) && !touched.count(t.c)) continue;
            boundary.clear();
            bool inserted = false;
            for (int e = 0; e < 3; ++e) {
                const uint64_t u = corners[e], v = corners[(e + 1) % 3];
                boundary.push_back({u, frame[e]});
                carriers.assign(1, ekey(u, v));
                for (uint64_t endpoint : {u, v}) {
                    auto it = state.vertex_carriers.find(endpoint);
                    if (it != state.vertex_carriers.end())
                        carriers.insert(carriers.end(), it->second.begin(), it->second.end());
                }
                const EdgeKey* carrier = nullptr;
                double tu = 0.0, tv = 0.0;
                for (const auto& c : carriers)
                    if (state.carriers.count(c) && parameter_on(c, u, tu) && parameter_on(c, v, tv)) {
                        carrier = &c;
                        break;
                    }
                if (!carrier) continue;
                if (std::fabs(tv - tu) <= mg::kF64Eps) continue;
                between.clear();
                for (const auto& en : state.carriers.at(*carrier)) {
                    if (en.second == u || en.second == v) continue;
                    const double rel = (en.first - tu) / (tv - tu);
                    if (rel > 1.0e-9 && rel < 1.0 - 1.0e-9) between.push_back({rel, en.second});
                }
                std::stable_sort(between.begin(), between.end(),
                                 [](const auto& x, const auto& y) { return total_less(x.first, y.first); });
                between.erase(std::unique(between.begin(), between.end(),
                                          [](const auto& x, const auto& y) { return x.second == y.second; }),
                              between.end());
                const V2 start = frame[e], end = frame[(e + 1) % 3];
                for (const auto& b : between) {
                    boundary.push_back({b.second, start + (end - start) * b.first});
                    inserted = true;
                }
            }
            if (!inserted) continue;
            Poly2 poly;
            for (const auto& b : boundary) poly.push_back(b.second);
            if (!ear_clip(poly, 1.0e-12, ears)) {
                part.failures += 1;
                continue;
            }
            bool degenerate = false;
            for (const auto& ear : ears) {
                const V3 a = position(boundary[ear[0]].first), b = position(boundary[ear[1]].first),
                         c = position(boundary[ear[2]].first);
                if (mg::norm3(mg::cross3(b - a, c - a)) <= mg::kF64Eps) {
                    degenerate = true;
                    break;
                }
            }
            if (degenerate) {
                part.failures += 1;
                continue;
            }
            std::vector<v3d_mesh_triangle> pieces;
            for (const auto& ear : ears)
                pieces.push_back(v3d_mesh_triangle{boundary[ear[0]].first, boundary[ear[1]].first,
                                                   boundary[ear[2]].first, t.confidence, 0});
            part.pieces.push_back({slot, std::move(pieces)});
        }
    };
    std::vector<std::thread> pool;
    for (size_t k = 0; k < n_threads; ++k) pool.emplace_back(work, k);
    for (auto& th : pool) th.join();
    split.clear();
    failures = 0;
    std::vector<v3d_mesh_triangle> appended;
    for (const Part& part : parts) {
        failures += part.failures;
        for (const auto& sp : part.pieces) {
            tris[sp.first] = sp.second[0];
            appended.insert(appended.end(), sp.second.begin() + 1, sp.second.end());
            split.push_back(sp.first);
        }
    }
    tris.insert(tris.end(), appended.begin(), appended.end());
    return true;
}

// ---- seam stitching (surface_merge_stitch.rs:299-660) ---------------------------------
constexpr size_t kMaxSeamVertices = 6;
constexpr size_t kMaxSeamsPerVertex = 16;
constexpr double kMaxUnobservedStitchShare = 1.0e-6;
constexpr double kMaxStitchOverlapShare = 1.0e-6;
constexpr double kInsideTolerance = 1.0e-6;

struct Removal {
    uint32_t triangle, footprint;
    double scale;
};

bool contains(const PT& t, V2 p) {
    const V2 a = t.p(0), b = t.p(1), c = t.p(2);
    const double det = mg::cross2(b - a, c - a);
    if (std::fabs(det) <= mg::kF64Eps) return false;
    const double wb = mg::cross2(p - a, c - a) / det;
    const double wc = mg::cross2(b - a, p - a) / det;
    return ((1.0 - wb) - wc) >= -kInsideTolerance && wb >= -kInsideTolerance && wc >= -kInsideTolerance;
}

double intersection_area(const Poly2& polygon, const PT& t) {
    const double o = mg::signum(mg::signed_image_area(t));
    Poly2 inside = polygon, next;
    for (int e = 0; e < 3; ++e) {
        split_polygon(inside, t.p(e), t.p((e + 1) % 3), o, next, nullptr);
        inside.swap(next);
        if (inside.empty()) return 0.0;
    }
    return poly_area(inside);
}

// unobserved_area (surface_merge_stitch.rs:203-251); false for None
bool unobserved_area(const PT& stitch, const std::vector<PT>& seams, double& out) {
    const double eps = std::fabs(mg::signed_image_area(stitch)) * 1.0e-12;
    std::vector<Poly2> remaining{Poly2{stitch.p(0), stitch.p(1), stitch.p(2)}};
    Poly2 inside, included, excluded;
    for (const PT& seam : seams) {
        const double o = mg::signum(mg::signed_image_area(seam));
        std::vector<Poly2> next;
        for (Poly2& polygon : remaining) {
            inside = std::move(polygon);
            std::vector<Poly2> outside;
            for (int e = 0; e < 3; ++e) {
                split_polygon(inside, seam.p(e), seam.p((e + 1) % 3), o, included, &excluded);
                if (poly_area(excluded) > eps) outside.push_back(excluded);
                inside.swap(included);
                if (inside.empty()) break;
            }
            if (poly_area(inside) > eps) {
                bool agrees = true;
                for (const V2& p : inside) {
                    double s, m;
                    if (!mg::inverse_depth(stitch, p, s) || !mg::inverse_depth(seam, p, m)) {
                        agrees = false;
                        break;
                    }
                    const double sd = 1.0 / s, md = 1.0 / m;
                    if (!(std::fabs(sd - md) <= kMaxRelativeDepthDisagreement * md)) {
                        agrees = false;
                        break;
                    }
                }
                if (!agrees) outside.push_back(inside);
            }
            for (auto& o2 : outside) next.push_back(std::move(o2));
            if (next.size() > kMaxUncoveredPieces) return false;
        }
        remaining = std::move(next);
        if (remaining.empty()) break;
    }
    double total = -0.0;
    for (const auto& p : remaining) total += poly_area(p);
    out = total;
    return true;
}

struct HalfEdge {
    uint32_t low, high, from, triangle;
    bool operator<(const HalfEdge& o) const {
        if (low != o.low) return low < o.low;
        if (high != o.high) return high < o.high;
        if (from != o.from) return from < o.from;
        return triangle < o.triangle;
    }
};

struct StitchInputs {
    const Inputs* in;
    const std::vector<uint8_t>* keep;
    const std::vector<int64_t>* patch_of;
    const std::vector<Removal>* removals;
    const Grid3* kept_grid;
    const std::vector<uint32_t>* all_kept;
    double tolerance, cell;
    double* stage_ms;  // [0] retained edges, [1] seams, [2] the greedy pass
};

std::vector<v3d_mesh_triangle> stitch_trimmed_seams(const StitchInputs& si, Tally& tally) {
    auto t0 = Clock::now();
    const Inputs& in = *si.in;
    const auto& tris = *in.triangles;
    const auto& removals = *si.removals;
    const auto& patch_of = *si.patch_of;
    const auto& fps = *in.footprints;
    const auto& geometry = *in.geometry;
    const auto& has_geometry = *in.has_geometry;
    std::vector<v3d_mesh_triangle> output;
    if (removals.empty() || in.n_points > UINT32_MAX || tris.size() > UINT32_MAX ||
        removals.size() > UINT32_MAX)
        return output;
    std::vector<HalfEdge> retained;
    retained.reserve(3 * tris.size());
    for (size_t i = 0; i < tris.size(); ++i) {
        if (!(*si.keep)[i]) continue;
        const uint32_t a = (uint32_t)tris[i].a, b = (uint32_t)tris[i].b, c = (uint32_t)tris[i].c;
        const uint32_t es[3][2] = {{a, b}, {b, c}, {c, a}};
        for (const auto& e : es)
            if (e[0] != e[1])
                retained.push_back({std::min(e[0], e[1]), std::max(e[0], e[1]), e[0], (uint32_t)i});
    }
    std::sort(retained.begin(), retained.end());
    std::vector<uint8_t> on_boundary(in.n_points, 0);
    std::vector<uint32_t> boundary;
    for (size_t s = 0; s < retained.size();) {
        size_t e = s;
        while (e < retained.size() && retained[e].low == retained[s].low &&
               retained[e].high == retained[s].high)
            ++e;
        if (e - s == 1) {
            on_boundary[retained[s].low] = 1;
            on_boundary[retained[s].high] = 1;
            boundary.push_back((uint32_t)s);
        }
        s = e;
    }
    struct Seam {
        uint32_t v[kMaxSeamVertices];
        uint8_t len;
        bool ok;
    };
    si.stage_ms[0] += ms_since(t0);
    t0 = Clock::now();
    std::vector<Seam> seams(removals.size());
    std::vector<std::pair<uint32_t, uint32_t>> seams_by_vertex;
    // each removal's seam is independent of the others: threads over removals,
    // the lookups' tallies folded after (max and sum are order-free)
    auto seam_of = [&](size_t slot, std::vector<uint32_t>& found, Tally& t) {
        const Removal& r = removals[slot];
        Seam& seam = seams[slot];
        seam.ok = false;
        seam.len = 0;
        if (r.footprint >= fps.size() || !has_geometry[r.triangle]) return;
        const Footprint& f = fps[r.footprint];
        PT projected;
        if (!f.project_candidate(geometry[r.triangle], projected)) return;
        const int64_t lower = patch_of[r.triangle];
        const v3d_mesh_triangle& removed = tris[r.triangle];
        // the stitchable vertices, ascending (a BTreeSet in the reference)
        uint64_t st[kMaxSeamVertices + 1];
        size_t n_st = 0;
        bool too_many = false;
        auto insert = [&](uint64_t v) {
            for (size_t i = 0; i < n_st; ++i)
                if (st[i] == v) return;
            if (n_st == kMaxSeamVertices) {
                too_many = true;
                return;
            }
            size_t j = n_st++;
            while (j > 0 && st[j - 1] > v) {
                st[j] = st[j - 1];
                --j;
            }
            st[j] = v;
        };
        auto has = [&](uint64_t v) {
            for (size_t i = 0; i < n_st; ++i)
                if (st[i] == v) return true;
            return false;
        };
        for (uint64_t v : {removed.a, removed.b, removed.c})
            if (on_boundary[v] && in.group(v) >= 0) insert(v);
        size_t used;
        const Limit q = f.lookup(projected, found, used);
        t.record(used, q);
        if (q != Limit::None) return;
        for (uint32_t kept : found) {
            if (too_many) break;
            if (!in.linked(r.triangle, f.comp[kept])) continue;
            for (uint32_t vertex : f.vert[kept]) {
                if (!on_boundary[vertex] || in.group(vertex) < 0 || in.group(vertex) == lower || has(vertex))
                    continue;
                double ix, iy, iz;
                if (mg::project(f.cam, in.position(vertex), ix, iy, iz) && contains(projected, V2{ix, iy}))
                    insert(vertex);
                if (too_many) break;
            }
        }
        // more than MAX_SEAM_VERTICES: no seam (the reference fails closed)
        if (too_many) return;
        seam.ok = true;
        for (size_t i = 0; i < n_st; ++i) seam.v[seam.len++] = (uint32_t)st[i];
    };
    {
        const size_t n_threads =
            std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), 16));
        const size_t chunk = (removals.size() + n_threads - 1) / n_threads;
        std::vector<Tally> tallies(n_threads);
        std::vector<std::thread> pool;
        for (size_t k = 0; k < n_threads; ++k)
            pool.emplace_back([&, k] {
                std::vector<uint32_t> found;
                const size_t lo = k * chunk, hi = std::min(removals.size(), lo + chunk);
                for (size_t slot = lo; slot < hi; ++slot) seam_of(slot, found, tallies[k]);
            });
        for (auto& th : pool) th.join();
        for (const Tally& t : tallies) {
            tally.max_postings = std::max(tally.max_postings, t.max_postings);
            tally.bound_hits += t.bound_hits;
        }
    }
    for (size_t slot = 0; slot < removals.size(); ++slot)
        for (uint8_t i = 0; i < seams[slot].len; ++i)
            seams_by_vertex.push_back({seams[slot].v[i], (uint32_t)slot});
    std::sort(seams_by_vertex.begin(), seams_by_vertex.end());
    si.stage_ms[1] += ms_since(t0);
    t0 = Clock::now();
    auto seams_of = [&](uint64_t vertex, std::vector<uint32_t>& out) {
        auto it = std::partition_point(seams_by_vertex.begin(), seams_by_vertex.end(),
                                       [&](const auto& e) { return e.first < vertex; });
        size_t taken = 0;
        for (; it != seams_by_vertex.end() && it->first == vertex && taken < kMaxSeamsPerVertex;
             ++it, ++taken)
            out.push_back(it->second);
    };
    std::unordered_map<uint64_t, std::pair<uint32_t, uint32_t>> stitched;  // edge -> (count, from)
    auto usage = [&](uint32_t a, uint32_t b, uint32_t& count, uint32_t& from) -> bool {
        const uint32_t lo = std::min(a, b), hi = std::max(a, b);
        auto it = stitched.find(((uint64_t)lo << 32) | hi);
        if (it != stitched.end()) {
            count = it->second.first;
            from = it->second.second;
            return true;
        }
        auto first = std::partition_point(retained.begin(), retained.end(), [&](const HalfEdge& e) {
            return e.low < lo || (e.low == lo && e.high < hi);
        });
        auto last = first;
        while (last != retained.end() && last->low == lo && last->high == hi) ++last;
        if (first == last) return false;
        count = (uint32_t)(last - first);
        from = first->from;
        return true;
    };
    auto length = [&](uint64_t a, uint64_t b) { return mg::norm3(in.position(a) - in.position(b)); };
    Grid3 stitch_grid(si.cell);
    // A stitch check (surface_merge_stitch.rs:253-297) in the reference's order
    // reads edge usage, then only inputs of this pass (geometry, the seams'
    // cover, the kept triangles), then the stitches made so far.  The part that
    // reads only inputs is evaluated for every boundary edge concurrently (in
    // candidate order, up to the first candidate it passes); the ordered pass
    // then replays each check: usage, the recorded outcome and lookup tally, and
    // for a recorded pass the lookup among earlier stitches, whose overlap adds
    // onto the recorded sum in the same order.  Stitches only add usage and
    // overlap, so the outcome and the tallies are the reference's.
    struct Static {
        uint8_t stage = 0;  // 0 failed before the kept-triangle lookup, 1 failed at or after it, 2 passed
        Limit q = Limit::None;
        size_t used = 0;
        uint32_t footprint = 0;
        double area = 0.0, overlap = 0.0;
        double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
        Poly2 polygon;
    };
    struct Scratch {
        std::vector<uint32_t> cover_v, nearby;
    };
    auto check_static = [&](const uint64_t corners[3], uint32_t slot, uint32_t adjacent, Scratch& sc,
                            Static& st) {
        const uint64_t a = corners[0], b = corners[1], c = corners[2];
        const V3 cs[3] = {in.position(a), in.position(b), in.position(c)};
        Geometry surface;
        if (!make_geometry(cs, surface)) return;
        const Removal& r = removals[slot];
        const Footprint& f = fps[r.footprint];
        const int64_t lower = patch_of[r.triangle];
        PT projected;
        if (!mg::project_triangle(f.cam, surface.c, projected)) return;
        double area = mg::signed_image_area(projected);
        if (!has_geometry[adjacent]) return;
        PT adj;
        if (!mg::project_triangle(f.cam, geometry[adjacent].c, adj)) return;
        const double adjacent_area = mg::signed_image_area(adj);
        if (std::fabs(area) <= mg::kF64Eps * mg::kF64Eps ||
            mg::signum(adjacent_area) != mg::signum(area))
            return;
        area = std::fabs(area);
        for (int i = 0; i < 3; ++i)
            if (in.group(corners[i]) != lower) projected.z[i] *= r.scale;
        auto& cover_v = sc.cover_v;
        cover_v.clear();
        for (int i = 0; i < 3; ++i) seams_of(corners[i], cover_v);
        std::sort(cover_v.begin(), cover_v.end());
        cover_v.erase(std::unique(cover_v.begin(), cover_v.end()), cover_v.end());
        std::vector<PT> cover;
        for (uint32_t s2 : cover_v) {
            if (!seams[s2].ok || removals[s2].footprint != r.footprint || patch_of[removals[s2].triangle] != lower)
                continue;
            const Removal& rs = removals[s2];
            if (rs.footprint >= fps.size() || !has_geometry[rs.triangle]) continue;
            PT pp;
            if (fps[rs.footprint].project_candidate(geometry[rs.triangle], pp)) cover.push_back(pp);
        }
        double unobserved;
        if (!unobserved_area(projected, cover, unobserved)) return;
        if (unobserved > kMaxUnobservedStitchShare * area) return;
        st.polygon = Poly2{projected.p(0), projected.p(1), projected.p(2)};
        surface.aabb(si.tolerance, st.lo, st.hi);
        auto& nearby = sc.nearby;
        nearby.clear();
        Budget budget;
        Limit q = si.kept_grid->query(st.lo, st.hi, kMaxGridCells, budget, nearby);
        if (q == Limit::Cells) q = budget.take(si.all_kept->data(), si.all_kept->size(), nearby);
        st.stage = 1;
        st.used = budget.used;
        st.q = q;
        if (q != Limit::None) return;
        std::sort(nearby.begin(), nearby.end());
        double overlap = 0.0;
        for (uint32_t other : nearby) {
            if (!has_geometry[other]) continue;
            PT pp;
            if (!mg::project_triangle(f.cam, geometry[other].c, pp)) return;
            overlap += intersection_area(st.polygon, pp);
        }
        st.stage = 2;
        st.footprint = (uint32_t)r.footprint;
        st.area = area;
        st.overlap = overlap;
    };
    struct Cand {
        double perimeter;
        std::array<uint64_t, 4> c;
    };
    // the boundary edges' candidates in the reference's order, and the static
    // checks up to the first pass, per thread over contiguous edge ranges
    struct Part {
        std::vector<uint32_t> start;  // per edge of the range: first candidate (+1 end entry)
        std::vector<uint8_t> stitchable;
        std::vector<Cand> cands;
        std::vector<Static> checked;  // per candidate; stage 255 = not evaluated
    };
    const size_t n_edges = boundary.size();
    const size_t n_threads = std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), 16));
    const size_t chunk = (n_edges + n_threads - 1) / n_threads;
    std::vector<Part> parts(n_threads);
    auto build = [&](size_t k) {
        Part& part = parts[k];
        const size_t lo = std::min(n_edges, k * chunk), hi = std::min(n_edges, lo + chunk);
        Scratch sc;
        std::vector<uint32_t> slots;
        std::vector<Cand> candidates;
        part.start.reserve(hi - lo + 1);
        for (size_t ei = lo; ei < hi; ++ei) {
            part.start.push_back((uint32_t)part.cands.size());
            const HalfEdge edge = retained[boundary[ei]];
            const uint64_t from = edge.from;
            const uint64_t to = edge.from == edge.low ? edge.high : edge.low;
            if (in.group(from) != in.group(to)) {
                part.stitchable.push_back(0);
                continue;
            }
            part.stitchable.push_back(1);
            slots.clear();
            seams_of(from, slots);
            seams_of(to, slots);
            std::sort(slots.begin(), slots.end());
            slots.erase(std::unique(slots.begin(), slots.end()), slots.end());
            std::set<uint64_t> seen;
            candidates.clear();
            for (uint32_t slot : slots) {
                if (!seams[slot].ok) continue;
                const int64_t lower = patch_of[removals[slot].triangle];
                const bool edge_is_lower = in.group(from) == lower;
                for (uint8_t i = 0; i < seams[slot].len; ++i) {
                    const uint64_t vertex = seams[slot].v[i];
                    if (vertex == from || vertex == to || (in.group(vertex) == lower) == edge_is_lower)
                        continue;
                    if (!seen.insert(vertex).second) continue;
                    const double perimeter = (length(from, to) + length(to, vertex)) + length(vertex, from);
                    candidates.push_back({perimeter, {to, from, vertex, slot}});
                }
            }
            std::stable_sort(candidates.begin(), candidates.end(), [](const Cand& l, const Cand& r) {
                if (total_less(l.perimeter, r.perimeter)) return true;
                if (total_less(r.perimeter, l.perimeter)) return false;
                return l.c < r.c;
            });
            bool passed = false;
            for (const Cand& cd : candidates) {
                part.cands.push_back(cd);
                part.checked.emplace_back();
                Static& st = part.checked.back();
                if (passed) {
                    st.stage = 255;
                    continue;
                }
                const uint64_t corners[3] = {cd.c[0], cd.c[1], cd.c[2]};
                check_static(corners, (uint32_t)cd.c[3], edge.triangle, sc, st);
                passed = st.stage == 2;
            }
        }
        part.start.push_back((uint32_t)part.cands.size());
    };
    {
        std::vector<std::thread> pool;
        for (size_t k = 1; k < n_threads; ++k) pool.emplace_back(build, k);
        build(0);
        for (auto& th : pool) th.join();
    }
    Scratch sc;
    std::vector<uint32_t> nearby;
    bool full = false;
    for (size_t k = 0; k < n_threads && !full; ++k) {
        Part& part = parts[k];
        const size_t lo = std::min(n_edges, k * chunk), hi = std::min(n_edges, lo + chunk);
        for (size_t ei = lo; ei < hi; ++ei) {
            if (output.size() >= removals.size()) {
                full = true;
                break;
            }
            const size_t e = ei - lo;
            if (!part.stitchable[e]) continue;
            const uint32_t adjacent = retained[boundary[ei]].triangle;
            for (uint32_t j = part.start[e]; j < part.start[e + 1]; ++j) {
                const Cand& cd = part.cands[j];
                const uint64_t corners[3] = {cd.c[0], cd.c[1], cd.c[2]};
                const uint64_t es[3][2] = {{corners[0], corners[1]}, {corners[1], corners[2]},
                                           {corners[2], corners[0]}};
                bool ok = true;
                for (const auto& ed : es) {
                    uint32_t count, from_;
                    if (usage((uint32_t)ed[0], (uint32_t)ed[1], count, from_) &&
                        !(count < 2 && from_ != (uint32_t)ed[0])) {
                        ok = false;
                        break;
                    }
                }
                if (!ok) continue;
                Static& st = part.checked[j];
                if (st.stage == 255) {
                    st = Static{};
                    check_static(corners, (uint32_t)cd.c[3], adjacent, sc, st);
                }
                if (st.stage == 0) continue;
                tally.record(st.used, st.q);
                if (st.stage == 1) continue;
                nearby.clear();
                Budget budget2;
                const Limit q = stitch_grid.query(st.lo, st.hi, kMaxGridCells, budget2, nearby);
                tally.record(budget2.used, q);
                if (q != Limit::None) continue;
                std::sort(nearby.begin(), nearby.end());
                const Footprint& f = fps[st.footprint];
                double overlap = st.overlap;
                for (uint32_t other : nearby) {
                    const v3d_mesh_triangle& o = output[other];
                    const V3 oc[3] = {in.position(o.a), in.position(o.b), in.position(o.c)};
                    PT pp;
                    if (!mg::project_triangle(f.cam, oc, pp)) {
                        ok = false;
                        break;
                    }
                    overlap += intersection_area(st.polygon, pp);
                }
                if (!ok || !(overlap <= kMaxStitchOverlapShare * st.area)) continue;
                for (const auto& ed : es) {
                    uint32_t count, from_;
                    const uint32_t f0 = (uint32_t)ed[0], t1 = (uint32_t)ed[1];
                    const bool had = usage(f0, t1, count, from_);
                    const uint32_t lo32 = std::min(f0, t1), hi32 = std::max(f0, t1);
                    stitched[((uint64_t)lo32 << 32) | hi32] = had ? std::make_pair(count + 1, from_)
                                                                  : std::make_pair(1u, f0);
                }
                stitch_grid.insert((uint32_t)output.size(), st.lo, st.hi);
                output.push_back(v3d_mesh_triangle{corners[0], corners[1], corners[2],
                                                   std::fmin(tris[adjacent].confidence,
                                                             tris[removals[cd.c[3]].triangle].confidence)});
                break;
            }
        }
    }
    si.stage_ms[2] += ms_since(t0);
    return output;
}

}  // namespace
}  // namespace merge
}  // namespace v3d

namespace v3d {
namespace merge {
namespace {

// ReconstructionControl (reconstruction/control.rs:5-27)
struct Control {
    v3d_cancel_fn fn;
    void* user;
    bool canceled = false;
    bool is_canceled() {
        canceled = canceled || (fn && fn(user) != 0);
        return canceled;
    }
};

struct Stats {
    v3d_merge_stats s{};
    std::vector<v3d_fusion_pair> uncalibrated;
    std::vector<uint64_t> retained_by_group;
    std::vector<v3d_triangle_source> sources;
};

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t cap = 0;
    cudaError_t ensure(size_t n, cudaStream_t st) {
        if (n <= cap) return cudaSuccess;
        if (p) cudaFreeAsync(p, st);
        p = nullptr;
        cap = std::max(n, cap * 2);
        return cudaMallocAsync(&p, sizeof(T) * std::max<size_t>(cap, 1), st);
    }
    void release(cudaStream_t st) {
        if (p) cudaFreeAsync(p, st);
        p = nullptr;
        cap = 0;
    }
};

// The device half: the footprint store and the per-patch job launches.
struct Device {
    v3d_context* ctx;
    cudaStream_t st;
    DevBuf<double> corners, fp_tri, ratios;
    DevBuf<uint32_t> fp_comp, fp_vert, items, anchors, omitted;
    DevBuf<Cand> cands;
    DevBuf<OwnerRef> owner_refs;
    DevBuf<PairOut> pair_outs;
    DevBuf<CandOut> cand_outs;
    size_t n_omitted = 0;
    DevBuf<mg::GridBucket> buckets;
    DevBuf<DevFootprint> fps;
    DevBuf<int32_t> cluster;
    DevBuf<Job> jobs;
    DevBuf<JobOut> outs;
    size_t n_tri = 0, n_buckets = 0, n_items = 0, n_fps = 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    float kernel_ms = 0.f;
    uint64_t launches = 0;
    double stage_ms[12] = {};

    ~Device() {
        corners.release(st);
        fp_tri.release(st);
        ratios.release(st);
        fp_comp.release(st);
        fp_vert.release(st);
        items.release(st);
        anchors.release(st);
        omitted.release(st);
        cands.release(st);
        owner_refs.release(st);
        pair_outs.release(st);
        cand_outs.release(st);
        buckets.release(st);
        fps.release(st);
        cluster.release(st);
        jobs.release(st);
        outs.release(st);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
    DevStore store() const {
        return DevStore{corners.p, fps.p, fp_tri.p, fp_comp.p, fp_vert.p, buckets.p, items.p, cluster.p,
                        omitted.p};
    }
    cudaError_t add_footprint(const Footprint& f, size_t capacity_tri, size_t n_groups) {
        cudaError_t e;
        if ((e = fp_tri.ensure(capacity_tri * 9, st)) || (e = fp_comp.ensure(capacity_tri, st)) ||
            (e = fp_vert.ensure(capacity_tri * 3, st)) || (e = items.ensure(capacity_tri, st)) ||
            (e = buckets.ensure(capacity_tri, st)) || (e = fps.ensure(n_groups, st)) ||
            (e = omitted.ensure(capacity_tri, st)))
            return e;
        DevFootprint d{};
        d.cam = f.cam;
        d.cell = f.cell;
        d.levels = f.levels;
        d.tri_off = (uint32_t)n_tri;
        d.n_tri = (uint32_t)f.tri.size();
        d.bucket_off = (uint32_t)n_buckets;
        d.n_buckets = (uint32_t)f.buckets.size();
        d.item_off = (uint32_t)n_items;
        d.n_bucketed = f.n_bucketed;
        d.n_unindexed = (uint32_t)(f.items.size() - f.n_bucketed);
        d.omit_off = (uint32_t)n_omitted;
        d.n_omit = (uint32_t)f.omitted.size();
        std::vector<uint32_t> omit_comp(f.omitted.size());
        for (size_t i = 0; i < f.omitted.size(); ++i) omit_comp[i] = f.omitted[i].first;
        static_assert(sizeof(PT) == 9 * sizeof(double), "PT is nine doubles");
        const size_t k = f.tri.size();
        if ((e = cudaMemcpyAsync(fp_tri.p + n_tri * 9, f.tri.data(), sizeof(PT) * k,
                                 cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(fp_comp.p + n_tri, f.comp.data(), 4 * k, cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(fp_vert.p + n_tri * 3, f.vert.data(), 12 * k, cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(buckets.p + n_buckets, f.buckets.data(),
                                 sizeof(mg::GridBucket) * f.buckets.size(), cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(items.p + n_items, f.items.data(), 4 * f.items.size(),
                                 cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(omitted.p + n_omitted, omit_comp.data(), 4 * omit_comp.size(),
                                 cudaMemcpyHostToDevice, st)) ||
            (e = cudaMemcpyAsync(fps.p + n_fps, &d, sizeof d, cudaMemcpyHostToDevice, st)))
            return e;
        // the host copies must outlive the transfers: wait here (one footprint a patch)
        if ((e = cudaStreamSynchronize(st))) return e;
        n_tri += k;
        n_buckets += f.buckets.size();
        n_items += f.items.size();
        n_omitted += f.omitted.size();
        n_fps += 1;
        return cudaSuccess;
    }
    // runs `launch` over the jobs, timed, and brings the outputs back
    template <class Launch>
    cudaError_t run(const std::vector<Job>& host_jobs, std::vector<JobOut>& host_out, Launch launch) {
        host_out.resize(host_jobs.size());
        if (host_jobs.empty()) return cudaSuccess;
        cudaError_t e;
        if ((e = jobs.ensure(host_jobs.size(), st)) || (e = outs.ensure(host_jobs.size(), st))) return e;
        if ((e = cudaMemcpyAsync(jobs.p, host_jobs.data(), sizeof(Job) * host_jobs.size(),
                                 cudaMemcpyHostToDevice, st)))
            return e;
        cudaEventRecord(e0, st);
        const uint32_t n = (uint32_t)host_jobs.size();
        launch(n);
        ++launches;
        ++::v3d::g_kernel_launches;
        cudaEventRecord(e1, st);
        if ((e = cudaGetLastError())) return e;
        if ((e = cudaMemcpyAsync(host_out.data(), outs.p, sizeof(JobOut) * n, cudaMemcpyDeviceToHost, st)))
            return e;
        if ((e = cudaStreamSynchronize(st))) return e;
        float ms = 0.f;
        if (cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) kernel_ms += ms;
        return cudaSuccess;
    }
};

}  // namespace
}  // namespace merge
}  // namespace v3d

namespace v3d {
namespace merge {
namespace {

// fn(lo, hi) over [0, n) in contiguous ranges on up to 16 host threads (the
// callers write disjoint elements, so the result does not depend on the split)
template <class F>
void parallel_ranges(size_t n, F&& fn) {
    const size_t n_threads = std::max<size_t>(
        1, std::min<size_t>({(size_t)std::thread::hardware_concurrency(), 16, (n + 65535) / 65536}));
    const size_t chunk = (n + n_threads - 1) / n_threads;
    std::vector<std::thread> pool;
    for (size_t k = 1; k < n_threads; ++k)
        pool.emplace_back([&, k] { fn(std::min(n, k * chunk), std::min(n, (k + 1) * chunk)); });
    fn(0, std::min(n, chunk));
    for (auto& th : pool) th.join();
}

size_t uf_find(std::vector<size_t>& parent, size_t i) {
    size_t r = i;
    while (parent[r] != r) r = parent[r];
    while (parent[i] != r) {
        const size_t n = parent[i];
        parent[i] = r;
        i = n;
    }
    return r;
}

// merge_impl (surface_merge.rs:355-1078) with clip_overlaps set.  Returns a
// v3d_status; *completed false when canceled (the reference's
// Default::default()), with `tris` possibly re-indexed already.
int32_t merge_impl(v3d_context* ctx, Device& dev, const v3d_point* points, uint64_t n_points,
                   std::vector<v3d_mesh_triangle>& tris, const int64_t* membership,
                   const v3d_fusion_pair* pairs, uint64_t n_pairs, const v3d_reference_camera* cams,
                   uint64_t n_cams, const int32_t* origins, uint64_t n_origins, Control& control,
                   Stats& stats, std::vector<Derived>& derived_out, bool& completed) {
    completed = false;
    stats = Stats();
    derived_out.clear();
    auto t_stage = Clock::now();
    auto group = [&](uint64_t v) -> int64_t { return v < n_points && membership[v] >= 0 ? membership[v] : -1; };
    const size_t nt = tris.size();
    for (const auto& t : tris)
        if (t.a >= n_points || t.b >= n_points || t.c >= n_points) {
            completed = true;
            return V3D_OK;
        }
    // original components
    std::vector<size_t> parent(n_points);
    for (size_t i = 0; i < n_points; ++i) parent[i] = i;
    for (const auto& t : tris) {
        if (control.is_canceled()) return V3D_OK;
        const int64_t g = group(t.a);
        if (g < 0 || g != group(t.b) || g != group(t.c)) continue;
        const size_t rep = uf_find(parent, t.a);
        for (uint64_t v : {t.b, t.c}) {
            const size_t root = uf_find(parent, v);
            parent[root] = rep;
        }
    }
    std::vector<uint32_t> comp_of_vertex(n_points);
    for (size_t v = 0; v < n_points; ++v) comp_of_vertex[v] = (uint32_t)uf_find(parent, v);
    std::vector<uint32_t> comp_of_tri(nt);
    for (size_t i = 0; i < nt; ++i) comp_of_tri[i] = comp_of_vertex[tris[i].a];
    // patches and priority
    std::vector<int64_t> patch_of(nt);
    int64_t max_group = -1;
    for (size_t v = 0; v < n_points; ++v) max_group = std::max(max_group, group(v));
    const size_t n_groups = (size_t)(max_group + 1);
    std::vector<uint64_t> counts(n_groups, 0);
    for (size_t i = 0; i < nt; ++i) {
        patch_of[i] = group(tris[i].a);
        if (patch_of[i] >= 0) counts[(size_t)patch_of[i]] += 1;
    }
    std::vector<size_t> order;
    for (size_t g = 0; g < n_groups; ++g)
        if (counts[g]) order.push_back(g);
    std::sort(order.begin(), order.end(), [&](size_t a, size_t b) {
        return counts[a] != counts[b] ? counts[a] > counts[b] : a < b;
    });
    std::vector<size_t> rank(n_groups, SIZE_MAX);
    for (size_t r = 0; r < order.size(); ++r) rank[order[r]] = r;
    auto rank_of = [&](uint64_t v) -> size_t {
        const int64_t g = group(v);
        return g < 0 ? SIZE_MAX : rank[(size_t)g];
    };
    // point_origins.get(v): absent beyond the slice
    auto origin_get = [&](uint64_t v) -> int64_t { return v < n_origins ? origins[v] : INT64_MIN; };
    std::vector<uint64_t> canonical(n_points);
    for (size_t i = 0; i < n_points; ++i) canonical[i] = i;
    std::vector<uint8_t> claimed(n_points, 0);
    std::vector<std::pair<uint64_t, uint64_t>> accepted;
    uint64_t fused_pairs = 0, provenance_separated = 0;
    for (uint64_t k = 0; k < n_pairs; ++k) {
        if (control.is_canceled()) return V3D_OK;
        const uint64_t first = pairs[k].first, second = pairs[k].second;
        if (first >= n_points || second >= n_points || group(first) < 0 ||
            group(first) == group(second) || claimed[first] || claimed[second])
            continue;
        claimed[first] = claimed[second] = 1;
        accepted.push_back({first, second});
        if (origin_get(first) != origin_get(second)) {
            provenance_separated += 1;
            continue;
        }
        const auto rf = std::make_pair(rank_of(first), first), rs = std::make_pair(rank_of(second), second);
        if (rf <= rs) canonical[second] = first;
        else canonical[first] = second;
        fused_pairs += 1;
    }
    std::set<std::pair<uint32_t, uint32_t>> linked_components;
    std::set<std::pair<size_t, size_t>> linked_patches;
    std::map<std::pair<size_t, size_t>, std::vector<uint32_t>> scale_anchors;
    for (const auto& pr : accepted) {
        const int64_t ga = group(pr.first), gb = group(pr.second);
        if (ga >= 0 && gb >= 0 && ga != gb) {
            const uint32_t a = comp_of_vertex[pr.first], b = comp_of_vertex[pr.second];
            linked_components.insert({std::min(a, b), std::max(a, b)});
            linked_patches.insert({(size_t)std::min(ga, gb), (size_t)std::max(ga, gb)});
        }
        if (ga >= 0 && gb >= 0) {
            auto& s = scale_anchors[{(size_t)std::min(ga, gb), (size_t)std::max(ga, gb)}];
            s.push_back((uint32_t)pr.first);
            s.push_back((uint32_t)pr.second);
        }
    }
    for (auto& kv : scale_anchors) {
        std::sort(kv.second.begin(), kv.second.end());
        kv.second.erase(std::unique(kv.second.begin(), kv.second.end()), kv.second.end());
    }
    std::vector<std::pair<uint64_t, std::array<uint64_t, 3>>> reindexed;
    for (size_t i = 0; i < nt; ++i) {
        if (control.is_canceled()) return V3D_OK;
        v3d_mesh_triangle& t = tris[i];
        const std::array<uint64_t, 3> orig{t.a, t.b, t.c};
        const std::array<uint64_t, 3> m{canonical[t.a], canonical[t.b], canonical[t.c]};
        if (m != orig && m[0] != m[1] && m[1] != m[2] && m[0] != m[2]) {
            t.a = m[0];
            t.b = m[1];
            t.c = m[2];
            reindexed.push_back({i, orig});
        }
    }
    // geometry
    auto position = [&](uint64_t v) { return V3{(double)points[v].x, (double)points[v].y, (double)points[v].z}; };
    std::vector<Geometry> geometry(nt);
    std::vector<uint8_t> has_geometry(nt, 0);
    parallel_ranges(nt, [&](size_t lo, size_t hi) {
        for (size_t i = lo; i < hi; ++i) {
            const V3 c[3] = {position(tris[i].a), position(tris[i].b), position(tris[i].c)};
            has_geometry[i] = make_geometry(c, geometry[i]) ? 1 : 0;
        }
    });
    double median_edge;
    {
        std::vector<double> edges;
        edges.reserve(3 * nt);
        for (size_t i = 0; i < nt; ++i)
            if (has_geometry[i]) edges.insert(edges.end(), geometry[i].e, geometry[i].e + 3);
        if (edges.empty()) {
            completed = true;
            return V3D_OK;
        }
        const size_t mid = edges.size() / 2;
        std::nth_element(edges.begin(), edges.begin() + mid, edges.end(), total_less);
        median_edge = edges[mid];
    }
    const double tolerance = median_edge * kMaxOverlapDistanceFraction;
    const double cell = std::fmax(median_edge * 2.0, mg::kGeomEps);
    std::vector<uint8_t> keep(nt, 1);
    Grid3 kept_grid(cell);
    std::vector<uint32_t> all_kept;
    uint64_t removed_dup = 0, remaining_overlap = 0, budget_exhausted = 0, trimmed = 0;
    Tally tally;
    double trimmed_area = 0.0;
    std::vector<Removal> removals;
    std::vector<ClipJob> clip_jobs;
    double total_area = -0.0;
    for (size_t i = 0; i < nt; ++i)
        if (has_geometry[i]) total_area += geometry[i].area();
    // linked clusters of original components (only their equality matters)
    std::vector<int32_t> cluster(n_points, -1);
    {
        std::map<uint32_t, size_t> dense;
        for (const auto& lc : linked_components) {
            dense.emplace(lc.first, dense.size());
            dense.emplace(lc.second, dense.size());
        }
        std::vector<size_t> up(dense.size());
        for (size_t i = 0; i < up.size(); ++i) up[i] = i;
        for (const auto& lc : linked_components) {
            const size_t a = uf_find(up, dense[lc.first]), b = uf_find(up, dense[lc.second]);
            up[a] = b;
        }
        for (const auto& kv : dense) cluster[kv.first] = (int32_t)uf_find(up, kv.second);
    }
    auto components_linked = [&](uint32_t t, uint32_t comp) {
        const uint32_t own = comp_of_tri[t];
        if (own == comp) return false;
        const int32_t c = cluster[own];
        return c >= 0 && cluster[comp] == c;
    };
    std::vector<Footprint> footprints;
    Inputs in{points, n_points, membership, origins, n_origins, &tris, &has_geometry, &geometry,
              &footprints, &comp_of_tri, &cluster, &reindexed};

    // device inputs: every triangle's world corners and the clusters
    {
        std::vector<double> corners(nt * 9, 0.0);
        parallel_ranges(nt, [&](size_t lo, size_t hi) {
            for (size_t i = lo; i < hi; ++i)
                if (has_geometry[i])
                    for (int k = 0; k < 3; ++k) {
                        corners[i * 9 + 3 * k] = geometry[i].c[k].x;
                        corners[i * 9 + 3 * k + 1] = geometry[i].c[k].y;
                        corners[i * 9 + 3 * k + 2] = geometry[i].c[k].z;
                    }
        });
        V3D_CTX_CK(dev.corners.ensure(nt * 9, dev.st));
        V3D_CTX_CK(dev.cluster.ensure(n_points, dev.st));
        V3D_CTX_CK(cudaMemcpyAsync(dev.corners.p, corners.data(), 8 * corners.size(),
                                   cudaMemcpyHostToDevice, dev.st));
        V3D_CTX_CK(cudaMemcpyAsync(dev.cluster.p, cluster.data(), 4 * n_points, cudaMemcpyHostToDevice,
                                   dev.st));
        V3D_CTX_CK(cudaStreamSynchronize(dev.st));
    }
    // members of each patch, ascending
    std::vector<std::vector<uint32_t>> members_of(n_groups);
    for (size_t i = 0; i < nt; ++i)
        if (patch_of[i] >= 0) members_of[(size_t)patch_of[i]].push_back((uint32_t)i);
    std::vector<uint8_t> has_footprint(n_groups, 0);
    // vertex -> triangles (re-indexed corners), to find each patch's anchored triangles
    std::vector<uint32_t> inc_off(n_points + 1, 0), inc_tri;
    {
        for (size_t i = 0; i < nt; ++i)
            for (uint64_t v : {tris[i].a, tris[i].b, tris[i].c}) inc_off[v + 1] += 1;
        for (size_t v = 0; v < n_points; ++v) inc_off[v + 1] += inc_off[v];
        inc_tri.resize(inc_off[n_points]);
        std::vector<uint32_t> fill(inc_off.begin(), inc_off.end() - 1);
        for (size_t i = 0; i < nt; ++i)
            for (uint64_t v : {tris[i].a, tris[i].b, tris[i].c}) inc_tri[fill[v]++] = (uint32_t)i;
    }
    std::vector<uint32_t> anchored;
    std::vector<Job> jobs;
    std::vector<JobOut> outs;
    std::vector<uint32_t> nearby;
    std::vector<double> ratio_buf;
    dev.stage_ms[0] += ms_since(t_stage);

    for (size_t pr = 0; pr < order.size(); ++pr) {
        const size_t patch = order[pr];
        if (control.is_canceled()) return V3D_OK;
        const std::vector<uint32_t>& members = members_of[patch];
        if (pr > 0) {
            t_stage = Clock::now();
            struct Owner {
                uint32_t slot;
                double scale;
            };
            std::vector<Owner> owners;
            std::vector<uint32_t> owner_slots;
            for (uint32_t slot = 0; slot < footprints.size(); ++slot) {
                const size_t fp = footprints[slot].patch;
                if (linked_patches.count({std::min(fp, patch), std::max(fp, patch)})) owner_slots.push_back(slot);
            }
            // relative depth scale of each owner pair: median of the anchored samples
            const auto t_scale = Clock::now();
            if (!owner_slots.empty()) {
                std::vector<uint32_t> anchors_all;
                jobs.clear();
                std::vector<size_t> first_job(owner_slots.size() + 1, 0);
                for (size_t k = 0; k < owner_slots.size(); ++k) {
                    const size_t fp = footprints[owner_slots[k]].patch;
                    auto it = scale_anchors.find({std::min(fp, patch), std::max(fp, patch)});
                    const uint32_t a_off = (uint32_t)anchors_all.size();
                    if (it != scale_anchors.end())
                        anchors_all.insert(anchors_all.end(), it->second.begin(), it->second.end());
                    const uint32_t n_a = (uint32_t)anchors_all.size() - a_off;
                    first_job[k] = jobs.size();
                    // this patch's triangles at an anchor vertex, ascending (the members the
                    // reference's scan over the patch finds anchored)
                    anchored.clear();
                    for (uint32_t q = a_off; q < a_off + n_a; ++q) {
                        const uint32_t v = anchors_all[q];
                        for (uint32_t e = inc_off[v]; e < inc_off[v + 1]; ++e) {
                            const uint32_t t = inc_tri[e];
                            if ((size_t)patch_of[t] == patch && has_geometry[t]) anchored.push_back(t);
                        }
                    }
                    std::sort(anchored.begin(), anchored.end());
                    anchored.erase(std::unique(anchored.begin(), anchored.end()), anchored.end());
                    for (uint32_t m : anchored)
                        jobs.push_back(Job{m, owner_slots[k], comp_of_tri[m], a_off, n_a, 0, 0, 0.0});
                }
                first_job[owner_slots.size()] = jobs.size();
                std::vector<double> scales(owner_slots.size(), 1.0);
                std::vector<uint32_t> totals(owner_slots.size(), 0);
                if (!jobs.empty()) {
                    V3D_CTX_CK(dev.anchors.ensure(anchors_all.size(), dev.st));
                    V3D_CTX_CK(cudaMemcpyAsync(dev.anchors.p, anchors_all.data(), 4 * anchors_all.size(),
                                               cudaMemcpyHostToDevice, dev.st));
                    const DevStore s = dev.store();
                    const uint32_t* anchors_d = dev.anchors.p;
                    V3D_CTX_CK(dev.run(jobs, outs, [&](uint32_t n) {
                        k_ratios<false><<<(n + kLookupWarps - 1) / kLookupWarps, 32 * kLookupWarps, 0, dev.st>>>(s, dev.jobs.p, n, anchors_d,
                                                                             dev.outs.p, nullptr);
                    }));
                    // members are taken in order until 4096 samples (surface_merge.rs:630-647)
                    std::vector<Job> writes;
                    for (size_t k = 0; k < owner_slots.size(); ++k) {
                        uint32_t prefix = 0;
                        for (size_t j = first_job[k]; j < first_job[k + 1]; ++j) {
                            if (prefix >= kMaxScaleSamples) break;
                            const JobOut& o = outs[j];
                            if (o.status == kUnprojectable) continue;
                            tally.record(o.used, o.status == kPostingBound ? Limit::Postings
                                                 : o.status == kTooManyCells ? Limit::Cells
                                                                             : Limit::None);
                            if (o.status != kJudged || o.count == 0) continue;
                            Job w = jobs[j];
                            w.out_off = (uint32_t)(k * kMaxScaleSamples) + prefix;
                            w.out_limit = (uint32_t)(k * kMaxScaleSamples) + kMaxScaleSamples;
                            writes.push_back(w);
                            prefix = std::min<uint32_t>(prefix + o.count, kMaxScaleSamples);
                        }
                        totals[k] = prefix;
                    }
                    if (!writes.empty()) {
                        V3D_CTX_CK(dev.ratios.ensure(owner_slots.size() * kMaxScaleSamples, dev.st));
                        std::vector<JobOut> unused;
                        double* ratios_d = dev.ratios.p;
                        V3D_CTX_CK(dev.run(writes, unused, [&](uint32_t n) {
                            k_ratios<true><<<(n + kLookupWarps - 1) / kLookupWarps, 32 * kLookupWarps, 0, dev.st>>>(s, dev.jobs.p, n, anchors_d,
                                                                                dev.outs.p, ratios_d);
                        }));
                        ratio_buf.resize(owner_slots.size() * kMaxScaleSamples);
                        V3D_CTX_CK(cudaMemcpyAsync(ratio_buf.data(), ratios_d, 8 * ratio_buf.size(),
                                                   cudaMemcpyDeviceToHost, dev.st));
                        V3D_CTX_CK(cudaStreamSynchronize(dev.st));
                    }
                }
                for (size_t k = 0; k < owner_slots.size(); ++k) {
                    if (totals[k] >= kMinScaleSamples) {
                        double* r = ratio_buf.data() + k * kMaxScaleSamples;
                        const size_t mid = totals[k] / 2;
                        std::nth_element(r, r + mid, r + totals[k], total_less);
                        scales[k] = r[mid];
                    } else {
                        stats.uncalibrated.push_back({footprints[owner_slots[k]].patch, patch});
                    }
                    owners.push_back({owner_slots[k], scales[k]});
                }
            }
            dev.stage_ms[8] += ms_since(t_scale);
            bool imageless_owner = false;
            for (size_t r = 0; r < pr && !imageless_owner; ++r) {
                const size_t o = order[r];
                if (linked_patches.count({std::min(o, patch), std::max(o, patch)}) && !has_footprint[o])
                    imageless_owner = true;
            }
            // every candidate against every linked owner on the device, and each
            // candidate's fold over its owners
            std::vector<uint32_t> cand;
            for (uint32_t m : members)
                if (has_geometry[m]) cand.push_back(m);
            std::vector<CandOut> folds(cand.size());
            std::vector<PairOut> pair_host;  // read only for candidates the 3D test takes
            const uint32_t n_own = (uint32_t)owners.size();
            if (n_own && !cand.empty()) {
                std::vector<Cand> cands(cand.size());
                for (size_t i = 0; i < cand.size(); ++i) cands[i] = Cand{cand[i], comp_of_tri[cand[i]]};
                std::vector<OwnerRef> refs(n_own);
                for (uint32_t k = 0; k < n_own; ++k) refs[k] = OwnerRef{owners[k].slot, 0, owners[k].scale};
                const size_t n_pairs = cands.size() * n_own;
                V3D_CTX_CK(dev.cands.ensure(cands.size(), dev.st));
                V3D_CTX_CK(dev.owner_refs.ensure(n_own, dev.st));
                V3D_CTX_CK(dev.pair_outs.ensure(n_pairs, dev.st));
                V3D_CTX_CK(dev.cand_outs.ensure(cands.size(), dev.st));
                V3D_CTX_CK(cudaMemcpyAsync(dev.cands.p, cands.data(), sizeof(Cand) * cands.size(),
                                           cudaMemcpyHostToDevice, dev.st));
                V3D_CTX_CK(cudaMemcpyAsync(dev.owner_refs.p, refs.data(), sizeof(OwnerRef) * n_own,
                                           cudaMemcpyHostToDevice, dev.st));
                const DevStore st = dev.store();
                cudaEventRecord(dev.e0, dev.st);
                k_ownership<<<(unsigned)((n_pairs + 127) / 128), 128, 0, dev.st>>>(
                    st, dev.cands.p, (uint32_t)cands.size(), dev.owner_refs.p, n_own, dev.pair_outs.p);
                k_fold<<<(unsigned)((cands.size() + 127) / 128), 128, 0, dev.st>>>(
                    st, dev.cands.p, (uint32_t)cands.size(), dev.owner_refs.p, n_own, dev.pair_outs.p,
                    dev.cand_outs.p);
                cudaEventRecord(dev.e1, dev.st);
                dev.launches += 2;
                ::v3d::g_kernel_launches += 2;
                V3D_CTX_CK(cudaGetLastError());
                V3D_CTX_CK(cudaMemcpyAsync(folds.data(), dev.cand_outs.p, sizeof(CandOut) * folds.size(),
                                           cudaMemcpyDeviceToHost, dev.st));
                V3D_CTX_CK(cudaStreamSynchronize(dev.st));
                float ms = 0.f;
                if (cudaEventElapsedTime(&ms, dev.e0, dev.e1) == cudaSuccess) dev.kernel_ms += ms;
                bool any_3d = false;
                for (const CandOut& f : folds)
                    if (!(f.flags & 1u) && !(f.share >= kMinImageOwnershipShare) &&
                        !((f.flags & 2u) && !imageless_owner))
                        any_3d = true;
                if (any_3d) {
                    pair_host.resize(n_pairs);
                    V3D_CTX_CK(cudaMemcpyAsync(pair_host.data(), dev.pair_outs.p, sizeof(PairOut) * n_pairs,
                                               cudaMemcpyDeviceToHost, dev.st));
                    V3D_CTX_CK(cudaStreamSynchronize(dev.st));
                }
            } else {
                for (CandOut& f : folds) f = CandOut{0.0, 0.0, 1.0, 0xffffffffu, 0u, 0u, n_own == 0 ? 2u : 0u};
            }
            dev.stage_ms[1] += ms_since(t_stage);
            t_stage = Clock::now();
            std::set<size_t> judged_patches;
            std::map<size_t, std::vector<uint32_t>> unjudged_triangles;
            std::vector<const Geometry*> surfaces;
            for (size_t ci = 0; ci < cand.size(); ++ci) {
                if (control.is_canceled()) return V3D_OK;
                const uint32_t index = cand[ci];
                const Geometry& candidate = geometry[index];
                const CandOut& fo = folds[ci];
                // the lookups this candidate's owners recorded
                if (n_own) {
                    tally.max_postings = std::max<size_t>(tally.max_postings, fo.max_used);
                    tally.bound_hits += fo.bound_hits;
                }
                if (fo.flags & 1u) continue;  // cut off at the posting bound: kept unjudged
                const double best_share = fo.share, best_surface = fo.surface, best_scale = fo.scale;
                const uint32_t best_slot = fo.slot;
                if (best_share >= kMinImageOwnershipShare) {
                    keep[index] = 0;
                    removed_dup += 1;
                    removals.push_back({index, best_slot, best_scale});
                    if (best_share < 1.0 - kOwnershipEpsilon) {
                        trimmed += 1;
                        trimmed_area += std::fmax(candidate.area() - best_surface, 0.0);
                    }
                    continue;
                }
                if ((fo.flags & 2u) && !imageless_owner) {
                    if (best_share > kOwnershipEpsilon) {
                        remaining_overlap += 1;
                        clip_jobs.push_back({index, best_slot, best_scale});
                    }
                    continue;
                }
                // which owners judged it, and the kept triangles the others could not project
                judged_patches.clear();
                unjudged_triangles.clear();
                for (uint32_t k = 0; k < n_own; ++k) {
                    const PairOut& o = pair_host[ci * n_own + k];
                    if (o.status != kJudged) continue;
                    const Footprint& f = footprints[owners[k].slot];
                    std::vector<uint32_t> unjudged;
                    if (o.share < kMinImageOwnershipShare)
                        for (const auto& om : f.omitted)
                            if (components_linked(index, om.first)) unjudged.push_back(om.second);
                    if (unjudged.empty()) judged_patches.insert(f.patch);
                    else unjudged_triangles[f.patch] = std::move(unjudged);
                }
                // the 3D test (surface_merge.rs:737-795)
                double lo[3], hi[3];
                candidate.aabb(0.0, lo, hi);
                nearby.clear();
                Budget budget;
                Limit q = kept_grid.query(lo, hi, kMaxGridCells, budget, nearby);
                if (q == Limit::Cells) q = budget.take(all_kept.data(), all_kept.size(), nearby);
                tally.record(budget.used, q);
                if (q != Limit::None) continue;
                std::sort(nearby.begin(), nearby.end());
                surfaces.clear();
                for (uint32_t other : nearby) {
                    if (!components_linked(index, comp_of_tri[other])) continue;
                    bool ok;
                    if (patch_of[other] >= 0) {
                        const size_t owner = (size_t)patch_of[other];
                        if (judged_patches.count(owner)) {
                            ok = false;
                        } else {
                            auto it = unjudged_triangles.find(owner);
                            ok = it == unjudged_triangles.end() ||
                                 std::find(it->second.begin(), it->second.end(), other) != it->second.end();
                        }
                    } else {
                        ok = true;
                    }
                    if (ok && has_geometry[other]) surfaces.push_back(&geometry[other]);
                }
                switch (coverage(candidate, surfaces, tolerance)) {
                    case Cover::Full:
                        keep[index] = 0;
                        removed_dup += 1;
                        break;
                    case Cover::Exhausted: budget_exhausted += 1; break;
                    case Cover::Partial: remaining_overlap += 1; break;
                    case Cover::Uncovered:
                        if (best_share > kOwnershipEpsilon) remaining_overlap += 1;
                        break;
                }
            }
        }
        if (pr > 0) dev.stage_ms[2] += ms_since(t_stage);
        t_stage = Clock::now();
        if (patch < n_cams && cams[patch].present) {
            Footprint f;
            f.patch = patch;
            std::memcpy(f.cam.R, cams[patch].rotation, sizeof f.cam.R);
            std::memcpy(f.cam.t, cams[patch].translation, sizeof f.cam.t);
            for (uint32_t m : members) {
                if (!keep[m] || !has_geometry[m]) continue;
                PT p;
                if (mg::project_triangle(f.cam, geometry[m].c, p) &&
                    mg::image_area(p) > mg::kGeomEps * mg::kGeomEps) {
                    f.tri.push_back(p);
                    f.comp.push_back(comp_of_tri[m]);
                    f.vert.push_back({(uint32_t)tris[m].a, (uint32_t)tris[m].b, (uint32_t)tris[m].c});
                    f.mesh.push_back(m);
                } else {
                    f.omitted.push_back({comp_of_tri[m], m});
                }
            }
            if (!f.tri.empty()) {
                build_footprint_grid(f);
                V3D_CTX_CK(dev.add_footprint(f, nt, n_groups));
                has_footprint[patch] = 1;
                footprints.push_back(std::move(f));
            }
        }
        for (uint32_t m : members) {
            if (!keep[m] || !has_geometry[m]) continue;
            all_kept.push_back(m);
            double lo[3], hi[3];
            geometry[m].aabb(tolerance, lo, hi);
            kept_grid.insert(m, lo, hi);
        }
        dev.stage_ms[3] += ms_since(t_stage);
    }
    // seams, clips, assembly (surface_merge.rs:848-1077)
    StitchInputs si{&in, &keep, &patch_of, &removals, &kept_grid, &all_kept, tolerance, cell, dev.stage_ms + 9};
    t_stage = Clock::now();
    std::vector<v3d_mesh_triangle> stitches = stitch_trimmed_seams(si, tally);
    dev.stage_ms[4] += ms_since(t_stage);
    t_stage = Clock::now();
    ClipState clip_state;
    clip_state.base = n_points;
    std::vector<std::pair<uint32_t, std::vector<std::array<uint64_t, 3>>>> clipped;
    uint64_t clip_failures = 0;
    std::vector<std::array<uint64_t, 3>> pieces;
    {
        // plan the clips concurrently (pure geometry), commit them in job order;
        // batches bound the plans held at once
        constexpr size_t kBatch = 8192;
        const size_t n_threads =
            std::max<size_t>(1, std::min<size_t>(std::thread::hardware_concurrency(), 16));
        std::vector<ClipPlan> plans;
        std::vector<uint8_t> planned;
        std::vector<Tally> tallies(n_threads);
        for (size_t b0 = 0; b0 < clip_jobs.size(); b0 += kBatch) {
            const size_t b1 = std::min(clip_jobs.size(), b0 + kBatch);
            plans.assign(b1 - b0, ClipPlan());
            planned.assign(b1 - b0, 0);
            std::atomic<size_t> next{b0};
            std::vector<std::thread> pool;
            for (size_t k = 0; k < n_threads; ++k)
                pool.emplace_back([&, k] {
                    for (;;) {
                        const size_t j = next.fetch_add(16);
                        if (j >= b1) break;
                        for (size_t i = j; i < std::min(j + 16, b1); ++i)
                            planned[i - b0] = plan_clip(in, clip_jobs[i], tallies[k], plans[i - b0]) ? 1 : 0;
                    }
                });
            for (auto& th : pool) th.join();
            for (size_t i = b0; i < b1; ++i) {
                if (control.is_canceled()) return V3D_OK;
                if (planned[i - b0] && commit_clip(in, clip_state, plans[i - b0], pieces))
                    clipped.push_back({clip_jobs[i].triangle, pieces});
                else
                    clip_failures += 1;
            }
        }
        for (const Tally& t : tallies) {
            tally.max_postings = std::max(tally.max_postings, t.max_postings);
            tally.bound_hits += t.bound_hits;
        }
    }
    dev.stage_ms[5] += ms_since(t_stage);
    t_stage = Clock::now();
    for (const auto& c : clipped) keep[c.first] = 0;
    stats.retained_by_group.assign(n_groups, 0);
    for (size_t i = 0; i < nt; ++i)
        if (keep[i] && patch_of[i] >= 0) stats.retained_by_group[(size_t)patch_of[i]] += 1;
    for (const auto& c : clipped)
        if (patch_of[c.first] >= 0) stats.retained_by_group[(size_t)patch_of[c.first]] += c.second.size();
    uint64_t shared_vertices = 0;
    {
        // per vertex: the patch of the first retained triangle using it, and
        // whether a retained triangle of another patch uses it too
        const int64_t kUnseen = INT64_MIN;
        std::vector<int64_t> first_patch(n_points, kUnseen);
        std::vector<uint8_t> shared(n_points, 0);
        for (size_t i = 0; i < nt; ++i) {
            if (!keep[i]) continue;
            for (uint64_t v : {tris[i].a, tris[i].b, tris[i].c}) {
                if (first_patch[v] == kUnseen) first_patch[v] = patch_of[i];
                else if (first_patch[v] != patch_of[i]) shared[v] = 1;
            }
        }
        for (size_t v = 0; v < n_points; ++v) shared_vertices += shared[v];
    }
    std::vector<float> clipped_confidence;
    for (const auto& c : clipped) clipped_confidence.push_back(tris[c.first].confidence);
    {
        size_t w = 0, next = 0, retained_before = 0;
        for (size_t i = 0; i < nt; ++i) {
            if (next < reindexed.size() && reindexed[next].first == i) {
                if (keep[i]) {
                    v3d_triangle_source src{retained_before, {}};
                    for (int k = 0; k < 3; ++k) src.corners[k] = reindexed[next].second[k];
                    stats.sources.push_back(src);
                }
                ++next;
            }
            retained_before += keep[i] ? 1 : 0;
            if (keep[i]) tris[w++] = tris[i];
        }
        tris.resize(w);
    }
    tris.insert(tris.end(), stitches.begin(), stitches.end());
    uint64_t clip_pieces = 0;
    for (size_t c = 0; c < clipped.size(); ++c) {
        clip_pieces += clipped[c].second.size();
        for (const auto& p : clipped[c].second)
            tris.push_back(v3d_mesh_triangle{p[0], p[1], p[2], clipped_confidence[c], 0});
    }
    uint64_t conformed = 0, conformance_failures = 0;
    dev.stage_ms[7] += ms_since(t_stage);
    t_stage = Clock::now();
    if (!clip_state.carriers.empty()) {
        auto derived_position = [&](uint64_t v) {
            if (v < n_points) return position(v);
            const v3d_point& p = clip_state.derived[v - n_points].point;
            return V3{(double)p.x, (double)p.y, (double)p.z};
        };
        std::vector<uint64_t> split;
        if (!conform_edges(clip_state, tris, derived_position, [&] { return control.is_canceled(); },
                           split, conformance_failures))
            return V3D_OK;
        conformed = split.size();
        std::sort(split.begin(), split.end());
        stats.sources.erase(std::remove_if(stats.sources.begin(), stats.sources.end(),
                                           [&](const v3d_triangle_source& s) {
                                               return std::binary_search(split.begin(), split.end(),
                                                                         s.triangle);
                                           }),
                            stats.sources.end());
    }
    dev.stage_ms[6] += ms_since(t_stage);
    t_stage = Clock::now();
    auto group_all = [&](uint64_t v) -> int64_t {
        if (v < n_points) return group(v);
        const uint64_t d = v - n_points;
        return d < clip_state.derived.size() ? clip_state.derived[d].group : -1;
    };
    std::vector<uint8_t> present(n_groups, 0);
    uint64_t cross_reference = 0;
    std::vector<std::pair<int64_t, int64_t>> links;
    for (const auto& t : tris) {
        if (control.is_canceled()) return V3D_OK;
        const int64_t g[3] = {group_all(t.a), group_all(t.b), group_all(t.c)};
        for (int k = 0; k < 3; ++k)
            if (g[k] >= 0) present[(size_t)g[k]] = 1;
        if (g[1] != g[0] || g[2] != g[0]) {
            cross_reference += 1;
            int64_t prev = -1;
            for (int k = 0; k < 3; ++k) {
                if (g[k] < 0) continue;
                if (prev >= 0) links.push_back({prev, g[k]});
                prev = g[k];
            }
        }
    }
    std::vector<size_t> slot_of(n_groups, SIZE_MAX);
    size_t n_present = 0;
    for (size_t g = 0; g < n_groups; ++g)
        if (present[g]) slot_of[g] = n_present++;
    std::vector<size_t> up(n_present);
    for (size_t i = 0; i < n_present; ++i) up[i] = i;
    for (const auto& l : links) {
        const size_t a = uf_find(up, slot_of[(size_t)l.first]), b = uf_find(up, slot_of[(size_t)l.second]);
        up[a] = b;
    }
    uint64_t components = 0;
    for (size_t i = 0; i < n_present; ++i) components += uf_find(up, i) == i ? 1 : 0;

    v3d_merge_stats& o = stats.s;
    o.fused_pairs = fused_pairs;
    o.shared_vertices = shared_vertices;
    o.cross_reference_triangles = cross_reference;
    o.removed_duplicate_triangles = removed_dup;
    o.remaining_overlap_triangles = remaining_overlap;
    o.provenance_separated_pairs = provenance_separated;
    o.trimmed_seam_triangles = trimmed;
    o.trimmed_seam_area_share = total_area > 0.0 ? trimmed_area / total_area : 0.0;
    o.stitched_seam_triangles = stitches.size();
    o.patch_components = components;
    o.meshed_patches = n_present;
    o.max_postings_per_query = tally.max_postings;
    o.posting_bound_hits = tally.bound_hits;
    o.clipping_budget_exhausted = budget_exhausted;
    o.clipped_overlap_triangles = clipped.size();
    o.clip_pieces = clip_pieces;
    o.derived_vertices = clip_state.derived.size();
    o.unclipped_overlap_triangles = clip_failures;
    o.conformed_triangles = conformed;
    o.conformance_failures = conformance_failures;
    derived_out = std::move(clip_state.derived);
    completed = true;
    dev.stage_ms[7] += ms_since(t_stage);
    return V3D_OK;
}

}  // namespace
}  // namespace merge
}  // namespace v3d

using namespace v3d;
using namespace v3d::merge;

extern "C" void v3d_merge_result_free(v3d_merge_result* r) {
    if (!r) return;
    std::free(r->points);
    std::free(r->triangles);
    std::free(r->derived_vertices);
    std::free(r->uncalibrated_patch_pairs);
    std::free(r->retained_by_group);
    std::free(r->triangle_sources);
    std::free(r);
}

extern "C" int32_t v3d_merge_fused_patches_owned(
    v3d_context* ctx, const v3d_point* points, uint64_t n_points, const v3d_mesh_triangle* triangles,
    uint64_t n_triangles, const int64_t* membership, const v3d_fusion_pair* pairs, uint64_t n_pairs,
    const v3d_reference_camera* cameras, uint64_t n_cameras, const int32_t* origins,
    uint64_t n_origins, v3d_cancel_fn cancel, void* cancel_user, v3d_merge_result** out) {
    if (!ctx || !out || (n_points && (!points || !membership)) || (n_triangles && !triangles) ||
        (n_pairs && !pairs) || (n_cameras && !cameras) || (n_origins && !origins))
        return V3D_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    // vertex indices travel as u32 (as the reference's stitch pass stores them)
    if (n_points >= 0xFFFFFFFFull || n_triangles >= 0x7FFFFFFFull) {
        ctx->last_error = "the surface merge takes fewer than 2^32 points and 2^31 triangles";
        return V3D_ERR_INVALID_ARGUMENT;
    }
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    Control control{cancel, cancel_user};
    if (control.is_canceled()) {
        ctx->last_error = "reconstruction canceled";
        return V3D_REJECTED;
    }
    const uint64_t launches0 = g_kernel_launches;
    Device dev;
    dev.ctx = ctx;
    dev.st = static_cast<cudaStream_t>(ctx->stream);
    V3D_CTX_CK(cudaEventCreate(&dev.e0));
    V3D_CTX_CK(cudaEventCreate(&dev.e1));
    std::vector<v3d_mesh_triangle> tris(triangles, triangles + n_triangles);
    Stats stats;
    std::vector<Derived> derived;
    bool completed = false;
    const int32_t status = merge_impl(ctx, dev, points, n_points, tris, membership, pairs, n_pairs,
                                      cameras, n_cameras, origins, n_origins, control, stats, derived,
                                      completed);
    if (status != V3D_OK) return status;
    if (!completed) {
        stats = Stats();
        derived.clear();
    }
    ctx->last_ms = dev.kernel_ms;
    ctx->last_launches = g_kernel_launches - launches0;
    for (int i = 0; i < 12; ++i) ctx->last_merge_stage_ms[i] = dev.stage_ms[i];
    if (control.is_canceled()) {
        ctx->last_error = "reconstruction canceled";
        return V3D_REJECTED;
    }
    if (stats.s.conformance_failures > 0) {
        ctx->last_error = "surface merge could not split " + std::to_string(stats.s.conformance_failures) +
                          " triangle(s) at clipped seam vertices; the merge is rejected rather than "
                          "published with T-junctions";
        return V3D_REJECTED;
    }
    auto* r = static_cast<v3d_merge_result*>(std::calloc(1, sizeof(v3d_merge_result)));
    auto alloc = [](size_t n, size_t size) { return std::malloc(std::max<size_t>(n, 1) * size); };
    r->stats = stats.s;
    r->n_points = n_points + derived.size();
    r->points = static_cast<v3d_point*>(alloc(r->n_points, sizeof(v3d_point)));
    if (n_points) std::memcpy(r->points, points, sizeof(v3d_point) * n_points);
    r->n_derived_vertices = derived.size();
    r->derived_vertices =
        static_cast<v3d_derived_vertex_source*>(alloc(derived.size(), sizeof(v3d_derived_vertex_source)));
    for (size_t i = 0; i < derived.size(); ++i) {
        r->points[n_points + i] = derived[i].point;
        r->derived_vertices[i] = derived[i].source;
    }
    r->n_triangles = tris.size();
    r->triangles = static_cast<v3d_mesh_triangle*>(alloc(tris.size(), sizeof(v3d_mesh_triangle)));
    if (!tris.empty()) std::memcpy(r->triangles, tris.data(), sizeof(v3d_mesh_triangle) * tris.size());
    r->n_uncalibrated_patch_pairs = stats.uncalibrated.size();
    r->uncalibrated_patch_pairs =
        static_cast<v3d_fusion_pair*>(alloc(stats.uncalibrated.size(), sizeof(v3d_fusion_pair)));
    if (!stats.uncalibrated.empty())
        std::memcpy(r->uncalibrated_patch_pairs, stats.uncalibrated.data(),
                    sizeof(v3d_fusion_pair) * stats.uncalibrated.size());
    r->n_retained_by_group = stats.retained_by_group.size();
    r->retained_by_group = static_cast<uint64_t*>(alloc(stats.retained_by_group.size(), 8));
    if (!stats.retained_by_group.empty())
        std::memcpy(r->retained_by_group, stats.retained_by_group.data(), 8 * stats.retained_by_group.size());
    r->n_triangle_sources = stats.sources.size();
    r->triangle_sources =
        static_cast<v3d_triangle_source*>(alloc(stats.sources.size(), sizeof(v3d_triangle_source)));
    if (!stats.sources.empty())
        std::memcpy(r->triangle_sources, stats.sources.data(), sizeof(v3d_triangle_source) * stats.sources.size());
    *out = r;
    return V3D_OK;
}
