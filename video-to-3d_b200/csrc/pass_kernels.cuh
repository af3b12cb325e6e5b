// Kernel-side records and launch entry points of the batched dense pass.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/v3d_dense.h"
#include "v3d_device.cuh"

namespace v3d {

// Per-site result of the depth sweep.
enum SiteStatus : uint8_t {
    kSiteInactive = 0,     // outside the grid of its reference
    kSiteLowContrast = 1,  // patch_contrast gate (dense_legacy.rs:277-281)
    kSiteNoCandidate = 2,  // no hypothesis had a passing source view
    kSiteGateRejected = 3, // photometric or ambiguity gate (dense_legacy.rs:350-362)
    kSiteAccepted = 4,     // goes to the reciprocal check
    kSitePending = 5,      // swept in plane chunks, waiting for their merge
};

struct SiteRank {
    int32_t support;
    int32_t plane;
    double error;
    double margin;
};

// A point entering the reciprocal check and fusion: a primary sweep winner or
// a surface-completion proposal.
struct Cand {
    uint32_t ref;
    uint32_t site;     // flat grid index inside its reference
    uint32_t x, y;     // pixel coordinates of the grid site
    D3 pos;            // best.position / predicted_position
    double depth;      // best.depth / predicted_depth (fusion radius)
    double error;      // best.error / direct_error
    double margin;     // ambiguity margin / mean neighbour depth margin
    double nconf;      // completion: mean neighbour confidence
    int32_t support;   // best.support / number of passing direct errors
    int32_t pad;
};

struct RecipObs {
    D3 pos;
    int32_t valid;
    int32_t pad;
};

// Output record of one accepted point.
struct OutPoint {
    v3d_point p;
    v3d_grid_site s;
    v3d_point_attributes a;
    uint32_t ref;
    uint32_t site;
    double error;
    double support;
    double observations;
};

// What the per-reference medians (dense_legacy.rs:459-462) read of one output
// point.  The photometric error is narrowed to f32 per point: the reference
// takes the median in f64 and narrows the result, and narrowing is monotone,
// so the order statistic is the same.  Support and fusion observations are
// small counts; only primary points enter the observation median.
struct MedianKey {
    float error;
    uint8_t support;
    uint8_t observations;
    uint8_t primary;
    uint8_t pad;
};

// Per-reference counters, accumulated with integer atomics.
struct RefCounters {
    unsigned long long sampled, checked, recip_rejected, consistent, fusion_input,
        fusion_rejected_obs, fusion_rejected_pts, primary_points;
    unsigned long long proposals, completed, rej_texture, rej_cross, rej_recip, rej_fusion,
        rej_footprint;
    unsigned long long pass_additions[2];
    unsigned long long recip_evals, candidates;
};

enum CandStatus : uint8_t {
    kCandNone = 0,
    kCandRecipRejected = 1,
    kCandFusionRejected = 2,
    kCandFootprintRejected = 3,
    kCandAccepted = 4,
};

// Completion proposal status per site.
enum PropStatus : uint8_t {
    kPropNone = 0,
    kPropTexture = 1,
    kPropCrossView = 2,
    kPropCandidate = 3,
    kPropSeed = 4,        // passed the neighbour tests, its costs still to come
};

struct BatchDev {
    const DevReference* refs;   // [n_refs]
    const uint64_t* site_off;   // [n_refs + 1] flat site offsets
    const float* src_inv;       // [n_refs][kMaxSources][planes] 1/depth of each source hypothesis
    int32_t n_refs;
    int32_t max_src;            // largest source count of the batch
    int32_t storage;            // StorageFormat
    DevProfile prof;
    bool exact;
    bool sums32;                // the box-filtered sweep's window sums in f32
};

// Launch wrappers (pass_kernels.cu).  All run on `stream`; none synchronises.
// Count-dependent stages read their item counts from device memory and loop
// grid-stride, so a whole batch is enqueued without host round trips.
cudaError_t launch_luma(const uint8_t* rgba, uint8_t* luma, size_t pixels, cudaStream_t stream);

cudaError_t launch_site_ref(const uint64_t* site_off, int32_t n_refs, uint64_t total_sites,
                            uint32_t* site_ref, cudaStream_t stream);

// Plane chunking of the tiled sweep: `n` CTAs per tile each sweep a
// contiguous share of the hypotheses and leave their running rank state in
// `partial` ([n][sites]); a merge folds the shares in plane order.  The rank
// merge is associative and commutative over disjoint plane sets, so the
// result is the one-CTA sweep's.
struct SweepChunks {
    int n = 1;
    Rank* partial = nullptr;
    int tile_x = 32;  // tile width: 32 (32x8 sites) or 16 (16x16)
};

// The gates of one swept site on its final rank state (dense_legacy.rs:332-362).
__device__ __forceinline__ void finish_site(const Rank& st, const DevProfile& prof, uint64_t g,
                                            SiteRank* rank, uint8_t* status) {
    SiteRank out;
    out.support = st.support;
    out.plane = st.plane;
    out.error = st.error;
    out.margin = isinf(st.second) ? __longlong_as_double(0x7ff0000000000000LL)
                                  : dsub(st.second, st.error);
    uint8_t code;
    if (st.support < 0)
        code = kSiteNoCandidate;
    else if (st.error > prof.max_error || out.margin < prof.min_margin)
        code = kSiteGateRejected;
    else
        code = kSiteAccepted;
    rank[g] = out;
    status[g] = code;
}

// `tiled` selects the box-filter ZNCC sweep (fast policy, all references share
// `uniform_stride`, optionally in plane chunks); otherwise the warp-per-site
// sweep runs.
cudaError_t launch_sweep_dispatch(const BatchDev& b, const uint32_t* site_ref,
                                  uint64_t total_sites, uint32_t max_nx, uint32_t max_ny,
                                  uint32_t uniform_stride, bool tiled, SiteRank* rank,
                                  uint8_t* status, RefCounters* counters, cudaStream_t stream,
                                  SweepChunks chunks = SweepChunks{});

// Order-preserving compaction of indices i in [0, n) with flags[i] == value.
// `scratch` needs compaction_scratch_bytes(n) bytes; *count_dev gets the count.
size_t compaction_scratch_bytes(uint64_t n);
cudaError_t launch_compact(const uint8_t* flags, uint8_t value, uint64_t n, uint32_t* out_idx,
                           uint32_t* count_dev, void* scratch, cudaStream_t stream);

cudaError_t launch_make_primary_cands(const BatchDev& b, const uint32_t* site_idx,
                                      const uint32_t* count_dev, uint64_t cap,
                                      const uint32_t* site_ref, const SiteRank* rank, Cand* cands,
                                      cudaStream_t stream);

// Work queue of the fast-policy reciprocal sweep: the prologue flags each
// (candidate, source) item that passed it (item = candidate * max_src +
// source; `cap_items` = the candidate capacity * max_src flags), a compaction
// lists the flagged items in order, and the sweep's warps take the list round
// robin, so every warp gets the same share of the pairs that need a sweep.
struct RecipQueue {
    uint8_t* flags;       // [cap_items]
    uint32_t* items;      // [cap_items]
    uint32_t* n_items;    // device count of listed items
    void* scratch;        // compaction_scratch_bytes(cap_items)
    uint64_t cap_items;
    // optional timing marks, recorded on the stream before the prologue, before
    // the single-view sweep and after it (the exact policy's one kernel counts as
    // the sweep)
    cudaEvent_t t_prepare = nullptr, t_sweep = nullptr, t_end = nullptr;
    // pairs whose band does not fit the banded sweep's stage, for the
    // per-hypothesis sweep: [cap_items] entries and their device count
    uint32_t* fallback = nullptr;
    uint32_t* n_fallback = nullptr;
};
cudaError_t launch_reciprocal(const BatchDev& b, const Cand* cands, const uint32_t* count_dev,
                              uint64_t cap, RecipObs* obs, RefCounters* counters,
                              const RecipQueue& queue, cudaStream_t stream);

cudaError_t launch_fuse(const BatchDev& b, const Cand* cands, const uint32_t* count_dev,
                        uint64_t cap, const RecipObs* obs, bool completion, int pass,
                        OutPoint* out, uint8_t* cand_status, RefCounters* counters,
                        cudaStream_t stream);

// Appends src[idx[i]] for i < *count_dev to pool[*pool_size ...], then
// advances *pool_size and stores it in *segment_end.
cudaError_t launch_append(const uint32_t* idx, const uint32_t* count_dev, uint64_t cap,
                          const OutPoint* src, OutPoint* pool, uint32_t* pool_size,
                          uint32_t* segment_end, cudaStream_t stream);

cudaError_t launch_occupancy_clear(int32_t* occ, uint64_t total_sites, cudaStream_t stream);
// occ[site of pool[i]] = i for i in [*begin (0 if null), *end).
cudaError_t launch_occupy(const BatchDev& b, const OutPoint* pool, const uint32_t* begin,
                          const uint32_t* end, uint64_t cap, int32_t* occ, cudaStream_t stream);

// complete_surface_samples (dense_legacy.rs:542-650) proposals of one pass, in
// two stages: a thread per site for the neighbour tests, then, over the
// compacted seeds (seed_idx, *seed_count, `scratch` for the compaction), a
// thread per seed for the contrast and cross-view costs.
cudaError_t launch_propose(const BatchDev& b, int pass, uint64_t total_sites,
                           const uint32_t* site_ref, const int32_t* occ, const OutPoint* pool,
                           uint8_t* prop_status, Cand* prop_cand, RefCounters* counters,
                           uint32_t* seed_idx, uint32_t* seed_count, void* scratch,
                           cudaStream_t stream);

cudaError_t launch_gather_cands(const uint32_t* idx, const uint32_t* count_dev, uint64_t cap,
                                const Cand* src, Cand* dst, cudaStream_t stream);

}  // namespace v3d
