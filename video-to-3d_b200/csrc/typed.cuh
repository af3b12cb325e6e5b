// Storage-typed launch entry points (typed_impl.cuh), one explicit
// instantiation per pixel storage type in typed_<type>.cu.
#pragma once

#include "pass_kernels.cuh"

namespace v3d {

template <class T>
struct Typed {
    static cudaError_t sweep_site(const BatchDev& b, const uint32_t* site_ref, uint64_t total,
                                  SiteRank* rank, uint8_t* status, RefCounters* ctr,
                                  cudaStream_t st);
    static cudaError_t sweep_tiled(const BatchDev& b, uint32_t max_nx, uint32_t max_ny,
                                   uint32_t stride, SiteRank* rank, uint8_t* status,
                                   RefCounters* ctr, cudaStream_t st, uint64_t total_sites,
                                   SweepChunks chunks);
    static cudaError_t reciprocal(const BatchDev& b, const Cand* cands, const uint32_t* count,
                                  RecipObs* obs, RefCounters* ctr, const RecipQueue& queue,
                                  cudaStream_t st);
    static cudaError_t propose(const BatchDev& b, const uint32_t* seed_idx,
                               const uint32_t* seed_count, uint64_t total, uint8_t* prop_status,
                               Cand* prop, RefCounters* ctr, cudaStream_t st);
};

extern template struct Typed<uint8_t>;
extern template struct Typed<float>;
extern template struct Typed<__half>;
extern template struct Typed<__nv_bfloat16>;

}  // namespace v3d
