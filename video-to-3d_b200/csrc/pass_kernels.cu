// Storage-independent kernels of the batched dense plane-sweep pass
// (dense_legacy.rs:149-737) and the launch entry points.
//
// One launch of each stage covers every reference of a batch:
//   sweep      -> per-site best hypothesis + gates        (dense_legacy.rs:272-362)
//   compact    -> accepted sites in (reference, raster) order
//   reciprocal -> per (candidate, source) reciprocal point (dense_legacy.rs:777-857, 887-949)
//   fuse       -> fusion, confidence, attributes           (dense_legacy.rs:379-412, 859-884)
//   propose    -> surface-completion proposals             (dense_legacy.rs:542-650)
// Counters are integer atomics, so every statistic is deterministic.  The
// storage-typed kernels live in typed_impl.cuh.
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>

#include "pass_kernels.cuh"
#include "typed.cuh"

namespace v3d {

thread_local uint64_t g_kernel_launches = 0;

namespace {

constexpr double kInf = __builtin_huge_val();

__device__ __forceinline__ void site_xy(const DevReference& ref, uint32_t local, uint32_t& x,
                                        uint32_t& y) {
    uint32_t gy = local / ref.nx, gx = local - gy * ref.nx;
    x = ref.border + gx * ref.stride;
    y = ref.border + gy * ref.stride;
}

// ---- K0: RGBA8 -> luma (dense_legacy.rs:1147-1157) ---------------------------
__global__ void k_luma(const uchar4* __restrict__ rgba, uint8_t* __restrict__ luma, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        uchar4 p = rgba[i];
        luma[i] = (uint8_t)((77u * p.x + 150u * p.y + 29u * p.z) >> 8);
    }
}

__global__ void k_site_ref(const uint64_t* __restrict__ off, int32_t n_refs, uint64_t total,
                           uint32_t* __restrict__ site_ref) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        int lo = 0, hi = n_refs - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (off[mid] <= i)
                lo = mid;
            else
                hi = mid - 1;
        }
        site_ref[i] = (uint32_t)lo;
    }
}


// ---- compaction ---------------------------------------------------------------
constexpr int kCompactThreads = 512;
constexpr int kCompactItems = 8;
constexpr int kCompactChunk = kCompactThreads * kCompactItems;

__global__ void k_compact_count(const uint8_t* __restrict__ flags, uint8_t value, uint64_t n,
                                uint32_t* __restrict__ block_counts) {
    using Scan = cub::BlockReduce<uint32_t, kCompactThreads>;
    __shared__ typename Scan::TempStorage tmp;
    uint64_t base = (uint64_t)blockIdx.x * kCompactChunk;
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < kCompactItems; ++k) {
        uint64_t i = base + (uint64_t)k * kCompactThreads + threadIdx.x;
        c += (i < n && flags[i] == value);
    }
    uint32_t total = Scan(tmp).Sum(c);
    if (threadIdx.x == 0) block_counts[blockIdx.x] = total;
}

__global__ void k_compact_scan(uint32_t* __restrict__ block_counts, uint32_t nblocks,
                               uint32_t* __restrict__ count_out) {
    using Scan = cub::BlockScan<uint32_t, 1024>;
    __shared__ typename Scan::TempStorage tmp;
    __shared__ uint32_t carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (uint32_t base = 0; base < nblocks; base += 1024) {
        uint32_t i = base + threadIdx.x;
        uint32_t v = i < nblocks ? block_counts[i] : 0;
        uint32_t excl, agg;
        Scan(tmp).ExclusiveSum(v, excl, agg);
        if (i < nblocks) block_counts[i] = excl + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry += agg;
        __syncthreads();
    }
    if (threadIdx.x == 0) *count_out = carry;
}

__global__ void k_compact_scatter(const uint8_t* __restrict__ flags, uint8_t value, uint64_t n,
                                  const uint32_t* __restrict__ block_offsets,
                                  uint32_t* __restrict__ out) {
    using Scan = cub::BlockScan<uint32_t, kCompactThreads>;
    __shared__ typename Scan::TempStorage tmp;
    uint64_t base = (uint64_t)blockIdx.x * kCompactChunk + (uint64_t)threadIdx.x * kCompactItems;
    uint32_t f[kCompactItems];
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < kCompactItems; ++k) {
        uint64_t i = base + k;
        f[k] = (i < n && flags[i] == value);
        c += f[k];
    }
    uint32_t excl;
    Scan(tmp).ExclusiveSum(c, excl);
    uint32_t pos = block_offsets[blockIdx.x] + excl;
#pragma unroll
    for (int k = 0; k < kCompactItems; ++k)
        if (f[k]) out[pos++] = (uint32_t)(base + k);
}

// ---- candidates -------------------------------------------------------------
__global__ void k_make_primary_cands(BatchDev b, const uint32_t* __restrict__ site_idx,
                                     const uint32_t* __restrict__ count,
                                     const uint32_t* __restrict__ site_ref,
                                     const SiteRank* __restrict__ rank, Cand* __restrict__ cands) {
    const uint32_t n = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t g = site_idx[i];
        uint32_t r = site_ref[g];
        const DevReference& ref = b.refs[r];
        uint32_t local = (uint32_t)(g - b.site_off[r]);
        uint32_t x, y;
        site_xy(ref, local, x, y);
        const SiteRank& sr = rank[g];
        Cand c;
        c.ref = r;
        c.site = local;
        c.x = x;
        c.y = y;
        c.depth = hypothesis_depth(sr.plane, ref.planes, ref.search_min, ref.search_max);
        c.pos = unproject_exact(ref.cam, (double)x, (double)y, c.depth, ref.img.width,
                                ref.img.height, ref.focal);
        c.error = sr.error;
        c.margin = sr.margin;
        c.nconf = 0.0;
        c.support = sr.support;
        c.pad = 0;
        cands[i] = c;
    }
}


// ---- fusion, confidence and attributes ----------------------------------------
__device__ __forceinline__ void sample_rgb(const DevReference& ref, int32_t storage, uint32_t x,
                                           uint32_t y, v3d_point& p) {
    size_t idx = (size_t)y * ref.img.width + x;
    if (ref.rgba) {
        const uint8_t* q = ref.rgba + idx * 4;
        p.r = q[0];
        p.g = q[1];
        p.b = q[2];
        return;
    }
    float v;
    if (storage == kF32)
        v = pix<float>(static_cast<const float*>(ref.img.data), idx);
    else if (storage == kF16)
        v = pix<__half>(static_cast<const __half*>(ref.img.data), idx);
    else if (storage == kBF16)
        v = pix<__nv_bfloat16>(static_cast<const __nv_bfloat16*>(ref.img.data), idx);
    else
        v = pix<uint8_t>(static_cast<const uint8_t*>(ref.img.data), idx) / 255.0f;
    double q = round(dmul((double)v, 255.0));
    if (!(q >= 0.0)) q = 0.0;
    if (q > 255.0) q = 255.0;
    p.r = p.g = p.b = (uint8_t)q;
}

// One candidate's contribution to its reference's counters.
struct FuseCounts {
    unsigned recip_rejected, consistent, fusion_input, fusion_rejected_obs, fusion_rejected,
        footprint_rejected, accepted;
};

// Adds every lane's FuseCounts to its reference's counters: one atomic per
// counter and warp when the warp's candidates share a reference (candidates
// are listed reference by reference), one per lane otherwise.  Every lane of
// the warp calls it.
__device__ __forceinline__ void add_fuse_counts(RefCounters* ctr, uint32_t r, bool valid, FuseCounts k,
                                                int completion, int pass) {
    const unsigned full = 0xFFFFFFFFu;
    unsigned cand = valid ? 1u : 0u;
    const uint32_t r0 = __shfl_sync(full, r, 0);
    if (__all_sync(full, !valid || r == r0)) {
        cand = __reduce_add_sync(full, cand);
        k.recip_rejected = __reduce_add_sync(full, k.recip_rejected);
        k.consistent = __reduce_add_sync(full, k.consistent);
        k.fusion_input = __reduce_add_sync(full, k.fusion_input);
        k.fusion_rejected_obs = __reduce_add_sync(full, k.fusion_rejected_obs);
        k.fusion_rejected = __reduce_add_sync(full, k.fusion_rejected);
        k.footprint_rejected = __reduce_add_sync(full, k.footprint_rejected);
        k.accepted = __reduce_add_sync(full, k.accepted);
        if ((threadIdx.x & 31) != 0) return;
        r = r0;
    } else if (!valid) {
        return;
    }
    RefCounters& c = ctr[r];
    auto add = [](unsigned long long* at, unsigned v) {
        if (v) atomicAdd(at, (unsigned long long)v);
    };
    add(&c.candidates, cand);
    if (!completion) add(&c.checked, cand);
    add(completion ? &c.rej_recip : &c.recip_rejected, k.recip_rejected);
    add(completion ? &c.rej_fusion : &c.fusion_rejected_pts, k.fusion_rejected);
    if (!completion) {
        add(&c.consistent, k.consistent);
        add(&c.fusion_input, k.fusion_input);
        add(&c.fusion_rejected_obs, k.fusion_rejected_obs);
        add(&c.primary_points, k.accepted);
    } else {
        add(&c.rej_footprint, k.footprint_rejected);
        add(&c.completed, k.accepted);
        add(&c.pass_additions[pass], k.accepted);
    }
}

// fuse_depth_observations (dense_legacy.rs:859-884) and the point's
// confidence and attributes for one candidate.
__device__ __forceinline__ void fuse_one(const BatchDev& b, const Cand& cd, uint32_t i,
                                         const RecipObs* __restrict__ o, int completion,
                                         OutPoint* __restrict__ out, uint8_t* __restrict__ cand_status,
                                         FuseCounts& k) {
    {
        const DevReference& ref = b.refs[cd.ref];
        int nrec = 0;
        for (int s = 0; s < ref.n_src; ++s) nrec += o[s].valid;
        if (nrec == 0) {
            k.recip_rejected = 1;
            cand_status[i] = kCandRecipRejected;
            return;
        }
        k.consistent = 1;
        k.fusion_input = (unsigned)(1 + nrec);
        // fuse_depth_observations (dense_legacy.rs:859-884)
        double radius = fmax(dmul(fabs(cd.depth), kMaxFusionRelativePositionError), 1.0e-4);
        D3 sum = cd.pos;
        int nobs = 1, rejected = 0;
        for (int s = 0; s < ref.n_src; ++s) {
            if (!o[s].valid) continue;
            D3 p = o[s].pos;
            double dx = dsub(p.x, cd.pos.x), dy = dsub(p.y, cd.pos.y), dz = dsub(p.z, cd.pos.z);
            double dist = __dsqrt_rn(dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz)));
            if (!finite3(p) || dist > radius) {
                ++rejected;
                continue;
            }
            sum.x = dadd(sum.x, p.x);
            sum.y = dadd(sum.y, p.y);
            sum.z = dadd(sum.z, p.z);
            ++nobs;
        }
        D3 fused{ddiv(sum.x, (double)nobs), ddiv(sum.y, (double)nobs), ddiv(sum.z, (double)nobs)};
        k.fusion_rejected_obs = (unsigned)rejected;
        if (nobs < kMinFusionObservations) {
            k.fusion_rejected = 1;
            cand_status[i] = kCandFusionRejected;
            return;
        }
        const double S = (double)ref.n_src;
        const double support_conf = ddiv((double)cd.support, S);
        const double recip_conf = clampd(ddiv((double)(nobs - 1), S), 0.0, 1.0);
        const double error_conf = ddiv(1.0, dadd(1.0, ddiv(cd.error, b.prof.error_scale)));
        OutPoint op;
        if (completion) {
            D3 fp;
            bool inside = project_exact(ref.cam, fused, ref.img.width, ref.img.height, ref.focal, fp);
            if (inside) {
                double limit = dmul((double)ref.stride, 0.5);
                inside = !(fabs(dsub(fp.x, (double)cd.x)) >= limit) &&
                         !(fabs(dsub(fp.y, (double)cd.y)) >= limit);
            }
            if (!inside) {
                k.footprint_rejected = 1;
                cand_status[i] = kCandFootprintRejected;
                return;
            }
            double conf = dmul(dmul(dmul(dmul(cd.nconf, support_conf), recip_conf), error_conf),
                               kSurfaceCompletionConfidenceScale);
            op.p.confidence = (float)clampd(conf, 0.05, 0.9);
            op.a.depth_margin = (float)clampd(cd.margin, 0.0, 1.0);
        } else {
            double dm = isfinite(cd.margin) ? clampd(ddiv(cd.margin, b.prof.margin_saturation), 0.0, 1.0)
                                            : 1.0;
            double mc = fmax(dm, 0.2);
            double conf = dmul(dmul(dmul(support_conf, recip_conf), error_conf), mc);
            op.p.confidence = (float)clampd(conf, 0.05, 1.0);
            op.a.depth_margin = (float)dm;
        }
        op.p.x = (float)fused.x;
        op.p.y = (float)fused.y;
        op.p.z = (float)fused.z;
        op.p.pad = 0;
        sample_rgb(ref, b.storage, cd.x, cd.y, op.p);
        op.s.x = cd.x;
        op.s.y = cd.y;
        op.a.reciprocal_consistency = (float)recip_conf;
        op.ref = cd.ref;
        op.site = cd.site;
        op.error = cd.error;
        op.support = (double)cd.support;
        op.observations = (double)nobs;
        out[i] = op;
        cand_status[i] = kCandAccepted;
        k.accepted = 1;
    }
}

__global__ void k_fuse(BatchDev b, const Cand* __restrict__ cands, const uint32_t* __restrict__ count,
                       const RecipObs* __restrict__ obs, int completion, int pass,
                       OutPoint* __restrict__ out, uint8_t* __restrict__ cand_status,
                       RefCounters* __restrict__ ctr) {
    const uint32_t n = *count;
    const unsigned lane = threadIdx.x & 31;
    // warp-aligned turns, so every lane reaches the counter reduction
    for (uint32_t i0 = blockIdx.x * blockDim.x + threadIdx.x - lane; i0 < n; i0 += gridDim.x * blockDim.x) {
        const uint32_t i = i0 + lane;
        FuseCounts k{};
        uint32_t r = 0;
        if (i < n) {
            const Cand cd = cands[i];
            r = cd.ref;
            fuse_one(b, cd, i, obs + (uint64_t)i * kMaxSources, completion, out, cand_status, k);
        }
        add_fuse_counts(ctr, r, i < n, k, completion, pass);
    }
}

__global__ void k_append(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ count,
                         const OutPoint* __restrict__ src, OutPoint* __restrict__ pool,
                         uint32_t* __restrict__ pool_size) {
    const uint32_t n = *count, base = *pool_size;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        pool[base + i] = src[idx[i]];
}

__global__ void k_bump(uint32_t* __restrict__ pool_size, const uint32_t* __restrict__ count,
                       uint32_t* __restrict__ segment_end) {
    *pool_size += *count;
    *segment_end = *pool_size;
}

__global__ void k_fill(int32_t* __restrict__ p, uint64_t n, int32_t v) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = v;
}

// Occupancy of pool points [begin, end): site -> pool index.
__global__ void k_occupy(BatchDev b, const OutPoint* __restrict__ pool,
                         const uint32_t* __restrict__ begin, const uint32_t* __restrict__ end,
                         int32_t* __restrict__ occ) {
    const uint32_t lo = begin ? *begin : 0u, hi = *end;
    for (uint32_t i = lo + blockIdx.x * blockDim.x + threadIdx.x; i < hi;
         i += gridDim.x * blockDim.x) {
        const OutPoint& p = pool[i];
        occ[b.site_off[p.ref] + p.site] = (int32_t)i;
    }
}


__global__ void k_gather_cands(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ count,
                               const Cand* __restrict__ src, Cand* __restrict__ dst) {
    const uint32_t n = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = src[idx[i]];
}


// Multiprocessors of the current device when first asked (a thread-safe
// static: server slots launch from several threads).
int sm_count() {
    static const int sms = [] {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n <= 0) {
            cudaGetLastError();
            n = 148;
        }
        return n;
    }();
    return sms;
}

unsigned grid_for(uint64_t cap, int threads) {
    uint64_t blocks = (cap + threads - 1) / threads;
    uint64_t lim = (uint64_t)sm_count() * 16;
    if (blocks > lim) blocks = lim;
    if (blocks == 0) blocks = 1;
    return (unsigned)blocks;
}


template <class F>
cudaError_t by_storage(int storage, F&& f) {
    switch (storage) {
        case kU8: return f(uint8_t{});
        case kF32: return f(float{});
        case kF16: return f(__half{});
        case kBF16: return f(__nv_bfloat16{});
    }
    return cudaErrorInvalidValue;
}

}  // namespace

cudaError_t launch_luma(const uint8_t* rgba, uint8_t* luma, size_t pixels, cudaStream_t stream) {
    if (!pixels) return cudaSuccess;
    V3D_COUNTED k_luma<<<grid_for(pixels, 256), 256, 0, stream>>>(reinterpret_cast<const uchar4*>(rgba), luma,
                                                      pixels);
    return cudaGetLastError();
}

cudaError_t launch_site_ref(const uint64_t* site_off, int32_t n_refs, uint64_t total_sites,
                            uint32_t* site_ref, cudaStream_t stream) {
    if (!total_sites) return cudaSuccess;
    V3D_COUNTED k_site_ref<<<grid_for(total_sites, 256), 256, 0, stream>>>(site_off, n_refs, total_sites,
                                                               site_ref);
    return cudaGetLastError();
}

namespace {
// Folds the plane chunks of every pending site in plane order and applies the gates.
__global__ void k_merge_chunks(DevProfile prof, uint64_t total, int n, const Rank* __restrict__ partial,
                               SiteRank* __restrict__ rank, uint8_t* __restrict__ status) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < total;
         g += (uint64_t)gridDim.x * blockDim.x) {
        if (status[g] != kSitePending) continue;
        Rank st = partial[g];
        for (int c = 1; c < n; ++c) st = rank_merge(st, partial[(uint64_t)c * total + g]);
        finish_site(st, prof, g, rank, status);
    }
}
}  // namespace

cudaError_t launch_sweep_dispatch(const BatchDev& b, const uint32_t* site_ref, uint64_t total_sites,
                                  uint32_t max_nx, uint32_t max_ny, uint32_t uniform_stride,
                                  bool tiled, SiteRank* rank, uint8_t* status,
                                  RefCounters* counters, cudaStream_t stream, SweepChunks chunks) {
    if (!total_sites) return cudaSuccess;
    if (!tiled) chunks = SweepChunks{};
    cudaError_t e = by_storage(b.storage, [&](auto t) {
        using T = decltype(t);
        if (tiled)
            return Typed<T>::sweep_tiled(b, max_nx, max_ny, uniform_stride, rank, status,
                                         counters, stream, total_sites, chunks);
        return Typed<T>::sweep_site(b, site_ref, total_sites, rank, status, counters, stream);
    });
    if (e != cudaSuccess || chunks.n <= 1) return e;
    V3D_COUNTED k_merge_chunks<<<grid_for(total_sites, 256), 256, 0, stream>>>(b.prof, total_sites, chunks.n,
                                                                chunks.partial, rank, status);
    return cudaGetLastError();
}

size_t compaction_scratch_bytes(uint64_t n) {
    uint64_t blocks = (n + kCompactChunk - 1) / kCompactChunk;
    return (blocks + 1) * sizeof(uint32_t);
}

cudaError_t launch_compact(const uint8_t* flags, uint8_t value, uint64_t n, uint32_t* out_idx,
                           uint32_t* count_dev, void* scratch, cudaStream_t stream) {
    uint64_t blocks = (n + kCompactChunk - 1) / kCompactChunk;
    if (blocks == 0) {
        return cudaMemsetAsync(count_dev, 0, sizeof(uint32_t), stream);
    }
    uint32_t* bc = static_cast<uint32_t*>(scratch);
    V3D_COUNTED k_compact_count<<<(unsigned)blocks, kCompactThreads, 0, stream>>>(flags, value, n, bc);
    V3D_COUNTED k_compact_scan<<<1, 1024, 0, stream>>>(bc, (uint32_t)blocks, count_dev);
    V3D_COUNTED k_compact_scatter<<<(unsigned)blocks, kCompactThreads, 0, stream>>>(flags, value, n, bc,
                                                                        out_idx);
    return cudaGetLastError();
}

cudaError_t launch_make_primary_cands(const BatchDev& b, const uint32_t* site_idx,
                                      const uint32_t* count_dev, uint64_t cap,
                                      const uint32_t* site_ref, const SiteRank* rank, Cand* cands,
                                      cudaStream_t stream) {
    V3D_COUNTED k_make_primary_cands<<<grid_for(cap, 256), 256, 0, stream>>>(b, site_idx, count_dev, site_ref,
                                                                  rank, cands);
    return cudaGetLastError();
}

cudaError_t launch_reciprocal(const BatchDev& b, const Cand* cands, const uint32_t* count_dev,
                              uint64_t /*cap*/, RecipObs* obs, RefCounters* counters,
                              const RecipQueue& queue, cudaStream_t stream) {
    return by_storage(b.storage, [&](auto t) {
        return Typed<decltype(t)>::reciprocal(b, cands, count_dev, obs, counters, queue, stream);
    });
}

cudaError_t launch_fuse(const BatchDev& b, const Cand* cands, const uint32_t* count_dev,
                        uint64_t cap, const RecipObs* obs, bool completion, int pass,
                        OutPoint* out, uint8_t* cand_status, RefCounters* counters,
                        cudaStream_t stream) {
    V3D_COUNTED k_fuse<<<grid_for(cap, 128), 128, 0, stream>>>(b, cands, count_dev, obs, completion ? 1 : 0,
                                                   pass, out, cand_status, counters);
    return cudaGetLastError();
}

cudaError_t launch_append(const uint32_t* idx, const uint32_t* count_dev, uint64_t cap,
                          const OutPoint* src, OutPoint* pool, uint32_t* pool_size,
                          uint32_t* segment_end, cudaStream_t stream) {
    V3D_COUNTED k_append<<<grid_for(cap, 256), 256, 0, stream>>>(idx, count_dev, src, pool, pool_size);
    V3D_COUNTED k_bump<<<1, 1, 0, stream>>>(pool_size, count_dev, segment_end);
    return cudaGetLastError();
}

cudaError_t launch_occupancy_clear(int32_t* occ, uint64_t total_sites, cudaStream_t stream) {
    if (!total_sites) return cudaSuccess;
    V3D_COUNTED k_fill<<<grid_for(total_sites, 256), 256, 0, stream>>>(occ, total_sites, -1);
    return cudaGetLastError();
}

cudaError_t launch_occupy(const BatchDev& b, const OutPoint* pool, const uint32_t* begin,
                          const uint32_t* end, uint64_t cap, int32_t* occ, cudaStream_t stream) {
    V3D_COUNTED k_occupy<<<grid_for(cap, 256), 256, 0, stream>>>(b, pool, begin, end, occ);
    return cudaGetLastError();
}

namespace {
// First stage of a completion pass (dense_legacy.rs:551-599): every empty site
// with at least 3 occupied grid neighbours whose depths spread by at most 6 %
// becomes a seed with its predicted depth (surface_depth_prediction,
// dense_legacy.rs:739-753) and its neighbours' mean confidence and margin.
__global__ void k_propose_seed(BatchDev b, int pass, uint64_t total,
                               const uint32_t* __restrict__ site_ref,
                               const int32_t* __restrict__ occ, const OutPoint* __restrict__ pool,
                               uint8_t* __restrict__ prop_status, Cand* __restrict__ prop,
                               RefCounters* __restrict__ ctr) {
    for (uint64_t g = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; g < total;
         g += (uint64_t)gridDim.x * blockDim.x) {
        prop_status[g] = kPropNone;
        const uint32_t r = site_ref[g];
        const DevReference& ref = b.refs[r];
        if (ref.n_src == 0 || ref.stride == 0) continue;
        if (pass > 0 && ctr[r].pass_additions[pass - 1] == 0) continue;
        if (occ[g] >= 0) continue;
        const uint32_t local = (uint32_t)(g - b.site_off[r]);
        const uint32_t gy = local / ref.nx, gx = local - gy * ref.nx;
        double depths[8], confs[8], margins[8];
        int n = 0;
        for (int oy = -1; oy <= 1; ++oy)
            for (int ox = -1; ox <= 1; ++ox) {
                if (ox == 0 && oy == 0) continue;
                int ngx = (int)gx + ox, ngy = (int)gy + oy;
                if (ngx < 0 || ngy < 0 || ngx >= (int)ref.nx || ngy >= (int)ref.ny) continue;
                int32_t pi = occ[b.site_off[r] + (uint64_t)ngy * ref.nx + ngx];
                if (pi < 0) continue;
                const OutPoint& pt = pool[pi];
                D3 pos{(double)pt.p.x, (double)pt.p.y, (double)pt.p.z};
                D3 q;
                if (!project_exact(ref.cam, pos, ref.img.width, ref.img.height, ref.focal, q))
                    continue;
                depths[n] = q.z;
                confs[n] = (double)pt.p.confidence;
                margins[n] = (double)pt.a.depth_margin;
                ++n;
            }
        if (n < kMinSurfaceNeighbors) continue;
        double sorted[8];
        for (int i = 0; i < n; ++i) sorted[i] = depths[i];
        const double predicted = median_of(sorted, n);
        const double mn = sorted[0], mx = sorted[n - 1];
        if (!isfinite(mn) || !isfinite(mx) || mn <= 0.0 || mx <= 0.0) continue;
        if (ddiv(dsub(mx, mn), mx) > kMaxSurfaceNeighborSpread) continue;
        atomicAdd(&ctr[r].proposals, 1ull);
        double csum = 0.0, msum = 0.0;
        for (int i = 0; i < n; ++i) csum = dadd(csum, confs[i]);
        for (int i = 0; i < n; ++i) msum = dadd(msum, margins[i]);
        Cand cd;
        cd.ref = r;
        cd.site = local;
        cd.x = ref.border + gx * ref.stride;
        cd.y = ref.border + gy * ref.stride;
        cd.pos = D3{0, 0, 0};
        cd.depth = predicted;
        cd.error = 0.0;
        cd.margin = ddiv(msum, (double)n);
        cd.nconf = ddiv(csum, (double)n);
        cd.support = 0;
        cd.pad = 0;
        prop[g] = cd;
        prop_status[g] = kPropSeed;
    }
}
}  // namespace

cudaError_t launch_propose(const BatchDev& b, int pass, uint64_t total_sites,
                           const uint32_t* site_ref, const int32_t* occ, const OutPoint* pool,
                           uint8_t* prop_status, Cand* prop_cand, RefCounters* counters,
                           uint32_t* seed_idx, uint32_t* seed_count, void* scratch,
                           cudaStream_t stream) {
    if (!total_sites) return cudaSuccess;
    V3D_COUNTED k_propose_seed<<<grid_for(total_sites, 256), 256, 0, stream>>>(
        b, pass, total_sites, site_ref, occ, pool, prop_status, prop_cand, counters);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    e = launch_compact(prop_status, kPropSeed, total_sites, seed_idx, seed_count, scratch, stream);
    if (e != cudaSuccess) return e;
    return by_storage(b.storage, [&](auto t) {
        return Typed<decltype(t)>::propose(b, seed_idx, seed_count, total_sites, prop_status,
                                           prop_cand, counters, stream);
    });
}

cudaError_t launch_gather_cands(const uint32_t* idx, const uint32_t* count_dev, uint64_t cap,
                                const Cand* src, Cand* dst, cudaStream_t stream) {
    V3D_COUNTED k_gather_cands<<<grid_for(cap, 256), 256, 0, stream>>>(idx, count_dev, src, dst);
    return cudaGetLastError();
}

}  // namespace v3d
