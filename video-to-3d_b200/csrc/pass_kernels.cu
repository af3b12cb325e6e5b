// Kernels of the batched dense plane-sweep pass (dense_legacy.rs:149-737).
//
// One launch of each stage covers every reference of a batch:
//   sweep      -> per-site best hypothesis + gates        (dense_legacy.rs:272-362)
//   compact    -> accepted sites in (reference, raster) order
//   reciprocal -> per (candidate, source) reciprocal point (dense_legacy.rs:777-857, 887-949)
//   fuse       -> fusion, confidence, attributes           (dense_legacy.rs:379-412, 859-884)
//   propose    -> surface-completion proposals             (dense_legacy.rs:542-650)
// Counters are integer atomics, so every statistic is deterministic.
#include <cub/block/block_reduce.cuh>
#include <cub/block/block_scan.cuh>

#include "pass_kernels.cuh"

namespace v3d {
namespace {

constexpr int kTileX = 32;
constexpr int kTileY = 8;
constexpr double kInf = __builtin_huge_val();

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

__device__ __forceinline__ void site_xy(const DevReference& ref, uint32_t local, uint32_t& x,
                                        uint32_t& y) {
    uint32_t gy = local / ref.nx, gx = local - gy * ref.nx;
    x = ref.border + gx * ref.stride;
    y = ref.border + gy * ref.stride;
}

// ---- fast window cost --------------------------------------------------------
// Window cost between fixed values pv (taps of the first image, row-major) and
// samples of `img` at H (x + dx, y + dy, 1); false where the reference's
// patch_error returns None (a tap behind the camera or outside the bilinear
// bounds, or a ZNCC window under the variance floor).
template <class T, int R>
__device__ __forceinline__ bool window_cost_fast(const DevProfile& prof, const float* pv,
                                                 float pmean, float pvar, const float* H,
                                                 float zmin, const DevImage& img, float x, float y,
                                                 float& cost) {
    constexpr int W = 2 * R + 1;
    constexpr int N = W * W;
    const T* data = static_cast<const T*>(img.data);
    const uint32_t w = img.width, h = img.height;
    if (prof.cost == 1) {
        float ss = 0.f, sss = 0.f, sps = 0.f;
#pragma unroll
        for (int dy = 0; dy < W; ++dy) {
            float Y = y + (float)(dy - R);
#pragma unroll
            for (int dx = 0; dx < W; ++dx) {
                float X = x + (float)(dx - R);
                float h2 = fmaf(H[6], X, fmaf(H[7], Y, H[8]));
                if (!(h2 > zmin)) return false;
                float inv = __frcp_rn(h2);
                float u = fmaf(H[0], X, fmaf(H[1], Y, H[2])) * inv;
                float v = fmaf(H[3], X, fmaf(H[4], Y, H[5])) * inv;
                if (!in_bounds_fast(u, v, w, h)) return false;
                float s = sample_fast<T>(data, w, u, v) - pmean;
                ss += s;
                sss = fmaf(s, s, sss);
                sps = fmaf(pv[dy * W + dx] - pmean, s, sps);
            }
        }
        const float n = (float)N;
        float vs = sss - ss * ss / n;
        float cov = sps;  // sum of (p - mean p) equals zero up to rounding
        if (!(pvar > 0.f) || !(vs > 0.f) || pvar / n < (float)prof.min_variance ||
            vs / n < (float)prof.min_variance)
            return false;
        cost = 1.0f - cov * rsqrtf(pvar * vs);
        return true;
    }
    float sv[N];
    float ss = 0.f;
#pragma unroll
    for (int dy = 0; dy < W; ++dy) {
        float Y = y + (float)(dy - R);
#pragma unroll
        for (int dx = 0; dx < W; ++dx) {
            float X = x + (float)(dx - R);
            float h2 = fmaf(H[6], X, fmaf(H[7], Y, H[8]));
            if (!(h2 > zmin)) return false;
            float inv = __frcp_rn(h2);
            float u = fmaf(H[0], X, fmaf(H[1], Y, H[2])) * inv;
            float v = fmaf(H[3], X, fmaf(H[4], Y, H[5])) * inv;
            if (!in_bounds_fast(u, v, w, h)) return false;
            float s = sample_fast<T>(data, w, u, v);
            sv[dy * W + dx] = s;
            ss += s;
        }
    }
    float ms = ss / (float)N;
    float acc = 0.f;
#pragma unroll
    for (int i = 0; i < N; ++i) acc += fabsf((pv[i] - pmean) - (sv[i] - ms));
    cost = acc / (float)N;
    return true;
}

// Fixed-window statistics for window_cost_fast: mean and sum of squared deviations.
template <int R>
__device__ __forceinline__ void window_stats(const float* pv, float& mean, float& var) {
    constexpr int N = (2 * R + 1) * (2 * R + 1);
    float s = 0.f;
#pragma unroll
    for (int i = 0; i < N; ++i) s += pv[i];
    mean = s / (float)N;
    float v = 0.f;
#pragma unroll
    for (int i = 0; i < N; ++i) v = fmaf(pv[i] - mean, pv[i] - mean, v);
    var = v;
}

// Homography ref->src (or src->ref) at inverse depth `inv`: A + inv * b e3^T.
__device__ __forceinline__ void plane_h(const float* A, const float* b, float inv, float* H) {
#pragma unroll
    for (int i = 0; i < 9; ++i) H[i] = A[i];
    H[2] = fmaf(inv, b[0], A[2]);
    H[5] = fmaf(inv, b[1], A[5]);
    H[8] = fmaf(inv, b[2], A[8]);
}

// f32 bilinear taps of a window at fractional centre (x, y); false if out of bounds.
template <class T, int R>
__device__ __forceinline__ bool load_window(const DevImage& img, float x, float y, float* pv) {
    constexpr int W = 2 * R + 1;
    const T* data = static_cast<const T*>(img.data);
#pragma unroll
    for (int dy = 0; dy < W; ++dy)
#pragma unroll
        for (int dx = 0; dx < W; ++dx) {
            float X = x + (float)(dx - R), Y = y + (float)(dy - R);
            if (!in_bounds_fast(X, Y, img.width, img.height)) return false;
            pv[dy * W + dx] = sample_fast<T>(data, img.width, X, Y);
        }
    return true;
}

// Integer-position window (exact pixel values).
template <class T, int R>
__device__ __forceinline__ void load_window_int(const DevImage& img, uint32_t x, uint32_t y,
                                                float* pv) {
    constexpr int W = 2 * R + 1;
    const T* data = static_cast<const T*>(img.data);
#pragma unroll
    for (int dy = 0; dy < W; ++dy)
#pragma unroll
        for (int dx = 0; dx < W; ++dx)
            pv[dy * W + dx] = pix<T>(data, (size_t)(y + dy - R) * img.width + (x + dx - R));
}

__device__ __forceinline__ float zmin_of(double inv_depth) { return (float)(1.0e-4 * inv_depth); }

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

// ---- sweep, warp per site ----------------------------------------------------
// Lanes take hypotheses lane, lane+32, ...; each lane keeps the running
// best/second state, and a warp merge reproduces the reference's sort.
template <class T, bool EXACT, int R>
__global__ void __launch_bounds__(256) k_sweep_site(BatchDev b, const uint32_t* __restrict__ site_ref,
                                                    uint64_t total, SiteRank* __restrict__ rank,
                                                    uint8_t* __restrict__ status,
                                                    RefCounters* __restrict__ ctr) {
    constexpr int W = 2 * R + 1;
    const uint64_t gw = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = lane_id();
    if (gw >= total) return;
    const uint32_t r = site_ref[gw];
    const DevReference& ref = b.refs[r];
    const uint32_t local = (uint32_t)(gw - b.site_off[r]);
    uint32_t x, y;
    site_xy(ref, local, x, y);
    const DevProfile& prof = b.prof;
    double contrast = 0.0;
    if (lane == 0) contrast = patch_contrast_exact<T>(ref.img, (double)x, (double)y, R);
    contrast = __shfl_sync(0xffffffffu, contrast, 0);
    if (contrast < prof.min_contrast) {
        if (lane == 0) status[gw] = kSiteLowContrast;
        return;
    }
    if (lane == 0) atomicAdd(&ctr[r].sampled, 1ull);
    float pv[W * W];
    float pmean = 0.f, pvar = 0.f;
    if (!EXACT) {
        load_window_int<T, R>(ref.img, x, y, pv);
        window_stats<R>(pv, pmean, pvar);
    }
    Rank st = rank_empty();
    const int n_src = ref.n_src;
    for (int k = lane; k < prof.planes; k += 32) {
        const double depth = hypothesis_depth(k, prof.planes, ref.search_min, ref.search_max);
        const double inv = ddiv(1.0, depth);
        double errs[kMaxSources];
        int n = 0;
        for (int s = 0; s < n_src; ++s) {
            const DevSource& src = ref.src[s];
            double e;
            bool ok;
            if (EXACT) {
                ok = patch_error_exact<T>(prof, ref.cam, ref.img, src.cam, src.img, ref.focal,
                                          (double)x, (double)y, depth, e);
            } else {
                float H[9];
                plane_h(src.fwd_A, src.fwd_b, (float)inv, H);
                float c;
                ok = window_cost_fast<T, R>(prof, pv, pmean, pvar, H, zmin_of(inv), src.img,
                                            (float)x, (float)y, c);
                e = c;
            }
            if (ok && e <= prof.max_error) errs[n++] = e;
        }
        if (n > 0) {
            Rank c;
            c.support = n;
            c.plane = k;
            c.error = median_of(errs, n);
            c.second = kInf;
            st = rank_merge(st, c);
        }
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) st = rank_shfl_merge(st, off);
    if (lane != 0) return;
    SiteRank out;
    out.support = st.support;
    out.plane = st.plane;
    out.error = st.error;
    out.margin = isinf(st.second) ? kInf : dsub(st.second, st.error);
    uint8_t code;
    if (st.support < 0)
        code = kSiteNoCandidate;
    else if (st.error > prof.max_error || out.margin < prof.min_margin)
        code = kSiteGateRejected;
    else
        code = kSiteAccepted;
    rank[gw] = out;
    status[gw] = code;
}

// ---- sweep, tiled ZNCC (fast policy) -----------------------------------------
// A CTA owns a 32x8 block of grid sites.  For every (plane, source) it warps
// the block's pixel footprint into the source once (f32 homography and f32
// bilinear), then forms the window sums of s, s^2 and r*s with separable box
// filters, so overlapping windows (stride < window) share every bilinear
// sample.  Products and sums are formed in f64: s^2 - (sum s)^2/n cancels
// badly in f32 on low-variance windows.  Invalid taps are NaN and poison
// their windows, which reproduces the reference's all-taps-valid rule.
template <class T, int R>
__global__ void __launch_bounds__(256) k_sweep_tiled(BatchDev b, uint64_t total_sites_unused,
                                                     SiteRank* __restrict__ rank,
                                                     uint8_t* __restrict__ status,
                                                     RefCounters* __restrict__ ctr) {
    constexpr int W = 2 * R + 1;
    constexpr int N = W * W;
    extern __shared__ double smem_d[];
    const uint32_t r = blockIdx.z;
    const DevReference& ref = b.refs[r];
    const DevProfile& prof = b.prof;
    const uint32_t gx0 = blockIdx.x * kTileX, gy0 = blockIdx.y * kTileY;
    if (gx0 >= ref.nx || gy0 >= ref.ny) return;
    const int s = (int)ref.stride;
    const int PX = (kTileX - 1) * s + W, PY = (kTileY - 1) * s + W;
    const int npx = PX * PY;
    double* hs = smem_d;                     // [PY][32] row sums of s
    double* hss = hs + PY * kTileX;          // [PY][32] row sums of s^2
    double* hrs = hss + PY * kTileX;         // [PY][32] row sums of r*s
    float* refv = reinterpret_cast<float*>(hrs + PY * kTileX);  // [PY][PX] reference values
    float* samp = refv + npx;                // [PY][PX] source samples (NaN = invalid)
    float* costs = samp + npx;               // [n_src][256]
    float* hA = costs + kMaxSources * 256;   // [n_src][12] homography parts
    float* pinv = hA + kMaxSources * 12;     // [planes] inverse depths
    const int tid = threadIdx.x;
    const T* rdata = static_cast<const T*>(ref.img.data);
    const int px0 = (int)(ref.border + gx0 * s) - R, py0 = (int)(ref.border + gy0 * s) - R;
    for (int i = tid; i < npx; i += 256) {
        int yy = i / PX, xx = i - yy * PX;
        int X = px0 + xx, Y = py0 + yy;
        float v = __int_as_float(0x7fc00000);
        if (X >= 0 && Y >= 0 && X < (int)ref.img.width && Y < (int)ref.img.height)
            v = pix<T>(rdata, (size_t)Y * ref.img.width + X);
        refv[i] = v;
    }
    const int n_src = ref.n_src;
    for (int i = tid; i < n_src * 12; i += 256) {
        int j = i / 12, c = i - j * 12;
        hA[i] = c < 9 ? ref.src[j].fwd_A[c] : ref.src[j].fwd_b[c - 9];
    }
    for (int k = tid; k < prof.planes; k += 256)
        pinv[k] = (float)ddiv(1.0, hypothesis_depth(k, prof.planes, ref.search_min, ref.search_max));
    __syncthreads();

    const int tx = tid & 31, ty = tid >> 5;
    const uint32_t gx = gx0 + tx, gy = gy0 + ty;
    const bool active = gx < ref.nx && gy < ref.ny;
    const uint64_t gsite = b.site_off[r] + (uint64_t)gy * ref.nx + gx;
    // reference window statistics and the contrast gate on exact pixel values
    double sr = 0.0, srr = 0.0;
    bool sampled = false;
    if (active) {
        float mn = 3.0e38f, mx = -3.0e38f;
        for (int dy = 0; dy < W; ++dy)
            for (int dx = 0; dx < W; ++dx) {
                float v = refv[(ty * s + dy) * PX + tx * s + dx];
                mn = fminf(mn, v);
                mx = fmaxf(mx, v);
                sr += (double)v;
                srr = fma((double)v, (double)v, srr);
            }
        double contrast = (double)mx - (double)mn;
        sampled = contrast >= prof.min_contrast;
        if (!sampled) status[gsite] = kSiteLowContrast;
        else atomicAdd(&ctr[r].sampled, 1ull);
    }
    const double n = (double)N;
    const double vr = srr - sr * sr / n;
    const double minvar_n = prof.min_variance * n;
    Rank st = rank_empty();
    for (int k = 0; k < prof.planes; ++k) {
        const float inv = pinv[k];
        const float zmin = 1.0e-4f * inv;
        for (int j = 0; j < n_src; ++j) {
            const float* A = hA + j * 12;
            const float H2 = fmaf(inv, A[9], A[2]);
            const float H5 = fmaf(inv, A[10], A[5]);
            const float H8 = fmaf(inv, A[11], A[8]);
            const DevImage si = ref.src[j].img;
            const T* sdata = static_cast<const T*>(si.data);
            const float wl = (float)(si.width - 1), hl = (float)(si.height - 1);
            for (int i = tid; i < npx; i += 256) {
                int yy = i / PX, xx = i - yy * PX;
                float X = (float)(px0 + xx), Y = (float)(py0 + yy);
                float h2 = fmaf(A[6], X, fmaf(A[7], Y, H8));
                float v = __int_as_float(0x7fc00000);
                if (h2 > zmin) {
                    float iv = __frcp_rn(h2);
                    float u = fmaf(A[0], X, fmaf(A[1], Y, H2)) * iv;
                    float q = fmaf(A[3], X, fmaf(A[4], Y, H5)) * iv;
                    if (u >= 0.f && q >= 0.f && u < wl && q < hl)
                        v = sample_fast<T>(sdata, si.width, u, q);
                }
                samp[i] = v;
            }
            __syncthreads();
            for (int i = tid; i < PY * kTileX; i += 256) {
                int row = i >> 5, col = i & 31;
                const float* sp = samp + row * PX + col * s;
                const float* rp = refv + row * PX + col * s;
                double a = 0.0, bb = 0.0, c = 0.0;
#pragma unroll
                for (int dx = 0; dx < W; ++dx) {
                    double v = (double)sp[dx];
                    a += v;
                    bb = fma(v, v, bb);
                    c = fma((double)rp[dx], v, c);
                }
                hs[i] = a;
                hss[i] = bb;
                hrs[i] = c;
            }
            __syncthreads();
            if (sampled) {
                double a = 0.0, bb = 0.0, c = 0.0;
#pragma unroll
                for (int dy = 0; dy < W; ++dy) {
                    int i = (ty * s + dy) * kTileX + tx;
                    a += hs[i];
                    bb += hss[i];
                    c += hrs[i];
                }
                double vs = bb - a * a / n;
                double cov = c - sr * a / n;
                float cost = __int_as_float(0x7fc00000);
                if (vs > 0.0 && vr > 0.0 && vs >= minvar_n && vr >= minvar_n)
                    cost = (float)(1.0 - cov / sqrt(vr * vs));
                costs[j * 256 + tid] = cost;  // NaN when invalid
            }
        }
        if (sampled) {
            double errs[kMaxSources];
            int cnt = 0;
            for (int j = 0; j < n_src; ++j) {
                float c = costs[j * 256 + tid];
                if ((double)c <= prof.max_error) errs[cnt++] = c;
            }
            if (cnt > 0) {
                Rank c;
                c.support = cnt;
                c.plane = k;
                c.error = median_of(errs, cnt);
                c.second = kInf;
                st = rank_merge(st, c);
            }
        }
    }
    if (!sampled) return;
    SiteRank out;
    out.support = st.support;
    out.plane = st.plane;
    out.error = st.error;
    out.margin = isinf(st.second) ? kInf : dsub(st.second, st.error);
    uint8_t code;
    if (st.support < 0)
        code = kSiteNoCandidate;
    else if (st.error > prof.max_error || out.margin < prof.min_margin)
        code = kSiteGateRejected;
    else
        code = kSiteAccepted;
    rank[gsite] = out;
    status[gsite] = code;
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
        c.depth = hypothesis_depth(sr.plane, b.prof.planes, ref.search_min, ref.search_max);
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

// ---- reciprocal check, warp per (candidate, source) ----------------------------
// reciprocal_depth_observations (dense_legacy.rs:777-857) for one source:
// direct cost at the re-projected reference position, projection into the
// source, then estimate_single_view_depth (dense_legacy.rs:887-949) with lanes
// over the source's hypotheses, and the reciprocal agreement test.
template <class T, bool EXACT, int R>
__global__ void __launch_bounds__(256) k_reciprocal(BatchDev b, const Cand* __restrict__ cands,
                                                    const uint32_t* __restrict__ count,
                                                    RecipObs* __restrict__ obs,
                                                    RefCounters* __restrict__ ctr) {
    constexpr int W = 2 * R + 1;
    const uint32_t lane = lane_id();
    const uint64_t items = (uint64_t)(*count) * kMaxSources;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const DevProfile& prof = b.prof;
    for (uint64_t it = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; it < items;
         it += nwarps) {
        const uint32_t ci = (uint32_t)(it / kMaxSources);
        const int si = (int)(it - (uint64_t)ci * kMaxSources);
        const Cand cd = cands[ci];
        const DevReference& ref = b.refs[cd.ref];
        RecipObs res;
        res.valid = 0;
        res.pad = 0;
        res.pos = D3{0, 0, 0};
        bool ok = si < ref.n_src;
        const DevSource& src = ref.src[ok ? si : 0];
        D3 rp, sp;
        if (ok) ok = project_exact(ref.cam, cd.pos, ref.img.width, ref.img.height, ref.focal, rp);
        // direct cost of the reference window at (rp.x, rp.y), depth rp.z
        if (ok) {
            bool dok = false;
            double de = 0.0;
            if (lane == 0) {
                if (EXACT) {
                    dok = patch_error_exact<T>(prof, ref.cam, ref.img, src.cam, src.img, ref.focal,
                                               rp.x, rp.y, rp.z, de);
                } else {
                    float pv[W * W];
                    if (load_window<T, R>(ref.img, (float)rp.x, (float)rp.y, pv)) {
                        float pm, pvv, c;
                        window_stats<R>(pv, pm, pvv);
                        float H[9];
                        double inv = ddiv(1.0, rp.z);
                        plane_h(src.fwd_A, src.fwd_b, (float)inv, H);
                        dok = window_cost_fast<T, R>(prof, pv, pm, pvv, H, zmin_of(inv), src.img,
                                                     (float)rp.x, (float)rp.y, c);
                        de = c;
                    }
                }
            }
            dok = __shfl_sync(0xffffffffu, dok, 0);
            de = __shfl_sync(0xffffffffu, de, 0);
            ok = dok && !(de > prof.max_error);
        }
        if (ok) ok = project_exact(src.cam, cd.pos, src.img.width, src.img.height, ref.focal, sp);
        if (ok) {
            double contrast = 0.0;
            if (lane == 0) contrast = patch_contrast_exact<T>(src.img, sp.x, sp.y, R);
            contrast = __shfl_sync(0xffffffffu, contrast, 0);
            ok = !(contrast < prof.min_contrast);
        }
        if (ok) {
            float pv[W * W];
            float pm = 0.f, pvv = 0.f;
            if (!EXACT) {
                // the f64 contrast check passed, so the f32 taps are in bounds
                // unless rounding moved one onto the edge
                ok = load_window<T, R>(src.img, (float)sp.x, (float)sp.y, pv);
                window_stats<R>(pv, pm, pvv);
            }
            double be = kInf;
            int bk = 0x7fffffff;
            if (ok && lane == 0) atomicAdd(&ctr[cd.ref].recip_evals, (unsigned long long)prof.planes);
            for (int k = lane; ok && k < prof.planes; k += 32) {
                double d = hypothesis_depth(k, prof.planes, src.search_min, src.search_max);
                double e;
                bool eok;
                if (EXACT) {
                    eok = patch_error_exact<T>(prof, src.cam, src.img, ref.cam, ref.img, ref.focal,
                                               sp.x, sp.y, d, e);
                } else {
                    double inv = ddiv(1.0, d);
                    float H[9];
                    plane_h(src.bwd_A, src.bwd_b, (float)inv, H);
                    float c;
                    eok = window_cost_fast<T, R>(prof, pv, pm, pvv, H, zmin_of(inv), ref.img,
                                                 (float)sp.x, (float)sp.y, c);
                    e = c;
                }
                if (eok && e <= prof.max_error && e < be) {
                    be = e;
                    bk = k;
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                double oe = __shfl_down_sync(0xffffffffu, be, off);
                int ok2 = __shfl_down_sync(0xffffffffu, bk, off);
                if (oe < be || (oe == be && ok2 < bk)) {
                    be = oe;
                    bk = ok2;
                }
            }
            bk = __shfl_sync(0xffffffffu, bk, 0);
            if (bk == 0x7fffffff) {
                ok = false;
            } else {
                double rd = hypothesis_depth(bk, prof.planes, src.search_min, src.search_max);
                // reciprocal_depth_agrees (dense_legacy.rs:951-957)
                double ex = sp.z;
                bool agree = isfinite(ex) && isfinite(rd) && ex > 0.0 && rd > 0.0;
                if (agree) {
                    double scale = fmax(fmax(ex, rd), 1.0e-9);
                    agree = ddiv(fabs(dsub(ex, rd)), scale) <= kMaxReciprocalRelativeDepthError;
                }
                if (agree) {
                    res.pos = unproject_exact(src.cam, sp.x, sp.y, rd, src.img.width,
                                              src.img.height, ref.focal);
                    res.valid = finite3(res.pos) ? 1 : 0;
                }
            }
        }
        if (lane == 0) obs[it] = res;
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

__global__ void k_fuse(BatchDev b, const Cand* __restrict__ cands, const uint32_t* __restrict__ count,
                       const RecipObs* __restrict__ obs, int completion, int pass,
                       OutPoint* __restrict__ out, uint8_t* __restrict__ cand_status,
                       RefCounters* __restrict__ ctr) {
    const uint32_t n = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Cand cd = cands[i];
        const DevReference& ref = b.refs[cd.ref];
        RefCounters& c = ctr[cd.ref];
        const RecipObs* o = obs + (uint64_t)i * kMaxSources;
        atomicAdd(&c.candidates, 1ull);
        int nrec = 0;
        for (int s = 0; s < ref.n_src; ++s) nrec += o[s].valid;
        if (!completion) atomicAdd(&c.checked, 1ull);
        if (nrec == 0) {
            atomicAdd(completion ? &c.rej_recip : &c.recip_rejected, 1ull);
            cand_status[i] = kCandRecipRejected;
            continue;
        }
        if (!completion) {
            atomicAdd(&c.consistent, 1ull);
            atomicAdd(&c.fusion_input, (unsigned long long)(1 + nrec));
        }
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
        if (!completion) atomicAdd(&c.fusion_rejected_obs, (unsigned long long)rejected);
        if (nobs < kMinFusionObservations) {
            atomicAdd(completion ? &c.rej_fusion : &c.fusion_rejected_pts, 1ull);
            cand_status[i] = kCandFusionRejected;
            continue;
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
                atomicAdd(&c.rej_footprint, 1ull);
                cand_status[i] = kCandFootprintRejected;
                continue;
            }
            double conf = dmul(dmul(dmul(dmul(cd.nconf, support_conf), recip_conf), error_conf),
                               kSurfaceCompletionConfidenceScale);
            op.p.confidence = (float)clampd(conf, 0.05, 0.9);
            op.a.depth_margin = (float)clampd(cd.margin, 0.0, 1.0);
            atomicAdd(&c.completed, 1ull);
            atomicAdd(&c.pass_additions[pass], 1ull);
        } else {
            double dm = isfinite(cd.margin) ? clampd(ddiv(cd.margin, b.prof.margin_saturation), 0.0, 1.0)
                                            : 1.0;
            double mc = fmax(dm, 0.2);
            double conf = dmul(dmul(dmul(support_conf, recip_conf), error_conf), mc);
            op.p.confidence = (float)clampd(conf, 0.05, 1.0);
            op.a.depth_margin = (float)dm;
            atomicAdd(&c.primary_points, 1ull);
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

// ---- surface completion proposals (dense_legacy.rs:542-650) ------------------
template <class T, bool EXACT, int R>
__global__ void __launch_bounds__(128) k_propose(BatchDev b, int pass, uint64_t total,
                                                 const uint32_t* __restrict__ site_ref,
                                                 const int32_t* __restrict__ occ,
                                                 const OutPoint* __restrict__ pool,
                                                 uint8_t* __restrict__ prop_status,
                                                 Cand* __restrict__ prop, RefCounters* __restrict__ ctr) {
    constexpr int W = 2 * R + 1;
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
        const uint32_t x = ref.border + gx * ref.stride, y = ref.border + gy * ref.stride;
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
        // surface_depth_prediction (dense_legacy.rs:739-753)
        if (n < kMinSurfaceNeighbors) continue;
        double sorted[8];
        for (int i = 0; i < n; ++i) sorted[i] = depths[i];
        double predicted = median_of(sorted, n);
        double mn = sorted[0], mx = sorted[n - 1];
        if (!isfinite(mn) || !isfinite(mx) || mn <= 0.0 || mx <= 0.0) continue;
        if (ddiv(dsub(mx, mn), mx) > kMaxSurfaceNeighborSpread) continue;
        RefCounters& c = ctr[r];
        atomicAdd(&c.proposals, 1ull);
        if (patch_contrast_exact<T>(ref.img, (double)x, (double)y, R) < b.prof.min_contrast) {
            atomicAdd(&c.rej_texture, 1ull);
            prop_status[g] = kPropTexture;
            continue;
        }
        D3 ppos = unproject_exact(ref.cam, (double)x, (double)y, predicted, ref.img.width,
                                  ref.img.height, ref.focal);
        double errs[kMaxSources];
        int ne = 0;
        float pv[W * W];
        float pm = 0.f, pvv = 0.f;
        double inv = ddiv(1.0, predicted);
        if (!EXACT) {
            load_window_int<T, R>(ref.img, x, y, pv);
            window_stats<R>(pv, pm, pvv);
        }
        for (int s = 0; s < ref.n_src; ++s) {
            const DevSource& src = ref.src[s];
            double e;
            bool ok;
            if (EXACT) {
                ok = patch_error_exact<T>(b.prof, ref.cam, ref.img, src.cam, src.img, ref.focal,
                                          (double)x, (double)y, predicted, e);
            } else {
                float H[9];
                plane_h(src.fwd_A, src.fwd_b, (float)inv, H);
                float cst;
                ok = window_cost_fast<T, R>(b.prof, pv, pm, pvv, H, zmin_of(inv), src.img,
                                            (float)x, (float)y, cst);
                e = cst;
            }
            if (ok && e <= b.prof.max_error) errs[ne++] = e;
        }
        if (ne == 0) {
            atomicAdd(&c.rej_cross, 1ull);
            prop_status[g] = kPropCrossView;
            continue;
        }
        double direct_error = median_of(errs, ne);
        double csum = 0.0, msum = 0.0;
        for (int i = 0; i < n; ++i) csum = dadd(csum, confs[i]);
        for (int i = 0; i < n; ++i) msum = dadd(msum, margins[i]);
        Cand cd;
        cd.ref = r;
        cd.site = local;
        cd.x = x;
        cd.y = y;
        cd.pos = ppos;
        cd.depth = predicted;
        cd.error = direct_error;
        cd.margin = ddiv(msum, (double)n);
        cd.nconf = ddiv(csum, (double)n);
        cd.support = ne;
        cd.pad = 0;
        prop[g] = cd;
        prop_status[g] = kPropCandidate;
    }
}

__global__ void k_gather_cands(const uint32_t* __restrict__ idx, const uint32_t* __restrict__ count,
                               const Cand* __restrict__ src, Cand* __restrict__ dst) {
    const uint32_t n = *count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        dst[i] = src[idx[i]];
}

int sm_count() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 148;
    }
    return sms;
}

// Dispatch helpers over (storage type, exactness, radius).
template <template <class, bool, int> class L, class... A>
cudaError_t dispatch(int storage, bool exact, int radius, A&&... a) {
#define V3D_CASE_R(T, E, RR) \
    if (radius == RR) return L<T, E, RR>::run(a...);
#define V3D_CASE_E(T, E) \
    V3D_CASE_R(T, E, 1) V3D_CASE_R(T, E, 2) V3D_CASE_R(T, E, 3) V3D_CASE_R(T, E, 4)
#define V3D_CASE_T(T)                  \
    if (exact) {                       \
        V3D_CASE_E(T, true)            \
    } else {                           \
        V3D_CASE_E(T, false)           \
    }
    switch (storage) {
        case kU8: V3D_CASE_T(uint8_t) break;
        case kF32: V3D_CASE_T(float) break;
        case kF16: V3D_CASE_T(__half) break;
        case kBF16: V3D_CASE_T(__nv_bfloat16) break;
    }
#undef V3D_CASE_T
#undef V3D_CASE_E
#undef V3D_CASE_R
    return cudaErrorInvalidValue;
}

template <class T, bool EXACT, int R>
struct SweepSiteL {
    static cudaError_t run(const BatchDev& b, const uint32_t* site_ref, uint64_t total,
                           SiteRank* rank, uint8_t* status, RefCounters* ctr, cudaStream_t st) {
        uint64_t threads = total * 32;
        uint64_t blocks = (threads + 255) / 256;
        k_sweep_site<T, EXACT, R><<<(unsigned)blocks, 256, 0, st>>>(b, site_ref, total, rank,
                                                                    status, ctr);
        return cudaGetLastError();
    }
};

template <class T, bool EXACT, int R>
struct SweepTiledL {
    static cudaError_t run(const BatchDev& b, uint32_t max_nx, uint32_t max_ny, uint32_t stride,
                           SiteRank* rank, uint8_t* status, RefCounters* ctr, cudaStream_t st) {
        constexpr int W = 2 * R + 1;
        int PX = (kTileX - 1) * (int)stride + W, PY = (kTileY - 1) * (int)stride + W;
        size_t smem = sizeof(double) * 3 * (size_t)PY * kTileX +
                      sizeof(float) * (2 * (size_t)PX * PY + kMaxSources * 256 +
                                       kMaxSources * 12 + kMaxPlanes);
        auto kern = k_sweep_tiled<T, R>;
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        dim3 grid((max_nx + kTileX - 1) / kTileX, (max_ny + kTileY - 1) / kTileY, b.n_refs);
        kern<<<grid, 256, smem, st>>>(b, 0, rank, status, ctr);
        return cudaGetLastError();
    }
};

template <class T, bool EXACT, int R>
struct ReciprocalL {
    static cudaError_t run(const BatchDev& b, const Cand* cands, const uint32_t* count,
                           RecipObs* obs, RefCounters* ctr, cudaStream_t st) {
        k_reciprocal<T, EXACT, R><<<sm_count() * 8, 256, 0, st>>>(b, cands, count, obs, ctr);
        return cudaGetLastError();
    }
};

template <class T, bool EXACT, int R>
struct ProposeL {
    static cudaError_t run(const BatchDev& b, int pass, uint64_t total, const uint32_t* site_ref,
                           const int32_t* occ, const OutPoint* pool, uint8_t* prop_status,
                           Cand* prop, RefCounters* ctr, cudaStream_t st) {
        uint64_t blocks = (total + 127) / 128;
        if (blocks > (uint64_t)sm_count() * 64) blocks = (uint64_t)sm_count() * 64;
        if (blocks == 0) blocks = 1;
        k_propose<T, EXACT, R><<<(unsigned)blocks, 128, 0, st>>>(b, pass, total, site_ref, occ,
                                                                 pool, prop_status, prop, ctr);
        return cudaGetLastError();
    }
};

unsigned grid_for(uint64_t cap, int threads) {
    uint64_t blocks = (cap + threads - 1) / threads;
    uint64_t lim = (uint64_t)sm_count() * 16;
    if (blocks > lim) blocks = lim;
    if (blocks == 0) blocks = 1;
    return (unsigned)blocks;
}

}  // namespace

cudaError_t launch_luma(const uint8_t* rgba, uint8_t* luma, size_t pixels, cudaStream_t stream) {
    if (!pixels) return cudaSuccess;
    k_luma<<<grid_for(pixels, 256), 256, 0, stream>>>(reinterpret_cast<const uchar4*>(rgba), luma,
                                                      pixels);
    return cudaGetLastError();
}

cudaError_t launch_site_ref(const uint64_t* site_off, int32_t n_refs, uint64_t total_sites,
                            uint32_t* site_ref, cudaStream_t stream) {
    if (!total_sites) return cudaSuccess;
    k_site_ref<<<grid_for(total_sites, 256), 256, 0, stream>>>(site_off, n_refs, total_sites,
                                                               site_ref);
    return cudaGetLastError();
}

cudaError_t launch_sweep_dispatch(const BatchDev& b, const uint32_t* site_ref, uint64_t total_sites,
                                  uint32_t max_nx, uint32_t max_ny, uint32_t uniform_stride,
                                  bool tiled, SiteRank* rank, uint8_t* status,
                                  RefCounters* counters, cudaStream_t stream) {
    if (!total_sites) return cudaSuccess;
    if (tiled)
        return dispatch<SweepTiledL>(b.storage, false, b.prof.radius, b, max_nx, max_ny,
                                     uniform_stride, rank, status, counters, stream);
    return dispatch<SweepSiteL>(b.storage, b.exact, b.prof.radius, b, site_ref, total_sites, rank,
                                status, counters, stream);
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
    k_compact_count<<<(unsigned)blocks, kCompactThreads, 0, stream>>>(flags, value, n, bc);
    k_compact_scan<<<1, 1024, 0, stream>>>(bc, (uint32_t)blocks, count_dev);
    k_compact_scatter<<<(unsigned)blocks, kCompactThreads, 0, stream>>>(flags, value, n, bc,
                                                                        out_idx);
    return cudaGetLastError();
}

cudaError_t launch_make_primary_cands(const BatchDev& b, const uint32_t* site_idx,
                                      const uint32_t* count_dev, uint64_t cap,
                                      const uint32_t* site_ref, const SiteRank* rank, Cand* cands,
                                      cudaStream_t stream) {
    k_make_primary_cands<<<grid_for(cap, 256), 256, 0, stream>>>(b, site_idx, count_dev, site_ref,
                                                                  rank, cands);
    return cudaGetLastError();
}

cudaError_t launch_reciprocal(const BatchDev& b, const Cand* cands, const uint32_t* count_dev,
                              uint64_t /*cap*/, RecipObs* obs, RefCounters* counters,
                              cudaStream_t stream) {
    return dispatch<ReciprocalL>(b.storage, b.exact, b.prof.radius, b, cands, count_dev, obs,
                                 counters, stream);
}

cudaError_t launch_fuse(const BatchDev& b, const Cand* cands, const uint32_t* count_dev,
                        uint64_t cap, const RecipObs* obs, bool completion, int pass,
                        OutPoint* out, uint8_t* cand_status, RefCounters* counters,
                        cudaStream_t stream) {
    k_fuse<<<grid_for(cap, 128), 128, 0, stream>>>(b, cands, count_dev, obs, completion ? 1 : 0,
                                                   pass, out, cand_status, counters);
    return cudaGetLastError();
}

cudaError_t launch_append(const uint32_t* idx, const uint32_t* count_dev, uint64_t cap,
                          const OutPoint* src, OutPoint* pool, uint32_t* pool_size,
                          uint32_t* segment_end, cudaStream_t stream) {
    k_append<<<grid_for(cap, 256), 256, 0, stream>>>(idx, count_dev, src, pool, pool_size);
    k_bump<<<1, 1, 0, stream>>>(pool_size, count_dev, segment_end);
    return cudaGetLastError();
}

cudaError_t launch_occupancy_clear(int32_t* occ, uint64_t total_sites, cudaStream_t stream) {
    if (!total_sites) return cudaSuccess;
    k_fill<<<grid_for(total_sites, 256), 256, 0, stream>>>(occ, total_sites, -1);
    return cudaGetLastError();
}

cudaError_t launch_occupy(const BatchDev& b, const OutPoint* pool, const uint32_t* begin,
                          const uint32_t* end, uint64_t cap, int32_t* occ, cudaStream_t stream) {
    k_occupy<<<grid_for(cap, 256), 256, 0, stream>>>(b, pool, begin, end, occ);
    return cudaGetLastError();
}

cudaError_t launch_propose(const BatchDev& b, int pass, uint64_t total_sites,
                           const uint32_t* site_ref, const int32_t* occ, const OutPoint* pool,
                           uint8_t* prop_status, Cand* prop_cand, RefCounters* counters,
                           cudaStream_t stream) {
    if (!total_sites) return cudaSuccess;
    return dispatch<ProposeL>(b.storage, b.exact, b.prof.radius, b, pass, total_sites, site_ref,
                              occ, pool, prop_status, prop_cand, counters, stream);
}

cudaError_t launch_gather_cands(const uint32_t* idx, const uint32_t* count_dev, uint64_t cap,
                                const Cand* src, Cand* dst, cudaStream_t stream) {
    k_gather_cands<<<grid_for(cap, 256), 256, 0, stream>>>(idx, count_dev, src, dst);
    return cudaGetLastError();
}

}  // namespace v3d
