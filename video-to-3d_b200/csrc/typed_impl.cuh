// Storage-typed kernels of the dense pass: the depth sweeps, the reciprocal
// check and the completion proposals, templated on the pixel storage type T,
// the exactness policy, the window radius R and (fast policy) the cost.
// typed_<type>.cu instantiate one storage type each so the kernels compile in
// parallel; pass_kernels.cu dispatches to them.
#pragma once

#include <map>
#include <mutex>
#include <utility>

#include "pass_kernels.cuh"
#include "typed.cuh"

namespace v3d {
namespace typed_detail {

// The tiled sweep's CTA: one thread per grid site of a TX x TY tile (32x8 or
// 16x16), eight warps.
constexpr int kTileThreads = 256;
constexpr int kTileWarps = kTileThreads / 32;
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
template <class T, int R, int COST>
__device__ __forceinline__ bool window_cost_fast(const DevProfile& prof, const float* pv,
                                                 float pmean, float pvar, const float* H,
                                                 float zmin, const DevImage& img, float x, float y,
                                                 float& cost) {
    constexpr int W = 2 * R + 1;
    constexpr int N = W * W;
    const T* data = static_cast<const T*>(img.data);
    const uint32_t w = img.width, h = img.height;
    if (COST == 1) {
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

// Bilinear sample at a non-negative coordinate below 2^22 (the caller checks
// the domain).  floor() is one round-down add of 2^23, which leaves floor(u)
// in the low mantissa bits: the same floor, integer and fraction as floorf.
template <class T>
__device__ __forceinline__ float sample_nonneg(const T* __restrict__ p, uint32_t w, float u,
                                               float v) {
    constexpr float kShift = 8388608.0f;  // 2^23
    const float tu = __fadd_rd(u, kShift), tv = __fadd_rd(v, kShift);
    const float fu = tu - kShift, fv = tv - kShift;
    const uint32_t ix = (uint32_t)(__float_as_int(tu) - __float_as_int(kShift));
    const uint32_t iy = (uint32_t)(__float_as_int(tv) - __float_as_int(kShift));
    const float tx = u - fu, ty = v - fv;
    // 32-bit element offsets (frames hold fewer than 2^32 pixels): each row's
    // address is then one wide multiply-add from the image base
    const uint32_t o0 = iy * w + ix, o1 = o0 + w;
    const float v00 = pix<T>(p + o0, 0), v10 = pix<T>(p + o0, 1);
    const float v01 = pix<T>(p + o1, 0), v11 = pix<T>(p + o1, 1);
    const float top = fmaf(v10 - v00, tx, v00);
    const float bot = fmaf(v11 - v01, tx, v01);
    return fmaf(bot - top, ty, top);
}



// Packed f32x2 forms (sm_100): each component is computed exactly as the
// scalar form with the same rounding.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

// The approximate reciprocal of the special-function unit, as __fdividef(1, x)
// computes it for the normal, positive denominators the sweeps pass.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

template <class T>
__device__ __forceinline__ float2 sample_nonneg_pair(const T* __restrict__ p, uint32_t w, float2 u,
                                                     float2 v) {
    const float2 shift = f2(8388608.0f, 8388608.0f);  // 2^23, as in sample_nonneg
    const float2 tu = __fadd2_rd(u, shift), tv = __fadd2_rd(v, shift);
    const float2 fu = __fadd2_rn(tu, neg2(shift)), fv = __fadd2_rn(tv, neg2(shift));
    const int sb = __float_as_int(8388608.0f);
    const uint32_t ixa = (uint32_t)(__float_as_int(tu.x) - sb), ixb = (uint32_t)(__float_as_int(tu.y) - sb);
    const uint32_t iya = (uint32_t)(__float_as_int(tv.x) - sb), iyb = (uint32_t)(__float_as_int(tv.y) - sb);
    const float2 tx = __fadd2_rn(u, neg2(fu)), ty = __fadd2_rn(v, neg2(fv));
    const uint32_t oa = iya * w + ixa, ob = iyb * w + ixb;  // as in sample_nonneg
    const T *qa0 = p + oa, *qb0 = p + ob, *qa1 = p + (oa + w), *qb1 = p + (ob + w);
    const float2 v00 = f2(pix<T>(qa0, 0), pix<T>(qb0, 0));
    const float2 v10 = f2(pix<T>(qa0, 1), pix<T>(qb0, 1));
    const float2 v01 = f2(pix<T>(qa1, 0), pix<T>(qb1, 0));
    const float2 v11 = f2(pix<T>(qa1, 1), pix<T>(qb1, 1));
    const float2 top = __ffma2_rn(__fadd2_rn(v10, neg2(v00)), tx, v00);
    const float2 bot = __ffma2_rn(__fadd2_rn(v11, neg2(v01)), tx, v01);
    return __ffma2_rn(__fadd2_rn(bot, neg2(top)), ty, top);
}

// ---- sweep, warp per site ----------------------------------------------------
// Lanes take hypotheses lane, lane+32, ...; each lane keeps the running
// best/second state, and a warp merge reproduces the reference's sort.
template <class T, bool EXACT, int R, int COST>
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
    for (int k = lane; k < ref.planes; k += 32) {
        const double depth = hypothesis_depth(k, ref.planes, ref.search_min, ref.search_max);
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
                ok = window_cost_fast<T, R, COST>(prof, pv, pmean, pvar, H, zmin_of(inv), src.img,
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

// True when every point (X, Y) of the rectangle [xa, xb] x [ya, yb] maps
// through H, by the per-tap f32 formula of the sweeps (h2 = H6 X + (H7 Y + H8),
// u = (H0 X + (H1 Y + H2)) / h2, v likewise), to a denominator above zmin and
// into [0, wl) x [0, hl).  The denominator is affine, so its minimum over the
// rectangle is at a corner, and a projective map with a positive denominator
// keeps the rectangle inside the hull of its mapped corners; the margins bound
// the f32 rounding of any point's evaluation (a few ulp of the magnitudes
// involved, taken at 2^-20 relative).
__device__ __forceinline__ bool rect_inside(const float* H, float zmin, float wl, float hl,
                                            float xa, float xb, float ya, float yb) {
    const float ax = fmaxf(fabsf(xa), fabsf(xb)), ay = fmaxf(fabsf(ya), fabsf(yb));
    const float su = fmaf(fabsf(H[0]), ax, fmaf(fabsf(H[1]), ay, fabsf(H[2])));
    const float sv = fmaf(fabsf(H[3]), ax, fmaf(fabsf(H[4]), ay, fabsf(H[5])));
    const float sz = fmaf(fabsf(H[6]), ax, fmaf(fabsf(H[7]), ay, fabsf(H[8])));
    constexpr float kRel = 9.5367431640625e-07f;  // 2^-20
    float hmin = 3.0e38f, umin = 3.0e38f, vmin = 3.0e38f, umax = -3.0e38f, vmax = -3.0e38f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float X = (c & 1) ? xb : xa;
        const float Y = (c & 2) ? yb : ya;
        const float h2 = fmaf(H[6], X, fmaf(H[7], Y, H[8]));
        const float iv = rcp_approx(h2);
        const float u = fmaf(H[0], X, fmaf(H[1], Y, H[2])) * iv;
        const float v = fmaf(H[3], X, fmaf(H[4], Y, H[5])) * iv;
        hmin = fminf(hmin, h2);
        umin = fminf(umin, u);
        umax = fmaxf(umax, u);
        vmin = fminf(vmin, v);
        vmax = fmaxf(vmax, v);
    }
    if (!(hmin > zmin + kRel * sz) || !(hmin > 0.f)) return false;
    const float m = 0.015625f + kRel * (fmaxf(su, sv) + fmaxf(wl, hl) * sz) / hmin;
    // NaN fails every comparison
    return umin >= m && vmin >= m && umax <= wl - m && vmax <= hl - m;
}

// Pair-steps of the tiled sweep's warp step per warp: every step of the
// CTA's warps covers 64 footprint slots each.
__host__ __device__ constexpr int tiled_steps(int np) { return (np + 2 * kTileThreads - 1) / (2 * kTileThreads); }

// ---- sweep, tiled ZNCC (fast policy) -----------------------------------------
// A CTA owns a TX x TY block of grid sites (32x8 or 16x16, the tuner's pick;
// the f64 window sums are formed tap by tap in the same order whatever the
// tile, so the shape never changes a result).  For every (plane, source) it warps
// the block's pixel footprint into the source once (f32 homography and f32
// bilinear), then forms the window sums of s, s^2 and r*s with separable box
// filters, so overlapping windows (stride < window) share every bilinear
// sample.  Products and sums are formed in f64: s^2 - (sum s)^2/n cancels
// badly in f32 on low-variance windows (Acc = double; with Acc = float, the
// FAST32_SUMS32 policy, the sums are f32 on values shifted by the tile's
// centre reference texel, which keeps the shifted values near the windows'
// means).  Invalid taps are NaN and poison their windows, which reproduces
// the reference's all-taps-valid rule.
//
// The footprint rows in shared memory keep their columns grouped by x mod
// stride (column x at slot (x % s) * PXs + x / s), so the stride-s reads of
// the horizontal box filter fall on consecutive words across the lanes.  The
// warp step runs over the flat footprint (slot f = row * PXp + column slot),
// 64 slots per warp and step with packed f32x2 arithmetic, their coordinates
// from a per-CTA table, so it converts no integers and leaves no lanes idle at
// row ends.  When the footprint's image in a source lies inside that image
// (tested once per plane and source on the rectangle's corners), the step
// skips the per-sample domain tests.
template <class T, int R, class Acc, int TX, int S>
__global__ void __launch_bounds__(kTileThreads, (S && R >= 4) ? 3 : 1024 / kTileThreads) k_sweep_tiled(BatchDev b, uint64_t total_sites,
                                                     SiteRank* __restrict__ rank,
                                                     uint8_t* __restrict__ status,
                                                     RefCounters* __restrict__ ctr, int n_chunks,
                                                     Rank* __restrict__ partial) {
    constexpr int W = 2 * R + 1;
    constexpr int N = W * W;
    constexpr int TY = kTileThreads / TX;
    extern __shared__ double smem_d[];
    // blockIdx.z = reference x plane chunk; the chunk sweeps planes [k0, k1)
    const uint32_t r = blockIdx.z / (uint32_t)n_chunks;
    const int chunk = (int)(blockIdx.z - r * (uint32_t)n_chunks);
    const DevReference& ref = b.refs[r];
    const DevProfile& prof = b.prof;
    const uint32_t gx0 = blockIdx.x * TX, gy0 = blockIdx.y * TY;
    if (gx0 >= ref.nx || gy0 >= ref.ny) return;
    const int per_chunk = (ref.planes + n_chunks - 1) / n_chunks;
    const int k0 = chunk * per_chunk, k1 = min(ref.planes, k0 + per_chunk);
    // S, when not 0, is the batch's grid stride at compile time (the tiled sweep
    // runs batches of one stride), so the footprint's shape and every tap
    // offset of the box filters fold into constants
    const int s = S ? S : (int)ref.stride;
    const int PX = (TX - 1) * s + W, PY = (TY - 1) * s + W;
    const int PXs = (PX + s - 1) / s, PXp = PXs * s;  // columns per residue, padded row
    const int np = PY * PXp;
    const int ms = b.max_src;
    Acc* hs = reinterpret_cast<Acc*>(smem_d);  // [PY][TX] row sums of s
    Acc* hss = hs + PY * TX;                   // [PY][TX] row sums of s^2
    Acc* hrs = hss + PY * TX;                  // [PY][TX] row sums of r*s
    float* refv = reinterpret_cast<float*>(hrs + PY * TX);  // [PY][PXp] reference values
    float* samp = refv + np;                 // [PY][PXp] source samples (NaN = invalid)
    float* costs = samp + np;                // [max_src][kTileThreads]
    float* hA = costs + ms * kTileThreads;   // [max_src][12] homography parts
    float* pinv = hA + ms * 12;              // [planes] inverse depths
    uint32_t* inmask = reinterpret_cast<uint32_t*>(pinv + b.prof.planes);  // [planes] inside sources
    int* rowmap = reinterpret_cast<int*>(inmask + b.prof.planes);  // [PY] horizontal pass rows
    // [steps * kTileY][32] (x_a, x_b, y_a, y_b) of the slots f and f + 32 of each lane step
    float4* slotxy = reinterpret_cast<float4*>(
        (reinterpret_cast<uintptr_t>(rowmap + PY) + 15) & ~(uintptr_t)15);
    const int n_steps = tiled_steps(np);
    const int tid = threadIdx.x;
    const T* rdata = static_cast<const T*>(ref.img.data);
    const int px0 = (int)(ref.border + gx0 * s) - R, py0 = (int)(ref.border + gy0 * s) - R;
    // padding slots (column PX and beyond) and slots past the footprint take
    // the footprint's last column: their samples are never read, and the
    // coordinates stay inside the rectangle that the inside test covers
    auto slot_xy = [&](int f, float& X, float& Y) {
        int yy = 0, x = PX - 1;
        if (f < np) {
            yy = f / PXp;
            const int t = f - yy * PXp;
            x = min((t % PXs) * s + t / PXs, PX - 1);
        }
        X = (float)(px0 + x);
        Y = (float)(py0 + yy);
    };
    for (int i = tid; i < n_steps * kTileThreads; i += kTileThreads) {
        const int fa = (i >> 5) * 64 + (i & 31);
        float4 e;
        slot_xy(fa, e.x, e.z);
        slot_xy(fa + 32, e.y, e.w);
        slotxy[i] = e;
    }
    for (int i = tid; i < np; i += kTileThreads) {
        const int yy = i / PXp, t = i - yy * PXp;
        const int x = (t % PXs) * s + t / PXs;
        const int X = px0 + x, Y = py0 + yy;
        float v = __int_as_float(0x7fc00000);
        if (x < PX && X >= 0 && Y >= 0 && X < (int)ref.img.width && Y < (int)ref.img.height)
            v = pix<T>(rdata, (size_t)Y * ref.img.width + X);
        refv[i] = v;
    }
    const int n_src = ref.n_src;
    for (int i = tid; i < n_src * 12; i += kTileThreads) {
        int j = i / 12, c = i - j * 12;
        hA[i] = c < 9 ? ref.src[j].fwd_A[c] : ref.src[j].fwd_b[c - 9];
    }
    for (int k = tid; k < ref.planes; k += kTileThreads)
        pinv[k] = (float)ddiv(1.0, hypothesis_depth(k, ref.planes, ref.search_min, ref.search_max));
    // sources whose image of the footprint rectangle lies inside, per plane of the chunk
    for (int kk = tid; kk < k1 - k0; kk += kTileThreads) {
        const float inv = (float)ddiv(1.0, hypothesis_depth(k0 + kk, ref.planes, ref.search_min,
                                                             ref.search_max));
        uint32_t m = 0;
        for (int j = 0; j < n_src; ++j) {
            const DevSource& sj = ref.src[j];
            const float H[9] = {sj.fwd_A[0], sj.fwd_A[1], fmaf(inv, sj.fwd_b[0], sj.fwd_A[2]),
                                sj.fwd_A[3], sj.fwd_A[4], fmaf(inv, sj.fwd_b[1], sj.fwd_A[5]),
                                sj.fwd_A[6], sj.fwd_A[7], fmaf(inv, sj.fwd_b[2], sj.fwd_A[8])};
            if (rect_inside(H, 1.0e-4f * inv, (float)(sj.img.width - 1), (float)(sj.img.height - 1),
                            (float)px0, (float)(px0 + PX - 1), (float)py0, (float)(py0 + PY - 1)))
                m |= 1u << j;
        }
        inmask[kk] = m;
    }
    // The horizontal pass of a 16-wide tile gives a warp's half-warps two rows;
    // rows pd apart, pd x PXp = 16 (mod 32) words, fall on the two halves of the
    // banks.  Rows pair up in blocks of 2 pd (the rows of a last partial block
    // in order); the row sums land at their own rows either way.
    if (TX == 16) {
        int pd = 0;
        for (int d = 1; d < 32 && !pd; ++d)
            if ((d * PXp) % 32 == 16) pd = d;
        for (int q = tid; q < PY; q += kTileThreads) {
            int row = q;
            if (pd) {
                const int blk = 2 * pd, bq = q / blk;
                if ((bq + 1) * blk <= PY) {
                    const int w = q - bq * blk;
                    row = bq * blk + (w >> 1) + (w & 1) * pd;
                }
            }
            rowmap[q] = row;
        }
    }
    // slot of tap dx of the window that starts at column 0 (add the window's start)
    int toff[W];
#pragma unroll
    for (int dx = 0; dx < W; ++dx) toff[dx] = (dx % s) * PXs + dx / s;
    __syncthreads();

    const int tx = tid % TX, ty = tid / TX;         // this thread's site in the tile
    const int lane = tid & 31, wid = tid >> 5;      // its place in the flat warp step
    const uint32_t gx = gx0 + tx, gy = gy0 + ty;
    const bool active = gx < ref.nx && gy < ref.ny;
    const uint64_t gsite = b.site_off[r] + (uint64_t)gy * ref.nx + gx;
    // reference window statistics and the contrast gate on exact pixel values
    double sr = 0.0, srr = 0.0;
    bool sampled = false;
    if (active) {
        float mn = 3.0e38f, mx = -3.0e38f;
        for (int dy = 0; dy < W; ++dy)
#pragma unroll
            for (int dx = 0; dx < W; ++dx) {
                float v = refv[(ty * s + dy) * PXp + toff[dx] + tx];
                mn = fminf(mn, v);
                mx = fmaxf(mx, v);
                sr += (double)v;
                srr = fma((double)v, (double)v, srr);
            }
        double contrast = (double)mx - (double)mn;
        sampled = contrast >= prof.min_contrast;
        if (chunk == 0) {  // one chunk records the gate
            if (!sampled) status[gsite] = kSiteLowContrast;
            else atomicAdd(&ctr[r].sampled, 1ull);
        }
    }
    const double n = (double)N;
    const double inv_n = 1.0 / n;
    const double vr = srr - sr * sr / n;
    const double minvar_n = prof.min_variance * n;
    const bool vr_ok = vr > 0.0 && vr >= minvar_n;
    const float vr_f = (float)vr;
    // f32 sums: every value shifted by the centre texel of the tile's middle
    // active site (cov and var are shift-invariant; the site is inside the
    // grid, so the texel is a pixel of the image); f64 sums: no shift
    constexpr bool kF32 = sizeof(Acc) == 4;
    float shift = 0.f;
    if (kF32) {
        const int cx = R + (int)min((uint32_t)TX / 2u, ref.nx - gx0 - 1) * s;
        const int cy = R + (int)min((uint32_t)TY / 2u, ref.ny - gy0 - 1) * s;
        shift = refv[cy * PXp + (cx % s) * PXs + cx / s];
    }
    const float sr_shift = (float)(sr - n * (double)shift);
    const float inv_nf = 1.0f / (float)N, minvar_nf = (float)minvar_n;
    // the reference taps of this thread's first horizontal windows, the same
    // for every plane and source: the stride-2 instantiation keeps one window's
    // in registers at four blocks an SM, and for 9x9 windows three blocks an SM
    // with three windows' taps (its measured best)
    constexpr int kRegWindows = S ? (R >= 4 ? 3 : 1) : 0;
    float rreg[(kRegWindows ? kRegWindows : 1) * W];
#pragma unroll
    for (int w = 0; w < kRegWindows; ++w) {
        const int i0 = tid + w * kTileThreads, i = i0 < PY * TX ? i0 : 0;
        const int yy = TX == 16 ? rowmap[i / TX] : i / TX;
        const float* rp = refv + yy * PXp + i % TX;
#pragma unroll
        for (int dx = 0; dx < W; ++dx) rreg[w * W + dx] = rp[toff[dx]];
    }
    Rank st = rank_empty();
    for (int k = k0; k < k1; ++k) {
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
            // the flat footprint, slots fa and fa + 32 per lane and step; the
            // reciprocal from the approximate unit; each component of the packed
            // arithmetic is the scalar computation, bit for bit
            const bool inside = (inmask[k - k0] >> j) & 1u;
            const float a0 = A[0], a1 = A[1], a3 = A[3], a4 = A[4], a6 = A[6], a7 = A[7];
            // inside the source: two pair-steps at a time, both steps' gathers
            // issued before either step's stores (every slot of the table has
            // coordinates inside the footprint rectangle, so a step past the
            // footprint samples harmlessly and only its stores are skipped)
            int p0 = 0;
            if (inside && R < 4) {
                auto step = [&](int ws) {
                    const float4 e = slotxy[ws * 32 + lane];
                    const float2 X2 = f2(e.x, e.y), Y2 = f2(e.z, e.w);
                    const float2 hx = __ffma2_rn(f2(a1, a1), Y2, f2(H2, H2));
                    const float2 hy = __ffma2_rn(f2(a4, a4), Y2, f2(H5, H5));
                    const float2 hz = __ffma2_rn(f2(a7, a7), Y2, f2(H8, H8));
                    const float2 h2 = __ffma2_rn(f2(a6, a6), X2, hz);
                    const float2 iv = f2(rcp_approx(h2.x), rcp_approx(h2.y));
                    const float2 u = __fmul2_rn(__ffma2_rn(f2(a0, a0), X2, hx), iv);
                    const float2 q = __fmul2_rn(__ffma2_rn(f2(a3, a3), X2, hy), iv);
                    return sample_nonneg_pair<T>(sdata, si.width, u, q);
                };
                for (; p0 + 1 < n_steps; p0 += 2) {
                    const int ws0 = p0 * kTileWarps + wid, ws1 = ws0 + kTileWarps;
                    const int fa0 = ws0 * 64 + lane, fa1 = ws1 * 64 + lane;
                    if (fa0 >= np) break;
                    const float2 s0 = step(ws0), s1 = step(ws1);
                    samp[fa0] = s0.x;
                    if (fa0 + 32 < np) samp[fa0 + 32] = s0.y;
                    if (fa1 < np) samp[fa1] = s1.x;
                    if (fa1 + 32 < np) samp[fa1 + 32] = s1.y;
                }
            }
            for (int p = p0; p < n_steps; ++p) {
                const int ws = p * kTileWarps + wid;
                const int fa = ws * 64 + lane;
                if (fa >= np) break;
                const int fb = fa + 32;
                const float4 e = slotxy[ws * 32 + lane];
                const float2 X2 = f2(e.x, e.y), Y2 = f2(e.z, e.w);
                const float2 hx = __ffma2_rn(f2(a1, a1), Y2, f2(H2, H2));
                const float2 hy = __ffma2_rn(f2(a4, a4), Y2, f2(H5, H5));
                const float2 hz = __ffma2_rn(f2(a7, a7), Y2, f2(H8, H8));
                const float2 h2 = __ffma2_rn(f2(a6, a6), X2, hz);
                const float2 iv = f2(rcp_approx(h2.x), rcp_approx(h2.y));
                const float2 u = __fmul2_rn(__ffma2_rn(f2(a0, a0), X2, hx), iv);
                const float2 q = __fmul2_rn(__ffma2_rn(f2(a3, a3), X2, hy), iv);
                float va = __int_as_float(0x7fc00000), vb = va;
                if (inside) {
                    const float2 sv = sample_nonneg_pair<T>(sdata, si.width, u, q);
                    va = sv.x;
                    vb = sv.y;
                } else {
                    const bool ia = h2.x > zmin && u.x >= 0.f && q.x >= 0.f && u.x < wl && q.x < hl;
                    const bool ib = h2.y > zmin && u.y >= 0.f && q.y >= 0.f && u.y < wl && q.y < hl;
                    if (ia && ib) {
                        const float2 sv = sample_nonneg_pair<T>(sdata, si.width, u, q);
                        va = sv.x;
                        vb = sv.y;
                    } else {
                        if (ia) va = sample_nonneg<T>(sdata, si.width, u.x, q.x);
                        if (ib) vb = sample_nonneg<T>(sdata, si.width, u.y, q.y);
                    }
                }
                samp[fa] = va;
                if (fb < np) samp[fb] = vb;
            }
            __syncthreads();
            // horizontal box filter: the window of column c of row yy at slot c,
            // TX windows a row (a warp takes one row of 32, or two rows of 16)
            // (a thread's first window takes its reference taps from registers)
            auto hwindow = [&](int i, const float* rtap) {
                const int c = i % TX;
                const int yy = TX == 16 ? rowmap[i / TX] : i / TX;
                const int o = yy * TX + c;
                const float* sp = samp + yy * PXp + c;
                const float* rp = refv + yy * PXp + c;
                if (kF32) {
                    // (sum s, sum s^2) as one packed FMA a tap: (s, s) * (1, s) + acc
                    float2 ab = f2(0.f, 0.f);
                    float c = 0.f;
#pragma unroll
                    for (int dx = 0; dx < W; ++dx) {
                        const float v = sp[toff[dx]] - shift;
                        ab = __ffma2_rn(f2(v, v), f2(1.0f, v), ab);
                        c = fmaf((rtap ? rtap[dx] : rp[toff[dx]]) - shift, v, c);
                    }
                    hs[o] = (Acc)ab.x;
                    hss[o] = (Acc)ab.y;
                    hrs[o] = (Acc)c;
                } else {
                    double a = 0.0, bb = 0.0, c = 0.0;
#pragma unroll
                    for (int dx = 0; dx < W; ++dx) {
                        const double v = (double)sp[toff[dx]];
                        a += v;
                        bb = fma(v, v, bb);
                        c = fma((double)(rtap ? rtap[dx] : rp[toff[dx]]), v, c);
                    }
                    hs[o] = (Acc)a;
                    hss[o] = (Acc)bb;
                    hrs[o] = (Acc)c;
                }
            };
#pragma unroll
            for (int w = 0; w < kRegWindows; ++w)
                if (tid + w * kTileThreads < PY * TX) hwindow(tid + w * kTileThreads, rreg + w * W);
            for (int i = tid + kRegWindows * kTileThreads; i < PY * TX; i += kTileThreads) hwindow(i, nullptr);
            __syncthreads();
            if (sampled) {
                float cost = __int_as_float(0x7fc00000);
                if (kF32) {
                    float a = 0.f, bb = 0.f, c = 0.f;
#pragma unroll
                    for (int dy = 0; dy < W; ++dy) {
                        const int i = (ty * s + dy) * TX + tx;
                        a += (float)hs[i];
                        bb += (float)hss[i];
                        c += (float)hrs[i];
                    }
                    const float vs = bb - a * a * inv_nf;
                    const float cov = c - sr_shift * a * inv_nf;
                    if (vs > 0.f && vs >= minvar_nf && vr_ok) cost = 1.0f - cov * rsqrtf(vr_f * vs);
                } else {
                    double a = 0.0, bb = 0.0, c = 0.0;
#pragma unroll
                    for (int dy = 0; dy < W; ++dy) {
                        const int i = (ty * s + dy) * TX + tx;
                        a += (double)hs[i];
                        bb += (double)hss[i];
                        c += (double)hrs[i];
                    }
                    // the cancelling differences in f64, the ratio in f32
                    const double vs = bb - a * a * inv_n;
                    const double cov = c - sr * a * inv_n;
                    if (vs > 0.0 && vs >= minvar_n && vr_ok)
                        cost = 1.0f - (float)cov * rsqrtf(vr_f * (float)vs);
                }
                costs[j * kTileThreads + tid] = cost;  // NaN when invalid
            }
        }
        if (sampled) {
            // the passing source costs, compacted and sorted in this thread's column
            float* col = costs + tid;
            int cnt = 0;
            for (int j = 0; j < n_src; ++j) {
                const float c = col[j * kTileThreads];
                if ((double)c <= prof.max_error) col[(cnt++) * kTileThreads] = c;
            }
            if (cnt > 0) {
                for (int i = 1; i < cnt; ++i) {
                    const float x = col[i * kTileThreads];
                    int m = i - 1;
                    while (m >= 0 && col[m * kTileThreads] > x) {
                        col[(m + 1) * kTileThreads] = col[m * kTileThreads];
                        --m;
                    }
                    col[(m + 1) * kTileThreads] = x;
                }
                Rank c;
                c.support = cnt;
                c.plane = k;
                c.error = (double)col[(cnt / 2) * kTileThreads];
                c.second = kInf;
                st = rank_merge(st, c);
            }
        }
    }
    if (!sampled) return;
    if (n_chunks > 1) {
        partial[(uint64_t)chunk * total_sites + gsite] = st;
        if (chunk == 0) status[gsite] = kSitePending;
        return;
    }
    finish_site(st, prof, gsite, rank, status);
}

// ---- reciprocal check, warp per (candidate, source) ----------------------------
// reciprocal_depth_observations (dense_legacy.rs:777-857) for one source:
// direct cost at the re-projected reference position, projection into the
// source, then estimate_single_view_depth (dense_legacy.rs:887-949) with lanes
// over the source's hypotheses, and the reciprocal agreement test.
template <class T, int R>
__global__ void __launch_bounds__(256) k_reciprocal_exact(BatchDev b, const Cand* __restrict__ cands,
                                                    const uint32_t* __restrict__ count,
                                                    RecipObs* __restrict__ obs,
                                                    RefCounters* __restrict__ ctr) {
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
            if (lane == 0)
                dok = patch_error_exact<T>(prof, ref.cam, ref.img, src.cam, src.img, ref.focal,
                                           rp.x, rp.y, rp.z, de);
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
            double be = kInf;
            int bk = 0x7fffffff;
            if (ok && lane == 0) atomicAdd(&ctr[cd.ref].recip_evals, (unsigned long long)ref.planes);
            for (int k = lane; ok && k < ref.planes; k += 32) {
                double d = hypothesis_depth(k, ref.planes, src.search_min, src.search_max);
                double e;
                const bool eok = patch_error_exact<T>(prof, src.cam, src.img, ref.cam, ref.img,
                                                      ref.focal, sp.x, sp.y, d, e);
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
                double rd = hypothesis_depth(bk, ref.planes, src.search_min, src.search_max);
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

// ---- reciprocal check, fast policy ---------------------------------------------
// Same contract as k_reciprocal_exact for the fast policy, split in two
// kernels so that the single-view sweep, where the time goes, is not sized
// by the registers of the exact-f64 prologue:
//  * k_recip_prepare, one warp per candidate: its reference window once, then
//    per source the direct cost and the source contrast gate (f32 on the
//    exact f64 taps' texels and fractions, the exact f64 contrast where the
//    f32 one lies near the gate), lane-parallel over the window taps with warp
//    reductions (max/min are order-free, so the gate's decision is the exact
//    one).  A pair that passes parks its source pixel in its RecipObs slot
//    with valid = kObsPending;
//  * k_recip_sweep, one warp per pending pair, lanes over hypotheses:
//    re-samples the source window (the same f64 taps, so the same f32
//    values), sweeps every hypothesis and writes the final RecipObs.
//    Per hypothesis the four window corners are mapped first; when they land
//    inside the bilinear domain with a margin that covers f32 rounding, every
//    tap does (the denominator is affine, so its minimum over the window is at
//    a corner, and a projective map with a positive denominator keeps the
//    window inside the hull of its mapped corners) and the taps skip their
//    bounds tests.
constexpr int32_t kObsPending = 2;
// rounds of 32 lanes that cover the taps of the largest window (9x9)
constexpr int kTapRounds = ((2 * V3D_MAX_PATCH_RADIUS + 1) * (2 * V3D_MAX_PATCH_RADIUS + 1) + 31) / 32;

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// True when every tap (x + dx, y + dy), |dx|, |dy| <= R, maps through H to a
// point with denominator above zmin and inside [0, wl) x [0, hl), as the f32
// per-tap tests of window_cost would compute it.  The margins bound the f32
// rounding of the corner and of any inner tap (a few ulp of the magnitudes
// involved, taken at 2^-20 relative).
template <int R>
__device__ __forceinline__ bool window_inside(const float* H, float zmin, float wl, float hl,
                                              float x, float y) {
    const float ax = fabsf(x) + (float)R, ay = fabsf(y) + (float)R;
    const float su = fmaf(fabsf(H[0]), ax, fmaf(fabsf(H[1]), ay, fabsf(H[2])));
    const float sv = fmaf(fabsf(H[3]), ax, fmaf(fabsf(H[4]), ay, fabsf(H[5])));
    const float sz = fmaf(fabsf(H[6]), ax, fmaf(fabsf(H[7]), ay, fabsf(H[8])));
    constexpr float kRel = 9.5367431640625e-07f;  // 2^-20
    float hmin = 3.0e38f, umin = 3.0e38f, vmin = 3.0e38f, umax = -3.0e38f, vmax = -3.0e38f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        const float X = x + ((c & 1) ? (float)R : -(float)R);
        const float Y = y + ((c & 2) ? (float)R : -(float)R);
        const float h2 = fmaf(H[6], X, fmaf(H[7], Y, H[8]));
        const float iv = rcp_approx(h2);
        const float u = fmaf(H[0], X, fmaf(H[1], Y, H[2])) * iv;
        const float v = fmaf(H[3], X, fmaf(H[4], Y, H[5])) * iv;
        hmin = fminf(hmin, h2);
        umin = fminf(umin, u);
        umax = fmaxf(umax, u);
        vmin = fminf(vmin, v);
        vmax = fmaxf(vmax, v);
    }
    if (!(hmin > zmin + kRel * sz) || !(hmin > 0.f)) return false;
    const float m = 0.015625f + kRel * (fmaxf(su, sv) + fmaxf(wl, hl) * sz) / hmin;
    // NaN fails every comparison
    return umin >= m && vmin >= m && umax <= wl - m && vmax <= hl - m;
}

// Bilinear samplers of the reference image for the single-view sweep, both
// with the floor, fraction and texels of sample_nonneg:
//  * ImageSampler reads the image in global memory;
//  * BandSampler reads a staged box of it in shared memory (a warp's band,
//    rows of kBandPitch entries starting at image texel (x0, y0); entry c of a
//    row holds texel c and the difference texel c+1 - texel c, the f32
//    subtraction the bilinear step makes, so a tap reads four words and
//    starts its interpolation with an FMA).  The floor is the same round-down
//    add with the box origin folded into the shift: u + (2^23 - x0) rounded
//    down is 2^23 - x0 + floor(u) exactly, whose bits are 2^23's plus
//    floor(u) - x0, the band column; so the entry's 32-bit shared address is
//    one shift-add of each coordinate's bits onto a per-band constant (the
//    2^23 bits folded in, modulo 2^32).  The fraction u - floor(u) and the
//    texel values are the image's, so the two samplers agree bit for bit.
constexpr int kBandPitch = 64;  // entries per staged band row
constexpr int kBandRows = 20;   // staged band rows
constexpr int kBandRowShift = 9;  // log2 of a row's bytes (kBandPitch 8-byte entries)
static_assert(8 * kBandPitch == (1 << kBandRowShift), "band row bytes");

// Shared-memory loads at a 32-bit shared address.
__device__ __forceinline__ float lds_f32(uint32_t a) {
    float x;
    asm volatile("ld.shared.f32 %0, [%1];" : "=f"(x) : "r"(a));
    return x;
}
__device__ __forceinline__ float2 lds_f32x2(uint32_t a) {
    float2 x;
    asm volatile("ld.shared.v2.f32 {%0, %1}, [%2];" : "=f"(x.x), "=f"(x.y) : "r"(a));
    return x;
}


template <class T>
struct ImageSampler {
    const T* __restrict__ img;
    uint32_t w;
    __device__ __forceinline__ float operator()(float u, float v) const {
        return sample_nonneg<T>(img, w, u, v);
    }
    __device__ __forceinline__ float2 pair(float2 u, float2 v) const {
        return sample_nonneg_pair<T>(img, w, u, v);
    }
};

struct BandSampler {
    uint32_t cbase;  // shared address of the band minus (8 + 8 kBandPitch) x bits(2^23), mod 2^32
    float sx, sy;    // 2^23 - x0, 2^23 - y0
    __device__ BandSampler(const float2* band, float sx_, float sy_) : sx(sx_), sy(sy_) {
        const uint32_t sb = (uint32_t)__float_as_int(8388608.0f);
        cbase = (uint32_t)__cvta_generic_to_shared(band) - (8u + 8u * kBandPitch) * sb;
    }
    // shared address of the entry under (tu, tv), the rounded-down shifted coordinates
    __device__ __forceinline__ uint32_t entry(float tu, float tv) const {
        return cbase + ((uint32_t)__float_as_int(tv) << kBandRowShift) +
               ((uint32_t)__float_as_int(tu) << 3);
    }
    __device__ __forceinline__ float operator()(float u, float v) const {
        const float tu = __fadd_rd(u, sx), tv = __fadd_rd(v, sy);
        const float fu = tu - sx, fv = tv - sy;
        const uint32_t a = entry(tu, tv);
        const float tx = u - fu, ty = v - fv;
        constexpr uint32_t kRow = 1u << kBandRowShift;
        const float v00 = lds_f32(a), d0 = lds_f32(a + 4);
        const float v01 = lds_f32(a + kRow), d1 = lds_f32(a + kRow + 4);
        const float top = fmaf(d0, tx, v00);
        const float bot = fmaf(d1, tx, v01);
        return fmaf(bot - top, ty, top);
    }
    // two taps at once: each tap's entries come as one 8-byte load a row, the
    // row interpolations are scalar FMAs whose results form the packed operands
    // of the last step (the same operations as the scalar sampler, per tap)
    __device__ __forceinline__ float2 pair(float2 u, float2 v) const {
        const float2 s2x = f2(sx, sx), s2y = f2(sy, sy);
        const float2 tu = __fadd2_rd(u, s2x), tv = __fadd2_rd(v, s2y);
        const float2 fu = __fadd2_rn(tu, neg2(s2x)), fv = __fadd2_rn(tv, neg2(s2y));
        const uint32_t aa = entry(tu.x, tv.x), ab = entry(tu.y, tv.y);
        const float2 tx = __fadd2_rn(u, neg2(fu)), ty = __fadd2_rn(v, neg2(fv));
        constexpr uint32_t kRow = 1u << kBandRowShift;
        const float2 a0 = lds_f32x2(aa), a1 = lds_f32x2(aa + kRow);
        const float2 b0 = lds_f32x2(ab), b1 = lds_f32x2(ab + kRow);
        const float2 top = f2(fmaf(a0.y, tx.x, a0.x), fmaf(b0.y, tx.y, b0.x));
        const float2 bot = f2(fmaf(a1.y, tx.x, a1.x), fmaf(b1.y, tx.y, b1.x));
        return __ffma2_rn(__fadd2_rn(bot, neg2(top)), ty, top);
    }
};

// Window cost against the window centred on its mean pm (pvc, squared
// deviation pvar), sampling the image through H at taps (x + dx, y + dy);
// the samples are shifted by pm too before their sums, as in the direct cost.  CHECK runs the
// per-tap domain tests; without it the caller has established the domain
// (window_inside, or the band box of every hypothesis).  The window rows run
// as a rolled loop with the taps of a row unrolled: a fully unrolled 7x7 or
// 9x9 body outgrows the instruction cache.
template <int R, int COST, bool CHECK, class S>
__device__ __forceinline__ bool window_cost(const float* pvc, float pm, float pvar, const float* H,
                                            float zmin, float wl, float hl, float minvar,
                                            const S& smp_of, float x, float y, float& cost) {
    constexpr int W = 2 * R + 1;
    constexpr int N = W * W;
    float sv[COST == 1 ? 1 : N];
    float ss = 0.f, sss = 0.f, sps = 0.f;
#pragma unroll 1
    for (int dy = 0; dy < W; ++dy) {
        const float Y = y + (float)(dy - R);
        const float hx = fmaf(H[1], Y, H[2]), hy = fmaf(H[4], Y, H[5]), hz = fmaf(H[7], Y, H[8]);
        const float* prow = pvc + dy * W;
#pragma unroll
        for (int dx = 0; dx < W; ++dx) {
            const float X = x + (float)(dx - R);
            const float h2 = fmaf(H[6], X, hz);
            if (CHECK && !(h2 > zmin)) return false;
            const float iv = rcp_approx(h2);
            const float u = fmaf(H[0], X, hx) * iv;
            const float v = fmaf(H[3], X, hy) * iv;
            if (CHECK && !(u >= 0.f && v >= 0.f && u < wl && v < hl)) return false;
            const float smp = smp_of(u, v);
            if (COST == 1) {
                const float s = smp - pm;
                ss += s;
                sss = fmaf(s, s, sss);
                sps = fmaf(prow[dx], s, sps);
            } else {
                sv[dy * W + dx] = smp;
                ss += smp;
            }
        }
    }
    if (COST == 1) {
        const float n = (float)N;
        const float vs = sss - ss * ss / n;
        if (!(pvar > 0.f) || !(vs > 0.f) || pvar / n < minvar || vs / n < minvar) return false;
        cost = 1.0f - sps * rsqrtf(pvar * vs);
        return true;
    }
    const float ms = ss / (float)N;
    float acc = 0.f;
#pragma unroll
    for (int i = 0; i < N; ++i) acc += fabsf(pvc[i] - (sv[i] - ms));
    cost = acc / (float)N;
    return true;
}

// The ZNCC window costs of two hypotheses at once, for windows whose domain
// the caller established: the same operations as window_cost<R, 1, false>,
// each done on both hypotheses by one packed f32x2 instruction (sm_100) with
// the scalar's rounding, so every component equals the scalar cost bit for
// bit while the pair costs about half the issue slots.  pvc2 holds the
// centred window with each value twice, so a tap loads its packed operand.
template <int R, class S>
__device__ __forceinline__ void window_cost_zncc_pair(const float2* pvc2, float pm, float pvar,
                                                      const float* Ha, const float* Hb,
                                                      float minvar, const S& smp_of, float x,
                                                      float y, bool& oka, float& ea, bool& okb,
                                                      float& eb) {
    constexpr int W = 2 * R + 1;
    constexpr int N = W * W;
    const float2 H0 = f2(Ha[0], Hb[0]), H3 = f2(Ha[3], Hb[3]), H6 = f2(Ha[6], Hb[6]);
    const float2 H1 = f2(Ha[1], Hb[1]), H4 = f2(Ha[4], Hb[4]), H7 = f2(Ha[7], Hb[7]);
    const float2 H2 = f2(Ha[2], Hb[2]), H5 = f2(Ha[5], Hb[5]), H8 = f2(Ha[8], Hb[8]);
    const float2 npm = f2(-pm, -pm);
    float2 ss = f2(0.f, 0.f), sss = f2(0.f, 0.f), sps = f2(0.f, 0.f);
#pragma unroll 1
    for (int dy = 0; dy < W; ++dy) {
        const float Y = y + (float)(dy - R);
        const float2 Y2 = f2(Y, Y);
        const float2 hx = __ffma2_rn(H1, Y2, H2), hy = __ffma2_rn(H4, Y2, H5),
                     hz = __ffma2_rn(H7, Y2, H8);
        const float2* prow = pvc2 + dy * W;
#pragma unroll
        for (int dx = 0; dx < W; ++dx) {
            const float X = x + (float)(dx - R);
            const float2 X2 = f2(X, X);
            const float2 h2 = __ffma2_rn(H6, X2, hz);
            const float2 iv = f2(rcp_approx(h2.x), rcp_approx(h2.y));
            const float2 u = __fmul2_rn(__ffma2_rn(H0, X2, hx), iv);
            const float2 v = __fmul2_rn(__ffma2_rn(H3, X2, hy), iv);
            const float2 s = __fadd2_rn(smp_of.pair(u, v), npm);
            ss = __fadd2_rn(ss, s);
            sss = __ffma2_rn(s, s, sss);
            sps = __ffma2_rn(prow[dx], s, sps);
        }
    }
    const float n = (float)N;
    auto finish = [&](float ssv, float sssv, float spsv, float& cost) {
        const float vs = sssv - ssv * ssv / n;
        if (!(pvar > 0.f) || !(vs > 0.f) || pvar / n < minvar || vs / n < minvar) return false;
        cost = 1.0f - spsv * rsqrtf(pvar * vs);
        return true;
    };
    oka = finish(ss.x, sss.x, sps.x, ea);
    okb = finish(ss.y, sss.y, sps.y, eb);
}

// The band of the reference that a pair's single-view sweep reads: the box of
// texels under every tap of every hypothesis.  For one hypothesis the window's
// image is the convex quadrilateral of its mapped corners (a projective map
// with a positive denominator); along the hypotheses each tap moves
// monotonically (u = (p + inv b0) / (q + inv b2) is monotone in inv), and the
// denominator minus the depth floor is affine in (X, Y, inv); so the corners
// at the first and last inverse depth bound everything.  The margin bounds the
// f32 rounding of any tap at any hypothesis (window_inside's, maximised over
// the two ends: the homography's magnitudes are largest, and the denominator
// smallest, at an end).  False when that box leaves the bilinear domain or
// exceeds kBandPitch x kBandRows texels; the caller then tests hypothesis by
// hypothesis.
template <int R>
__device__ __forceinline__ bool band_box(const float* A, const float* bv, float inv_a, float inv_b,
                                         float wl, float hl, float x, float y, int& bx0, int& by0,
                                         int& cols, int& rows) {
    constexpr float kRel = 9.5367431640625e-07f;  // 2^-20
    float umin = 3.0e38f, vmin = 3.0e38f, umax = -3.0e38f, vmax = -3.0e38f, m = 0.f;
    const float ax = fabsf(x) + (float)R, ay = fabsf(y) + (float)R;
#pragma unroll
    for (int e = 0; e < 2; ++e) {
        float H[9];
        const float inv = e ? inv_b : inv_a;
        plane_h(A, bv, inv, H);
        const float su = fmaf(fabsf(H[0]), ax, fmaf(fabsf(H[1]), ay, fabsf(H[2])));
        const float sv = fmaf(fabsf(H[3]), ax, fmaf(fabsf(H[4]), ay, fabsf(H[5])));
        const float sz = fmaf(fabsf(H[6]), ax, fmaf(fabsf(H[7]), ay, fabsf(H[8])));
        float hmin = 3.0e38f;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const float X = x + ((c & 1) ? (float)R : -(float)R);
            const float Y = y + ((c & 2) ? (float)R : -(float)R);
            const float h2 = fmaf(H[6], X, fmaf(H[7], Y, H[8]));
            const float iv = rcp_approx(h2);
            const float u = fmaf(H[0], X, fmaf(H[1], Y, H[2])) * iv;
            const float v = fmaf(H[3], X, fmaf(H[4], Y, H[5])) * iv;
            hmin = fminf(hmin, h2);
            umin = fminf(umin, u);
            umax = fmaxf(umax, u);
            vmin = fminf(vmin, v);
            vmax = fmaxf(vmax, v);
        }
        if (!(hmin > 1.0e-4f * inv + kRel * sz) || !(hmin > 0.f)) return false;
        m = fmaxf(m, 0.015625f + kRel * (fmaxf(su, sv) + fmaxf(wl, hl) * sz) / hmin);
    }
    // NaN fails every comparison
    if (!(umin >= m && vmin >= m && umax <= wl - m && vmax <= hl - m)) return false;
    bx0 = (int)floorf(umin - m);
    by0 = (int)floorf(vmin - m);
    cols = (int)floorf(umax + m) + 2 - bx0;
    rows = (int)floorf(vmax + m) + 2 - by0;
    return cols <= kBandPitch && rows <= kBandRows;
}

template <class T, int R, int COST>
__global__ void __launch_bounds__(256, 3) k_recip_prepare(BatchDev b, const Cand* __restrict__ cands,
                                                       const uint32_t* __restrict__ count,
                                                       RecipObs* __restrict__ obs,
                                                       RefCounters* __restrict__ ctr,
                                                       uint8_t* __restrict__ pending) {
    constexpr int W = 2 * R + 1;
    constexpr int N = W * W;
    const uint32_t lane = lane_id();
    const uint32_t ms = (uint32_t)b.max_src;
    const uint32_t n_cands = *count;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const DevProfile& prof = b.prof;
    const float n = (float)N;
    // a warp per candidate: the reference window (its re-projection, taps, mean
    // and squared deviation) once, then its sources in order
    for (uint32_t ci = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; ci < n_cands; ci += nwarps) {
        const Cand cd = cands[ci];
        const DevReference& ref = b.refs[cd.ref];
        D3 rp;
        bool rok = project_exact(ref.cam, cd.pos, ref.img.width, ref.img.height, ref.focal, rp);
        // the reference window at (rp.x, rp.y); taps beyond N are exact zeros in every sum
        float dr[kTapRounds], vr = 0.f;
        if (rok) {
            const T* rdata = static_cast<const T*>(ref.img.data);
            float rv[kTapRounds];
            bool tv = true;
#pragma unroll
            for (int h = 0; h < kTapRounds; ++h) {
                rv[h] = 0.f;
                const int t = lane + 32 * h;
                if (t >= N) continue;
                const float X = (float)rp.x + (float)(t % W - R);
                const float Y = (float)rp.y + (float)(t / W - R);
                if (!in_bounds_fast(X, Y, ref.img.width, ref.img.height)) {
                    tv = false;
                    continue;
                }
                rv[h] = sample_fast<T>(rdata, ref.img.width, X, Y);
            }
            rok = __all_sync(0xffffffffu, tv);
            if (rok) {
                float sr = 0.f;
#pragma unroll
                for (int h = 0; h < kTapRounds; ++h) sr += rv[h];
                const float mr = warp_sum(sr) / n;
                float r2 = 0.f;
#pragma unroll
                for (int h = 0; h < kTapRounds; ++h) {
                    dr[h] = lane + 32 * h < N ? rv[h] - mr : 0.f;
                    r2 += dr[h] * dr[h];
                }
                if (COST == 1) vr = warp_sum(r2);
            }
        }
        const double inv = rok ? ddiv(1.0, rp.z) : 0.0;
        const float zmin = zmin_of(inv);
        unsigned long long evals = 0;
        for (uint32_t si = 0; si < ms; ++si) {
            const uint64_t item = (uint64_t)ci * ms + si;
            const uint64_t it = (uint64_t)ci * kMaxSources + si;
            RecipObs res;
            res.valid = 0;
            res.pad = 0;
            res.pos = D3{0, 0, 0};
            bool ok = rok && (int)si < ref.n_src;
            const DevSource& src = ref.src[(int)si < ref.n_src ? si : 0];
            D3 sp;
            // direct cost of the reference window at depth rp.z in this source; lanes over taps
            if (ok) {
                float H[9];
                plane_h(src.fwd_A, src.fwd_b, (float)inv, H);
                const T* sdata = static_cast<const T*>(src.img.data);
                float sv2[kTapRounds];
                bool tv = true;
#pragma unroll
                for (int h = 0; h < kTapRounds; ++h) {
                    sv2[h] = 0.f;
                    const int t = lane + 32 * h;
                    if (t >= N) continue;
                    const float X = (float)rp.x + (float)(t % W - R);
                    const float Y = (float)rp.y + (float)(t / W - R);
                    const float h2 = fmaf(H[6], X, fmaf(H[7], Y, H[8]));
                    if (!(h2 > zmin)) {
                        tv = false;
                        continue;
                    }
                    const float iv = __frcp_rn(h2);
                    const float u = fmaf(H[0], X, fmaf(H[1], Y, H[2])) * iv;
                    const float v = fmaf(H[3], X, fmaf(H[4], Y, H[5])) * iv;
                    if (!in_bounds_fast(u, v, src.img.width, src.img.height)) {
                        tv = false;
                        continue;
                    }
                    sv2[h] = sample_fast<T>(sdata, src.img.width, u, v);
                }
                ok = __all_sync(0xffffffffu, tv);
                if (ok) {
                    float ssv = 0.f;
#pragma unroll
                    for (int h = 0; h < kTapRounds; ++h) ssv += sv2[h];
                    const float mss = warp_sum(ssv) / n;
                    float ds[kTapRounds];
#pragma unroll
                    for (int h = 0; h < kTapRounds; ++h) ds[h] = lane + 32 * h < N ? sv2[h] - mss : 0.f;
                    float cost;
                    if (COST == 1) {
                        float c = 0.f, s2 = 0.f;
#pragma unroll
                        for (int h = 0; h < kTapRounds; ++h) {
                            c += dr[h] * ds[h];
                            s2 += ds[h] * ds[h];
                        }
                        const float cov = warp_sum(c);
                        const float vs = warp_sum(s2);
                        if (!(vr > 0.f) || !(vs > 0.f) || vr / n < (float)prof.min_variance ||
                            vs / n < (float)prof.min_variance)
                            ok = false;
                        cost = 1.0f - cov * rsqrtf(vr * vs);
                    } else {
                        float a = 0.f;
#pragma unroll
                        for (int h = 0; h < kTapRounds; ++h) a += fabsf(dr[h] - ds[h]);
                        cost = warp_sum(a) / n;
                    }
                    ok = ok && !((double)cost > prof.max_error);
                }
            }
            if (ok) ok = project_exact(src.cam, cd.pos, src.img.width, src.img.height, ref.focal, sp);
            // patch_contrast of the source window at (sp.x, sp.y), lanes over taps:
            // first in f32 on the exact texels and fractions of the f64 taps, whose
            // error is below M 2^-19 (M the largest texel magnitude read); the
            // exact f64 contrast decides when that leaves the gate open
            if (ok) {
                const T* sdata = static_cast<const T*>(src.img.data);
                const uint32_t sw = src.img.width;
                float mnf = 3.0e38f, mxf = -3.0e38f, mag = 0.f;
                bool inb = true;
#pragma unroll
                for (int h = 0; h < kTapRounds; ++h) {
                    const int t = lane + 32 * h;
                    if (t >= N) continue;
                    const double x = dadd(sp.x, (double)(t % W - R)), y = dadd(sp.y, (double)(t / W - R));
                    if (!in_bilinear_bounds(x, y, sw, src.img.height)) {
                        inb = false;
                        continue;
                    }
                    const uint32_t x0 = (uint32_t)floor(x), y0 = (uint32_t)floor(y);
                    const float tx = (float)dsub(x, (double)x0), ty = (float)dsub(y, (double)y0);
                    const size_t r0 = (size_t)y0 * sw + x0;
                    const float v00 = pix<T>(sdata, r0), v10 = pix<T>(sdata, r0 + 1);
                    const float v01 = pix<T>(sdata, r0 + sw), v11 = pix<T>(sdata, r0 + sw + 1);
                    const float top = fmaf(v10 - v00, tx, v00);
                    const float bot = fmaf(v11 - v01, tx, v01);
                    const float v = fmaf(bot - top, ty, top);
                    mnf = fminf(mnf, v);
                    mxf = fmaxf(mxf, v);
                    mag = fmaxf(mag, fmaxf(fmaxf(fabsf(v00), fabsf(v10)), fmaxf(fabsf(v01), fabsf(v11))));
                }
                ok = __all_sync(0xffffffffu, inb);
                if (ok) {
#pragma unroll
                    for (int o = 16; o > 0; o >>= 1) {
                        mnf = fminf(mnf, __shfl_xor_sync(0xffffffffu, mnf, o));
                        mxf = fmaxf(mxf, __shfl_xor_sync(0xffffffffu, mxf, o));
                        mag = fmaxf(mag, __shfl_xor_sync(0xffffffffu, mag, o));
                    }
                    const double c = (double)mxf - (double)mnf;
                    const double eps = (double)mag * 1.52587890625e-05;  // 2^-16: 8 x the bound
                    if (c >= prof.min_contrast + eps) {
                        ok = true;
                    } else if (c < prof.min_contrast - eps) {
                        ok = false;
                    } else {
                        // exact patch_contrast near the gate
                        double mn = kInf, mx = -kInf;
#pragma unroll
                        for (int h = 0; h < kTapRounds; ++h) {
                            const int t = lane + 32 * h;
                            if (t >= N) continue;
                            double v = 0.0;
                            sample_exact<T>(src.img, dadd(sp.x, (double)(t % W - R)),
                                            dadd(sp.y, (double)(t / W - R)), v);
                            mn = fmin(mn, v);
                            mx = fmax(mx, v);
                        }
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) {
                            mn = fmin(mn, __shfl_xor_sync(0xffffffffu, mn, o));
                            mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
                        }
                        ok = !(dsub(mx, mn) < prof.min_contrast);
                    }
                }
            }
            if (ok) {
                res.pos = sp;
                res.valid = kObsPending;
                evals += (unsigned long long)ref.planes;
            }
            if (lane == 0 && (int)si < ref.n_src) obs[it] = res;
            if (lane == 0) pending[item] = ok ? 1 : 0;
        }
        if (lane == 0 && evals) atomicAdd(&ctr[cd.ref].recip_evals, evals);
    }
}

// MODE kRecipBanded takes the pairs whose band fits the stage and appends the
// others to `fallback`; kRecipPerHypothesis takes a list with the per-hypothesis
// domain tests only.  The banded kernel needs fewer registers and runs three
// blocks per SM.
constexpr int kRecipBanded = 1, kRecipPerHypothesis = 2;

// The banded kernel runs 4 warps a block (their bands of texel pairs fill the
// static shared memory), the per-hypothesis one 8.
template <int MODE>
struct RecipBounds {
    static constexpr int kWarps = MODE == kRecipBanded ? 4 : 8;
    static constexpr int kThreads = 32 * kWarps;
    static constexpr int kBlocks = MODE == kRecipBanded ? 4 : 2;
};

template <class T, int R, int COST, int MODE>
__global__ void __launch_bounds__(RecipBounds<MODE>::kThreads, RecipBounds<MODE>::kBlocks) k_recip_sweep(
    BatchDev b, const Cand* __restrict__ cands, const uint32_t* __restrict__ list,
    const uint32_t* __restrict__ list_count, RecipObs* __restrict__ obs,
    uint32_t* __restrict__ fallback, uint32_t* __restrict__ n_fallback) {
    constexpr int W = 2 * R + 1;
    constexpr int N = W * W;
    constexpr int kWarps = RecipBounds<MODE>::kWarps;
    __shared__ float pvc_all[kWarps][N];
    __shared__ float2 pvc2_all[kWarps][N];  // the same values twice, a packed operand each
    // the warps' bands of texel pairs (banded kernel only), with a guard row
    // before the first and after the last
    __shared__ float2 band_all[MODE == kRecipBanded ? (kWarps * kBandRows + 2) * kBandPitch : 1];
    const uint32_t lane = lane_id(), wid = threadIdx.x >> 5;
    float* pvc = pvc_all[wid];
    float2* pvc2 = pvc2_all[wid];
    float2* band = band_all + (MODE == kRecipBanded ? (1 + wid * kBandRows) * kBandPitch : 0);
    const uint32_t ms = (uint32_t)b.max_src;
    const uint32_t n_list = *list_count;
    const uint32_t nwarps = (gridDim.x * blockDim.x) >> 5;
    const DevProfile& prof = b.prof;
    // the pending (candidate, source) items, listed in order by the compaction
    for (uint32_t li = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; li < n_list; li += nwarps) {
        const uint32_t item = list[li];
        const uint32_t ci = item / ms;
        const int si = (int)(item - ci * ms);
        const uint64_t it = (uint64_t)ci * kMaxSources + si;
        const uint32_t r = cands[ci].ref;
        const DevReference& ref = b.refs[r];
        const D3 sp = obs[it].pos;
        const DevSource& src = ref.src[si];
        // the source window as the contrast gate sampled it, centred; taps
        // beyond N contribute exact zeros to the sums
        float p[kTapRounds];
        float psum = 0.f;
#pragma unroll
        for (int h = 0; h < kTapRounds; ++h) {
            const int t = lane + 32 * h;
            double v = 0.0;
            if (t < N)
                sample_exact<T>(src.img, dadd(sp.x, (double)(t % W - R)),
                                dadd(sp.y, (double)(t / W - R)), v);
            p[h] = (float)v;
            psum += p[h];
        }
        const float pm = warp_sum(psum) / (float)N;
        float dsq = 0.f;
#pragma unroll
        for (int h = 0; h < kTapRounds; ++h) {
            const int t = lane + 32 * h;
            const float d = t < N ? p[h] - pm : 0.f;
            dsq += d * d;
            if (t < N) {
                pvc[t] = d;
                pvc2[t] = f2(d, d);
            }
        }
        const float pvar = warp_sum(dsq);
        const float* inv_tab = b.src_inv + ref.inv_off + (size_t)si * ref.planes;
        const T* rimg = static_cast<const T*>(ref.img.data);
        const uint32_t rw = ref.img.width;
        const float wl = (float)(ref.img.width - 1), hl = (float)(ref.img.height - 1);
        const float x0 = (float)sp.x, y0 = (float)sp.y;
        const float minvar = (float)prof.min_variance;
        float be = 3.0e38f;
        int bk = 0x7fffffff;
        auto take = [&](bool ok, float e, int k) {
            if (ok && (double)e <= prof.max_error && e < be) {
                be = e;
                bk = k;
            }
        };
        // every hypothesis's window inside one staged box of the reference
        int bx0 = 0, by0 = 0, cols = 0, rows = 0;
        const bool banded =
            MODE == kRecipBanded && band_box<R>(src.bwd_A, src.bwd_b, inv_tab[0],
                                                inv_tab[ref.planes - 1], wl, hl, x0, y0, bx0,
                                                by0, cols, rows);
        if (MODE == kRecipBanded && !banded) {
            // the per-hypothesis kernel takes this pair
            if (lane == 0) fallback[atomicAdd(n_fallback, 1u)] = item;
            __syncwarp();
            continue;
        }
        if (banded) {
            // entry c: texel c of the row and texel c + 1 minus texel c; the last
            // column is read only as a right neighbour.  The lanes run over the
            // flat rows x (cols - 1) entries; the row of entry e is
            // floor((e + 1/2) / (cols - 1)), exact in f32 since e < 2^11 and the
            // fraction lies at least 1/128 from an integer
            const int c1 = cols - 1;
            const float inv_c1 = 1.0f / (float)c1;
            const T* base = rimg + (size_t)by0 * rw + bx0;
            for (int e = lane; e < rows * c1; e += 32) {
                const int rr = (int)(((float)e + 0.5f) * inv_c1);
                const int c = e - rr * c1;
                const T* row = base + (size_t)rr * rw;
                const float t0 = pix<T>(row, c), t1 = pix<T>(row, c + 1);
                band[rr * kBandPitch + c] = f2(t0, t1 - t0);
            }
        }
        __syncwarp();
        if (banded) {
            const BandSampler smp{band, 8388608.0f - (float)bx0, 8388608.0f - (float)by0};
            // this lane's hypotheses in the order lane, lane + 32, lane + 64, ...,
            // two at a time (k, k + 32) on the packed ZNCC path
            for (int k = lane; k < ref.planes; k += 64) {
                const int k2 = k + 32;
                float Ha[9], Hb[9];
                plane_h(src.bwd_A, src.bwd_b, inv_tab[k], Ha);
                if (COST == 1 && k2 < ref.planes) {
                    plane_h(src.bwd_A, src.bwd_b, inv_tab[k2], Hb);
                    bool oka, okb;
                    float ea, eb;
                    window_cost_zncc_pair<R>(pvc2, pm, pvar, Ha, Hb, minvar, smp, x0, y0, oka, ea,
                                             okb, eb);
                    take(oka, ea, k);
                    take(okb, eb, k2);
                } else {
                    float e;
                    bool ok = window_cost<R, COST, false>(pvc, pm, pvar, Ha, 0.f, wl, hl, minvar,
                                                          smp, x0, y0, e);
                    take(ok, e, k);
                    if (k2 < ref.planes) {
                        plane_h(src.bwd_A, src.bwd_b, inv_tab[k2], Hb);
                        ok = window_cost<R, COST, false>(pvc, pm, pvar, Hb, 0.f, wl, hl, minvar,
                                                         smp, x0, y0, e);
                        take(ok, e, k2);
                    }
                }
            }
        } else {
            const ImageSampler<T> smp{rimg, rw};
            // one hypothesis alone, through the scalar paths
            auto single = [&](int k, const float* H, bool inside) {
                const float zmin = 1.0e-4f * inv_tab[k];
                float e;
                const bool ok =
                    inside ? window_cost<R, COST, false>(pvc, pm, pvar, H, zmin, wl, hl, minvar,
                                                         smp, x0, y0, e)
                           : window_cost<R, COST, true>(pvc, pm, pvar, H, zmin, wl, hl, minvar,
                                                        smp, x0, y0, e);
                take(ok, e, k);
            };
            for (int k = lane; k < ref.planes; k += 64) {
                const int k2 = k + 32;
                float Ha[9], Hb[9];
                plane_h(src.bwd_A, src.bwd_b, inv_tab[k], Ha);
                const bool ina = window_inside<R>(Ha, 1.0e-4f * inv_tab[k], wl, hl, x0, y0);
                bool inb = false;
                if (k2 < ref.planes) {
                    plane_h(src.bwd_A, src.bwd_b, inv_tab[k2], Hb);
                    inb = window_inside<R>(Hb, 1.0e-4f * inv_tab[k2], wl, hl, x0, y0);
                }
                if (COST == 1 && ina && inb) {
                    bool oka, okb;
                    float ea, eb;
                    window_cost_zncc_pair<R>(pvc2, pm, pvar, Ha, Hb, minvar, smp, x0, y0, oka, ea,
                                             okb, eb);
                    take(oka, ea, k);
                    take(okb, eb, k2);
                } else {
                    single(k, Ha, ina);
                    if (k2 < ref.planes) single(k2, Hb, inb);
                }
            }
        }
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) {
            const float oe = __shfl_down_sync(0xffffffffu, be, off);
            const int ok2 = __shfl_down_sync(0xffffffffu, bk, off);
            if (oe < be || (oe == be && ok2 < bk)) {
                be = oe;
                bk = ok2;
            }
        }
        if (lane == 0) {
            RecipObs res;
            res.valid = 0;
            res.pad = 0;
            res.pos = D3{0, 0, 0};
            if (bk != 0x7fffffff) {
                const double rd = hypothesis_depth(bk, ref.planes, src.search_min, src.search_max);
                const double ex = sp.z;
                // reciprocal_depth_agrees (dense_legacy.rs:951-957)
                bool agree = isfinite(ex) && isfinite(rd) && ex > 0.0 && rd > 0.0;
                if (agree) {
                    const double scale = fmax(fmax(ex, rd), 1.0e-9);
                    agree = ddiv(fabs(dsub(ex, rd)), scale) <= kMaxReciprocalRelativeDepthError;
                }
                if (agree) {
                    res.pos = unproject_exact(src.cam, sp.x, sp.y, rd, src.img.width,
                                              src.img.height, ref.focal);
                    res.valid = finite3(res.pos) ? 1 : 0;
                }
            }
            obs[it] = res;
        }
        __syncwarp();
    }
}


// ---- surface completion proposals (dense_legacy.rs:600-650) ------------------
// Second stage of a completion pass, a thread per seed left by the first stage
// (the seed Cand holds the site, the predicted depth and the neighbours' mean
// margin and confidence): the reference window's contrast, then the predicted
// point's cost in every source view.  Seeds are compacted in site order, so the
// warps run full.
template <class T, bool EXACT, int R, int COST>
__global__ void __launch_bounds__(128) k_propose_costs(BatchDev b,
                                                       const uint32_t* __restrict__ seed_idx,
                                                       const uint32_t* __restrict__ seed_count,
                                                       uint8_t* __restrict__ prop_status,
                                                       Cand* __restrict__ prop,
                                                       RefCounters* __restrict__ ctr) {
    constexpr int W = 2 * R + 1;
    const uint32_t count = *seed_count;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count;
         i += gridDim.x * blockDim.x) {
        const uint32_t g = seed_idx[i];
        Cand cd = prop[g];
        const uint32_t r = cd.ref;
        const DevReference& ref = b.refs[r];
        const uint32_t x = cd.x, y = cd.y;
        const double predicted = cd.depth;
        RefCounters& c = ctr[r];
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
                ok = window_cost_fast<T, R, COST>(b.prof, pv, pm, pvv, H, zmin_of(inv), src.img,
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
        cd.pos = ppos;
        cd.error = median_of(errs, ne);
        cd.support = ne;
        prop[g] = cd;
        prop_status[g] = kPropCandidate;
    }
}


// Raises a kernel's dynamic shared memory limit on the current device to at
// least `bytes`, never lowering it: the server's slots launch the same kernel
// from several threads with different sizes, and a limit lowered by one
// thread between another's setting and launch would refuse that launch.
inline cudaError_t raise_dynamic_smem_limit(const void* kern, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, const void*>, size_t> limit;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> lock(mu);
    size_t& have = limit[{dev, kern}];
    if (bytes <= have) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) have = bytes;
    return e;
}

// Multiprocessors of the current device when first asked (a thread-safe
// static: server slots launch from several threads).
inline int sm_count() {
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

// Dispatch helpers over (storage type, exactness, radius).

}  // namespace typed_detail

template <class T>
cudaError_t Typed<T>::sweep_site(const BatchDev& b, const uint32_t* site_ref, uint64_t total,
                                 SiteRank* rank, uint8_t* status, RefCounters* ctr,
                                 cudaStream_t st) {
    using namespace typed_detail;
    const unsigned blocks = (unsigned)((total * 32 + 255) / 256);
#define V3D_SITE(E, RR, C)                                                                   \
    if (b.exact == E && b.prof.radius == RR && (E || b.prof.cost == C)) {                     \
        V3D_COUNTED k_sweep_site<T, E, RR, C><<<blocks, 256, 0, st>>>(b, site_ref, total, rank, status, ctr); \
        return cudaGetLastError();                                                           \
    }
#define V3D_SITE_R(RR) V3D_SITE(true, RR, 0) V3D_SITE(false, RR, 0) V3D_SITE(false, RR, 1)
    V3D_SITE_R(1) V3D_SITE_R(2) V3D_SITE_R(3) V3D_SITE_R(4)
#undef V3D_SITE_R
#undef V3D_SITE
    return cudaErrorInvalidValue;
}

template <class T>
cudaError_t Typed<T>::sweep_tiled(const BatchDev& b, uint32_t max_nx, uint32_t max_ny,
                                  uint32_t stride, SiteRank* rank, uint8_t* status,
                                  RefCounters* ctr, cudaStream_t st, uint64_t total_sites,
                                  SweepChunks chunks) {
    using namespace typed_detail;
    const int TX = chunks.tile_x == 16 ? 16 : 32, TY = kTileThreads / TX;
    auto run = [&](auto kern, int W) -> cudaError_t {
        const int s = (int)stride;
        const int PX = (TX - 1) * s + W, PY = (TY - 1) * s + W;
        const size_t PXp = (size_t)((PX + s - 1) / s) * s, np = PXp * PY;
        const size_t smem = (b.sums32 ? sizeof(float) : sizeof(double)) * 3 * (size_t)PY * TX +
                            sizeof(float) * (2 * np + (size_t)b.max_src * (kTileThreads + 12) +
                                             2 * (size_t)b.prof.planes + PY) +
                            16 + sizeof(float4) * (size_t)tiled_steps((int)np) * kTileThreads;
        cudaError_t e = raise_dynamic_smem_limit(reinterpret_cast<const void*>(kern), smem);
        if (e != cudaSuccess) return e;
        const int n = chunks.n > 1 ? chunks.n : 1;
        dim3 grid((max_nx + TX - 1) / TX, (max_ny + TY - 1) / TY, (unsigned)b.n_refs * (unsigned)n);
        V3D_COUNTED kern<<<grid, kTileThreads, smem, st>>>(b, total_sites, rank, status, ctr, n, chunks.partial);
        return cudaGetLastError();
    };
    // grid stride 2, the ZNCC profiles' usual stride, has its own instantiation
    auto pick = [&](auto k2, auto k0, int W) { return stride == 2 ? run(k2, W) : run(k0, W); };
    auto by_acc = [&](auto tx_tag) -> cudaError_t {
        constexpr int X = decltype(tx_tag)::value;
        switch (b.prof.radius * 2 + (b.sums32 ? 1 : 0)) {
            case 2: return pick(k_sweep_tiled<T, 1, double, X, 2>, k_sweep_tiled<T, 1, double, X, 0>, 3);
            case 4: return pick(k_sweep_tiled<T, 2, double, X, 2>, k_sweep_tiled<T, 2, double, X, 0>, 5);
            case 6: return pick(k_sweep_tiled<T, 3, double, X, 2>, k_sweep_tiled<T, 3, double, X, 0>, 7);
            case 8: return pick(k_sweep_tiled<T, 4, double, X, 2>, k_sweep_tiled<T, 4, double, X, 0>, 9);
            case 3: return pick(k_sweep_tiled<T, 1, float, X, 2>, k_sweep_tiled<T, 1, float, X, 0>, 3);
            case 5: return pick(k_sweep_tiled<T, 2, float, X, 2>, k_sweep_tiled<T, 2, float, X, 0>, 5);
            case 7: return pick(k_sweep_tiled<T, 3, float, X, 2>, k_sweep_tiled<T, 3, float, X, 0>, 7);
            case 9: return pick(k_sweep_tiled<T, 4, float, X, 2>, k_sweep_tiled<T, 4, float, X, 0>, 9);
        }
        return cudaErrorInvalidValue;
    };
    return TX == 16 ? by_acc(std::integral_constant<int, 16>{})
                    : by_acc(std::integral_constant<int, 32>{});
}

template <class T>
cudaError_t Typed<T>::reciprocal(const BatchDev& b, const Cand* cands, const uint32_t* count,
                                 RecipObs* obs, RefCounters* ctr, const RecipQueue& q,
                                 cudaStream_t st) {
    using namespace typed_detail;
    const unsigned blocks = (unsigned)sm_count() * 8;
    // the banded sweep: four waves of its resident blocks (a whole number of
    // waves, so the grid-stride loop leaves no partial last wave)
    const unsigned rblocks3 = (unsigned)sm_count() * 4 * RecipBounds<kRecipBanded>::kBlocks;
#define V3D_CK_RET(x)                                \
    do {                                             \
        const cudaError_t e_ = (x);                  \
        if (e_ != cudaSuccess) return e_;            \
    } while (0)
    auto mark = [&](cudaEvent_t e) {
        if (e) cudaEventRecord(e, st);
    };
    mark(q.t_prepare);
    // prologue, then the list of its pending items, then the sweep over the list
    auto prep_and_list = [&](auto prep) -> cudaError_t {
        cudaError_t e = cudaMemsetAsync(q.flags, 0, q.cap_items, st);
        if (e != cudaSuccess) return e;
        // three waves of the prologue's three resident blocks an SM
        V3D_COUNTED prep<<<(unsigned)sm_count() * 9, 256, 0, st>>>(b, cands, count, obs, ctr, q.flags);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        return launch_compact(q.flags, 1, q.cap_items, q.items, q.n_items, q.scratch, st);
    };
#define V3D_REC(RR)                                                                            \
    if (b.prof.radius == RR) {                                                                 \
        if (b.exact) {                                                                         \
            mark(q.t_sweep);                                                                   \
            V3D_COUNTED k_reciprocal_exact<T, RR><<<blocks, 256, 0, st>>>(b, cands, count, obs, ctr);      \
        } else if (b.prof.cost == 1) {                                                         \
            const cudaError_t e = prep_and_list(k_recip_prepare<T, RR, 1>);                    \
            if (e != cudaSuccess) return e;                                                    \
            mark(q.t_sweep);                                                                   \
            V3D_CK_RET(cudaMemsetAsync(q.n_fallback, 0, sizeof(uint32_t), st));               \
            V3D_COUNTED k_recip_sweep<T, RR, 1, kRecipBanded><<<rblocks3, 128, 0, st>>>(        \
                b, cands, q.items, q.n_items, obs, q.fallback, q.n_fallback);                 \
            V3D_COUNTED k_recip_sweep<T, RR, 1, kRecipPerHypothesis><<<blocks, 256, 0, st>>>(   \
                b, cands, q.fallback, q.n_fallback, obs, nullptr, nullptr);                    \
        } else {                                                                               \
            const cudaError_t e = prep_and_list(k_recip_prepare<T, RR, 0>);                    \
            if (e != cudaSuccess) return e;                                                    \
            mark(q.t_sweep);                                                                   \
            V3D_CK_RET(cudaMemsetAsync(q.n_fallback, 0, sizeof(uint32_t), st));               \
            V3D_COUNTED k_recip_sweep<T, RR, 0, kRecipBanded><<<rblocks3, 128, 0, st>>>(        \
                b, cands, q.items, q.n_items, obs, q.fallback, q.n_fallback);                 \
            V3D_COUNTED k_recip_sweep<T, RR, 0, kRecipPerHypothesis><<<blocks, 256, 0, st>>>(   \
                b, cands, q.fallback, q.n_fallback, obs, nullptr, nullptr);                    \
        }                                                                                      \
        mark(q.t_end);                                                                         \
        return cudaGetLastError();                                                             \
    }
    V3D_REC(1) V3D_REC(2) V3D_REC(3) V3D_REC(4)
#undef V3D_REC
#undef V3D_CK_RET
    return cudaErrorInvalidValue;
}

template <class T>
cudaError_t Typed<T>::propose(const BatchDev& b, const uint32_t* seed_idx,
                              const uint32_t* seed_count, uint64_t total, uint8_t* prop_status,
                              Cand* prop, RefCounters* ctr, cudaStream_t st) {
    using namespace typed_detail;
    uint64_t blocks = (total + 127) / 128;
    if (blocks > (uint64_t)sm_count() * 16) blocks = (uint64_t)sm_count() * 16;
    if (blocks == 0) blocks = 1;
#define V3D_PROP(E, RR, C)                                                                  \
    if (b.exact == E && b.prof.radius == RR && (E || b.prof.cost == C)) {                    \
        V3D_COUNTED k_propose_costs<T, E, RR, C><<<(unsigned)blocks, 128, 0, st>>>(b, seed_idx, seed_count, \
                                                                       prop_status, prop, ctr); \
        return cudaGetLastError();                                                          \
    }
#define V3D_PROP_R(RR) V3D_PROP(true, RR, 0) V3D_PROP(false, RR, 0) V3D_PROP(false, RR, 1)
    V3D_PROP_R(1) V3D_PROP_R(2) V3D_PROP_R(3) V3D_PROP_R(4)
#undef V3D_PROP_R
#undef V3D_PROP
    return cudaErrorInvalidValue;
}

}  // namespace v3d
