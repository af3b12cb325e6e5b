// Measured ceiling of the depth sweep's inner step: homography-warped f32
// bilinear samples per second on this GPU (v3d_measure_gather_rate; the
// reference has no counterpart, it is a diagnostic for the gather roofline).
//
// Each CTA owns a 70x21 footprint of an f32 image, the size of a 32x8-site
// tile at stride 2 with a 7x7 window, and its warps sample it the way the
// sweep's warp step does: rows over warps, consecutive columns over lanes, a
// fresh plane homography per pass.  Nothing else happens: no shared-memory
// stores, no box filters, so the rate is what gathers alone sustain.
#include <cuda_runtime.h>

#include "../../include/v3d_dense.h"
#include "host.hpp"

namespace {

constexpr int kFootX = 70, kFootY = 21;
constexpr int kImgW = 1024, kImgH = 512;

__device__ __forceinline__ float bilinear(const float* __restrict__ p, uint32_t w, float u, float v) {
    const float kShift = 8388608.0f;
    const float tu = __fadd_rd(u, kShift), tv = __fadd_rd(v, kShift);
    const float fu = tu - kShift, fv = tv - kShift;
    const uint32_t ix = (uint32_t)(__float_as_int(tu) - __float_as_int(kShift));
    const uint32_t iy = (uint32_t)(__float_as_int(tv) - __float_as_int(kShift));
    const float tx = u - fu, ty = v - fv;
    const size_t r0 = (size_t)iy * w + ix;
    const float v00 = __ldg(p + r0), v10 = __ldg(p + r0 + 1);
    const float v01 = __ldg(p + r0 + w), v11 = __ldg(p + r0 + w + 1);
    const float top = fmaf(v10 - v00, tx, v00);
    const float bot = fmaf(v11 - v01, tx, v01);
    return fmaf(bot - top, ty, top);
}

__global__ void __launch_bounds__(256) k_gather_rate(const float* __restrict__ img, int passes,
                                                     float* __restrict__ sink) {
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    // the CTA's footprint origin, inside the image with a margin for the warp
    const float ox = (float)(8 + (blockIdx.x * 37) % (kImgW - kFootX - 40));
    const float oy = (float)(8 + (blockIdx.x * 11) % (kImgH - kFootY - 40));
    float acc = 0.f;
    for (int k = 0; k < passes; ++k) {
        // a mild homography that changes with the pass: scale, shear, offset
        const float a0 = 1.0f + 0.001f * (k & 15), a1 = 0.002f * ((k >> 4) & 7);
        const float a3 = 0.0015f * (k & 7), a4 = 1.0f - 0.0007f * (k & 31);
        const float a6 = 1.0e-5f * (k & 3), a7 = 2.0e-5f * (k & 5);
        const float b0 = ox + 0.37f * (k & 31), b1 = oy + 0.21f * (k & 15);
        for (int yy = ty; yy < kFootY; yy += 8) {
            const float Y = (float)yy;
            const float hx = fmaf(a1, Y, b0), hy = fmaf(a4, Y, b1), hz = fmaf(a7, Y, 1.0f);
            for (int xx = tx; xx < kFootX; xx += 32) {
                const float X = (float)xx;
                const float iv = __fdividef(1.0f, fmaf(a6, X, hz));
                const float u = fmaf(a0, X, hx) * iv;
                const float v = fmaf(a3, X, hy) * iv;
                acc += bilinear(img, kImgW, u, v);
            }
        }
    }
    if (acc == -1.0f) sink[blockIdx.x] = acc;  // keeps the loads without writing
}

}  // namespace

extern "C" int32_t v3d_measure_gather_rate(v3d_context* ctx, double* samples_per_second) {
    if (!ctx || !samples_per_second) return V3D_ERR_INVALID_ARGUMENT;
    *samples_per_second = 0.0;
    std::lock_guard<std::mutex> lock(ctx->mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(ctx->stream);
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ctx->device) != cudaSuccess)
        return V3D_ERR_CUDA;
    float* img = nullptr;
    float* sink = nullptr;
    const int blocks = sms * 8;
    if (cudaMalloc(&img, sizeof(float) * kImgW * kImgH) != cudaSuccess) return V3D_ERR_OUT_OF_MEMORY;
    if (cudaMalloc(&sink, sizeof(float) * blocks) != cudaSuccess) {
        cudaFree(img);
        return V3D_ERR_OUT_OF_MEMORY;
    }
    cudaMemsetAsync(img, 0x3e, sizeof(float) * kImgW * kImgH, st);  // about 0.19 everywhere
    const int passes = 256;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    k_gather_rate<<<blocks, 256, 0, st>>>(img, passes, sink);  // warm-up
    cudaEventRecord(e0, st);
    for (int rep = 0; rep < 4; ++rep) k_gather_rate<<<blocks, 256, 0, st>>>(img, passes, sink);
    cudaEventRecord(e1, st);
    const cudaError_t err = cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(img);
    cudaFree(sink);
    if (err != cudaSuccess || ms <= 0.f) return V3D_ERR_CUDA;
    const double samples = 4.0 * blocks * (double)passes * kFootX * kFootY;
    *samples_per_second = samples / (ms * 1e-3);
    return V3D_OK;
}
