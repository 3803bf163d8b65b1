// accumulate.cu — AccumulatePass (AccumulatePass.cpp:167-218) and its kernel
// accumulate.slang:21-46: FP32 running mean, reset when the camera moved or
// nothing is accumulated yet. `image_count` frames are folded per launch, in
// order, with each pixel's accumulator kept in registers between frames.
// The optional FP64 per-pixel sum is the RMSE judge buffer.

#include "rr_internal.h"

namespace rr {
namespace {

__global__ void __launch_bounds__(256) accumulate_kernel(const float4* __restrict__ rad, uint32_t images,
                                                         float4* __restrict__ acc, double4* __restrict__ sum64,
                                                         uint32_t pixels, uint32_t camera_moved,
                                                         uint32_t spp0) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pixels) return;
    const bool reset0 = camera_moved != 0 || spp0 == 0;
    float4 a = reset0 ? make_float4(0.f, 0.f, 0.f, 0.f) : acc[i];
    double4 d = make_double4(0.0, 0.0, 0.0, 0.0);
    if (sum64 && !reset0) d = sum64[i];
    uint32_t spp_before = spp0;
    for (uint32_t k = 0; k < images; ++k) {
        const float4 r = __ldcs(rad + size_t(k) * pixels + i);
        if ((k == 0 && reset0)) {
            a = r;
            spp_before = 0;
        } else {
            const float spp = float(spp_before);
            const float weight = 1.0f / (spp + 1.0f);
            const float keep = spp / (spp + 1.0f);
            a.x = a.x * keep + r.x * weight;
            a.y = a.y * keep + r.y * weight;
            a.z = a.z * keep + r.z * weight;
            a.w = a.w * keep + r.w * weight;
        }
        d.x += double(r.x); d.y += double(r.y); d.z += double(r.z); d.w += double(r.w);
        spp_before += 1;
    }
    acc[i] = a;
    if (sum64) sum64[i] = d;
}

} // namespace
} // namespace rr

extern "C" rr_status rr_accumulate_execute(rr_ctx* ctx, const float* radiance, uint32_t image_count,
                                           float* accumulated, double* oracle_sum,
                                           const rr_acc_params* p, void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!radiance || !accumulated || !p || image_count == 0)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_accumulate_execute: bad argument");
    const uint64_t px = uint64_t(p->width) * p->height;
    if (px == 0 || px >= (1ull << 31)) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "bad image size");
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    const uint32_t blocks = uint32_t((px + 255) / 256);
    rr::accumulate_kernel<<<blocks, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const float4*>(radiance), image_count, reinterpret_cast<float4*>(accumulated),
        reinterpret_cast<double4*>(oracle_sum), uint32_t(px), p->camera_moved, p->accumulated_spp);
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}
