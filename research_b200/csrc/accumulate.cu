// accumulate.cu — AccumulatePass (AccumulatePass.cpp:167-218) and its kernel
// accumulate.slang:21-46: FP32 running mean, reset when the camera moved or
// nothing is accumulated yet. `image_count` frames are folded per launch, in
// order, with each channel's accumulator kept in registers between frames.
// The optional FP64 per-pixel sum is the RMSE judge buffer.

#include "rr_internal.h"

namespace rr {
namespace {

// One thread per channel of a pixel (the channels' running means and sums
// are independent): element e of every image is channel e % 4 of pixel
// e / 4, so a warp reads 32 consecutive floats of an image. An image's
// weights 1/(spp+1) and spp/(spp+1) are the same for every pixel; each
// block computes those of kChunk images at a time into shared memory, and
// each thread folds the images in in order, reading kBatch of them at a time
// (their loads in flight together). The operations per channel are those of
// folding one image at a time.
constexpr uint32_t kAccThreads = 256;
constexpr uint32_t kChunk = kAccThreads;
constexpr uint32_t kBatch = 16;
static_assert(kChunk % kBatch == 0, "batches inside a chunk");

__global__ void __launch_bounds__(kAccThreads) accumulate_kernel(const float* __restrict__ rad, uint32_t images,
                                                                 float* __restrict__ acc, double* __restrict__ sum64,
                                                                 uint32_t elems, uint32_t camera_moved,
                                                                 uint32_t spp0) {
    __shared__ float s_weight[kChunk], s_keep[kChunk];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < elems;
    const bool reset0 = camera_moved != 0 || spp0 == 0;
    float a = 0.0f;
    double d = 0.0;
    if (valid && !reset0) {
        a = acc[i];
        if (sum64) d = sum64[i];
    }
    #pragma unroll 1
    for (uint32_t c0 = 0; c0 < images; c0 += kChunk) {
        {
            // image k = c0 + t is folded with spp_before = k (after a reset
            // at image 0) or spp0 + k
            const uint32_t k = c0 + threadIdx.x;
            const float spp = float(reset0 ? k : spp0 + k);
            s_weight[threadIdx.x] = 1.0f / (spp + 1.0f);
            s_keep[threadIdx.x] = spp / (spp + 1.0f);
        }
        __syncthreads();
        const uint32_t n = min(kChunk, images - c0);
        if (valid) {
            #pragma unroll 1
            for (uint32_t b0 = 0; b0 < n; b0 += kBatch) {
                float rb[kBatch];
                #pragma unroll
                for (uint32_t u = 0; u < kBatch; ++u)
                    if (b0 + u < n) rb[u] = __ldcs(rad + size_t(c0 + b0 + u) * elems + i);
                #pragma unroll
                for (uint32_t u = 0; u < kBatch; ++u) {
                    if (b0 + u >= n) break;
                    const float r = rb[u];
                    if (c0 + b0 + u == 0 && reset0) a = r;
                    else a = a * s_keep[b0 + u] + r * s_weight[b0 + u];
                    d += double(r);
                }
            }
        }
        __syncthreads();
    }
    if (valid) {
        acc[i] = a;
        if (sum64) sum64[i] = d;
    }
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
    // one thread per channel: 4 px elements indexed in 32 bits
    if (px == 0 || px >= (1ull << 30)) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "bad image size");
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    const uint64_t elems = px * 4;
    const uint32_t blocks = uint32_t((elems + rr::kAccThreads - 1) / rr::kAccThreads);
    rr::accumulate_kernel<<<blocks, rr::kAccThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        radiance, image_count, accumulated, oracle_sum, uint32_t(elems), p->camera_moved, p->accumulated_spp);
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}
