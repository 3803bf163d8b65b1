// accumulate.cu — AccumulatePass (AccumulatePass.cpp:167-218) and its kernel
// accumulate.slang:21-46: FP32 running mean, reset when the camera moved or
// nothing is accumulated yet. `image_count` frames are folded per launch, in
// order, with each pixel's (or channel's) accumulator kept in registers
// between frames.
// The optional FP64 per-pixel sum is the RMSE judge buffer.

#include "rr_internal.h"

namespace rr {
namespace {

// An image's weights 1/(spp+1) and spp/(spp+1) are the same for every
// pixel: each block computes those of up to kChunk images at a time into
// shared memory. Each thread folds the images in in order, reading a batch
// of them at a time (their loads in flight together), so the operations per
// channel are those of folding one image at a time. A thread owns one
// pixel (T = float4) or, for small images, one channel of a pixel (T =
// float: element e is channel e % 4 of pixel e / 4), which gives a 64 x 64
// image four times the threads.
constexpr uint32_t kAccThreads = 256;
constexpr uint32_t kChunk = kAccThreads;
constexpr uint64_t kSmallPixels = 1u << 18;   // below: one thread per channel
// images in flight per thread: 16 floats, or 4 float4 (more would cost the
// pixel form its occupancy, which a large image's stream needs)
template <class T> __host__ __device__ constexpr uint32_t batch_of() { return sizeof(T) == 16 ? 4u : 16u; }
static_assert(kChunk % batch_of<float>() == 0 && kChunk % batch_of<float4>() == 0, "batches inside a chunk");

__device__ __forceinline__ float acc_zero(float) { return 0.0f; }
__device__ __forceinline__ float4 acc_zero(float4) { return make_float4(0.f, 0.f, 0.f, 0.f); }
__device__ __forceinline__ double acc_zero64(float) { return 0.0; }
__device__ __forceinline__ double4 acc_zero64(float4) { return make_double4(0.0, 0.0, 0.0, 0.0); }
__device__ __forceinline__ float fold(float a, float r, float keep, float weight) { return a * keep + r * weight; }
__device__ __forceinline__ float4 fold(float4 a, float4 r, float keep, float weight) {
    return make_float4(a.x * keep + r.x * weight, a.y * keep + r.y * weight, a.z * keep + r.z * weight,
                       a.w * keep + r.w * weight);
}
__device__ __forceinline__ void add64(double& d, float r) { d += double(r); }
__device__ __forceinline__ void add64(double4& d, float4 r) {
    d.x += double(r.x); d.y += double(r.y); d.z += double(r.z); d.w += double(r.w);
}

template <class T, class D>
__global__ void __launch_bounds__(kAccThreads) accumulate_kernel(const T* __restrict__ rad, uint32_t images,
                                                                 T* __restrict__ acc, D* __restrict__ sum64,
                                                                 uint32_t items, uint32_t camera_moved,
                                                                 uint32_t spp0) {
    constexpr uint32_t kBatch = batch_of<T>();
    __shared__ float s_weight[kChunk], s_keep[kChunk];
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool valid = i < items;
    const bool reset0 = camera_moved != 0 || spp0 == 0;
    T a = acc_zero(T{});
    D d = acc_zero64(T{});
    if (valid && !reset0) {
        a = acc[i];
        if (sum64) d = sum64[i];
    }
    #pragma unroll 1
    for (uint32_t c0 = 0; c0 < images; c0 += kChunk) {
        const uint32_t n = min(kChunk, images - c0);
        if (threadIdx.x < n) {
            // image k = c0 + t is folded with spp_before = k (after a reset
            // at image 0) or spp0 + k
            const uint32_t k = c0 + threadIdx.x;
            const float spp = float(reset0 ? k : spp0 + k);
            s_weight[threadIdx.x] = 1.0f / (spp + 1.0f);
            s_keep[threadIdx.x] = spp / (spp + 1.0f);
        }
        __syncthreads();
        if (valid) {
            #pragma unroll 1
            for (uint32_t b0 = 0; b0 < n; b0 += kBatch) {
                T rb[kBatch];
                #pragma unroll
                for (uint32_t u = 0; u < kBatch; ++u)
                    if (b0 + u < n) rb[u] = __ldcs(rad + size_t(c0 + b0 + u) * items + i);
                #pragma unroll
                for (uint32_t u = 0; u < kBatch; ++u) {
                    if (b0 + u >= n) break;
                    const T r = rb[u];
                    if (c0 + b0 + u == 0 && reset0) a = r;
                    else a = fold(a, r, s_keep[b0 + u], s_weight[b0 + u]);
                    add64(d, r);
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
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (px < rr::kSmallPixels) {
        const uint64_t elems = px * 4;
        const uint32_t blocks = uint32_t((elems + rr::kAccThreads - 1) / rr::kAccThreads);
        rr::accumulate_kernel<float, double><<<blocks, rr::kAccThreads, 0, st>>>(
            radiance, image_count, accumulated, oracle_sum, uint32_t(elems), p->camera_moved, p->accumulated_spp);
    } else {
        const uint32_t blocks = uint32_t((px + rr::kAccThreads - 1) / rr::kAccThreads);
        rr::accumulate_kernel<float4, double4><<<blocks, rr::kAccThreads, 0, st>>>(
            reinterpret_cast<const float4*>(radiance), image_count, reinterpret_cast<float4*>(accumulated),
            reinterpret_cast<double4*>(oracle_sum), uint32_t(px), p->camera_moved, p->accumulated_spp);
    }
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}
