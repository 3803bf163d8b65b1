// image.cu — output-format utilities of the reference app on the device:
//   rr_tonemap_execute: exposure, ACES filmic approximation (Narkowicz),
//     clamp, gamma 1/2.2, 8-bit RGBA (Application.cpp:853-866, the same math
//     as tonemap.slang:40-69), for PNG output;
//   rr_image_mse: mean squared error over the RGB channels of a window of two
//     RGBA32F images in FP64 (Application::compute_mse, Application.cpp:
//     892-949, which reads back a 64x64 centre crop). The reduction order is
//     fixed (per-thread strided sums, fixed tree, one final block), so the
//     result is deterministic.

#include "rr_internal.h"

namespace rr {
namespace {

__global__ void __launch_bounds__(256) tonemap_kernel(const float4* __restrict__ in, uchar4* __restrict__ out,
                                                      uint32_t n, float exposure) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 h = in[i];
    float c[3] = {h.x, h.y, h.z};
    unsigned char b[3];
    #pragma unroll
    for (int k = 0; k < 3; ++k) {
        float v = c[k] * exposure;
        v = (v * (2.51f * v + 0.03f)) / (v * (2.43f * v + 0.59f) + 0.14f);
        v = fminf(fmaxf(v, 0.0f), 1.0f);
        v = powf(v, 1.0f / 2.2f);
        b[k] = static_cast<unsigned char>(v * 255.0f + 0.5f);
    }
    out[i] = make_uchar4(b[0], b[1], b[2], 255);
}

constexpr int kMseBlocks = 296;
constexpr int kMseThreads = 256;

__global__ void __launch_bounds__(kMseThreads) mse_partial_kernel(const float4* __restrict__ a, const float4* __restrict__ b,
                                                                  uint32_t W, uint32_t x0, uint32_t y0, uint32_t w,
                                                                  uint32_t h, double* __restrict__ partial) {
    __shared__ double red[kMseThreads];
    const uint64_t n = uint64_t(w) * h;
    double acc = 0.0;
    for (uint64_t k = uint64_t(blockIdx.x) * kMseThreads + threadIdx.x; k < n; k += uint64_t(kMseBlocks) * kMseThreads) {
        const uint32_t y = y0 + uint32_t(k / w), x = x0 + uint32_t(k % w);
        const float4 p = a[size_t(y) * W + x], q = b[size_t(y) * W + x];
        const double dx = double(p.x) - double(q.x), dy = double(p.y) - double(q.y), dz = double(p.z) - double(q.z);
        acc += dx * dx;
        acc += dy * dy;
        acc += dz * dz;
    }
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = kMseThreads / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) partial[blockIdx.x] = red[0];
}

__global__ void __launch_bounds__(32) mse_final_kernel(const double* __restrict__ partial, double denom,
                                                       double* __restrict__ out) {
    if (threadIdx.x != 0) return;
    double s = 0.0;
    for (int k = 0; k < kMseBlocks; ++k) s += partial[k];
    *out = s / denom;
}

} // namespace
} // namespace rr

extern "C" rr_status rr_tonemap_execute(rr_ctx* ctx, const float* hdr, uint32_t width, uint32_t height,
                                        float exposure, uint8_t* rgba8_out, void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!hdr || !rgba8_out || width == 0 || height == 0)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_tonemap_execute: bad argument");
    const uint64_t n = uint64_t(width) * height;
    if (n >= (1ull << 31)) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_tonemap_execute: image too large");
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    rr::tonemap_kernel<<<uint32_t((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const float4*>(hdr), reinterpret_cast<uchar4*>(rgba8_out), uint32_t(n), exposure);
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

extern "C" rr_status rr_image_mse(rr_ctx* ctx, const float* a, const float* b, uint32_t width, uint32_t height,
                                  uint32_t x0, uint32_t y0, uint32_t w, uint32_t h, double* mse_out_dev,
                                  void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!a || !b || !mse_out_dev || w == 0 || h == 0 || uint64_t(x0) + w > width || uint64_t(y0) + h > height)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_image_mse: bad argument or window");
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    if (!ctx->mse_partial) RR_TRY_CUDA(ctx, cudaMalloc(&ctx->mse_partial, sizeof(double) * rr::kMseBlocks));
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    rr::mse_partial_kernel<<<rr::kMseBlocks, rr::kMseThreads, 0, s>>>(
        reinterpret_cast<const float4*>(a), reinterpret_cast<const float4*>(b), width, x0, y0, w, h, ctx->mse_partial);
    RR_CHECK_LAUNCH(ctx);
    rr::mse_final_kernel<<<1, 32, 0, s>>>(ctx->mse_partial, double(w) * double(h) * 3.0, mse_out_dev);
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 2;
    return RR_OK;
}
