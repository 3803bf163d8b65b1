// atrous_static.cu — A-trous denoiser that performs no device allocation.
//
// Some callers cannot allocate device memory at all: an engine that hands the
// library only buffers from its own fixed memory budget, a host that forbids
// cudaMalloc while it renders frames, or a plugin running where the CUDA
// allocator is owned by someone else. rr_atrous_execute needs two caller
// buffers for its ping-pong; this variant needs only the input and the
// output. The one intermediate image it still needs lives in the file-scope
// array below, which the CUDA runtime places in device memory when the module
// is loaded on a device and keeps there until the process exits.
//
// Host code must not hand `g_atrous_scratch` to a kernel: in host code the
// name denotes a host-side stand-in, not a device address. Its device address
// is looked up once per device with cudaGetSymbolAddress (with that device
// current) and cached.
//
// Nothing in the scratch needs to start at zero: every pass writes every
// pixel of its target before the next pass reads it. All calls share the one
// array and it keeps the last call's contents, so two calls whose kernels
// overlap on the GPU (different streams without ordering) race on it.

#include "rr_cuda.h"
#include "rr_dev.cuh"

#include <algorithm>
#include <atomic>
#include <mutex>

namespace {

using namespace rr;

__device__ __align__(256) float4 g_atrous_scratch[RR_ATROUS_STATIC_MAX_PIXELS];

constexpr int kMaxDevices = 64;
std::atomic<float4*> g_scratch_addr[kMaxDevices];
std::mutex g_scratch_mutex;

// Device address of the scratch on the current device (set-up on first use).
cudaError_t scratch_address(float4** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    float4* p = g_scratch_addr[dev].load(std::memory_order_acquire);
    if (!p) {
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        p = g_scratch_addr[dev].load(std::memory_order_relaxed);
        if (!p) {
            e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_atrous_scratch);
            if (e != cudaSuccess) return e;
            g_scratch_addr[dev].store(p, std::memory_order_release);
        }
    }
    *out = p;
    return cudaSuccess;
}

RR_D float luma601(float3 c) { return dot(c, f3(0.299f, 0.587f, 0.114f)); }
RR_D float b3_weight(int o) { return (o == 2 || o == -2) ? 1.0f : ((o == 1 || o == -1) ? 4.0f : 6.0f); }

// One atrous.slang:cs_main pass (atrous.slang:41-106).
__global__ void __launch_bounds__(128) atrous_static_kernel(const float4* __restrict__ in,
                                                            const float4* __restrict__ gpos,
                                                            const float4* __restrict__ gnrm,
                                                            float4* __restrict__ out, int W, int H, int stride,
                                                            float sp2, float sn2, float sl2) {
    const int x = blockIdx.x * 16 + (threadIdx.x & 15);
    const int y = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (x >= W || y >= H) return;
    const size_t ci = size_t(y) * W + x;
    const float4 cpos = gpos[ci];
    const float4 crad = in[ci];
    if (cpos.w < 0.0f) { out[ci] = crad; return; }
    const float3 cn = normalize(xyz(gnrm[ci]));
    const float cl = luma601(xyz(crad));
    float3 acc = f3(0.0f, 0.0f, 0.0f);
    float wsum = 0.0f;
    for (int ty = -2; ty <= 2; ++ty) {
        const int sy = min(max(y + ty * stride, 0), H - 1);
        for (int tx = -2; tx <= 2; ++tx) {
            const int sx = min(max(x + tx * stride, 0), W - 1);
            const size_t si = size_t(sy) * W + sx;
            const float4 spos = gpos[si];
            if (spos.w < 0.0f) continue;
            const float base_w = (b3_weight(tx) * b3_weight(ty)) / 256.0f;
            const float3 pd = xyz(spos) - xyz(cpos);
            const float pos_w = rr_expf(-dot(pd, pd) / sp2);
            const float3 sn = normalize(xyz(gnrm[si]));
            const float normal_w = rr_expf(-mx(0.0f, 1.0f - dot(cn, sn)) / sn2);
            const float3 srad = xyz(in[si]);
            const float ld = luma601(srad) - cl;
            const float luma_w = rr_expf(-(ld * ld) / sl2);
            const float w = base_w * pos_w * normal_w * luma_w;
            acc = acc + srad * w;
            wsum += w;
        }
    }
    const float3 o = wsum > 0.0f ? acc / wsum : xyz(crad);
    out[ci] = make_float4(o.x, o.y, o.z, crad.w);
}

} // namespace

extern "C" rr_status rr_atrous_execute_static(const float* input, const float* gbuf_pos, const float* gbuf_norm,
                                              float* output, const rr_atrous_params* p, void* stream_v) {
    if (!input || !gbuf_pos || !gbuf_norm || !output || !p) return RR_ERR_INVALID_ARGUMENT;
    if (p->width == 0 || p->height == 0) return RR_ERR_INVALID_ARGUMENT;
    if (uint64_t(p->width) * p->height > RR_ATROUS_STATIC_MAX_PIXELS) return RR_ERR_UNSUPPORTED;
    if (input == output) return RR_ERR_INVALID_ARGUMENT;
    float4* scratch = nullptr;
    if (scratch_address(&scratch) != cudaSuccess) return RR_ERR_CUDA;
    const uint32_t iters = std::min(std::max(p->iterations, 1u), 7u);  // AtrousPass.cpp:265
    const float sp2 = std::max(p->sigma_position * p->sigma_position, 1.0e-6f);
    const float sn2 = std::max(p->sigma_normal * p->sigma_normal, 1.0e-6f);
    const float sl2 = std::max(p->sigma_luminance * p->sigma_luminance, 1.0e-6f);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    const dim3 grid((p->width + 15) / 16, (p->height + 7) / 8);
    // Pass i writes the output when (iters-1-i) is even and the scratch
    // otherwise, so the last pass always lands in `output`.
    const float4* read = reinterpret_cast<const float4*>(input);
    for (uint32_t i = 0; i < iters; ++i) {
        float4* write = ((iters - 1u - i) & 1u) == 0u ? reinterpret_cast<float4*>(output) : scratch;
        atrous_static_kernel<<<grid, 128, 0, stream>>>(read, reinterpret_cast<const float4*>(gbuf_pos),
                                                       reinterpret_cast<const float4*>(gbuf_norm), write,
                                                       int(p->width), int(p->height), int(1u << i), sp2, sn2, sl2);
        if (cudaGetLastError() != cudaSuccess) return RR_ERR_CUDA;
        read = write;
    }
    return RR_OK;
}
