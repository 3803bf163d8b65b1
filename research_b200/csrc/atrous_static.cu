// atrous_static.cu — A-trous denoiser that performs no device allocation.
//
// Some callers cannot allocate device memory at all: an engine that hands the
// library only buffers from its own fixed memory budget, a host that forbids
// cudaMalloc while it renders frames, or a plugin running where the CUDA
// allocator is owned by someone else. rr_atrous_execute needs two caller
// buffers for its ping-pong and a library buffer for the unit normals; this
// variant needs only the input and the output. The one intermediate image it
// still needs lives in the file-scope array below, which the CUDA runtime
// places in device memory when the module is loaded on a device and keeps
// there until the process exits. Normals are normalized at each tap (the same
// values the other entry point computes once per call).
//
// Host code must not hand `g_atrous_scratch` to a kernel: in host code the
// name denotes a host-side stand-in, not a device address. Its device address
// is looked up with cudaGetSymbolAddress, with the device current, and cached
// per device together with the unique id of the CUDA context it was looked up
// in; a call in another context (after cudaDeviceReset, for one) looks it up
// again.
//
// Nothing in the scratch needs to start at zero: every pass writes every
// pixel of its target before the next pass reads it. All calls share the one
// array and it keeps the last call's contents, so two calls whose kernels
// overlap on the GPU (different streams without ordering) race on it.

#include "rr_cuda.h"
#include "rr_atrous.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <mutex>

namespace {

using namespace rr;

__device__ __align__(256) float4 g_atrous_scratch[RR_ATROUS_STATIC_MAX_PIXELS];

constexpr int kMaxDevices = 64;

struct ScratchSlot {
    float4* addr = nullptr;
    unsigned long long context_id = 0;  // cuCtxGetId of the context the address belongs to
};
ScratchSlot g_scratch[kMaxDevices];
std::mutex g_scratch_mutex;

// cuCtxGetCurrent / cuCtxGetId from the driver (no link-time dependency).
struct ContextIdFns {
    PFN_cuCtxGetCurrent_v4000 get_current = nullptr;
    PFN_cuCtxGetId_v12000 get_id = nullptr;
};

const ContextIdFns& context_id_fns() {
    static const ContextIdFns fns = [] {
        ContextIdFns f;
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            f.get_current = reinterpret_cast<PFN_cuCtxGetCurrent_v4000>(p);
        p = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            f.get_id = reinterpret_cast<PFN_cuCtxGetId_v12000>(p);
        return f;
    }();
    return fns;
}

// Unique id of the calling thread's current CUDA context; 0 if none is
// current or the driver cannot say (the address is then never cached).
unsigned long long current_context_id() {
    const ContextIdFns& f = context_id_fns();
    if (!f.get_current || !f.get_id) return 0;
    CUcontext c = nullptr;
    unsigned long long id = 0;
    if (f.get_current(&c) != CUDA_SUCCESS || !c) return 0;
    if (f.get_id(c, &id) != CUDA_SUCCESS) return 0;
    return id;
}

// Device address of the scratch in the current context of the current device.
cudaError_t scratch_address(float4** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    unsigned long long id = current_context_id();
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    ScratchSlot& s = g_scratch[dev];
    if (s.addr && id != 0 && s.context_id == id) {
        *out = s.addr;
        return cudaSuccess;
    }
    float4* p = nullptr;
    e = cudaGetSymbolAddress(reinterpret_cast<void**>(&p), g_atrous_scratch);
    if (e != cudaSuccess) return e;
    if (id == 0) id = current_context_id();  // the lookup may have made the primary context current
    s.addr = p;
    s.context_id = id;
    *out = p;
    return cudaSuccess;
}

// The caller's images in global memory; normals normalized at each read
// (normalize is deterministic: the values normalize_kernel would store).
struct NormalizingFetch {
    const float4* __restrict__ rad_g;
    const float4* __restrict__ pos_g;
    const float4* __restrict__ nrm_g;
    int W;
    RR_D float4 rad(int x, int y) const { return __ldg(rad_g + size_t(y) * W + x); }
    RR_D float4 pos(int x, int y) const { return __ldg(pos_g + size_t(y) * W + x); }
    RR_D float4 nrm(int x, int y) const {
        const float3 v = normalize(xyz(__ldg(nrm_g + size_t(y) * W + x)));
        return make_float4(v.x, v.y, v.z, 0.0f);
    }
};

// One atrous.slang:cs_main pass (atrous.slang:41-106).
__global__ void __launch_bounds__(128) atrous_static_kernel(const float4* __restrict__ in,
                                                            const float4* __restrict__ gpos,
                                                            const float4* __restrict__ gnrm,
                                                            float4* __restrict__ out, int W, int H, int stride,
                                                            float sp2, float sn2, float sl2) {
    const int x = blockIdx.x * 16 + (threadIdx.x & 15);
    const int y = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (x >= W || y >= H) return;
    out[size_t(y) * W + x] = atrous_pixel(NormalizingFetch{in, gpos, gnrm, W}, x, y, W, H, stride, sp2, sn2, sl2);
}

// Byte ranges [a, a+n) and [b, b+n) share a byte.
bool overlaps(const void* a, const void* b, size_t n) {
    const uintptr_t x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    return x < y + n && y < x + n;
}

} // namespace

extern "C" rr_status rr_atrous_execute_static(const float* input, const float* gbuf_pos, const float* gbuf_norm,
                                              float* output, const rr_atrous_params* p, void* stream_v) {
    if (!input || !gbuf_pos || !gbuf_norm || !output || !p) return RR_ERR_INVALID_ARGUMENT;
    // the same image-size limits as rr_atrous_execute (grid of 16 x 8 blocks)
    if (p->width == 0 || p->height == 0 || p->width > 65535u * 16u || p->height > 65535u * 8u)
        return RR_ERR_INVALID_ARGUMENT;
    if (uint64_t(p->width) * p->height > RR_ATROUS_STATIC_MAX_PIXELS) return RR_ERR_UNSUPPORTED;
    const size_t bytes = size_t(p->width) * p->height * sizeof(float4);
    if (overlaps(input, output, bytes) || overlaps(gbuf_pos, output, bytes) || overlaps(gbuf_norm, output, bytes))
        return RR_ERR_INVALID_ARGUMENT;
    float4* scratch = nullptr;
    if (scratch_address(&scratch) != cudaSuccess) return RR_ERR_CUDA;
    const uint32_t iters = std::min(std::max(p->iterations, 1u), 7u);  // AtrousPass.cpp:265
    const float sp2 = std::max(p->sigma_position * p->sigma_position, 1.0e-6f);
    const float sn2 = std::max(p->sigma_normal * p->sigma_normal, 1.0e-6f);
    const float sl2 = std::max(p->sigma_luminance * p->sigma_luminance, 1.0e-6f);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    const dim3 grid((p->width + 15) / 16, (p->height + 7) / 8);
    int W = int(p->width), H = int(p->height);
    const float4* pos = reinterpret_cast<const float4*>(gbuf_pos);
    const float4* nrm = reinterpret_cast<const float4*>(gbuf_norm);
    // Pass i writes the output when (iters-1-i) is even and the scratch
    // otherwise, so the last pass always lands in `output`.
    const float4* read = reinterpret_cast<const float4*>(input);
    for (uint32_t i = 0; i < iters; ++i) {
        float4* write = ((iters - 1u - i) & 1u) == 0u ? reinterpret_cast<float4*>(output) : scratch;
        int stride = int(1u << i);
        float a_sp2 = sp2, a_sn2 = sn2, a_sl2 = sl2;
        void* args[] = {&read, &pos, &nrm, &write, &W, &H, &stride, &a_sp2, &a_sn2, &a_sl2};
        // the launch's own status: an error left by earlier, unrelated work
        // on this thread is neither reported here nor cleared
        if (cudaLaunchKernel(reinterpret_cast<const void*>(&atrous_static_kernel), grid, dim3(128), args, 0,
                             stream) != cudaSuccess) {
            cudaGetLastError();  // the failed launch's error, recorded by the runtime
            return RR_ERR_CUDA;
        }
        read = write;
    }
    return RR_OK;
}
