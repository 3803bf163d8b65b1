// atrous.cu — edge-aware A-trous wavelet filter (AtrousPass.cpp:243-306,
// kernel atrous.slang:41-106): 5x5 B3 taps (1,4,6,4,1)/16 per axis at
// stride 1<<iter, clamped to the image, skipping G-buffer misses, weighted by
// exp(-|dp|^2/sp^2) * exp(-max(0, 1-n.n')/sn^2) * exp(-dl^2/sl^2).

#include "rr_internal.h"
#include "rr_atrous.cuh"
#include "rr_tc.cuh"

#include <cuda.h>
#include <cudaTypedefs.h>

namespace rr {
namespace {

// The G-buffer normals normalized once per call (the filter reads each
// pixel's normal for up to 25 taps per iteration; normalize is deterministic,
// so the taps see the same values as normalizing on the spot).
__global__ void __launch_bounds__(256) normalize_kernel(const float4* __restrict__ gnrm, float4* __restrict__ out,
                                                        size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float3 v = normalize(xyz(gnrm[i]));
    out[i] = make_float4(v.x, v.y, v.z, 0.0f);
}

// Direct-load filter, one iteration in two launches. A pixel's tap on a
// neighbour has the same weight as the neighbour's opposite tap on the pixel
// (tap_weight), so the 24 neighbour weights of every pixel need only 12
// evaluations, each with three divisions and three exponentials:
//   atrous_pair_weights_kernel: for every pixel, the weights of its 12
//     forward taps (kPairFwd: (1,0), (2,0), then ty = 1, 2 with tx = -2..2),
//     on the clamped neighbour, -1 where either pixel is a G-buffer miss,
//     into 12 planes of W x H floats;
//   atrous_pair_sum_kernel: every pixel's 25 taps in atrous_pixel's order;
//     a forward tap reads its own weight, a backward tap whose neighbour is
//     in the image reads the neighbour's forward weight, and the centre and
//     backward taps clamped at the border are evaluated on the spot.
// The sums see the same weights in the same order as atrous_pixel: the
// same bits. `nrm`: unit normals (from normalize_kernel).
constexpr int kPairFwd = 12;
RR_D int2 pair_offset(int j) { return j < 2 ? make_int2(j + 1, 0) : make_int2((j - 2) % 5 - 2, (j - 2) / 5 + 1); }
RR_D bool pair_forward(int tx, int ty) { return ty > 0 || (ty == 0 && tx > 0); }
RR_D int pair_index(int tx, int ty) { return ty == 0 ? tx - 1 : 2 + (ty - 1) * 5 + (tx + 2); }

__global__ void __launch_bounds__(128) atrous_pair_weights_kernel(const float4* __restrict__ in,
                                                                  const float4* __restrict__ gpos,
                                                                  const float4* __restrict__ nrm,
                                                                  float* __restrict__ wt, int W, int H, int stride,
                                                                  float sp2, float sn2, float sl2) {
    const int x = blockIdx.x * 16 + (threadIdx.x & 15);
    const int y = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (x >= W || y >= H) return;
    const size_t plane = size_t(W) * H;
    const size_t i = size_t(y) * W + x;
    const float4 cpos = __ldg(gpos + i);
    if (cpos.w < 0.0f) {
        #pragma unroll
        for (int j = 0; j < kPairFwd; ++j) wt[j * plane + i] = -1.0f;
        return;
    }
    const float3 cn = xyz(__ldg(nrm + i));
    const float cl = luminance601(xyz(__ldg(in + i)));
    #pragma unroll
    for (int j = 0; j < kPairFwd; ++j) {
        const int2 o = pair_offset(j);
        const int sx = min(max(x + o.x * stride, 0), W - 1);
        const int sy = min(max(y + o.y * stride, 0), H - 1);
        const size_t k = size_t(sy) * W + sx;
        // the neighbour's three values are loaded whether or not it is a miss
        // (the address is in the image), so the loads of all taps can be in
        // flight together
        const float4 spos = __ldg(gpos + k);
        const float3 sn = xyz(__ldg(nrm + k));
        const float3 srad = xyz(__ldg(in + k));
        const float w = tap_weight(o.x, o.y, xyz(cpos), cn, cl, xyz(spos), sn, srad, sp2, sn2, sl2);
        wt[j * plane + i] = spos.w < 0.0f ? -1.0f : w;
    }
}

__global__ void __launch_bounds__(128) atrous_pair_sum_kernel(const float4* __restrict__ in,
                                                              const float4* __restrict__ gpos,
                                                              const float4* __restrict__ nrm,
                                                              const float* __restrict__ wt,
                                                              float4* __restrict__ out, int W, int H, int stride,
                                                              float sp2, float sn2, float sl2) {
    const int x = blockIdx.x * 16 + (threadIdx.x & 15);
    const int y = blockIdx.y * 8 + (threadIdx.x >> 4);
    if (x >= W || y >= H) return;
    const size_t plane = size_t(W) * H;
    const size_t i = size_t(y) * W + x;
    const float4 cpos = __ldg(gpos + i);
    const float4 crad = __ldg(in + i);
    if (cpos.w < 0.0f) {
        out[i] = crad;
        return;
    }
    const float3 cn = xyz(__ldg(nrm + i));
    const float cl = luminance601(xyz(crad));
    float3 filtered = f3(0.0f, 0.0f, 0.0f);
    float wsum = 0.0f;
    #pragma unroll
    for (int ty = -2; ty <= 2; ++ty) {
        const int uy = y + ty * stride;
        const int sy = min(max(uy, 0), H - 1);
        #pragma unroll
        for (int tx = -2; tx <= 2; ++tx) {
            const int ux = x + tx * stride;
            const int sx = min(max(ux, 0), W - 1);
            const size_t k = size_t(sy) * W + sx;
            float w;
            if (tx == 0 && ty == 0) {
                w = tap_weight(0, 0, xyz(cpos), cn, cl, xyz(cpos), cn, xyz(crad), sp2, sn2, sl2);
            } else if (pair_forward(tx, ty)) {
                w = __ldg(wt + pair_index(tx, ty) * plane + i);
            } else if (ux == sx && uy == sy) {
                w = __ldg(wt + pair_index(-tx, -ty) * plane + k);
            } else {
                const float4 spos = __ldg(gpos + k);
                w = spos.w < 0.0f ? -1.0f
                                  : tap_weight(tx, ty, xyz(cpos), cn, cl, xyz(spos), xyz(__ldg(nrm + k)),
                                               xyz(__ldg(in + k)), sp2, sn2, sl2);
            }
            // loaded before the weight is known (the address is in the image)
            const float3 srad = xyz(__ldg(in + k));
            if (!(w < 0.0f)) {   // w < 0: a G-buffer miss
                filtered = filtered + srad * w;
                wsum += w;
            }
        }
    }
    const float3 o = wsum > 0.0f ? filtered / wsum : xyz(crad);
    out[i] = make_float4(o.x, o.y, o.z, crad.w);
}

// TMA-staged form of the filter for strides 1, 2 and 4: a block of 32 x 8
// output pixels first loads its halo tile (the 5x5 taps reach 2*S pixels
// beyond the block on every side) of radiance, position and unit normal
// with three 3-D tensor copies (cp.async.bulk.tensor, box (4 floats,
// 32 + 4S, 8 + 4S), started 2S pixels up-left of the block, so at negative
// coordinates on the image's top and left edges) completing on one
// mbarrier. A tap clamped to the image lies inside the tile, so each tap
// reads the tile at its clamped coordinate; the box's out-of-image part
// (zero-filled) is never read. The arithmetic is atrous_kernel's, on the
// same values: the results are the same bits.
template <int S>
struct AtrousTile {
    static constexpr int W = 32 + 4 * S, H = 8 + 4 * S;
    static constexpr uint32_t kBytes = uint32_t(W * H * 16);   // one image's box
    static constexpr uint32_t kSmem = 3 * kBytes + 16;
    static_assert(kBytes % 128 == 0, "tiles stay 128-byte aligned");
};

// The images in a block's halo tile in shared memory.
template <int S>
struct TileFetch {
    const float4* rad_t;
    const float4* pos_t;
    const float4* nrm_t;
    int tx0, ty0;
    RR_D int at(int x, int y) const { return (y - ty0) * AtrousTile<S>::W + (x - tx0); }
    RR_D float4 rad(int x, int y) const { return rad_t[at(x, y)]; }
    RR_D float4 pos(int x, int y) const { return pos_t[at(x, y)]; }
    RR_D float4 nrm(int x, int y) const { return nrm_t[at(x, y)]; }
};

__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, int c0, int c1, int c2,
                                            uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4}], [%5];"
        ::"r"(tc::smem_addr(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2),
          "r"(tc::smem_addr(bar))
        : "memory");
}

template <int S>
__global__ void __launch_bounds__(256) atrous_tma_kernel(const __grid_constant__ CUtensorMap m_rad,
                                                         const __grid_constant__ CUtensorMap m_pos,
                                                         const __grid_constant__ CUtensorMap m_nrm,
                                                         const float4* __restrict__ in_g,
                                                         const float4* __restrict__ pos_g,
                                                         const float4* __restrict__ nrm_g,
                                                         float4* __restrict__ out, int W, int H, float sp2,
                                                         float sn2, float sl2, int* error, uint32_t wait_tries) {
    using T = AtrousTile<S>;
    extern __shared__ __align__(128) unsigned char sm[];
    const float4* t_rad = reinterpret_cast<const float4*>(sm);
    const float4* t_pos = t_rad + T::W * T::H;
    const float4* t_nrm = t_pos + T::W * T::H;
    uint64_t* bar = reinterpret_cast<uint64_t*>(sm + 3 * T::kBytes);
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 8;
    const int tx0 = x0 - 2 * S, ty0 = y0 - 2 * S;
    if (threadIdx.x == 0) {
        tc::mbar_init(bar, 1);
        tc::fence_proxy_async();
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(tc::smem_addr(bar)),
                     "r"(3 * T::kBytes)
                     : "memory");
        tma_load_3d(sm, &m_rad, 0, tx0, ty0, bar);
        tma_load_3d(sm + T::kBytes, &m_pos, 0, tx0, ty0, bar);
        tma_load_3d(sm + 2 * T::kBytes, &m_nrm, 0, tx0, ty0, bar);
    }
    __syncthreads();
    const bool staged = tc::mbar_wait(bar, 0, wait_tries);
    if (!staged) {
        // the copies did not complete within the bounded wait: report it in
        // the host-mapped flag, give them one more bounded wait so that none
        // is left writing this block's shared memory after it leaves, and
        // filter this thread's pixel from global memory instead (same bits)
        *reinterpret_cast<volatile int*>(error) = 1;
        tc::mbar_wait(bar, 0);
    }
    const int x = x0 + int(threadIdx.x & 31u), y = y0 + int(threadIdx.x >> 5);
    if (x >= W || y >= H) return;
    const size_t ci = size_t(y) * W + x;
    if (staged) {
        const TileFetch<S> f{t_rad, t_pos, t_nrm, tx0, ty0};
        out[ci] = atrous_pixel(f, x, y, W, H, S, sp2, sn2, sl2);
    } else {
        out[ci] = atrous_pixel(GlobalFetch{in_g, pos_g, nrm_g, W}, x, y, W, H, S, sp2, sn2, sl2);
    }
}

} // namespace
} // namespace rr

// cuTensorMapEncodeTiled from the driver (no link-time dependency on it).
PFN_cuTensorMapEncodeTiled_v12000 rr_tensor_map_encoder() {
    // looked up once (a function-local static: initialised once, thread-safe)
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
        return static_cast<PFN_cuTensorMapEncodeTiled_v12000>(nullptr);
    }();
    return fn;
}

// A W x H RGBA32F image as a 3-D tensor (4 floats, W, H) with a box of
// (4, bw, bh); false if the driver refuses it (the caller then uses the
// direct-load kernel).
static bool image_map(CUtensorMap* m, const void* img, uint32_t W, uint32_t H, uint32_t bw, uint32_t bh) {
    PFN_cuTensorMapEncodeTiled_v12000 enc = rr_tensor_map_encoder();
    if (!enc || (reinterpret_cast<uintptr_t>(img) & 15u) != 0) return false;
    const cuuint64_t dims[3] = {4, W, H};
    const cuuint64_t strides[2] = {16, cuuint64_t(W) * 16};
    const cuuint32_t box[3] = {4, bw, bh};
    const cuuint32_t estr[3] = {1, 1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 3, const_cast<void*>(img), dims, strides, box, estr,
               CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
               CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <int S>
static bool atrous_tma_launch(rr_ctx* ctx, const float* input, const float* gpos, const float4* nrm, float* output,
                              uint32_t W, uint32_t H, float sp2, float sn2, float sl2, cudaStream_t stream) {
    using T = rr::AtrousTile<S>;
    CUtensorMap mr, mp, mn;
    if (!image_map(&mr, input, W, H, T::W, T::H) || !image_map(&mp, gpos, W, H, T::W, T::H) ||
        !image_map(&mn, nrm, W, H, T::W, T::H))
        return false;
    if (cudaFuncSetAttribute(rr::atrous_tma_kernel<S>, cudaFuncAttributeMaxDynamicSharedMemorySize, T::kSmem) !=
        cudaSuccess)
        return false;
    const dim3 grid((W + 31) / 32, (H + 7) / 8);
    rr::atrous_tma_kernel<S><<<grid, 256, T::kSmem, stream>>>(
        mr, mp, mn, reinterpret_cast<const float4*>(input), reinterpret_cast<const float4*>(gpos), nrm,
        reinterpret_cast<float4*>(output), int(W), int(H), sp2, sn2, sl2, ctx->atrous_error_dev,
        ctx->atrous_wait_tries);
    return true;
}

// Unit normals of `gnrm` into the context's scratch image.
static rr_status atrous_normals(rr_ctx* ctx, const float* gnrm, uint32_t W, uint32_t H, cudaStream_t stream,
                                const float4** out) {
    const size_t n = size_t(W) * H;
    if (ctx->atrous_nrm_px < n) {
        cudaFree(ctx->atrous_nrm);
        ctx->atrous_nrm = nullptr;
        ctx->atrous_nrm_px = 0;
        RR_TRY_CUDA(ctx, cudaMalloc(&ctx->atrous_nrm, n * sizeof(float4)));
        ctx->atrous_nrm_px = n;
    }
    rr::normalize_kernel<<<unsigned((n + 255) / 256), 256, 0, stream>>>(reinterpret_cast<const float4*>(gnrm),
                                                                        ctx->atrous_nrm, n);
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    *out = ctx->atrous_nrm;
    return RR_OK;
}

static rr_status atrous_launch(rr_ctx* ctx, const float* input, const float* gpos, const float4* nrm,
                               float* output, uint32_t W, uint32_t H, uint32_t stride, float sp, float sn,
                               float sl, cudaStream_t stream) {
    const float sp2 = std::max(sp * sp, 1.0e-6f), sn2 = std::max(sn * sn, 1.0e-6f), sl2 = std::max(sl * sl, 1.0e-6f);
    if (ctx->atrous_tma && (stride == 1 || stride == 2 || stride == 4)) {
        if (!ctx->atrous_error) {
            // one host-mapped word: a block that gives up writes it, and the
            // next A-trous call reads it without synchronizing
            int* h = nullptr;
            RR_TRY_CUDA(ctx, cudaHostAlloc(reinterpret_cast<void**>(&h), sizeof(int), cudaHostAllocMapped));
            *reinterpret_cast<volatile int*>(h) = 0;
            void* d = nullptr;
            cudaError_t e = cudaHostGetDevicePointer(&d, h, 0);
            if (e != cudaSuccess) {
                cudaFreeHost(h);
                RR_TRY_CUDA(ctx, e);
            }
            ctx->atrous_error = h;
            ctx->atrous_error_dev = static_cast<int*>(d);
        }
        bool launched = false;
        if (stride == 1) launched = atrous_tma_launch<1>(ctx, input, gpos, nrm, output, W, H, sp2, sn2, sl2, stream);
        else if (stride == 2) launched = atrous_tma_launch<2>(ctx, input, gpos, nrm, output, W, H, sp2, sn2, sl2, stream);
        else launched = atrous_tma_launch<4>(ctx, input, gpos, nrm, output, W, H, sp2, sn2, sl2, stream);
        if (launched) {
            RR_CHECK_LAUNCH(ctx);
            ctx->launches += 1;
            return RR_OK;
        }
    }
    const size_t need = size_t(rr::kPairFwd) * W * H;
    if (ctx->atrous_wt_floats < need) {
        cudaFree(ctx->atrous_wt);
        ctx->atrous_wt = nullptr;
        ctx->atrous_wt_floats = 0;
        RR_TRY_CUDA(ctx, cudaMalloc(&ctx->atrous_wt, need * sizeof(float)));
        ctx->atrous_wt_floats = need;
    }
    dim3 grid((W + 15) / 16, (H + 7) / 8);
    rr::atrous_pair_weights_kernel<<<grid, 128, 0, stream>>>(
        reinterpret_cast<const float4*>(input), reinterpret_cast<const float4*>(gpos), nrm, ctx->atrous_wt, int(W),
        int(H), int(stride), sp2, sn2, sl2);
    RR_CHECK_LAUNCH(ctx);
    rr::atrous_pair_sum_kernel<<<grid, 128, 0, stream>>>(
        reinterpret_cast<const float4*>(input), reinterpret_cast<const float4*>(gpos), nrm, ctx->atrous_wt,
        reinterpret_cast<float4*>(output), int(W), int(H), int(stride), sp2, sn2, sl2);
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 2;
    return RR_OK;
}

// An earlier call's tile copies missed their bounded wait (the flag the
// blocks write into host-mapped memory): reported once, here, at the next
// call, which then does no work. The earlier call's output is complete: the
// blocks that gave up filtered their pixels from global memory.
static rr_status atrous_report_give_up(rr_ctx* ctx, const char* who) {
    if (!ctx->atrous_error || *reinterpret_cast<volatile int*>(ctx->atrous_error) == 0) return RR_OK;
    *reinterpret_cast<volatile int*>(ctx->atrous_error) = 0;
    return rr_fail(ctx, RR_ERR_TIMEOUT,
                   "%s: an earlier A-trous call's TMA tile copies did not complete within the bounded wait "
                   "(that call's output was filtered from global memory instead); this call did no work",
                   who);
}

extern "C" rr_status rr_atrous_iteration(rr_ctx* ctx, const float* input, const float* gpos,
                                         const float* gnrm, float* output, const rr_atrous_params* p,
                                         void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!input || !gpos || !gnrm || !output || !p) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_atrous_iteration: null argument");
    if (p->width == 0 || p->height == 0 || p->width > 65535u * 16u || p->height > 65535u * 8u)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_atrous_iteration: bad image size");
    if (input == output) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_atrous_iteration: input aliases output");
    if (rr_status g = atrous_report_give_up(ctx, "rr_atrous_iteration")) return g;
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    const float4* nrm = nullptr;
    rr_status st = atrous_normals(ctx, gnrm, p->width, p->height, static_cast<cudaStream_t>(stream), &nrm);
    if (st != RR_OK) return st;
    return atrous_launch(ctx, input, gpos, nrm, output, p->width, p->height, p->stride, p->sigma_position,
                         p->sigma_normal, p->sigma_luminance, static_cast<cudaStream_t>(stream));
}

extern "C" rr_status rr_atrous_execute(rr_ctx* ctx, const float* input, const float* gpos, const float* gnrm,
                                       float* ping0, float* ping1, const rr_atrous_params* p,
                                       uint32_t* out_slot, void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!input || !gpos || !gnrm || !ping0 || !ping1 || !p)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_atrous_execute: null argument");
    if (p->width == 0 || p->height == 0 || p->width > 65535u * 16u || p->height > 65535u * 8u)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_atrous_execute: bad image size");
    if (input == ping0 || input == ping1 || ping0 == ping1)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_atrous_execute: buffers alias");
    if (rr_status g = atrous_report_give_up(ctx, "rr_atrous_execute")) return g;
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    // AtrousPass.cpp:265 clamps to 1..7; slot (iterations-1)&1 holds the result.
    const uint32_t iters = std::min(std::max(p->iterations, 1u), 7u);
    const float4* nrm = nullptr;
    rr_status st0 = atrous_normals(ctx, gnrm, p->width, p->height, static_cast<cudaStream_t>(stream), &nrm);
    if (st0 != RR_OK) return st0;
    const float* read = input;
    float* ping[2] = {ping0, ping1};
    for (uint32_t it = 0; it < iters; ++it) {
        float* write = ping[it & 1u];
        rr_status st = atrous_launch(ctx, read, gpos, nrm, write, p->width, p->height, 1u << it,
                                     p->sigma_position, p->sigma_normal, p->sigma_luminance,
                                     static_cast<cudaStream_t>(stream));
        if (st != RR_OK) return st;
        read = write;
    }
    if (out_slot) *out_slot = (iters - 1u) & 1u;
    return RR_OK;
}

extern "C" rr_status rr_atrous_set_tma(rr_ctx* ctx, int enable) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    ctx->atrous_tma = enable != 0;
    return RR_OK;
}

extern "C" rr_status rr_atrous_tma_error(rr_ctx* ctx, int* error_out) {
    if (!ctx || !error_out) return RR_ERR_INVALID_ARGUMENT;
    *error_out = 0;
    if (!ctx->atrous_error) return RR_OK;
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    RR_TRY_CUDA(ctx, cudaDeviceSynchronize());
    *error_out = *reinterpret_cast<volatile int*>(ctx->atrous_error);
    *reinterpret_cast<volatile int*>(ctx->atrous_error) = 0;
    return RR_OK;
}

extern "C" rr_status rr_atrous_set_tma_wait_tries(rr_ctx* ctx, uint32_t tries) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    ctx->atrous_wait_tries = tries;
    return RR_OK;
}
