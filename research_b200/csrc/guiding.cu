// guiding.cu — world-space vMF guiding grid (assets/shaders/include/
// GuidingGrid.slang; host side ReSTIRPTPass.cpp:311-341, 602-611, 784-810).
//   splat : fixed-point (2^20) direction sums + count per hashed cell with
//           four 32-bit integer atomics (GuidingGrid.slang:73-90); integer
//           addition makes the accumulators order-independent (bit-exact)
//   fit   : Banerjee closed form per cell, resets the accumulator
//           (GuidingGrid.slang:100-137, cs_fit_guiding restir_pt.slang:1005-1015)
//   sample: one-sample MIS of the fitted lobe and a cosine lobe at a surface
//           point (sample_primary_dir, restir_pt.slang:520-563)

#include "rr_grid.cuh"

namespace rr {
namespace {

__global__ void __launch_bounds__(256) splat_kernel(uint32_t* __restrict__ accum, const float4* __restrict__ pos,
                                                    const float4* __restrict__ dir,
                                                    const uint32_t* __restrict__ bsdf, uint32_t n, GridParams g) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i], d = dir[i];
    splat_dir(accum, cell_index(xyz(p), bsdf[i], g), xyz(d));
}

__global__ void __launch_bounds__(256) fit_kernel(int4* __restrict__ accum, float4* __restrict__ fitted, GridParams g) {
    const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= g.cell_count) return;
    const int4 a = accum[cell];
    accum[cell] = make_int4(0, 0, 0, 0);
    const uint32_t n = uint32_t(a.w);
    if (n < (g.min_samples > 1u ? g.min_samples : 1u)) {
        // only kappa is written; mu keeps its previous value (GuidingGrid.slang:120)
        reinterpret_cast<float*>(fitted + cell)[3] = -1.0f;
        return;
    }
    const float3 sum = f3(float(a.x), float(a.y), float(a.z)) * (1.0f / 1048576.0f);
    const float len = length(sum);
    float r = len / float(n);
    r = clampf(r, 1.0e-4f, 0.9999f);
    const float3 mu = len > 1.0e-6f ? sum / len : f3(0.0f, 0.0f, 1.0f);
    float kappa = r * (3.0f - r * r) / (1.0f - r * r);
    kappa = clampf(kappa, 0.5f, g.kappa_max);
    fitted[cell] = make_float4(mu.x, mu.y, mu.z, kappa);
}

__global__ void __launch_bounds__(256) sample_kernel(const float4* __restrict__ fitted, const float4* __restrict__ pos,
                                                     const float4* __restrict__ nrm, const uint32_t* __restrict__ bsdf,
                                                     uint32_t* __restrict__ seeds, uint32_t n, GridParams g,
                                                     float4* __restrict__ wi_out, float* __restrict__ pdf_out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    uint32_t seed = seeds[i];
    float pdf;
    const float3 wi = sample_primary_dir(fitted, xyz(pos[i]), xyz(nrm[i]), bsdf[i], g, seed, pdf);
    wi_out[i] = make_float4(wi.x, wi.y, wi.z, 0.0f);
    pdf_out[i] = pdf;
    seeds[i] = seed;
}

} // namespace
} // namespace rr

using namespace rr;

extern "C" rr_status rr_guiding_splat(rr_ctx* ctx, int32_t* accum, const float* pos, const float* dir,
                                      const uint32_t* bsdf, uint32_t count, const float cam[3],
                                      const rr_guiding_params* p, void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!accum || !p || !cam || (count && (!pos || !dir || !bsdf)) || p->cell_count == 0)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_guiding_splat: bad argument");
    if (count == 0) return RR_OK;
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    splat_kernel<<<(count + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<uint32_t*>(accum), reinterpret_cast<const float4*>(pos),
        reinterpret_cast<const float4*>(dir), bsdf, count, to_grid(p, cam));
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

extern "C" rr_status rr_guiding_fit(rr_ctx* ctx, int32_t* accum, float* fitted, const rr_guiding_params* p,
                                    void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!accum || !fitted || !p || p->cell_count == 0) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_guiding_fit: bad argument");
    if (p->enabled == 0u) return RR_OK;  // restir_pt.slang:1010
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    fit_kernel<<<(p->cell_count + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<int4*>(accum), reinterpret_cast<float4*>(fitted), to_grid(p, nullptr));
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

extern "C" rr_status rr_guiding_sample(rr_ctx* ctx, const float* fitted, const float* pos, const float* nrm,
                                       const uint32_t* bsdf, uint32_t* seeds, uint32_t count, const float cam[3],
                                       const rr_guiding_params* p, float* wi_out, float* pdf_out, void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!fitted || !p || !cam || p->cell_count == 0 || (count && (!pos || !nrm || !bsdf || !seeds || !wi_out || !pdf_out)))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_guiding_sample: bad argument");
    if (count == 0) return RR_OK;
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    sample_kernel<<<(count + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const float4*>(fitted), reinterpret_cast<const float4*>(pos),
        reinterpret_cast<const float4*>(nrm), bsdf, seeds, count, to_grid(p, cam),
        reinterpret_cast<float4*>(wi_out), pdf_out);
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

extern "C" rr_status rr_guiding_reset(rr_ctx* ctx, int32_t* accum, float* fitted, const rr_guiding_params* p,
                                      void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!accum || !fitted || !p) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_guiding_reset: bad argument");
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t bytes = size_t(p->cell_count) * 16;
    RR_TRY_CUDA(ctx, cudaMemsetAsync(accum, 0, bytes, static_cast<cudaStream_t>(stream)));
    RR_TRY_CUDA(ctx, cudaMemsetAsync(fitted, 0, bytes, static_cast<cudaStream_t>(stream)));
    return RR_OK;
}

// ── batched closest-hit queries ───────────────────────────────────────────
namespace rr {
namespace {
__global__ void __launch_bounds__(128) trace_batch_kernel(DevScene s, const float4* __restrict__ o,
                                                          const float4* __restrict__ d, float tmin, float tmax,
                                                          uint32_t n, float4* __restrict__ hits,
                                                          uint32_t* __restrict__ prims) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = o[i], b = d[i];
    HitRec h;
    if (trace<false>(s, make_ray(xyz(a), xyz(b)), tmin, tmax, h)) {
        hits[i] = make_float4(h.t, h.u, h.v, __uint_as_float(h.inst));
        prims[i] = h.prim;
    } else {
        hits[i] = make_float4(-1.0f, 0.0f, 0.0f, __uint_as_float(kNoIndex));
        prims[i] = kNoIndex;
    }
}
template <bool AnyHit, bool Wide>
__global__ void __launch_bounds__(128) trace_counted_kernel(DevScene s, const float4* __restrict__ o,
                                                            const float4* __restrict__ d, float tmin, float tmax,
                                                            uint32_t n, float4* __restrict__ hits,
                                                            uint32_t* __restrict__ prims, uint2* __restrict__ work) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 a = o[i], b = d[i];
    HitRec h;
    TraceWork w;
    const Ray ray = make_ray(xyz(a), xyz(b));
    const bool found = Wide ? trace4<AnyHit, true>(s, ray, tmin, tmax, h, &w) : trace<AnyHit, true>(s, ray, tmin, tmax, h, &w);
    if (found) {
        hits[i] = make_float4(h.t, AnyHit ? 0.0f : h.u, AnyHit ? 0.0f : h.v,
                              __uint_as_float(AnyHit ? 0u : h.inst));
        prims[i] = AnyHit ? 0u : h.prim;
    } else {
        hits[i] = make_float4(-1.0f, 0.0f, 0.0f, __uint_as_float(kNoIndex));
        prims[i] = kNoIndex;
    }
    work[i] = make_uint2(w.nodes, w.tris);
}
} // namespace
} // namespace rr

extern "C" rr_status rr_trace_counted(rr_ctx* ctx, const rr_scene* scene, const float* origins, const float* dirs,
                                      float tmin, float tmax, uint32_t count, int flags, float* hits,
                                      uint32_t* prims, uint32_t* work, void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!scene || (count && (!origins || !dirs || !hits || !prims || !work)) ||
        (flags & ~(RR_TRACE_ANY_HIT | RR_TRACE_WIDE)))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_trace_counted: bad argument");
    if (count == 0) return RR_OK;
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    const auto o = reinterpret_cast<const float4*>(origins);
    const auto d = reinterpret_cast<const float4*>(dirs);
    const auto st = static_cast<cudaStream_t>(stream);
    auto launch = [&](auto kernel) {
        kernel<<<(count + 127) / 128, 128, 0, st>>>(scene->dev, o, d, tmin, tmax, count, reinterpret_cast<float4*>(hits),
                                                    prims, reinterpret_cast<uint2*>(work));
    };
    switch (flags) {
    case 0: launch(rr::trace_counted_kernel<false, false>); break;
    case RR_TRACE_ANY_HIT: launch(rr::trace_counted_kernel<true, false>); break;
    case RR_TRACE_WIDE: launch(rr::trace_counted_kernel<false, true>); break;
    default: launch(rr::trace_counted_kernel<true, true>); break;
    }
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

extern "C" rr_status rr_scene_copy_bvh(rr_ctx* ctx, const rr_scene* scene, float* nodes_out, float* tris_out) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!scene || !nodes_out || !tris_out) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_scene_copy_bvh: bad argument");
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    RR_TRY_CUDA(ctx, cudaMemcpy(nodes_out, scene->dev.nodes, size_t(scene->dev.num_nodes) * 4 * sizeof(float4),
                                cudaMemcpyDeviceToHost));
    RR_TRY_CUDA(ctx, cudaMemcpy(tris_out, scene->dev.tris, size_t(scene->dev.num_tris) * 3 * sizeof(float4),
                                cudaMemcpyDeviceToHost));
    return RR_OK;
}

extern "C" rr_status rr_scene_copy_bvh4(rr_ctx* ctx, const rr_scene* scene, float* nodes4_out) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!scene || !nodes4_out) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_scene_copy_bvh4: bad argument");
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    RR_TRY_CUDA(ctx, cudaMemcpy(nodes4_out, scene->dev.nodes4, size_t(scene->dev.num_nodes4) * 8 * sizeof(float4),
                                cudaMemcpyDeviceToHost));
    return RR_OK;
}

extern "C" rr_status rr_trace_closest(rr_ctx* ctx, const rr_scene* scene, const float* origins, const float* dirs,
                                      float tmin, float tmax, uint32_t count, float* hits, uint32_t* prims,
                                      void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!scene || (count && (!origins || !dirs || !hits || !prims)))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_trace_closest: bad argument");
    if (count == 0) return RR_OK;
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    rr::trace_batch_kernel<<<(count + 127) / 128, 128, 0, static_cast<cudaStream_t>(stream)>>>(
        scene->dev, reinterpret_cast<const float4*>(origins), reinterpret_cast<const float4*>(dirs), tmin, tmax,
        count, reinterpret_cast<float4*>(hits), prims);
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}
