// guiding.cu — world-space vMF guiding grid (assets/shaders/include/
// GuidingGrid.slang; host side ReSTIRPTPass.cpp:311-341, 602-611, 784-810).
//   splat : fixed-point (2^20) direction sums + count per hashed cell with
//           four 32-bit integer atomics (GuidingGrid.slang:73-90); integer
//           addition makes the accumulators order-independent (bit-exact)
//   fit   : Banerjee closed form per cell, resets the accumulator
//           (GuidingGrid.slang:100-137, cs_fit_guiding restir_pt.slang:1005-1015)
//   sample: one-sample MIS of the fitted lobe and a cosine lobe at a surface
//           point (sample_primary_dir, restir_pt.slang:520-563)

#include "rr_internal.h"
#include "rr_vmf.cuh"

namespace rr {
namespace {

struct GridParams {
    float base_cell_size, distance_slope;
    uint32_t cell_count, enabled, min_samples;
    float kappa_max, alpha;
    float cam_x, cam_y, cam_z;
};

// GuidingGrid.slang:54-67
RR_D uint32_t cell_index(float3 p, uint32_t bsdf, const GridParams& g) {
    const float view_dist = length(p - f3(g.cam_x, g.cam_y, g.cam_z));
    const float cell = mx(g.base_cell_size + g.distance_slope * view_dist, 1.0e-4f);
    const int qx = int(floorf(p.x / cell)), qy = int(floorf(p.y / cell)), qz = int(floorf(p.z / cell));
    const uint32_t h = pcg_hash(uint32_t(qx) * 73856093u ^ uint32_t(qy) * 19349663u ^
                                uint32_t(qz) * 83492791u ^ bsdf * 2654435761u);
    return h % (g.cell_count > 0u ? g.cell_count : 1u);
}

__global__ void __launch_bounds__(256) splat_kernel(uint32_t* __restrict__ accum, const float4* __restrict__ pos,
                                                    const float4* __restrict__ dir,
                                                    const uint32_t* __restrict__ bsdf, uint32_t n, GridParams g) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 p = pos[i], d = dir[i];
    const uint32_t cell = cell_index(xyz(p), bsdf[i], g);
    uint32_t* a = accum + size_t(cell) * 4;
    // round() to the nearest integer, ties to even (HLSL round); the scale is
    // a power of two, so the product is exact.
    atomicAdd(a + 0, uint32_t(int(rintf(d.x * 1048576.0f))));
    atomicAdd(a + 1, uint32_t(int(rintf(d.y * 1048576.0f))));
    atomicAdd(a + 2, uint32_t(int(rintf(d.z * 1048576.0f))));
    atomicAdd(a + 3, 1u);
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
    const float3 p = xyz(pos[i]), nn = xyz(nrm[i]);
    uint32_t seed = seeds[i];
    float alpha = 0.0f;
    bool valid = false;
    float3 mu = f3(0.0f, 0.0f, 0.0f);
    float kappa = 0.0f;
    if (g.enabled != 0u && g.alpha > 0.0f) {
        const float4 f = __ldg(fitted + cell_index(p, bsdf[i], g));
        mu = xyz(f);
        kappa = f.w;
        valid = kappa > 0.0f && dot(mu, mu) > 0.25f;
        if (valid) alpha = g.alpha;
    }
    float3 T, B;
    build_onb(nn, T, B);
    float3 wi;
    if (rand_float(seed) < alpha) {
        const float ux = rand_float(seed);
        const float uy = rand_float(seed);
        float vpdf;
        wi = vmf_sample(mu, kappa, ux, uy, vpdf);
    } else {
        const float u0 = rand_float(seed);
        const float u1 = rand_float(seed);
        float cpdf;
        wi = tangent_to_world(sample_cosine_hemisphere(u0, u1, cpdf), T, B, nn);
    }
    const float cos_i = dot(nn, wi);
    const float p_cos = cos_i > 0.0f ? cos_i * kInvPi : 0.0f;
    const float p_vmf = valid ? vmf_pdf(mu, kappa, wi) : 0.0f;
    wi_out[i] = make_float4(wi.x, wi.y, wi.z, 0.0f);
    pdf_out[i] = alpha * p_vmf + (1.0f - alpha) * p_cos;
    seeds[i] = seed;
}

GridParams to_grid(const rr_guiding_params* p, const float* cam) {
    GridParams g;
    g.base_cell_size = p->base_cell_size; g.distance_slope = p->distance_slope;
    g.cell_count = p->cell_count; g.enabled = p->enabled; g.min_samples = p->min_samples;
    g.kappa_max = p->kappa_max; g.alpha = p->alpha;
    g.cam_x = cam ? cam[0] : 0.0f; g.cam_y = cam ? cam[1] : 0.0f; g.cam_z = cam ? cam[2] : 0.0f;
    return g;
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
} // namespace
} // namespace rr

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
