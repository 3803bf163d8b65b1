// rr_grid.cuh — the world-space vMF guiding grid's device helpers
// (assets/shaders/include/GuidingGrid.slang), shared by the stand-alone
// guiding entry points (guiding.cu) and ReSTIR PT (restir_pt.cu):
//   cell_index         GuidingGrid.slang:54-67
//   splat_dir          GuidingGrid.slang:73-90 (guiding_splat)
//   sample_primary_dir restir_pt.slang:520-563 (one-sample MIS of the cell's
//                      fitted vMF lobe and a cosine lobe)
#pragma once

#include "rr_internal.h"
#include "rr_vmf.cuh"

namespace rr {

struct GridParams {
    float base_cell_size, distance_slope;
    uint32_t cell_count, enabled, min_samples;
    float kappa_max, alpha;
    float cam_x, cam_y, cam_z;
};

inline GridParams to_grid(const rr_guiding_params* p, const float* cam) {
    GridParams g;
    g.base_cell_size = p->base_cell_size; g.distance_slope = p->distance_slope;
    g.cell_count = p->cell_count; g.enabled = p->enabled; g.min_samples = p->min_samples;
    g.kappa_max = p->kappa_max; g.alpha = p->alpha;
    g.cam_x = cam ? cam[0] : 0.0f; g.cam_y = cam ? cam[1] : 0.0f; g.cam_z = cam ? cam[2] : 0.0f;
    return g;
}

// GuidingGrid.slang:54-67
RR_D uint32_t cell_index(float3 p, uint32_t bsdf, const GridParams& g) {
    const float view_dist = length(p - f3(g.cam_x, g.cam_y, g.cam_z));
    const float cell = mx(g.base_cell_size + g.distance_slope * view_dist, 1.0e-4f);
    const int qx = int(floorf(p.x / cell)), qy = int(floorf(p.y / cell)), qz = int(floorf(p.z / cell));
    const uint32_t h = pcg_hash(uint32_t(qx) * 73856093u ^ uint32_t(qy) * 19349663u ^
                                uint32_t(qz) * 83492791u ^ bsdf * 2654435761u);
    return h % (g.cell_count > 0u ? g.cell_count : 1u);
}

// GuidingGrid.slang:73-90: fixed-point (2^20) direction sums and a count per
// cell with four 32-bit integer atomics; integer addition makes the
// accumulators independent of the order of the splats. round() is ties to
// even (HLSL round); the scale is a power of two, so the product is exact.
RR_D void splat_dir(uint32_t* accum, uint32_t cell, float3 d) {
    uint32_t* a = accum + size_t(cell) * 4;
    atomicAdd(a + 0, uint32_t(int(rintf(d.x * 1048576.0f))));
    atomicAdd(a + 1, uint32_t(int(rintf(d.y * 1048576.0f))));
    atomicAdd(a + 2, uint32_t(int(rintf(d.z * 1048576.0f))));
    atomicAdd(a + 3, 1u);
}

// restir_pt.slang:520-563. A lobe is valid iff kappa > 0 and |mu|^2 > 0.25
// (guiding_load_lobe, GuidingGrid.slang:140-157); the first random number
// picks the vMF lobe with probability alpha (when valid), the next two sample
// the chosen lobe. Returns wi; src_pdf = alpha p_vmf + (1 - alpha) p_cos.
RR_D float3 sample_primary_dir(const float4* __restrict__ fitted, float3 p, float3 n, uint32_t bsdf,
                               const GridParams& g, uint32_t& seed, float& src_pdf) {
    float alpha = 0.0f;
    bool valid = false;
    float3 mu = f3(0.0f, 0.0f, 0.0f);
    float kappa = 0.0f;
    if (g.enabled != 0u && g.alpha > 0.0f) {
        const float4 f = __ldg(fitted + cell_index(p, bsdf, g));
        mu = xyz(f);
        kappa = f.w;
        valid = kappa > 0.0f && dot(mu, mu) > 0.25f;
        if (valid) alpha = g.alpha;
    }
    float3 T, B;
    build_onb(n, T, B);
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
        wi = tangent_to_world(sample_cosine_hemisphere(u0, u1, cpdf), T, B, n);
    }
    const float cos_i = dot(n, wi);
    const float p_cos = cos_i > 0.0f ? cos_i * kInvPi : 0.0f;
    const float p_vmf = valid ? vmf_pdf(mu, kappa, wi) : 0.0f;
    src_pdf = alpha * p_vmf + (1.0f - alpha) * p_cos;
    return wi;
}

} // namespace rr
