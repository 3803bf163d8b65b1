// rr_vmf.cuh — von Mises-Fisher lobe sampling and density
// (GuidingGrid.slang:160-189), shared by the hash-grid guide and the guided
// path tracer's mixture guides.
#pragma once

#include "rr_dev.cuh"

namespace rr {

// GuidingGrid.slang:160-180 — inverse-CDF sample of cos(theta) about +z,
// rotated into the frame of mu.
RR_D float3 vmf_sample(float3 mu, float kappa, float ux, float uy, float& pdf) {
    const float k = mx(kappa, 1.0e-3f);
    float w = 1.0f + (1.0f / k) * rr_logf(ux + (1.0f - ux) * rr_expf(-2.0f * k));
    w = clampf(w, -1.0f, 1.0f);
    const float s = sqrtf(mx(0.0f, 1.0f - w * w));
    const float phi = kTwoPi * uy;
    const float3 local = f3(s * rr_cosf(phi), s * rr_sinf(phi), w);
    float3 T, B;
    build_onb(mu, T, B);
    const float3 dir = tangent_to_world(local, T, B, mu);
    const float denom = kTwoPi * (1.0f - rr_expf(-2.0f * k));
    pdf = k * rr_expf(k * (w - 1.0f)) / mx(denom, 1.0e-8f);
    return dir;
}

// GuidingGrid.slang:183-189
RR_D float vmf_pdf(float3 mu, float kappa, float3 dir) {
    const float k = mx(kappa, 1.0e-3f);
    const float w = clampf(dot(mu, dir), -1.0f, 1.0f);
    const float denom = kTwoPi * (1.0f - rr_expf(-2.0f * k));
    return k * rr_expf(k * (w - 1.0f)) / mx(denom, 1.0e-8f);
}

// Density of brdf_sample's direction at an arbitrary wi: the p_spec-weighted
// mixture of the GGX-VNDF and cosine lobes evaluated exactly as
// BRDF.slang:229-283 evaluates it for the sampled direction.
RR_D float brdf_sample_pdf(float3 wo, float3 n, float3 base, float metallic, float roughness, float3 wi) {
    const float r = clampf(roughness, 0.04f, 1.0f);
    const float3 F0 = lerp(f3(0.04f, 0.04f, 0.04f), base, metallic);
    const float3 kS = fresnel_schlick(mx(dot(n, wo), 0.0f), F0);
    const float p_spec = clampf((kS.x + kS.y + kS.z) / 3.0f, 0.1f, 0.9f);
    float3 T, B;
    build_onb(n, T, B);
    const float3 wo_l = world_to_tangent(wo, T, B, n);
    const float3 wi_l = world_to_tangent(wi, T, B, n);
    const float NdotWI = mx(wi_l.z, 0.0f);
    const float3 h = normalize(wo_l + wi_l);
    const float NdotH = mx(h.z, 1e-6f);
    const float VdotH = mx(dot(wo_l, h), 1e-6f);
    const float D = distribution_ggx(NdotH, r * r);
    const float pdf_spec = D * NdotH / mx(4.0f * VdotH, 1e-6f);
    return p_spec * pdf_spec + (1.0f - p_spec) * (NdotWI * kInvPi);
}

constexpr int kMaxLobes = 8;

// Mixture of up to kMaxLobes vMF lobes: lobe[j] = (mu.xyz, kappa), weight[j]
// normalised to sum 1 (a weight of 0 disables a lobe).
struct VmfMixture {
    float4 lobe[kMaxLobes];
    float weight[kMaxLobes];
};

RR_D float mixture_pdf(const VmfMixture& m, int lobes, float3 dir) {
    float p = 0.0f;
    for (int j = 0; j < lobes; ++j)
        if (m.weight[j] > 0.0f) p += m.weight[j] * vmf_pdf(xyz(m.lobe[j]), m.lobe[j].w, dir);
    return p;
}

// Picks a lobe with u_pick, samples it with (ux, uy).
RR_D float3 mixture_sample(const VmfMixture& m, int lobes, float u_pick, float ux, float uy) {
    int j = 0;
    float c = 0.0f;
    for (int k = 0; k < lobes; ++k) {
        if (m.weight[k] <= 0.0f) continue;
        j = k;
        c += m.weight[k];
        if (u_pick < c) break;
    }
    float pdf;
    return vmf_sample(xyz(m.lobe[j]), m.lobe[j].w, ux, uy, pdf);
}

} // namespace rr
