// rr_vmf.cuh — von Mises-Fisher lobe sampling and density
// (GuidingGrid.slang:160-189) for the hash-grid guide and the grid guide's EM,
// and the guided path tracer's mixtures (fast forms, below).
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

// Two densities of brdf_sample's direction at an arbitrary wi (cos > 0):
//  ref    — the value brdf_sample returns as its pdf (BRDF.slang:229-283): the
//           p_spec-weighted mixture of D*NdotH/(4 VdotH) and the cosine lobe,
//           clamped at 1e-6 exactly as the reference clamps it;
//  actual — the density brdf_sample really draws from: its specular branch
//           samples the GGX distribution of visible normals, whose reflected
//           density is G1(wo) D(h) / (4 wo.z) (Heitz 2018, "Sampling the GGX
//           Distribution of Visible Normals", eq. 17 with the GGX Smith G1),
//           written as D / (2 (wo.z + sqrt(a^2 (wo.x^2 + wo.y^2) + wo.z^2)))
//           so that it stays finite at grazing wo.
// The reference tracer weights a bounce by f cos / ref, whose expectation is
// the integral of f cos actual/ref; a guided estimator that samples from
// another density reproduces that expectation with f cos (actual/ref) / p_mix.
struct BrdfPdfs {
    float ref;
    float actual;
};

RR_D BrdfPdfs brdf_sample_pdfs(float3 wo, float3 n, float3 base, float metallic, float roughness, float3 wi) {
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
    const float a = r * r;
    const float D = distribution_ggx(NdotH, a);
    const float pdf_diff = NdotWI * kInvPi;
    const float pdf_spec_ref = D * NdotH / mx(4.0f * VdotH, 1e-6f);
    const float vz = mx(wo_l.z, 0.0f);
    const float lam = sqrtf(a * a * (wo_l.x * wo_l.x + wo_l.y * wo_l.y) + vz * vz);
    const float pdf_spec_vndf = D / mx(2.0f * (vz + lam), 1e-12f);
    BrdfPdfs p;
    p.ref = mx(p_spec * pdf_spec_ref + (1.0f - p_spec) * pdf_diff, 1e-6f);
    p.actual = p_spec * pdf_spec_vndf + (1.0f - p_spec) * pdf_diff;
    return p;
}

constexpr int kMaxLobes = 8;

// Mixture of up to kMaxLobes vMF lobes: lobe[j] = (mu.xyz, kappa), weight[j]
// normalised to sum 1 (a weight of 0 disables a lobe).
struct VmfMixture {
    float4 lobe[kMaxLobes];
    float weight[kMaxLobes];
};

// The guided tracer's mixtures (no reference counterpart) use the same vMF
// formulas with the hardware approximations (__expf, __logf, __sincosf,
// __fdividef) instead of the deterministic functions the reference-parity
// paths need: the guided estimator only needs the density it evaluates to
// be the one it samples, and both use these forms. Per lobe the density is
// w_j k_j e^{k_j (mu_j.dir - 1)} / (2 pi (1 - e^{-2 k_j})).
RR_D float vmf_pdf_fast(float3 mu, float kappa, float3 dir) {
    const float k = mx(kappa, 1.0e-3f);
    const float w = clampf(dot(mu, dir), -1.0f, 1.0f);
    const float denom = kTwoPi * (1.0f - __expf(-2.0f * k));
    return __fdividef(k * __expf(k * (w - 1.0f)), mx(denom, 1.0e-8f));
}

RR_D float3 vmf_sample_fast(float3 mu, float kappa, float ux, float uy) {
    const float k = mx(kappa, 1.0e-3f);
    float w = 1.0f + __fdividef(__logf(ux + (1.0f - ux) * __expf(-2.0f * k)), k);
    w = clampf(w, -1.0f, 1.0f);
    const float s = sqrtf(mx(0.0f, 1.0f - w * w));
    float sp, cp;
    __sincosf(kTwoPi * uy, &sp, &cp);
    float3 T, B;
    build_onb(mu, T, B);
    return tangent_to_world(f3(s * cp, s * sp, w), T, B, mu);
}

RR_D float mixture_pdf(const VmfMixture& m, int lobes, float3 dir) {
    float p = 0.0f;
    for (int j = 0; j < lobes; ++j)
        if (m.weight[j] > 0.0f) p += m.weight[j] * vmf_pdf_fast(xyz(m.lobe[j]), m.lobe[j].w, dir);
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
    return vmf_sample_fast(xyz(m.lobe[j]), m.lobe[j].w, ux, uy);
}

} // namespace rr
