// rr_dev.cuh — device-side restatement of the reference shader math.
//
// Mirrors assets/shaders/include/{Common,Sampling,BRDF}.slang and the shared
// helpers of passes/pathtracer_reference/pathtracer.slang. The library is
// built with -fmad=false and IEEE division/square root, and the expression
// order below is the order of the Slang source, so every value matches the
// CPU checker bit for bit. sin/cos/exp/log are the rr_detmath.h functions.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>
#include "rr_detmath.h"
#include "rr_layouts.h"

#define RR_D __device__ __forceinline__

namespace rr {

// ── vector helpers (HLSL semantics) ───────────────────────────────────────
RR_D float3 f3(float x, float y, float z) { return make_float3(x, y, z); }
RR_D float3 operator+(float3 a, float3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
RR_D float3 operator-(float3 a, float3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
RR_D float3 operator*(float3 a, float3 b) { return f3(a.x * b.x, a.y * b.y, a.z * b.z); }
RR_D float3 operator*(float3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
RR_D float3 operator*(float s, float3 a) { return f3(s * a.x, s * a.y, s * a.z); }
RR_D float3 operator/(float3 a, float s) { return f3(a.x / s, a.y / s, a.z / s); }
RR_D float3 operator-(float3 a) { return f3(-a.x, -a.y, -a.z); }
RR_D float dot(float3 a, float3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
RR_D float length(float3 a) { return sqrtf(dot(a, a)); }
RR_D float3 normalize(float3 a) { const float inv = 1.0f / sqrtf(dot(a, a)); return a * inv; }
RR_D float3 cross(float3 a, float3 b) {
    return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
// max/min without NaN propagation games: same as the checker's a > b ? a : b
RR_D float mx(float a, float b) { return a > b ? a : b; }
RR_D float mn(float a, float b) { return a < b ? a : b; }
RR_D float clampf(float x, float lo, float hi) { return mn(mx(x, lo), hi); }
RR_D float3 lerp(float3 a, float3 b, float t) { return a + (b - a) * t; }  // x + s*(y-x)
RR_D float3 reflect(float3 i, float3 n) { const float d2 = 2.0f * dot(i, n); return i - n * d2; }
RR_D float3 xyz(float4 v) { return f3(v.x, v.y, v.z); }

// mul(M, float4(v, w)) for a row-major 4x4 given as 4 row float4s
RR_D float3 mul_rows_point(float4 r0, float4 r1, float4 r2, float3 v, float w) {
    return f3(r0.x * v.x + r0.y * v.y + r0.z * v.z + r0.w * w,
              r1.x * v.x + r1.y * v.y + r1.z * v.z + r1.w * w,
              r2.x * v.x + r2.y * v.y + r2.z * v.z + r2.w * w);
}
// mul((float3x3)M, v)
RR_D float3 mul_rows_dir(float4 r0, float4 r1, float4 r2, float3 v) {
    return f3(r0.x * v.x + r0.y * v.y + r0.z * v.z,
              r1.x * v.x + r1.y * v.y + r1.z * v.z,
              r2.x * v.x + r2.y * v.y + r2.z * v.z);
}

constexpr float kPi = 3.14159265358979323846f;
constexpr float kTwoPi = 6.28318530717958647692f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float kEpsilon = 1e-4f;
constexpr uint32_t kNoIndex = 0xffffffffu;

// ── RNG: Common.slang:18-28, Sampling.slang:11-30 ─────────────────────────
RR_D uint32_t pcg_hash(uint32_t seed) {
    const uint32_t state = seed * 747796405u + 2891336453u;
    const uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
RR_D float rand_float(uint32_t& seed) {
    seed = pcg_hash(seed);
    return float(seed >> 8) * (1.0f / float(1u << 24));
}
RR_D uint32_t make_seed(uint32_t px, uint32_t py, uint32_t frame) {
    return pcg_hash(px ^ (py * 1000003u) ^ (frame * 2654435761u));
}

// ── Sampling.slang:37-78 ───────────────────────────────────────────────────
RR_D float3 sample_cosine_hemisphere(float u0, float u1, float& pdf) {
    const float r = sqrtf(u0);
    const float phi = kTwoPi * u1;
    const float x = r * rr_cosf(phi);
    const float y = r * rr_sinf(phi);
    const float z = sqrtf(mx(0.0f, 1.0f - u0));
    pdf = z * kInvPi;
    return f3(x, y, z);
}
RR_D void build_onb(float3 n, float3& T, float3& B) {
    const float3 up = (fabsf(n.x) < 0.9f) ? f3(1.0f, 0.0f, 0.0f) : f3(0.0f, 1.0f, 0.0f);
    T = normalize(cross(up, n));
    B = cross(n, T);
}
RR_D float3 tangent_to_world(float3 v, float3 T, float3 B, float3 N) { return v.x * T + v.y * B + v.z * N; }
RR_D float3 world_to_tangent(float3 v, float3 T, float3 B, float3 N) { return f3(dot(v, T), dot(v, B), dot(v, N)); }

// ── BRDF.slang:16-187 ──────────────────────────────────────────────────────
RR_D float3 fresnel_schlick(float cos_theta, float3 F0) {
    const float x = clampf(1.0f - cos_theta, 0.0f, 1.0f);
    const float x2 = x * x;
    const float p = x2 * x2 * x;
    return f3(F0.x + (1.0f - F0.x) * p, F0.y + (1.0f - F0.y) * p, F0.z + (1.0f - F0.z) * p);
}
RR_D float distribution_ggx(float NdotH, float alpha) {
    const float a2 = alpha * alpha;
    const float d = NdotH * NdotH * (a2 - 1.0f) + 1.0f;
    return a2 / mx(kPi * d * d, kEpsilon);
}
RR_D float geometry_smith_ggx(float NdotV, float NdotL, float alpha) {
    const float k = alpha * 0.5f;
    const float gv = NdotV / mx(NdotV * (1.0f - k) + k, kEpsilon);
    const float gl = NdotL / mx(NdotL * (1.0f - k) + k, kEpsilon);
    return gv * gl;
}
RR_D float3 brdf_specular_ggx(float3 n, float3 wo, float3 wi, float3 F0, float roughness) {
    const float alpha = roughness * roughness;
    const float3 h = normalize(wo + wi);
    const float NdotH = mx(dot(n, h), 0.0f);
    const float NdotV = mx(dot(n, wo), 0.0f);
    const float NdotL = mx(dot(n, wi), 0.0f);
    const float VdotH = mx(dot(wo, h), 0.0f);
    const float3 F = fresnel_schlick(VdotH, F0);
    const float D = distribution_ggx(NdotH, alpha);
    const float G = geometry_smith_ggx(NdotV, NdotL, alpha);
    const float DG = D * G;
    const float den = mx(4.0f * NdotV * NdotL, kEpsilon);
    return f3((DG * F.x) / den, (DG * F.y) / den, (DG * F.z) / den);
}
RR_D float3 brdf_eval(float3 n, float3 wo, float3 wi, float3 base, float metallic, float roughness) {
    const float r = clampf(roughness, 0.04f, 1.0f);
    const float3 F0 = lerp(f3(0.04f, 0.04f, 0.04f), base, metallic);
    const float3 kS = fresnel_schlick(mx(dot(n, wo), 0.0f), F0);
    const float om = 1.0f - metallic;
    const float3 kD = f3((1.0f - kS.x) * om, (1.0f - kS.y) * om, (1.0f - kS.z) * om);
    const float3 diffuse = kD * (base * kInvPi);
    const float3 specular = brdf_specular_ggx(n, wo, wi, F0, r);
    return diffuse + specular;
}
RR_D float3 sample_ggx_vndf(float3 wo, float roughness, float u0, float u1) {
    const float alpha = roughness * roughness;
    const float3 Vh = normalize(f3(alpha * wo.x, alpha * wo.y, wo.z));
    const float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
    float3 T1;
    if (lensq > 0.0f) { const float s = sqrtf(lensq); T1 = f3(-Vh.y / s, Vh.x / s, 0.0f / s); }
    else T1 = f3(1.0f, 0.0f, 0.0f);
    const float3 T2 = cross(Vh, T1);
    const float r2 = sqrtf(u0);
    const float phi = kTwoPi * u1;
    const float t1 = r2 * rr_cosf(phi);
    float t2 = r2 * rr_sinf(phi);
    const float s = 0.5f * (1.0f + Vh.z);
    t2 = (1.0f - s) * sqrtf(1.0f - t1 * t1) + s * t2;
    const float sq = sqrtf(mx(0.0f, 1.0f - t1 * t1 - t2 * t2));
    const float3 Nh = t1 * T1 + t2 * T2 + sq * Vh;
    return normalize(f3(alpha * Nh.x, alpha * Nh.y, mx(0.0f, Nh.z)));
}
// BRDF.slang:116-172
RR_D float3 brdf_sample(float3 wo, float3 n, float3 base, float metallic, float roughness,
                        float ux, float uy, float3& wi, float& pdf) {
    const float r = clampf(roughness, 0.04f, 1.0f);
    const float3 F0 = lerp(f3(0.04f, 0.04f, 0.04f), base, metallic);
    const float3 kS = fresnel_schlick(mx(dot(n, wo), 0.0f), F0);
    float p_spec = (kS.x + kS.y + kS.z) / 3.0f;
    p_spec = clampf(p_spec, 0.1f, 0.9f);
    float3 T, B;
    build_onb(n, T, B);
    const float3 wo_l = world_to_tangent(wo, T, B, n);
    float3 wi_l;
    if (ux < p_spec) {
        const float3 h_l = sample_ggx_vndf(wo_l, r, ux / p_spec, uy);
        wi_l = reflect(-wo_l, h_l);
        if (wi_l.z <= 0.0f) { wi = f3(0.0f, 1.0f, 0.0f); pdf = 1.0f; return f3(0.0f, 0.0f, 0.0f); }
    } else {
        float pdf_l;
        wi_l = sample_cosine_hemisphere((ux - p_spec) / (1.0f - p_spec), uy, pdf_l);
    }
    wi = tangent_to_world(wi_l, T, B, n);
    const float NdotWI = mx(wi_l.z, 0.0f);
    const float3 h = normalize(wo_l + wi_l);
    const float NdotH = mx(h.z, 1e-6f);
    const float VdotH = mx(dot(wo_l, h), 1e-6f);
    const float D = distribution_ggx(NdotH, r * r);
    const float pdf_spec = D * NdotH / mx(4.0f * VdotH, 1e-6f);
    const float pdf_diff = NdotWI * kInvPi;
    pdf = p_spec * pdf_spec + (1.0f - p_spec) * pdf_diff;
    pdf = mx(pdf, 1e-6f);
    return brdf_eval(n, wo, wi, base, metallic, roughness);
}
RR_D float brdf_pdf(float3 wo, float3 wi, float3 n, float roughness) {
    const float r = clampf(roughness, 0.04f, 1.0f);
    const float3 h = normalize(wo + wi);
    const float NdotH = mx(dot(n, h), 1e-6f);
    const float VdotH = mx(dot(wo, h), 1e-6f);
    const float NdotL = mx(dot(n, wi), 0.0f);
    const float D = distribution_ggx(NdotH, r * r);
    const float pdf_spec = D * NdotH / mx(4.0f * VdotH, 1e-6f);
    const float pdf_diff = NdotL * kInvPi;
    return 0.5f * pdf_spec + 0.5f * pdf_diff;
}

// pathtracer.slang:216-217
RR_D float3 sky_radiance(float3 dir) {
    const float t = 0.5f * (dir.y + 1.0f);
    return lerp(f3(0.1f, 0.1f, 0.1f), f3(0.2f, 0.3f, 0.5f), t);
}

// Primary ray direction (pathtracer.slang:195-204). inv_proj/inv_view rows.
RR_D float3 primary_dir(const GpuCameraData& cam, float fx, float fy) {
    const float ndcx = fx / float(cam.screen_width) * 2.0f - 1.0f;
    const float ndcy = fy / float(cam.screen_height) * 2.0f - 1.0f;
    const float* P = cam.inv_proj;
    const float vx = P[0] * ndcx + P[1] * ndcy + P[2] * 1.0f + P[3] * 1.0f;
    const float vy = P[4] * ndcx + P[5] * ndcy + P[6] * 1.0f + P[7] * 1.0f;
    const float vz = -1.0f, vw = 0.0f;
    const float* V = cam.inv_view;
    const float3 w = f3(V[0] * vx + V[1] * vy + V[2] * vz + V[3] * vw,
                        V[4] * vx + V[5] * vy + V[6] * vz + V[7] * vw,
                        V[8] * vx + V[9] * vy + V[10] * vz + V[11] * vw);
    return normalize(w);
}

} // namespace rr
