// rr_oracle.cpp — CPU checker (test infrastructure only; see rr_oracle.h).
//
// A scalar restatement of the reference's Slang light-transport kernels.
// Paths in citations are relative to the reference project root; shader
// files live under assets/shaders/. Expression order follows the Slang source
// so that binary32 results are reproducible; compile with -ffp-contract=off.

#include "rr_oracle.h"
#include "rr_detmath.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <thread>
#include <vector>

namespace {

// ── float3 / float4 shim with HLSL semantics ──────────────────────────────

struct V3 { float x, y, z; };
struct V4 { float x, y, z, w; };

inline V3 v3(float x, float y, float z) { return V3{x, y, z}; }
inline V3 operator+(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 operator-(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 operator*(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
inline V3 operator*(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
inline V3 operator*(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
inline V3 operator/(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
inline V3 operator/(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
inline V3 operator-(V3 a) { return v3(-a.x, -a.y, -a.z); }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float length(V3 a) { return sqrtf(dot(a, a)); }
inline V3 normalize(V3 a) { const float inv = 1.0f / sqrtf(dot(a, a)); return a * inv; }
inline V3 cross(V3 a, V3 b) {
    return v3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float fmaxs(float a, float b) { return a > b ? a : b; }  // max(a,b), no NaN
inline float fmins(float a, float b) { return a < b ? a : b; }
inline float clampf(float x, float lo, float hi) { return fmins(fmaxs(x, lo), hi); }
// HLSL lerp(x, y, s) = x + s * (y - x)
inline V3 lerp(V3 a, V3 b, float t) { return a + (b - a) * t; }
inline V3 reflect(V3 i, V3 n) { const float d2 = 2.0f * dot(i, n); return i - n * d2; }
inline V3 load3(const float* p) { return v3(p[0], p[1], p[2]); }

// mul(M, v) for a row-major float4x4 (Scene.cpp:87-90)
inline V4 mul44(const float* M, V4 v) {
    V4 r;
    r.x = M[0] * v.x + M[1] * v.y + M[2] * v.z + M[3] * v.w;
    r.y = M[4] * v.x + M[5] * v.y + M[6] * v.z + M[7] * v.w;
    r.z = M[8] * v.x + M[9] * v.y + M[10] * v.z + M[11] * v.w;
    r.w = M[12] * v.x + M[13] * v.y + M[14] * v.z + M[15] * v.w;
    return r;
}
// mul((float3x3)M, v)
inline V3 mul33(const float* M, V3 v) {
    return v3(M[0] * v.x + M[1] * v.y + M[2] * v.z,
              M[4] * v.x + M[5] * v.y + M[6] * v.z,
              M[8] * v.x + M[9] * v.y + M[10] * v.z);
}

inline float asfloat(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
inline uint32_t asuint(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

// ── constants (BRDF.slang:8-11) ────────────────────────────────────────────
constexpr float kPi      = 3.14159265358979323846f;
constexpr float kTwoPi   = 6.28318530717958647692f;
constexpr float kInvPi   = 0.31830988618379067154f;
constexpr float kEpsilon = 1e-4f;

// ── RNG (Common.slang:18-28; Sampling.slang:11-30) ────────────────────────
inline uint32_t pcg_hash(uint32_t seed) {
    uint32_t state = seed * 747796405u + 2891336453u;
    uint32_t word = ((state >> ((state >> 28u) + 4u)) ^ state) * 277803737u;
    return (word >> 22u) ^ word;
}
inline float uint_to_float01(uint32_t v) { return float(v >> 8) * (1.0f / float(1u << 24)); }
inline float rand_float(uint32_t& seed) { seed = pcg_hash(seed); return uint_to_float01(seed); }
inline uint32_t make_seed(uint32_t px, uint32_t py, uint32_t frame) {
    uint32_t h = px ^ (py * 1000003u) ^ (frame * 2654435761u);
    return pcg_hash(h);
}

// ── Sampling.slang:37-85 ───────────────────────────────────────────────────
inline V3 sample_cosine_hemisphere(float u0, float u1, float& pdf) {
    float r = sqrtf(u0);
    float phi = 6.28318530717958647692f * u1;
    float x = r * rr_cosf(phi);
    float y = r * rr_sinf(phi);
    float z = sqrtf(fmaxs(0.0f, 1.0f - u0));
    pdf = z * 0.31830988618379067154f;
    return v3(x, y, z);
}
inline void build_onb(V3 n, V3& T, V3& B) {
    V3 up = (fabsf(n.x) < 0.9f) ? v3(1.0f, 0.0f, 0.0f) : v3(0.0f, 1.0f, 0.0f);
    T = normalize(cross(up, n));
    B = cross(n, T);
}
inline V3 tangent_to_world(V3 v, V3 T, V3 B, V3 N) { return v.x * T + v.y * B + v.z * N; }
inline V3 world_to_tangent(V3 v, V3 T, V3 B, V3 N) { return v3(dot(v, T), dot(v, B), dot(v, N)); }

// ── BRDF.slang:16-187 ──────────────────────────────────────────────────────
inline V3 fresnel_schlick(float cos_theta, V3 F0) {           // BRDF.slang:16-21
    float x = clampf(1.0f - cos_theta, 0.0f, 1.0f);
    float x2 = x * x;
    float p = x2 * x2 * x;
    return v3(F0.x + (1.0f - F0.x) * p, F0.y + (1.0f - F0.y) * p, F0.z + (1.0f - F0.z) * p);
}
inline float distribution_ggx(float NdotH, float alpha) {     // BRDF.slang:25-30
    float a2 = alpha * alpha;
    float d = NdotH * NdotH * (a2 - 1.0f) + 1.0f;
    return a2 / fmaxs(kPi * d * d, kEpsilon);
}
inline float geometry_smith_ggx(float NdotV, float NdotL, float alpha) {  // :34-40
    float k = alpha * 0.5f;
    float gv = NdotV / fmaxs(NdotV * (1.0f - k) + k, kEpsilon);
    float gl = NdotL / fmaxs(NdotL * (1.0f - k) + k, kEpsilon);
    return gv * gl;
}
inline V3 brdf_specular_ggx(V3 n, V3 wo, V3 wi, V3 F0, float roughness) {  // :44-59
    float alpha = roughness * roughness;
    V3 h = normalize(wo + wi);
    float NdotH = fmaxs(dot(n, h), 0.0f);
    float NdotV = fmaxs(dot(n, wo), 0.0f);
    float NdotL = fmaxs(dot(n, wi), 0.0f);
    float VdotH = fmaxs(dot(wo, h), 0.0f);
    V3 F = fresnel_schlick(VdotH, F0);
    float D = distribution_ggx(NdotH, alpha);
    float G = geometry_smith_ggx(NdotV, NdotL, alpha);
    float DG = D * G;
    float den = fmaxs(4.0f * NdotV * NdotL, kEpsilon);
    return v3((DG * F.x) / den, (DG * F.y) / den, (DG * F.z) / den);
}
inline V3 brdf_eval(V3 n, V3 wo, V3 wi, V3 base, float metallic, float roughness) {  // :71-83
    float r = clampf(roughness, 0.04f, 1.0f);
    V3 F0 = lerp(v3(0.04f, 0.04f, 0.04f), base, metallic);
    V3 kS = fresnel_schlick(fmaxs(dot(n, wo), 0.0f), F0);
    float om = 1.0f - metallic;
    V3 kD = v3((1.0f - kS.x) * om, (1.0f - kS.y) * om, (1.0f - kS.z) * om);
    V3 lam = base * kInvPi;
    V3 diffuse = kD * lam;
    V3 specular = brdf_specular_ggx(n, wo, wi, F0, r);
    return diffuse + specular;
}
inline V3 sample_ggx_vndf(V3 wo, float roughness, float u0, float u1) {  // :87-108
    float alpha = roughness * roughness;
    V3 Vh = normalize(v3(alpha * wo.x, alpha * wo.y, wo.z));
    float lensq = Vh.x * Vh.x + Vh.y * Vh.y;
    V3 T1;
    if (lensq > 0.0f) { float s = sqrtf(lensq); T1 = v3(-Vh.y / s, Vh.x / s, 0.0f / s); }
    else T1 = v3(1.0f, 0.0f, 0.0f);
    V3 T2 = cross(Vh, T1);
    float r2 = sqrtf(u0);
    float phi = kTwoPi * u1;
    float t1 = r2 * rr_cosf(phi);
    float t2 = r2 * rr_sinf(phi);
    float s = 0.5f * (1.0f + Vh.z);
    t2 = (1.0f - s) * sqrtf(1.0f - t1 * t1) + s * t2;
    float sq = sqrtf(fmaxs(0.0f, 1.0f - t1 * t1 - t2 * t2));
    V3 Nh = t1 * T1 + t2 * T2 + sq * Vh;
    return normalize(v3(alpha * Nh.x, alpha * Nh.y, fmaxs(0.0f, Nh.z)));
}
// BRDF.slang:116-172. Returns f; writes wi and pdf.
inline V3 brdf_sample(V3 wo, V3 n, V3 base, float metallic, float roughness,
                      float ux, float uy, V3& wi, float& pdf) {
    float r = clampf(roughness, 0.04f, 1.0f);
    V3 F0 = lerp(v3(0.04f, 0.04f, 0.04f), base, metallic);
    V3 kS_approx = fresnel_schlick(fmaxs(dot(n, wo), 0.0f), F0);
    float p_spec = (kS_approx.x + kS_approx.y + kS_approx.z) / 3.0f;
    p_spec = clampf(p_spec, 0.1f, 0.9f);
    V3 T, B;
    build_onb(n, T, B);
    V3 wo_local = world_to_tangent(wo, T, B, n);
    V3 wi_local;
    if (ux < p_spec) {
        float u2x = ux / p_spec;
        V3 h_local = sample_ggx_vndf(wo_local, r, u2x, uy);
        wi_local = reflect(-wo_local, h_local);
        if (wi_local.z <= 0.0f) { wi = v3(0.0f, 1.0f, 0.0f); pdf = 1.0f; return v3(0.0f, 0.0f, 0.0f); }
        // pdf_local of the chosen lobe is recomputed below for the mixture.
    } else {
        float u2x = (ux - p_spec) / (1.0f - p_spec);
        float pdf_local;
        wi_local = sample_cosine_hemisphere(u2x, uy, pdf_local);
    }
    wi = tangent_to_world(wi_local, T, B, n);
    float NdotWI = fmaxs(wi_local.z, 0.0f);
    V3 h = normalize(wo_local + wi_local);
    float NdotH = fmaxs(h.z, 1e-6f);
    float VdotH = fmaxs(dot(wo_local, h), 1e-6f);
    float D = distribution_ggx(NdotH, r * r);
    float pdf_spec_lobe = D * NdotH / fmaxs(4.0f * VdotH, 1e-6f);
    float pdf_diff_lobe = NdotWI * kInvPi;
    pdf = p_spec * pdf_spec_lobe + (1.0f - p_spec) * pdf_diff_lobe;
    pdf = fmaxs(pdf, 1e-6f);
    return brdf_eval(n, wo, wi, base, metallic, roughness);
}
inline float brdf_pdf(V3 wo, V3 wi, V3 n, float roughness) {  // BRDF.slang:176-187
    float r = clampf(roughness, 0.04f, 1.0f);
    V3 h = normalize(wo + wi);
    float NdotH = fmaxs(dot(n, h), 1e-6f);
    float VdotH = fmaxs(dot(wo, h), 1e-6f);
    float NdotL = fmaxs(dot(n, wi), 0.0f);
    float D = distribution_ggx(NdotH, r * r);
    float pdf_spec = D * NdotH / fmaxs(4.0f * VdotH, 1e-6f);
    float pdf_diff = NdotL * kInvPi;
    return 0.5f * pdf_spec + 0.5f * pdf_diff;
}

// The two densities of brdf_sample's direction wi (the library's
// brdf_sample_pdfs): `ref`, the value brdf_sample returns as its pdf, and
// `actual`, the density it really draws from (its specular branch samples
// the GGX distribution of visible normals, G1(wo) D(h) / (4 wo.z), Heitz 2018,
// written D / (2 (wo.z + sqrt(a^2 (wo.x^2 + wo.y^2) + wo.z^2)))). Not in the
// reference: the emitter-sampling mode weights bounces by `actual`.
struct BrdfPdfs { float ref, actual; };
inline BrdfPdfs brdf_sample_pdfs(V3 wo, V3 n, V3 base, float metallic, float roughness, V3 wi) {
    const float r = clampf(roughness, 0.04f, 1.0f);
    const V3 F0 = lerp(v3(0.04f, 0.04f, 0.04f), base, metallic);
    const V3 kS = fresnel_schlick(fmaxs(dot(n, wo), 0.0f), F0);
    const float p_spec = clampf((kS.x + kS.y + kS.z) / 3.0f, 0.1f, 0.9f);
    V3 T, B;
    build_onb(n, T, B);
    const V3 wo_l = world_to_tangent(wo, T, B, n);
    const V3 wi_l = world_to_tangent(wi, T, B, n);
    const float NdotWI = fmaxs(wi_l.z, 0.0f);
    const V3 h = normalize(wo_l + wi_l);
    const float NdotH = fmaxs(h.z, 1e-6f);
    const float VdotH = fmaxs(dot(wo_l, h), 1e-6f);
    const float a = r * r;
    const float D = distribution_ggx(NdotH, a);
    const float pdf_diff = NdotWI * kInvPi;
    const float pdf_spec_ref = D * NdotH / fmaxs(4.0f * VdotH, 1e-6f);
    const float vz = fmaxs(wo_l.z, 0.0f);
    const float lam = sqrtf(a * a * (wo_l.x * wo_l.x + wo_l.y * wo_l.y) + vz * vz);
    const float pdf_spec_vndf = D / fmaxs(2.0f * (vz + lam), 1e-12f);
    BrdfPdfs q;
    q.ref = fmaxs(p_spec * pdf_spec_ref + (1.0f - p_spec) * pdf_diff, 1e-6f);
    q.actual = p_spec * pdf_spec_vndf + (1.0f - p_spec) * pdf_diff;
    return q;
}

inline V3 sky(V3 dir) {  // pathtracer.slang:216-217
    float t = 0.5f * (dir.y + 1.0f);
    return lerp(v3(0.1f, 0.1f, 0.1f), v3(0.2f, 0.3f, 0.5f), t);
}

// ── Ray/triangle: watertight test (Woop, Benthin, Wald, JCGT 2013) ─────────
struct RayPre {
    V3 o, d;
    int kx, ky, kz;
    float Sx, Sy, Sz;
    V3 inv;  // for box tests
};
inline float comp(V3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }
inline RayPre ray_pre(V3 o, V3 d) {
    RayPre r;
    r.o = o; r.d = d;
    int kz = 0;
    if (fabsf(d.y) > fabsf(comp(d, kz))) kz = 1;
    if (fabsf(d.z) > fabsf(comp(d, kz))) kz = 2;
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    if (comp(d, kz) < 0.0f) std::swap(kx, ky);
    r.kx = kx; r.ky = ky; r.kz = kz;
    r.Sx = comp(d, kx) / comp(d, kz);
    r.Sy = comp(d, ky) / comp(d, kz);
    r.Sz = 1.0f / comp(d, kz);
    auto safe = [](float x) { return fabsf(x) < 1e-20f ? copysignf(1e-20f, x) : x; };
    r.inv = v3(1.0f / safe(d.x), 1.0f / safe(d.y), 1.0f / safe(d.z));
    return r;
}
// Returns true and t, (bu, bv) = weights of v1, v2 when the ray hits the
// triangle with tmin <= t <= tmax. Two-sided (AccelStructure.cpp:90 disables
// facing culling for every instance).
inline bool intersect_tri(const RayPre& r, V3 p0, V3 p1, V3 p2, float tmin, float tmax,
                          float& t, float& bu, float& bv) {
    V3 A = p0 - r.o, B = p1 - r.o, C = p2 - r.o;
    const float Az0 = comp(A, r.kz), Bz0 = comp(B, r.kz), Cz0 = comp(C, r.kz);
    const float Ax = comp(A, r.kx) - r.Sx * Az0, Ay = comp(A, r.ky) - r.Sy * Az0;
    const float Bx = comp(B, r.kx) - r.Sx * Bz0, By = comp(B, r.ky) - r.Sy * Bz0;
    const float Cx = comp(C, r.kx) - r.Sx * Cz0, Cy = comp(C, r.ky) - r.Sy * Cz0;
    const float U = Cx * By - Cy * Bx;
    const float V = Ax * Cy - Ay * Cx;
    const float W = Bx * Ay - By * Ax;
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = U + V + W;
    if (det == 0.0f) return false;
    const float Az = r.Sz * Az0, Bz = r.Sz * Bz0, Cz = r.Sz * Cz0;
    const float T = U * Az + V * Bz + W * Cz;
    const float rcp = 1.0f / det;
    const float tt = T * rcp;
    if (!(tt >= tmin && tt <= tmax)) return false;
    t = tt; bu = V * rcp; bv = W * rcp;
    return true;
}

// ── Scene ──────────────────────────────────────────────────────────────────
struct Tri { V3 p0, p1, p2; uint32_t inst, prim; };
struct BNode { float lo[3], hi[3]; int left, right; uint32_t first, count; };

} // namespace

struct OracleScene {
    std::vector<GpuVertex> vertices;
    std::vector<uint32_t> indices;
    std::vector<GpuMesh> meshes;
    std::vector<GpuMaterial> materials;
    std::vector<GpuInstance> instances;
    std::vector<GpuLight> lights;
    std::vector<Tri> tris;           // world space, instance-major (key = index)
    std::vector<uint32_t> order;     // BVH leaf order -> tri index
    std::vector<BNode> nodes;
    bool use_bvh = false;
    // emitter table (the emitter-sampling mode): every triangle of an emissive
    // material with non-zero area, instance-major; 12 floats each,
    // (p0, Le.r), (e1, Le.g), (e2, Le.b), and the inclusive prefix sums of
    // power = luminance(Le) * area
    std::vector<float> emit;             // 12 floats per emitter
    std::vector<float> emit_prob;        // alias table over the emitters' powers
    std::vector<uint32_t> emit_alias;
    float emit_total = 0.0f;
    uint32_t num_emitters() const { return (uint32_t)emit_prob.size(); }
};

namespace {

void bounds_of(const Tri& t, float lo[3], float hi[3]) {
    const V3 ps[3] = {t.p0, t.p1, t.p2};
    for (int a = 0; a < 3; ++a) { lo[a] = INFINITY; hi[a] = -INFINITY; }
    for (const V3& p : ps)
        for (int a = 0; a < 3; ++a) {
            float c = comp(p, a);
            lo[a] = std::min(lo[a], c); hi[a] = std::max(hi[a], c);
        }
}

// Median-split BVH over triangle centroids (independent of the product's
// binned-SAH builder; only its closest-hit answers are compared).
int build_node(OracleScene& s, uint32_t first, uint32_t count, std::vector<float>& cent) {
    BNode n;
    for (int a = 0; a < 3; ++a) { n.lo[a] = INFINITY; n.hi[a] = -INFINITY; }
    float clo[3] = {INFINITY, INFINITY, INFINITY}, chi[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (uint32_t i = first; i < first + count; ++i) {
        float lo[3], hi[3];
        bounds_of(s.tris[s.order[i]], lo, hi);
        for (int a = 0; a < 3; ++a) {
            n.lo[a] = std::min(n.lo[a], lo[a]); n.hi[a] = std::max(n.hi[a], hi[a]);
            float c = cent[s.order[i] * 3 + a];
            clo[a] = std::min(clo[a], c); chi[a] = std::max(chi[a], c);
        }
    }
    const int idx = (int)s.nodes.size();
    s.nodes.push_back(n);
    if (count <= 4) {
        s.nodes[idx].left = s.nodes[idx].right = -1;
        s.nodes[idx].first = first; s.nodes[idx].count = count;
        return idx;
    }
    int axis = 0;
    for (int a = 1; a < 3; ++a) if (chi[a] - clo[a] > chi[axis] - clo[axis]) axis = a;
    const uint32_t mid = first + count / 2;
    std::nth_element(s.order.begin() + first, s.order.begin() + mid, s.order.begin() + first + count,
                     [&](uint32_t a, uint32_t b) {
                         float ca = cent[a * 3 + axis], cb = cent[b * 3 + axis];
                         return ca < cb || (ca == cb && a < b);
                     });
    int l = build_node(s, first, mid - first, cent);
    int r = build_node(s, mid, first + count - mid, cent);
    s.nodes[idx].left = l; s.nodes[idx].right = r;
    s.nodes[idx].first = 0; s.nodes[idx].count = 0;
    return idx;
}

// Conservative slab test (Ize, "Robust BVH ray traversal", JCGT 2013): the
// far distance is widened by 1 + 2*gamma(3) so rounding never culls a box
// that holds a hit.
inline bool box_hit(const RayPre& r, const float lo[3], const float hi[3], float tmin, float tmax) {
    float tn = tmin, tf = tmax;
    const float o[3] = {r.o.x, r.o.y, r.o.z}, inv[3] = {r.inv.x, r.inv.y, r.inv.z};
    float bn = -INFINITY, bf = INFINITY;
    for (int a = 0; a < 3; ++a) {
        float t0 = (lo[a] - o[a]) * inv[a];
        float t1 = (hi[a] - o[a]) * inv[a];
        bn = std::max(bn, std::min(t0, t1));
        bf = std::min(bf, std::max(t0, t1));
    }
    bf = bf * 1.0000006f;
    // the closest-hit bound is widened too, so that a box holding a triangle
    // at exactly the current t is still opened: ties then go to the lowest
    // key whatever the visiting order
    tn = std::max(tn, bn); tf = std::min(tf * 1.00001f, bf);
    return tn <= tf;
}

struct Hit { bool hit; float t, u, v; uint32_t key; };

// Closest hit; ties on t resolve to the lowest (instance, primitive).
template <bool AnyHit>
Hit trace_scene(const OracleScene& s, V3 o, V3 d, float tmin, float tmax) {
    Hit best{false, tmax, 0.0f, 0.0f, 0xffffffffu};
    const RayPre r = ray_pre(o, d);
    auto test = [&](uint32_t key) -> bool {
        const Tri& tr = s.tris[key];
        float t, u, v;
        if (intersect_tri(r, tr.p0, tr.p1, tr.p2, tmin, best.t, t, u, v)) {
            if (!best.hit || t < best.t || (t == best.t && key < best.key)) {
                best.hit = true; best.t = t; best.u = u; best.v = v; best.key = key;
            }
            return true;
        }
        return false;
    };
    if (!s.use_bvh) {
        for (uint32_t k = 0; k < (uint32_t)s.tris.size(); ++k)
            if (test(k) && AnyHit) return best;
        return best;
    }
    if (s.nodes.empty()) return best;
    int stack[128];
    int sp = 0;
    stack[sp++] = 0;
    while (sp > 0) {
        const BNode& n = s.nodes[stack[--sp]];
        if (!box_hit(r, n.lo, n.hi, tmin, best.t)) continue;
        if (n.left < 0) {
            for (uint32_t i = n.first; i < n.first + n.count; ++i)
                if (test(s.order[i]) && AnyHit) return best;
        } else {
            stack[sp++] = n.right;
            stack[sp++] = n.left;
        }
    }
    return best;
}

// Hit attributes (pathtracer.slang:69-118).
struct Surf { V3 pos, normal; uint32_t material; };
Surf hit_surface(const OracleScene& s, const Hit& h) {
    const Tri& tr = s.tris[h.key];
    const GpuInstance& inst = s.instances[tr.inst];
    const GpuMesh& mesh = s.meshes[inst.mesh_index];
    const uint32_t base = mesh.index_byte_offset / 4u + tr.prim * 3u;
    const uint32_t i0 = s.indices[base], i1 = s.indices[base + 1], i2 = s.indices[base + 2];
    const GpuVertex& v0 = s.vertices[mesh.vertex_base + i0];
    const GpuVertex& v1 = s.vertices[mesh.vertex_base + i1];
    const GpuVertex& v2 = s.vertices[mesh.vertex_base + i2];
    V3 b3 = v3(1.0f - h.u - h.v, h.u, h.v);
    V3 lp = b3.x * load3(v0.pos) + b3.y * load3(v1.pos) + b3.z * load3(v2.pos);
    V3 ln = normalize(b3.x * load3(v0.normal) + b3.y * load3(v1.normal) + b3.z * load3(v2.normal));
    V4 wp = mul44(inst.transform, V4{lp.x, lp.y, lp.z, 1.0f});
    V3 wn = normalize(mul33(inst.transform, ln));
    return Surf{v3(wp.x, wp.y, wp.z), wn, mesh.material_index};
}

// Primary ray (pathtracer.slang:192-205; restir_di.slang:196-206).
void primary_ray(const GpuCameraData& cam, uint32_t px, uint32_t py, float jx, float jy,
                 V3& o, V3& d) {
    float ndcx = (float(px) + jx) / float(cam.screen_width) * 2.0f - 1.0f;
    float ndcy = (float(py) + jy) / float(cam.screen_height) * 2.0f - 1.0f;
    V4 rv = mul44(cam.inv_proj, V4{ndcx, ndcy, 1.0f, 1.0f});
    rv.z = -1.0f; rv.w = 0.0f;
    V4 rw = mul44(cam.inv_view, rv);
    d = normalize(v3(rw.x, rw.y, rw.z));
    o = load3(cam.position);
}

template <class F>
void parallel_rows(uint32_t rows, int threads, F&& fn) {
    if (threads <= 1 || rows < 2) { for (uint32_t y = 0; y < rows; ++y) fn(y); return; }
    std::atomic<uint32_t> next{0};
    std::vector<std::thread> pool;
    for (int t = 0; t < threads; ++t)
        pool.emplace_back([&]() { for (uint32_t y; (y = next.fetch_add(1)) < rows;) fn(y); });
    for (auto& th : pool) th.join();
}

// NEE (pathtracer.slang:124-177)
V3 sample_lights(const OracleScene& s, V3 hit_pos, V3 normal, V3 wo, const GpuMaterial& mat,
                 uint32_t& seed, uint64_t& shadow_rays) {
    const uint32_t N = (uint32_t)s.lights.size();
    if (N == 0) return v3(0, 0, 0);
    uint32_t light_idx = uint32_t(rand_float(seed) * float(N)) % N;
    const GpuLight& light = s.lights[light_idx];
    V3 light_dir; float dist; float pdf_light;
    if (light.type == 0) {
        V3 to_light = load3(light.position) - hit_pos;
        dist = length(to_light);
        light_dir = to_light / dist;
        float r2 = dist * dist;
        pdf_light = r2;
    } else {
        light_dir = normalize(-load3(light.direction));
        dist = 1e9f;
        pdf_light = 1.0f;
    }
    if (dot(light_dir, normal) <= 0.0f) return v3(0, 0, 0);
    ++shadow_rays;
    Hit sh = trace_scene<true>(s, hit_pos + normal * 1e-4f, light_dir, 0.001f, dist - 0.01f);
    if (sh.hit) return v3(0, 0, 0);
    V3 brdf_val = brdf_eval(normal, wo, light_dir, load3(mat.base_color), mat.metallic, mat.roughness);
    float n_dot_l = fmaxs(dot(normal, light_dir), 0.0f);
    float denom = light.type == 0 ? (pdf_light + 1e-6f) : 1.0f;
    V3 irradiance = v3(light.emission[0] * light.intensity / denom,
                       light.emission[1] * light.intensity / denom,
                       light.emission[2] * light.intensity / denom);
    float mis_weight = 1.0f;
    if (light.type != 0) {
        float pdf_bsdf = brdf_pdf(wo, light_dir, normal, mat.roughness);
        mis_weight = (pdf_light * pdf_light) / (pdf_light * pdf_light + pdf_bsdf * pdf_bsdf + 1e-10f);
    }
    V3 r = brdf_val * irradiance;
    r = r * n_dot_l;
    r = r * mis_weight;
    return r * float(N);
}

inline bool any_positive(const float* e) { return e[0] > 0.0f || e[1] > 0.0f || e[2] > 0.0f; }

// pathtracer.slang:181-265 for one pixel and one frame seed.
V3 trace_path(const OracleScene& s, const GpuCameraData& cam, uint32_t px, uint32_t py,
              uint32_t frame_seed, uint32_t max_bounces, uint64_t& ext, uint64_t& shd) {
    uint32_t seed = make_seed(px, py, frame_seed);
    float jx = rand_float(seed);
    float jy = rand_float(seed);
    V3 ray_orig, ray_dir;
    primary_ray(cam, px, py, jx, jy, ray_orig, ray_dir);
    V3 radiance = v3(0, 0, 0), throughput = v3(1, 1, 1);
    for (uint32_t bounce = 0; bounce < max_bounces; ++bounce) {
        ++ext;
        Hit h = trace_scene<false>(s, ray_orig, ray_dir, 0.001f, 1e9f);
        if (!h.hit) { radiance = radiance + throughput * sky(ray_dir); break; }
        Surf sf = hit_surface(s, h);
        const GpuMaterial& mat = s.materials[sf.material];
        if (any_positive(mat.emissive)) { radiance = radiance + throughput * load3(mat.emissive); break; }
        V3 wo = -ray_dir;
        V3 n = sf.normal;
        if (dot(n, wo) < 0.0f) n = -n;
        radiance = radiance + throughput * sample_lights(s, sf.pos, n, wo, mat, seed, shd);
        float u0 = rand_float(seed);
        float u1 = rand_float(seed);
        V3 wi; float pdf;
        V3 f = brdf_sample(wo, n, load3(mat.base_color), mat.metallic, mat.roughness, u0, u1, wi, pdf);
        if (pdf < 1e-6f) break;
        float n_dot_wi = fmaxs(dot(n, wi), 0.0f);
        throughput = throughput * ((f * n_dot_wi) / pdf);
        if (bounce >= 3) {
            float survive = fmins(fmaxs(throughput.x, fmaxs(throughput.y, throughput.z)), 0.95f);
            if (rand_float(seed) > survive) break;
            throughput = throughput / survive;
        }
        ray_orig = sf.pos + n * 1e-4f;
        ray_dir = wi;
    }
    return radiance;
}

// ── Emitter sampling (no reference counterpart; the library's
// RR_PT_FLAG_EMITTERS mode) ──────────────────────────────────────────────
// Next-event estimation over the GpuLights (the reference's point and
// directional lights, picked as sample_lights picks them) and the scene's
// emissive triangles (picked in proportion to luminance(Le) * area, a point
// uniform on the triangle), one group per vertex (each with probability 1/2
// when both exist); bounces weighted by brdf_sample's actual density, and
// emissive surfaces reached by a bounce weighted against the emitter sample
// by the power heuristic.
inline float lum709(V3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

// Solid-angle density of the emitter sample at a point of emission Le seen
// at squared distance d2 under |cos| cos_y from the shading point.
inline float emitter_pdf(float p_group, float lum, float total, float d2, float cos_y) {
    return p_group * (lum / total) * d2 / cos_y;
}

// The emitter a pair of uniforms picks from the alias table: column
// min(floor(u n), n - 1), kept when uc < its probability, else its alias.
inline uint32_t emitter_pick(const OracleScene& s, float u, float uc) {
    const uint32_t n = s.num_emitters();
    const uint32_t k = std::min((uint32_t)(u * (float)n), n - 1u);
    return uc < s.emit_prob[k] ? k : s.emit_alias[k];
}

// sample_lights (pathtracer.slang:124-177) with its light-count factor N
// replaced by `scale` (N / probability of the GpuLight group).
V3 sample_lights_scaled(const OracleScene& s, V3 hit_pos, V3 normal, V3 wo, const GpuMaterial& mat, uint32_t& seed,
                        uint64_t& shadow_rays, float scale) {
    const uint32_t N = (uint32_t)s.lights.size();
    uint32_t light_idx = uint32_t(rand_float(seed) * float(N)) % N;
    const GpuLight& light = s.lights[light_idx];
    V3 light_dir; float dist; float pdf_light;
    if (light.type == 0) {
        V3 to_light = load3(light.position) - hit_pos;
        dist = length(to_light);
        light_dir = to_light / dist;
        float r2 = dist * dist;
        pdf_light = r2;
    } else {
        light_dir = normalize(-load3(light.direction));
        dist = 1e9f;
        pdf_light = 1.0f;
    }
    if (dot(light_dir, normal) <= 0.0f) return v3(0, 0, 0);
    ++shadow_rays;
    Hit sh = trace_scene<true>(s, hit_pos + normal * 1e-4f, light_dir, 0.001f, dist - 0.01f);
    if (sh.hit) return v3(0, 0, 0);
    V3 brdf_val = brdf_eval(normal, wo, light_dir, load3(mat.base_color), mat.metallic, mat.roughness);
    float n_dot_l = fmaxs(dot(normal, light_dir), 0.0f);
    float denom = light.type == 0 ? (pdf_light + 1e-6f) : 1.0f;
    V3 irradiance = v3(light.emission[0] * light.intensity / denom,
                       light.emission[1] * light.intensity / denom,
                       light.emission[2] * light.intensity / denom);
    float mis_weight = 1.0f;
    if (light.type != 0) {
        float pdf_bsdf = brdf_pdf(wo, light_dir, normal, mat.roughness);
        mis_weight = (pdf_light * pdf_light) / (pdf_light * pdf_light + pdf_bsdf * pdf_bsdf + 1e-10f);
    }
    V3 r = brdf_val * irradiance;
    r = r * n_dot_l;
    r = r * mis_weight;
    return r * scale;
}

V3 trace_path_emitters(const OracleScene& s, const GpuCameraData& cam, uint32_t px, uint32_t py,
                       uint32_t frame_seed, uint32_t max_bounces, uint64_t& ext, uint64_t& shd) {
    uint32_t seed = make_seed(px, py, frame_seed);
    float jx = rand_float(seed);
    float jy = rand_float(seed);
    V3 ray_orig, ray_dir;
    primary_ray(cam, px, py, jx, jy, ray_orig, ray_dir);
    V3 radiance = v3(0, 0, 0), throughput = v3(1, 1, 1);
    const uint32_t NL = (uint32_t)s.lights.size(), NE = s.num_emitters();
    const float pe = NE == 0 ? 0.0f : (NL == 0 ? 1.0f : 0.5f);
    float prev_pdf = 0.0f;   // bounce density of the ray (0: a camera ray)
    for (uint32_t bounce = 0; bounce < max_bounces; ++bounce) {
        ++ext;
        Hit h = trace_scene<false>(s, ray_orig, ray_dir, 0.001f, 1e9f);
        if (!h.hit) { radiance = radiance + throughput * sky(ray_dir); break; }
        Surf sf = hit_surface(s, h);
        const GpuMaterial& mat = s.materials[sf.material];
        if (any_positive(mat.emissive)) {
            const V3 Le = load3(mat.emissive);
            float w = 1.0f;
            if (prev_pdf > 0.0f) {
                const Tri& t = s.tris[h.key];
                const V3 ng = normalize(cross(t.p1 - t.p0, t.p2 - t.p0));
                const float cos_y = fabsf(dot(ng, ray_dir));
                const V3 dd = sf.pos - ray_orig;
                const float pl = cos_y > 0.0f ? emitter_pdf(pe, lum709(Le), s.emit_total, dot(dd, dd), cos_y) : 0.0f;
                const float a = prev_pdf * prev_pdf;
                w = a / (a + pl * pl);
            }
            radiance = radiance + throughput * (Le * w);
            break;
        }
        V3 wo = -ray_dir;
        V3 n = sf.normal;
        if (dot(n, wo) < 0.0f) n = -n;
        const V3 base = load3(mat.base_color);
        if (NL + NE > 0) {
            const bool use_e = NE > 0 && (NL == 0 || rand_float(seed) < 0.5f);
            if (use_e) {
                const float u = rand_float(seed);
                const float uc = rand_float(seed);
                const float u1 = rand_float(seed);
                const float u2 = rand_float(seed);
                const uint32_t k = emitter_pick(s, u, uc);
                const float* e = &s.emit[size_t(k) * 12];
                const V3 p0 = v3(e[0], e[1], e[2]), E1 = v3(e[4], e[5], e[6]), E2 = v3(e[8], e[9], e[10]);
                const V3 Le = v3(e[3], e[7], e[11]);
                const float su = sqrtf(u1);
                const float b1 = su * (1.0f - u2), b2 = su * u2;
                const V3 y = p0 + E1 * b1 + E2 * b2;
                const V3 to = y - sf.pos;
                const float d2 = dot(to, to);
                const float dist = sqrtf(d2);
                const V3 l = to / dist;
                const float cos_x = dot(n, l);
                const V3 ny = normalize(cross(E1, E2));
                const float cos_y = fabsf(dot(ny, l));
                if (cos_x > 0.0f && cos_y > 0.0f && d2 > 0.0f) {
                    const float pl = emitter_pdf(pe, lum709(Le), s.emit_total, d2, cos_y);
                    const V3 f = brdf_eval(n, wo, l, base, mat.metallic, mat.roughness);
                    const float pb = brdf_sample_pdfs(wo, n, base, mat.metallic, mat.roughness, l).actual;
                    const float a = pl * pl;
                    // the last vertex traces no bounce that could reach the
                    // emitter: its sample carries the whole weight there
                    const float wl = bounce + 1 == max_bounces ? 1.0f : a / (a + pb * pb);
                    ++shd;
                    Hit sh = trace_scene<true>(s, sf.pos + n * 1e-4f, l, 0.001f, dist - 0.01f);
                    if (!sh.hit) {
                        V3 c = f * Le;
                        c = c * (cos_x * wl / pl);
                        radiance = radiance + throughput * c;
                    }
                }
            } else {
                radiance = radiance + throughput * sample_lights_scaled(s, sf.pos, n, wo, mat, seed, shd,
                                                                        float(NL) / (1.0f - pe));
            }
        }
        float u0 = rand_float(seed);
        float u1 = rand_float(seed);
        V3 wi; float pdf;
        V3 f = brdf_sample(wo, n, base, mat.metallic, mat.roughness, u0, u1, wi, pdf);
        if (pdf < 1e-6f) break;
        const float pa = brdf_sample_pdfs(wo, n, base, mat.metallic, mat.roughness, wi).actual;
        if (!(pa > 0.0f)) break;
        float n_dot_wi = fmaxs(dot(n, wi), 0.0f);
        throughput = throughput * ((f * n_dot_wi) / pa);
        if (bounce >= 3) {
            float survive = fmins(fmaxs(throughput.x, fmaxs(throughput.y, throughput.z)), 0.95f);
            if (rand_float(seed) > survive) break;
            throughput = throughput / survive;
        }
        prev_pdf = pa;
        ray_orig = sf.pos + n * 1e-4f;
        ray_dir = wi;
    }
    return radiance;
}

// ── ReSTIR DI helpers (restir_di.slang:57-178) ────────────────────────────
inline void pack_reservoir(float* out, uint32_t sel, float w_sum, float W, uint32_t M) {
    out[0] = asfloat(sel); out[1] = w_sum; out[2] = W; out[3] = asfloat(M);
}
float compute_p_hat(const OracleScene& s, uint32_t light_idx, V3 hit_pos, V3 normal) {
    if (light_idx >= (uint32_t)s.lights.size()) return 0.0f;
    const GpuLight& light = s.lights[light_idx];
    V3 l, irr;
    if (light.type == 0) {
        V3 to = load3(light.position) - hit_pos;
        float d2 = fmaxs(dot(to, to), 1e-6f);
        l = normalize(to);
        irr = v3(light.emission[0] * light.intensity / d2, light.emission[1] * light.intensity / d2,
                 light.emission[2] * light.intensity / d2);
    } else {
        l = normalize(-load3(light.direction));
        irr = load3(light.emission) * light.intensity;
    }
    float n_dot_l = fmaxs(dot(normal, l), 0.0f);
    float lum = 0.2126f * irr.x + 0.7152f * irr.y + 0.0722f * irr.z;
    return n_dot_l * lum;
}

// ── ReSTIR DI emitter candidates (ORACLE_DI_EMITTERS; no reference
// counterpart). A candidate is a 32-bit RNG state; the light sample it names
// is decoded from it: the group (GpuLights or emissive triangles, 1/2 each
// when both exist), then a GpuLight picked as the reference picks one, or an
// emissive triangle picked by power and a point on it. inv_src is 1 / the
// sample's source density (a probability for a GpuLight, an area density
// for a point on an emitter); the target is the reference's p_hat for a
// GpuLight and max(n.l, 0) luminance(Le |cos_y| / d^2) for an emitter point.
struct DiLightSample {
    bool emitter;
    uint32_t li;
    V3 y, Le, ny;
    float inv_src;
};
DiLightSample di_decode(const OracleScene& s, uint32_t c) {
    uint32_t st = c;
    const uint32_t NL = (uint32_t)s.lights.size(), NE = s.num_emitters();
    const float pe = NE == 0 ? 0.0f : (NL == 0 ? 1.0f : 0.5f);
    DiLightSample r{};
    r.emitter = NE > 0 && (NL == 0 || rand_float(st) < 0.5f);
    if (r.emitter) {
        const float u = rand_float(st);
        const float uc = rand_float(st);
        const float u1 = rand_float(st);
        const float u2 = rand_float(st);
        const uint32_t k = emitter_pick(s, u, uc);
        const float* e = &s.emit[size_t(k) * 12];
        const V3 E1 = v3(e[4], e[5], e[6]), E2 = v3(e[8], e[9], e[10]);
        const float su = sqrtf(u1);
        r.y = v3(e[0], e[1], e[2]) + E1 * (su * (1.0f - u2)) + E2 * (su * u2);
        r.Le = v3(e[3], e[7], e[11]);
        r.ny = normalize(cross(E1, E2));
        r.inv_src = s.emit_total / (pe * lum709(r.Le));
    } else {
        r.li = uint32_t(rand_float(st) * float(NL)) % NL;
        r.inv_src = float(NL) / (1.0f - pe);
    }
    return r;
}
float di_p_hat_emit(const OracleScene& s, const DiLightSample& d, V3 pos, V3 n) {
    if (!d.emitter) return compute_p_hat(s, d.li, pos, n);
    const V3 to = d.y - pos;
    const float d2 = fmaxs(dot(to, to), 1e-6f);
    const V3 l = normalize(to);
    const float cos_y = fabsf(dot(d.ny, l));
    const V3 irr = d.Le * (cos_y / d2);
    return fmaxs(dot(n, l), 0.0f) * lum709(irr);
}
// A candidate state: the RNG's next state (never the empty marker).
inline uint32_t di_candidate(uint32_t& seed) {
    (void)rand_float(seed);
    return seed == 0xffffffffu ? 0xfffffffeu : seed;
}

// A-trous (atrous.slang:21-39)
inline float luminance601(V3 c) { return dot(c, v3(0.299f, 0.587f, 0.114f)); }
inline float kernel_weight(int offset) {
    switch (offset) { case -2: case 2: return 1.0f; case -1: case 1: return 4.0f; default: return 6.0f; }
}

// GuidingGrid.slang:54-67
uint32_t cell_index(V3 p, uint32_t bsdf_id, V3 cam, const OracleGuidingParams& gp) {
    float view_dist = length(p - cam);
    float cell = fmaxs(gp.base_cell_size + gp.distance_slope * view_dist, 1.0e-4f);
    int qx = (int)floorf(p.x / cell), qy = (int)floorf(p.y / cell), qz = (int)floorf(p.z / cell);
    uint32_t h = pcg_hash((uint32_t)qx * 73856093u ^ (uint32_t)qy * 19349663u ^
                          (uint32_t)qz * 83492791u ^ bsdf_id * 2654435761u);
    return h % std::max(gp.cell_count, 1u);
}
// GuidingGrid.slang:160-189
V3 vmf_sample(V3 mu, float kappa, float ux, float uy, float& pdf) {
    float k = fmaxs(kappa, 1.0e-3f);
    float w = 1.0f + (1.0f / k) * rr_logf(ux + (1.0f - ux) * rr_expf(-2.0f * k));
    w = clampf(w, -1.0f, 1.0f);
    float s = sqrtf(fmaxs(0.0f, 1.0f - w * w));
    float phi = 6.28318530717958647692f * uy;
    V3 local = v3(s * rr_cosf(phi), s * rr_sinf(phi), w);
    V3 T, B;
    build_onb(mu, T, B);
    V3 dir = tangent_to_world(local, T, B, mu);
    float denom = 6.28318530717958647692f * (1.0f - rr_expf(-2.0f * k));
    pdf = k * rr_expf(k * (w - 1.0f)) / fmaxs(denom, 1.0e-8f);
    return dir;
}
float vmf_pdf(V3 mu, float kappa, V3 dir) {
    float k = fmaxs(kappa, 1.0e-3f);
    float w = clampf(dot(mu, dir), -1.0f, 1.0f);
    float denom = 6.28318530717958647692f * (1.0f - rr_expf(-2.0f * k));
    return k * rr_expf(k * (w - 1.0f)) / fmaxs(denom, 1.0e-8f);
}

// sample_primary_dir (restir_pt.slang:520-563)
V3 sample_primary_dir(const float* fitted, V3 p, V3 nn, uint32_t bsdf, V3 cam, const OracleGuidingParams& gp,
                      uint32_t& seed, float& src_pdf) {
    float alpha = 0.0f;
    bool valid = false;
    V3 mu = v3(0, 0, 0);
    float kappa = 0.0f;
    if (gp.enabled != 0u && gp.alpha > 0.0f) {
        uint32_t cell = cell_index(p, bsdf, cam, gp);
        const float* f = fitted + (size_t)cell * 4;
        mu = v3(f[0], f[1], f[2]);
        kappa = f[3];
        valid = (kappa > 0.0f) && (dot(mu, mu) > 0.25f);   // guiding_load_lobe, GuidingGrid.slang:140-157
        if (valid) alpha = gp.alpha;
    }
    V3 T, B;
    build_onb(nn, T, B);
    V3 wi;
    if (rand_float(seed) < alpha) {
        float ux = rand_float(seed);   // rand_float2: x then y
        float uy = rand_float(seed);
        float vpdf;
        wi = vmf_sample(mu, kappa, ux, uy, vpdf);
    } else {
        float u0 = rand_float(seed);   // arguments evaluate left to right
        float u1 = rand_float(seed);
        float cpdf;
        V3 local = sample_cosine_hemisphere(u0, u1, cpdf);
        wi = tangent_to_world(local, T, B, nn);
    }
    float cos_i = dot(nn, wi);
    float p_cos = (cos_i > 0.0f) ? (cos_i * kInvPi) : 0.0f;
    float p_vmf = valid ? vmf_pdf(mu, kappa, wi) : 0.0f;
    src_pdf = alpha * p_vmf + (1.0f - alpha) * p_cos;
    return wi;
}

// ── ReSTIR PT (restir_pt.slang) ────────────────────────────────────────────
struct PtRes {   // Reservoir (restir_pt.slang:231-261)
    V3 rc_pos, rc_normal, suffix_rad, prefix_thp;
    float w_sum, W;
    uint32_t M;
    float valid;
};
inline PtRes pt_load(float* const* img, size_t px) {
    const float* p = img[0] + 4 * px; const float* n = img[1] + 4 * px;
    const float* r = img[2] + 4 * px; const float* e = img[3] + 4 * px;
    PtRes res;
    res.rc_pos = load3(p); res.w_sum = p[3];
    res.rc_normal = load3(n); res.M = asuint(n[3]);
    res.suffix_rad = load3(r); res.W = r[3];
    res.prefix_thp = load3(e); res.valid = e[3];
    return res;
}
inline void put4(float* d, V3 v, float w) { d[0] = v.x; d[1] = v.y; d[2] = v.z; d[3] = w; }
inline void pt_store(float* const* img, size_t px, const PtRes& r) {
    put4(img[0] + 4 * px, r.rc_pos, r.w_sum);
    put4(img[1] + 4 * px, r.rc_normal, asfloat(r.M));
    put4(img[2] + 4 * px, r.suffix_rad, r.W);
    put4(img[3] + 4 * px, r.prefix_thp, r.valid);
}
inline void pt_store_empty(float* const* img, size_t px) {   // write_empty_reservoir (:223-229)
    put4(img[0] + 4 * px, v3(0, 0, 0), 0.0f);
    put4(img[1] + 4 * px, v3(0, 0, 0), asfloat(0u));
    put4(img[2] + 4 * px, v3(0, 0, 0), 0.0f);
    put4(img[3] + 4 * px, v3(0, 0, 0), 0.0f);
}
inline float rsqrt_hlsl(float x) { return 1.0f / sqrtf(x); }   // restated as 1 / sqrt, both correctly rounded
inline float frac_hlsl(float x) { return x - floorf(x); }
inline float luminance709(V3 c) { return dot(c, v3(0.2126f, 0.7152f, 0.0722f)); }   // :161-164

// load_surface_from_images (:287-305)
bool pt_surface(const OracleScene& s, const float* pos_img, const float* nrm_img, size_t px, V3& pos, V3& n,
                uint32_t& mat) {
    const float* p4 = pos_img + 4 * px;
    const float* n4 = nrm_img + 4 * px;
    if (p4[3] < 0.0f) return false;
    pos = load3(p4);
    n = normalize(load3(n4));
    mat = asuint(n4[3]);
    return mat < s.materials.size();
}

// sample_lights (:172-221)
V3 pt_sample_lights(const OracleScene& s, V3 hit_pos, V3 normal, V3 wo, const GpuMaterial& mat, float bias,
                    uint32_t& seed) {
    const uint32_t N = (uint32_t)s.lights.size();
    if (N == 0) return v3(0, 0, 0);
    uint32_t light_idx = uint32_t(rand_float(seed) * float(N)) % N;
    const GpuLight& light = s.lights[light_idx];
    V3 light_dir; float dist; float pdf_light;
    if (light.type == 0) {
        V3 to_light = load3(light.position) - hit_pos;
        dist = length(to_light);
        light_dir = to_light / fmaxs(dist, 1e-6f);
        pdf_light = dist * dist;
    } else {
        light_dir = normalize(-load3(light.direction));
        dist = 1e9f;
        pdf_light = 1.0f;
    }
    if (dot(light_dir, normal) <= 0.0f) return v3(0, 0, 0);
    Hit sh = trace_scene<true>(s, hit_pos + normal * bias, light_dir, bias, dist - 0.01f);
    if (sh.hit) return v3(0, 0, 0);
    V3 brdf_val = brdf_eval(normal, wo, light_dir, load3(mat.base_color), mat.metallic, mat.roughness);
    float n_dot_l = fmaxs(dot(normal, light_dir), 0.0f);
    float denom = light.type == 0 ? (pdf_light + 1e-6f) : 1.0f;
    V3 irradiance = v3(light.emission[0] * light.intensity / denom, light.emission[1] * light.intensity / denom,
                       light.emission[2] * light.intensity / denom);
    float pdf_bsdf = brdf_pdf(wo, light_dir, normal, mat.roughness);
    float mis_weight = (light.type == 0) ? 1.0f
                                         : (pdf_light * pdf_light) / (pdf_light * pdf_light + pdf_bsdf * pdf_bsdf + 1e-10f);
    return brdf_val * irradiance * n_dot_l * mis_weight * float(N);
}

// evaluate_contribution / target_function (:474-503)
V3 pt_contribution(V3 pp, V3 pn, const GpuMaterial& pm, V3 cam, const PtRes& r) {
    V3 to_rc = r.rc_pos - pp;
    float dist2 = dot(to_rc, to_rc);
    if (dist2 <= 1e-8f) return v3(0, 0, 0);
    V3 wi = to_rc * rsqrt_hlsl(dist2);
    float cos_x = fmaxs(dot(pn, wi), 0.0f);
    if (cos_x <= 0.0f) return v3(0, 0, 0);
    V3 wo = normalize(cam - pp);
    V3 brdf_val = brdf_eval(pn, wo, wi, load3(pm.base_color), pm.metallic, pm.roughness);
    return brdf_val * cos_x * r.prefix_thp * r.suffix_rad;
}
float pt_target(V3 pp, V3 pn, const GpuMaterial& pm, V3 cam, const PtRes& r) {
    return luminance709(pt_contribution(pp, pn, pm, cam, r));
}

// reconnection_jacobian (:437-457)
float pt_jacobian(V3 src, V3 tgt, V3 rc_pos, V3 rc_n) {
    V3 sd = rc_pos - src, td = rc_pos - tgt;
    float sd2 = dot(sd, sd), td2 = dot(td, td);
    if (sd2 <= 1e-8f || td2 <= 1e-8f) return 0.0f;
    V3 sdir = sd * rsqrt_hlsl(sd2), tdir = td * rsqrt_hlsl(td2);
    float scos = fabsf(dot(rc_n, -sdir)), tcos = fabsf(dot(rc_n, -tdir));
    if (scos <= 0.05f || tcos <= 0.05f) return 0.0f;
    float j = (tcos * sd2) / (scos * td2);
    return clampf(j, 0.0f, 3.0f);
}

// trace_visibility (:459-469)
bool pt_visible(const OracleScene& s, V3 origin, V3 normal, V3 target, float bias) {
    V3 delta = target - origin;
    float dist = length(delta);
    if (dist <= bias) return false;
    V3 dir = delta / dist;
    return !trace_scene<true>(s, origin + normal * bias, dir, bias, dist - bias).hit;
}

// ── ReSTIR GI (restir_gi.slang) ────────────────────────────────────────────
struct GiRes {   // three-image reservoir (restir_gi.slang:3-7, 199-238)
    V3 pos, rad, nrm;
    float w_sum, W;
    uint32_t M;
};
inline GiRes gi_load(float* const* img, size_t px) {
    const float* a = img[0] + 4 * px; const float* b = img[1] + 4 * px; const float* c = img[2] + 4 * px;
    return GiRes{load3(a), load3(b), load3(c), a[3], b[3], asuint(c[3])};
}
inline void gi_store(float* const* img, size_t px, const GiRes& r) {
    put4(img[0] + 4 * px, r.pos, r.w_sum);
    put4(img[1] + 4 * px, r.rad, r.W);
    put4(img[2] + 4 * px, r.nrm, asfloat(r.M));
}
inline void gi_store_empty(float* const* img, size_t px) {   // write_empty_reservoir (:192-197)
    put4(img[0] + 4 * px, v3(0, 0, 0), 0.0f);
    put4(img[1] + 4 * px, v3(0, 0, 0), 0.0f);
    put4(img[2] + 4 * px, v3(0, 0, 0), asfloat(0u));
}
// evaluate_indirect_radiance (:487-508)
V3 gi_indirect(V3 pp, V3 pn, const GpuMaterial& pm, V3 cam, V3 spos, V3 srad) {
    V3 to_sample = spos - pp;
    float dist2 = dot(to_sample, to_sample);
    if (dist2 <= 1e-8f) return v3(0, 0, 0);
    V3 wi = to_sample * rsqrt_hlsl(dist2);
    float cos_x = fmaxs(dot(pn, wi), 0.0f);
    if (cos_x <= 0.0f) return v3(0, 0, 0);
    V3 wo = normalize(cam - pp);
    V3 brdf_val = brdf_eval(pn, wo, wi, load3(pm.base_color), pm.metallic, pm.roughness);
    return brdf_val * srad * cos_x;
}
// compute_target_function (:524-537)
float gi_target(V3 pp, V3 pn, const GpuMaterial& pm, V3 cam, V3 spos, V3 srad) {
    return luminance709(gi_indirect(pp, pn, pm, cam, spos, srad));
}
// sample_primary_pdf (:510-522)
float gi_primary_pdf(V3 pp, V3 pn, V3 spos) {
    V3 delta = spos - pp;
    float dist2 = dot(delta, delta);
    if (dist2 <= 1e-8f) return 0.0f;
    V3 wi = delta * rsqrt_hlsl(dist2);
    float cos_x = fmaxs(dot(pn, wi), 0.0f);
    return fmaxs(cos_x * kInvPi, 0.0f);
}
// find_reprojected_history_surface (:358-433) with reproject_to_prev_pixel (:306-336)
bool gi_find_history(const GpuCameraData& cam, float* const* hist_prev, V3 pp, V3 pn, uint32_t pmat, V3 cp,
                     size_t& hist, V3& hpos) {
    const uint32_t W = cam.screen_width, H = cam.screen_height;
    V4 clip = mul44(cam.prev_view_proj, V4{pp.x, pp.y, pp.z, 1.0f});
    if (clip.w <= 1.0e-6f) return false;
    float nx = clip.x / clip.w, ny = clip.y / clip.w;
    if (fabsf(nx) > 1.0f || fabsf(ny) > 1.0f) return false;
    float fx = (nx * 0.5f + 0.5f) * float(W) - 0.5f;
    float fy = (ny * 0.5f + 0.5f) * float(H) - 0.5f;
    int cx = (int)floorf(fx + 0.5f), cy = (int)floorf(fy + 0.5f);
    if (cx < 0 || cy < 0 || cx >= (int)W || cy >= (int)H) return false;
    bool found = false;
    float best = 1e30f;
    hist = 0;
    hpos = v3(0, 0, 0);
    for (int oy = -1; oy <= 1; ++oy)
        for (int ox = -1; ox <= 1; ++ox) {
            int qx = cx + ox, qy = cy + oy;
            if (qx < 0 || qy < 0 || qx >= (int)W || qy >= (int)H) continue;
            size_t j = (size_t)qy * W + qx;
            const float* h4 = hist_prev[0] + 4 * j;
            const float* hn4 = hist_prev[1] + 4 * j;
            if (h4[3] < 0.0f) continue;
            V3 cpos = load3(h4), cn = normalize(load3(hn4));
            // is_reprojected_history_compatible (:338-356)
            if (pmat != asuint(hn4[3])) continue;
            if (dot(pn, cn) < 0.9f) continue;
            float view_dist = fmaxs(length(pp - cp), 1.0f);
            float plane = fabsf(dot(cpos - pp, pn));
            float dpos = length(cpos - pp);
            if (!(plane <= 0.01f * view_dist && dpos <= 0.05f * view_dist)) continue;
            float err = plane * 4.0f + dpos;
            if (err < best) { best = err; hist = j; hpos = cpos; found = true; }
        }
    return found;
}

} // namespace

// ═══════════════════════════════ C API ═════════════════════════════════════

extern "C" {

uint32_t oracle_pcg_hash(uint32_t seed) { return pcg_hash(seed); }
uint32_t oracle_make_seed(uint32_t px, uint32_t py, uint32_t f) { return make_seed(px, py, f); }
float oracle_rand_float(uint32_t* seed) { return rand_float(*seed); }

void oracle_detmath_eval(int which, const float* x, float* y, size_t n) {
    for (size_t i = 0; i < n; ++i) {
        switch (which) {
        case 0: y[i] = rr_sinf(x[i]); break;
        case 1: y[i] = rr_cosf(x[i]); break;
        case 2: y[i] = rr_expf(x[i]); break;
        default: y[i] = rr_logf(x[i]); break;
        }
    }
}

OracleScene* oracle_scene_create(const GpuVertex* vertices, uint32_t vertex_count,
                                 const uint32_t* indices, uint32_t index_count,
                                 const GpuMesh* meshes, uint32_t mesh_count,
                                 const GpuMaterial* materials, uint32_t material_count,
                                 const GpuInstance* instances, uint32_t instance_count,
                                 const GpuLight* lights, uint32_t light_count, int use_bvh) {
    OracleScene* s = new OracleScene;
    s->vertices.assign(vertices, vertices + vertex_count);
    s->indices.assign(indices, indices + index_count);
    s->meshes.assign(meshes, meshes + mesh_count);
    s->materials.assign(materials, materials + material_count);
    s->instances.assign(instances, instances + instance_count);
    if (light_count) s->lights.assign(lights, lights + light_count);
    // World-space triangles: instance i, mesh-local primitive j, vertex
    // position transformed by mul(transform, float4(p, 1)).
    for (uint32_t i = 0; i < instance_count; ++i) {
        const GpuInstance& inst = instances[i];
        const GpuMesh& m = meshes[inst.mesh_index];
        const uint32_t ntri = m.index_count / 3u;
        for (uint32_t j = 0; j < ntri; ++j) {
            Tri t;
            V3 p[3];
            for (int k = 0; k < 3; ++k) {
                const GpuVertex& v = vertices[m.vertex_base + indices[m.index_byte_offset / 4u + j * 3u + k]];
                V4 w = mul44(inst.transform, V4{v.pos[0], v.pos[1], v.pos[2], 1.0f});
                p[k] = v3(w.x, w.y, w.z);
            }
            t.p0 = p[0]; t.p1 = p[1]; t.p2 = p[2]; t.inst = i; t.prim = j;
            s->tris.push_back(t);
        }
    }
    {
        double acc = 0.0;
        std::vector<double> power;
        for (const Tri& t : s->tris) {
            const GpuMaterial& mat = materials[meshes[instances[t.inst].mesh_index].material_index];
            if (!any_positive(mat.emissive)) continue;
            const V3 e1 = t.p1 - t.p0, e2 = t.p2 - t.p0;
            const V3 c = cross(e1, e2);
            const float area = 0.5f * sqrtf(dot(c, c));
            if (!(area > 0.0f)) continue;
            const float lum = 0.2126f * mat.emissive[0] + 0.7152f * mat.emissive[1] + 0.0722f * mat.emissive[2];
            acc += double(lum) * double(area);
            const float rec[12] = {t.p0.x, t.p0.y, t.p0.z, mat.emissive[0], e1.x, e1.y, e1.z, mat.emissive[1],
                                   e2.x, e2.y, e2.z, mat.emissive[2]};
            s->emit.insert(s->emit.end(), rec, rec + 12);
            power.push_back(double(lum) * double(area));
        }
        s->emit_total = float(acc);
        // Vose's alias table over the powers (FP64): column k keeps a draw with
        // probability prob_k, else hands it to alias_k; columns paired in stack
        // order, the last "small" with the last "large"; leftovers keep all.
        const size_t n = power.size();
        s->emit_prob.assign(n, 1.0f);
        s->emit_alias.resize(n);
        for (size_t i = 0; i < n; ++i) s->emit_alias[i] = (uint32_t)i;
        if (n > 0) {
            double total = 0.0;
            for (double x : power) total += x;
            std::vector<double> sc(n);
            std::vector<uint32_t> small, large;
            for (size_t i = 0; i < n; ++i) {
                sc[i] = power[i] * double(n) / total;
                (sc[i] < 1.0 ? small : large).push_back((uint32_t)i);
            }
            while (!small.empty() && !large.empty()) {
                const uint32_t a = small.back();
                small.pop_back();
                const uint32_t b = large.back();
                large.pop_back();
                s->emit_prob[a] = (float)sc[a];
                s->emit_alias[a] = b;
                sc[b] = (sc[b] + sc[a]) - 1.0;
                (sc[b] < 1.0 ? small : large).push_back(b);
            }
        }
    }
    s->use_bvh = use_bvh != 0;
    if (s->use_bvh && !s->tris.empty()) {
        std::vector<float> cent(s->tris.size() * 3);
        for (size_t i = 0; i < s->tris.size(); ++i) {
            float lo[3], hi[3];
            bounds_of(s->tris[i], lo, hi);
            for (int a = 0; a < 3; ++a) cent[i * 3 + a] = 0.5f * (lo[a] + hi[a]);
        }
        s->order.resize(s->tris.size());
        for (size_t i = 0; i < s->order.size(); ++i) s->order[i] = (uint32_t)i;
        s->nodes.reserve(s->tris.size());
        build_node(*s, 0, (uint32_t)s->tris.size(), cent);
    }
    return s;
}

void oracle_scene_destroy(OracleScene* s) { delete s; }

uint32_t oracle_emitters(const OracleScene* s, float* records_out, float* prob_out, uint32_t* alias_out,
                         float* total_out) {
    if (records_out) std::memcpy(records_out, s->emit.data(), s->emit.size() * sizeof(float));
    if (prob_out) std::memcpy(prob_out, s->emit_prob.data(), s->emit_prob.size() * sizeof(float));
    if (alias_out) std::memcpy(alias_out, s->emit_alias.data(), s->emit_alias.size() * sizeof(uint32_t));
    if (total_out) *total_out = s->emit_total;
    return s->num_emitters();
}
uint32_t oracle_scene_triangle_count(const OracleScene* s) { return (uint32_t)s->tris.size(); }

int oracle_trace(const OracleScene* s, const float origin[3], const float dir[3], float tmin,
                 float tmax, float* t, float* bu, float* bv, uint32_t* inst, uint32_t* prim) {
    Hit h = trace_scene<false>(*s, load3(origin), load3(dir), tmin, tmax);
    if (!h.hit) { *inst = 0xffffffffu; *prim = 0xffffffffu; return 0; }
    *t = h.t; *bu = h.u; *bv = h.v;
    *inst = s->tris[h.key].inst; *prim = s->tris[h.key].prim;
    return 1;
}

void oracle_trace_batch(const OracleScene* s, const float* origins, const float* dirs, float tmin,
                        float tmax, size_t n, float* hits, uint32_t* prims, int threads) {
    const uint32_t rows = (uint32_t)((n + 255) / 256);
    parallel_rows(rows, threads, [&](uint32_t row) {
        for (size_t i = (size_t)row * 256; i < std::min(n, (size_t)row * 256 + 256); ++i) {
            Hit h = trace_scene<false>(*s, load3(origins + 4 * i), load3(dirs + 4 * i), tmin, tmax);
            if (h.hit) {
                hits[4 * i] = h.t; hits[4 * i + 1] = h.u; hits[4 * i + 2] = h.v;
                hits[4 * i + 3] = asfloat(s->tris[h.key].inst); prims[i] = s->tris[h.key].prim;
            } else {
                hits[4 * i] = -1.0f; hits[4 * i + 1] = 0; hits[4 * i + 2] = 0;
                hits[4 * i + 3] = asfloat(0xffffffffu); prims[i] = 0xffffffffu;
            }
        }
    });
}

void oracle_primary_ray(const GpuCameraData* cam, uint32_t px, uint32_t py, uint32_t frame_seed,
                        float origin[3], float dir[3], uint32_t* seed_out) {
    uint32_t seed = make_seed(px, py, frame_seed);
    float jx = rand_float(seed);
    float jy = rand_float(seed);
    V3 o, d;
    primary_ray(*cam, px, py, jx, jy, o, d);
    origin[0] = o.x; origin[1] = o.y; origin[2] = o.z;
    dir[0] = d.x; dir[1] = d.y; dir[2] = d.z;
    if (seed_out) *seed_out = seed;
}

void oracle_pathtrace(const OracleScene* s, const GpuCameraData* cam, uint32_t frame_seed,
                      uint32_t max_bounces, uint32_t spp, uint32_t x0, uint32_t y0, uint32_t w,
                      uint32_t h, float* out, int threads, uint64_t* stats) {
    oracle_pathtrace_ex(s, cam, frame_seed, max_bounces, spp, x0, y0, w, h, out, threads, stats, 0u);
}

void oracle_pathtrace_ex(const OracleScene* s, const GpuCameraData* cam, uint32_t frame_seed,
                         uint32_t max_bounces, uint32_t spp, uint32_t x0, uint32_t y0, uint32_t w,
                         uint32_t h, float* out, int threads, uint64_t* stats, uint32_t flags) {
    std::atomic<uint64_t> ext_total{0}, shd_total{0};
    const bool emitters = (flags & ORACLE_PT_EMITTERS) != 0;
    parallel_rows(h * spp, threads, [&](uint32_t row) {
        const uint32_t sidx = row / h, y = row % h;
        uint64_t ext = 0, shd = 0;
        for (uint32_t x = 0; x < w; ++x) {
            V3 r = emitters ? trace_path_emitters(*s, *cam, x0 + x, y0 + y, frame_seed + sidx, max_bounces, ext, shd)
                            : trace_path(*s, *cam, x0 + x, y0 + y, frame_seed + sidx, max_bounces, ext, shd);
            float* o = out + (((size_t)sidx * h + y) * w + x) * 4;
            o[0] = r.x; o[1] = r.y; o[2] = r.z; o[3] = 1.0f;
        }
        ext_total += ext; shd_total += shd;
    });
    if (stats) { stats[0] = ext_total; stats[1] = shd_total; }
}

void oracle_accumulate(const float* radiance, float* acc, size_t pixels, uint32_t camera_moved,
                       uint32_t accumulated_spp) {
    // accumulate.slang:33-45
    for (size_t i = 0; i < pixels * 4; ++i) {
        if (camera_moved != 0 || accumulated_spp == 0) {
            acc[i] = radiance[i];
        } else {
            float spp = float(accumulated_spp);
            float weight = 1.0f / (spp + 1.0f);
            acc[i] = acc[i] * (spp / (spp + 1.0f)) + radiance[i] * weight;
        }
    }
}

void oracle_restir_di_initial(const OracleScene* s, const GpuCameraData* cam, const OracleDIParams* p,
                              float* gbuf_pos, float* gbuf_norm, float* res, int threads) {
    // restir_di.slang:186-262
    const uint32_t W = cam->screen_width, H = cam->screen_height;
    const uint32_t N = (uint32_t)s->lights.size();
    const bool E = (p->flags & ORACLE_DI_EMITTERS) != 0;
    const uint32_t NE = E ? s->num_emitters() : 0u;
    parallel_rows(H, threads, [&](uint32_t y) {
        for (uint32_t x = 0; x < W; ++x) {
            const size_t i = ((size_t)y * W + x) * 4;
            uint32_t seed = make_seed(x, y, p->frame_seed);
            float jx = rand_float(seed);
            float jy = rand_float(seed);
            V3 o, d;
            primary_ray(*cam, x, y, jx, jy, o, d);
            Hit h = trace_scene<false>(*s, o, d, 0.001f, 1e9f);
            if (!h.hit) {
                gbuf_pos[i] = 0; gbuf_pos[i + 1] = 0; gbuf_pos[i + 2] = 0; gbuf_pos[i + 3] = -1.0f;
                gbuf_norm[i] = 0; gbuf_norm[i + 1] = 0; gbuf_norm[i + 2] = 0; gbuf_norm[i + 3] = 0;
                pack_reservoir(res + i, 0xffffffffu, 0.0f, 0.0f, 0);
                continue;
            }
            Surf sf = hit_surface(*s, h);
            V3 normal = sf.normal;
            if (dot(normal, -d) < 0.0f) normal = -normal;
            gbuf_pos[i] = sf.pos.x; gbuf_pos[i + 1] = sf.pos.y; gbuf_pos[i + 2] = sf.pos.z;
            gbuf_pos[i + 3] = h.t;
            gbuf_norm[i] = normal.x; gbuf_norm[i + 1] = normal.y; gbuf_norm[i + 2] = normal.z;
            gbuf_norm[i + 3] = asfloat(sf.material);
            if (E ? N + NE == 0 : N == 0) { pack_reservoir(res + i, 0xffffffffu, 0.0f, 0.0f, 0); continue; }
            uint32_t sel = 0xffffffffu;
            float w_sum = 0.0f;
            uint32_t M_count = 0;
            for (uint32_t c = 0; c < p->num_initial_candidates; ++c) {
                uint32_t cand;
                float w_i;
                if (E) {
                    cand = di_candidate(seed);
                    const DiLightSample ds = di_decode(*s, cand);
                    w_i = di_p_hat_emit(*s, ds, sf.pos, normal) * ds.inv_src;
                } else {
                    cand = uint32_t(rand_float(seed) * float(N)) % N;
                    float ph = compute_p_hat(*s, cand, sf.pos, normal);
                    w_i = ph * float(N);
                }
                w_sum += w_i;
                M_count++;
                if (w_sum > 0.0f && rand_float(seed) < w_i / w_sum) sel = cand;
            }
            float W_final = 0.0f;
            if (sel != 0xffffffffu) {
                float ph_y = E ? di_p_hat_emit(*s, di_decode(*s, sel), sf.pos, normal)
                               : compute_p_hat(*s, sel, sf.pos, normal);
                W_final = (ph_y > 1e-10f) ? (w_sum / (float(M_count) * ph_y)) : 0.0f;
            }
            pack_reservoir(res + i, sel, w_sum, W_final, M_count);
        }
    });
}

void oracle_restir_di_temporal(const OracleScene* s, const GpuCameraData* cam, const OracleDIParams* p,
                               const float* gbuf_pos, const float* gbuf_norm, float* res,
                               const float* prev, int threads) {
    // restir_di.slang:266-335
    if (!p->temporal_enable) return;
    const uint32_t W = cam->screen_width, H = cam->screen_height;
    const bool E = (p->flags & ORACLE_DI_EMITTERS) != 0;
    auto phat = [&](uint32_t sel, V3 pos, V3 n) {
        return E ? di_p_hat_emit(*s, di_decode(*s, sel), pos, n) : compute_p_hat(*s, sel, pos, n);
    };
    parallel_rows(H, threads, [&](uint32_t y) {
        for (uint32_t x = 0; x < W; ++x) {
            const size_t i = ((size_t)y * W + x) * 4;
            if (gbuf_pos[i + 3] < 0.0f) continue;
            V3 hit_pos = load3(gbuf_pos + i);
            V3 normal = load3(gbuf_norm + i);
            uint32_t curr_sel = asuint(res[i]); float curr_wsum = res[i + 1];
            uint32_t curr_M = asuint(res[i + 3]);
            uint32_t prev_sel = asuint(prev[i]); float prev_W = prev[i + 2];
            uint32_t prev_M = asuint(prev[i + 3]);
            if (prev_sel == 0xffffffffu || prev_M == 0) continue;
            uint32_t m_cap = std::min(std::max(p->m_cap_factor * p->num_initial_candidates, 1u), 8192u);
            prev_M = std::min(prev_M, m_cap);
            float ph_prev = phat(prev_sel, hit_pos, normal);
            float contrib = ph_prev * prev_W * float(prev_M);
            curr_wsum += contrib;
            uint32_t new_M = curr_M + prev_M;
            if (new_M > m_cap) {
                float scale = float(m_cap) / float(new_M);
                curr_wsum *= scale;
                curr_M = m_cap;
            } else {
                curr_M = new_M;
            }
            uint32_t seed = make_seed(x, y, p->frame_seed + 1u);
            if (contrib > 0.0f && rand_float(seed) < contrib / curr_wsum) curr_sel = prev_sel;
            float W_new = 0.0f;
            if (curr_sel != 0xffffffffu) {
                float ph_y = phat(curr_sel, hit_pos, normal);
                W_new = (ph_y > 1e-10f) ? (curr_wsum / (float(curr_M) * ph_y)) : 0.0f;
                W_new = fmins(W_new, 1e4f);
            }
            pack_reservoir(res + i, curr_sel, curr_wsum, W_new, curr_M);
        }
    });
}

void oracle_restir_di_spatial_shade(const OracleScene* s, const GpuCameraData* cam,
                                    const OracleDIParams* p, const float* gbuf_pos,
                                    const float* gbuf_norm, const float* res, float* output,
                                    int threads) {
    // restir_di.slang:339-472
    const uint32_t W = cam->screen_width, H = cam->screen_height;
    const uint32_t N = (uint32_t)s->lights.size();
    const bool E = (p->flags & ORACLE_DI_EMITTERS) != 0;
    const uint32_t NA = E ? N + s->num_emitters() : N;   // lights the reservoirs can name
    auto phat = [&](uint32_t sel, V3 pos, V3 n) {
        return E ? di_p_hat_emit(*s, di_decode(*s, sel), pos, n) : compute_p_hat(*s, sel, pos, n);
    };
    parallel_rows(H, threads, [&](uint32_t y) {
        for (uint32_t x = 0; x < W; ++x) {
            const size_t i = ((size_t)y * W + x) * 4;
            float* out = output + i;
            if (gbuf_pos[i + 3] < 0.0f) {
                float ndcx = (float(x) + 0.5f) / float(W) * 2.0f - 1.0f;
                float ndcy = (float(y) + 0.5f) / float(H) * 2.0f - 1.0f;
                V4 rv = mul44(cam->inv_proj, V4{ndcx, ndcy, 1.0f, 1.0f});
                rv.z = -1.0f; rv.w = 0.0f;
                V4 rw = mul44(cam->inv_view, rv);
                V3 dir = normalize(v3(rw.x, rw.y, rw.z));
                V3 c = sky(dir);
                out[0] = c.x; out[1] = c.y; out[2] = c.z; out[3] = 1.0f;
                continue;
            }
            V3 hit_pos = load3(gbuf_pos + i);
            V3 normal = load3(gbuf_norm + i);
            uint32_t mat_idx = asuint(gbuf_norm[i + 3]);
            const GpuMaterial& mat = s->materials[mat_idx];
            if (any_positive(mat.emissive)) {
                out[0] = mat.emissive[0]; out[1] = mat.emissive[1]; out[2] = mat.emissive[2]; out[3] = 1.0f;
                continue;
            }
            uint32_t r_sel = asuint(res[i]); float r_wsum = res[i + 1]; float r_W = res[i + 2];
            uint32_t r_M = asuint(res[i + 3]);
            if (p->spatial_enable && p->spatial_num_neighbors > 0 && NA > 0) {
                uint32_t seed = make_seed(x, y, p->frame_seed + 2u);
                for (uint32_t k = 0; k < p->spatial_num_neighbors; ++k) {
                    float angle = rand_float(seed) * 6.28318530717958f;
                    float radius = rand_float(seed) * float(p->spatial_radius);
                    int ox = int(radius * rr_cosf(angle)), oy = int(radius * rr_sinf(angle));
                    int nx = std::min(std::max((int)x + ox, 0), (int)W - 1);
                    int ny = std::min(std::max((int)y + oy, 0), (int)H - 1);
                    const size_t j = ((size_t)ny * W + nx) * 4;
                    if (gbuf_pos[j + 3] < 0.0f) continue;
                    uint32_t nb_sel = asuint(res[j]); float nb_W = res[j + 2];
                    uint32_t nb_M = asuint(res[j + 3]);
                    if (nb_sel == 0xffffffffu || nb_M == 0) continue;
                    float ph_nb = phat(nb_sel, hit_pos, normal);
                    float contrib = ph_nb * nb_W * float(nb_M);
                    r_wsum += contrib;
                    r_M += nb_M;
                    if (contrib > 0.0f && rand_float(seed) < contrib / r_wsum) r_sel = nb_sel;
                }
                if (r_sel != 0xffffffffu) {
                    float ph_y = phat(r_sel, hit_pos, normal);
                    r_W = (ph_y > 1e-10f) ? (r_wsum / (float(r_M) * ph_y)) : 0.0f;
                }
            }
            V3 o = v3(0, 0, 0);
            DiLightSample ds{};
            if (E && r_sel != 0xffffffffu && NA > 0) ds = di_decode(*s, r_sel);
            if (E && r_sel != 0xffffffffu && NA > 0 && ds.emitter && r_W > 0.0f) {
                // a point on an emissive triangle: irradiance Le |cos_y| / d^2
                V3 to = ds.y - hit_pos;
                float dist = length(to);
                V3 l = to / fmaxs(dist, 1e-6f);
                float dd = fmaxs(dist * dist, 1e-6f);
                float cos_y = fabsf(dot(ds.ny, l));
                V3 irr = ds.Le * (cos_y / dd);
                float n_dot_l = fmaxs(dot(normal, l), 0.0f);
                if (n_dot_l > 0.0f) {
                    Hit sh = trace_scene<true>(*s, hit_pos + normal * 1e-4f, l, 0.001f, dist - 0.01f);
                    if (!sh.hit) {
                        V3 wo = normalize(load3(cam->position) - hit_pos);
                        V3 bv = brdf_eval(normal, wo, l, load3(mat.base_color), mat.metallic, mat.roughness);
                        o = ((bv * irr) * n_dot_l) * r_W;
                    }
                }
            } else if (E ? (r_sel != 0xffffffffu && NA > 0 && !ds.emitter && r_W > 0.0f && N > 0)
                         : (r_sel != 0xffffffffu && r_sel < N && r_W > 0.0f && N > 0)) {
                const GpuLight& light = s->lights[E ? ds.li : r_sel];
                V3 l, irr; float dist;
                if (light.type == 0) {
                    V3 to = load3(light.position) - hit_pos;
                    dist = length(to);
                    l = to / fmaxs(dist, 1e-6f);
                    float dd = fmaxs(dist * dist, 1e-6f);
                    irr = v3(light.emission[0] * light.intensity / dd, light.emission[1] * light.intensity / dd,
                             light.emission[2] * light.intensity / dd);
                } else {
                    l = normalize(-load3(light.direction));
                    dist = 1e9f;
                    irr = load3(light.emission) * light.intensity;
                }
                float n_dot_l = fmaxs(dot(normal, l), 0.0f);
                if (n_dot_l > 0.0f) {
                    Hit sh = trace_scene<true>(*s, hit_pos + normal * 1e-4f, l, 0.001f, dist - 0.01f);
                    if (!sh.hit) {
                        V3 wo = normalize(load3(cam->position) - hit_pos);
                        V3 bv = brdf_eval(normal, wo, l, load3(mat.base_color), mat.metallic, mat.roughness);
                        o = ((bv * irr) * n_dot_l) * r_W;
                    }
                }
            }
            out[0] = o.x; out[1] = o.y; out[2] = o.z; out[3] = 1.0f;
        }
    });
}

// The weight of tap (tx, ty) of a centre pixel (position cp, unit normal cn,
// luminance cl) on a neighbour (sp, sn, radiance srad) (atrous.slang:70-95).
inline float atrous_tap_weight(int tx, int ty, V3 cp, V3 cn, float cl, V3 sp, V3 sn, V3 srad, float sigma_pos_sq,
                               float sigma_norm_sq, float sigma_luma_sq) {
    float base_w = (kernel_weight(tx) * kernel_weight(ty)) / 256.0f;
    V3 pd = sp - cp;
    float pos_w = rr_expf(-dot(pd, pd) / sigma_pos_sq);
    float nd = fmaxs(0.0f, 1.0f - dot(cn, sn));
    float normal_w = rr_expf(-nd / sigma_norm_sq);
    float ld = luminance601(srad) - cl;
    float luma_w = rr_expf(-(ld * ld) / sigma_luma_sq);
    return base_w * pos_w * normal_w * luma_w;
}

float oracle_atrous_tap_weight(const float cp[3], const float cn[3], float cl, const float sp[3], const float sn[3],
                               const float srad[3], int tx, int ty, float sp2, float sn2, float sl2) {
    return atrous_tap_weight(tx, ty, load3(cp), load3(cn), cl, load3(sp), load3(sn), load3(srad), sp2, sn2, sl2);
}

void oracle_atrous_iteration(const float* input, const float* gpos, const float* gnrm, float* output,
                             uint32_t width, uint32_t height, uint32_t stride_u, float sp, float sn,
                             float sl, int threads) {
    // atrous.slang:41-106
    parallel_rows(height, threads, [&](uint32_t y) {
        for (uint32_t x = 0; x < width; ++x) {
            const size_t i = ((size_t)y * width + x) * 4;
            const float* cpos = gpos + i;
            const float* crad = input + i;
            float* out = output + i;
            if (cpos[3] < 0.0f) { out[0] = crad[0]; out[1] = crad[1]; out[2] = crad[2]; out[3] = crad[3]; continue; }
            V3 center_normal = normalize(load3(gnrm + i));
            float center_luma = luminance601(load3(crad));
            float sigma_pos_sq = fmaxs(sp * sp, 1.0e-6f);
            float sigma_norm_sq = fmaxs(sn * sn, 1.0e-6f);
            float sigma_luma_sq = fmaxs(sl * sl, 1.0e-6f);
            V3 filtered = v3(0, 0, 0);
            float weight_sum = 0.0f;
            const int mx = (int)width - 1, my = (int)height - 1;
            const int stride = (int)stride_u;
            for (int ty = -2; ty <= 2; ++ty) {
                for (int tx = -2; tx <= 2; ++tx) {
                    int sx = std::min(std::max((int)x + tx * stride, 0), mx);
                    int sy = std::min(std::max((int)y + ty * stride, 0), my);
                    const size_t j = ((size_t)sy * width + sx) * 4;
                    if (gpos[j + 3] < 0.0f) continue;
                    float weight = atrous_tap_weight(tx, ty, load3(cpos), center_normal, center_luma,
                                                     load3(gpos + j), normalize(load3(gnrm + j)),
                                                     load3(input + j), sigma_pos_sq, sigma_norm_sq, sigma_luma_sq);
                    filtered = filtered + load3(input + j) * weight;
                    weight_sum += weight;
                }
            }
            V3 o = (weight_sum > 0.0f) ? (filtered / weight_sum) : load3(crad);
            out[0] = o.x; out[1] = o.y; out[2] = o.z; out[3] = crad[3];
        }
    });
}

uint32_t oracle_guiding_cell_index(const float pos[3], uint32_t bsdf_id, const float cam_pos[3],
                                   const OracleGuidingParams* gp) {
    return cell_index(load3(pos), bsdf_id, load3(cam_pos), *gp);
}

void oracle_guiding_splat(int32_t* accum, const float* pos, const float* dir, const uint32_t* bsdf,
                          size_t n, const float cam_pos[3], const OracleGuidingParams* gp) {
    // GuidingGrid.slang:73-90 at the call site restir_pt.slang:982-994
    for (size_t i = 0; i < n; ++i) {
        uint32_t cell = cell_index(load3(pos + 4 * i), bsdf[i], load3(cam_pos), *gp);
        const float* d = dir + 4 * i;
        uint32_t* a = reinterpret_cast<uint32_t*>(accum) + (size_t)cell * 4;
        for (int c = 0; c < 3; ++c) a[c] += (uint32_t)(int32_t)rintf(d[c] * 1048576.0f);
        a[3] += 1u;
    }
}

void oracle_guiding_fit(int32_t* accum, float* fitted, const OracleGuidingParams* gp) {
    // GuidingGrid.slang:100-137 via cs_fit_guiding (restir_pt.slang:1005-1015)
    if (gp->enabled == 0u) return;
    for (uint32_t cell = 0; cell < gp->cell_count; ++cell) {
        int32_t* a = accum + (size_t)cell * 4;
        float* f = fitted + (size_t)cell * 4;
        int32_t ix = a[0], iy = a[1], iz = a[2];
        uint32_t n = (uint32_t)a[3];
        a[0] = a[1] = a[2] = a[3] = 0;
        if (n < std::max(gp->min_samples, 1u)) { f[3] = -1.0f; continue; }
        V3 sum = v3(float(ix), float(iy), float(iz)) * (1.0f / 1048576.0f);
        float len = length(sum);
        float r = len / float(n);
        r = clampf(r, 1.0e-4f, 0.9999f);
        V3 mu = (len > 1.0e-6f) ? (sum / len) : v3(0.0f, 0.0f, 1.0f);
        float kappa = r * (3.0f - r * r) / (1.0f - r * r);
        kappa = clampf(kappa, 0.5f, gp->kappa_max);
        f[0] = mu.x; f[1] = mu.y; f[2] = mu.z; f[3] = kappa;
    }
}

void oracle_guiding_sample(const float* fitted, const float* pos, const float* normal,
                           const uint32_t* bsdf, uint32_t* seeds, size_t n, const float cam_pos[3],
                           const OracleGuidingParams* gp, float* wi_out, float* pdf_out) {
    for (size_t i = 0; i < n; ++i) {
        uint32_t seed = seeds[i];
        float src_pdf;
        V3 wi = sample_primary_dir(fitted, load3(pos + 4 * i), load3(normal + 4 * i), bsdf[i], load3(cam_pos), *gp,
                                   seed, src_pdf);
        wi_out[4 * i] = wi.x; wi_out[4 * i + 1] = wi.y; wi_out[4 * i + 2] = wi.z; wi_out[4 * i + 3] = 0.0f;
        pdf_out[i] = src_pdf;
        seeds[i] = seed;
    }
}

float oracle_vmf_pdf(const float mu[3], float kappa, const float dir[3]) {
    return vmf_pdf(load3(mu), kappa, load3(dir));
}

void oracle_brdf_eval(const float n[3], const float wo[3], const float wi[3], const float base[3],
                      float metallic, float roughness, float out[3]) {
    V3 r = brdf_eval(load3(n), load3(wo), load3(wi), load3(base), metallic, roughness);
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

void oracle_brdf_sample(const float wo[3], const float n[3], const float base[3], float metallic,
                        float roughness, float u0, float u1, float wi[3], float* pdf, float f[3]) {
    V3 w;
    V3 r = brdf_sample(load3(wo), load3(n), load3(base), metallic, roughness, u0, u1, w, *pdf);
    wi[0] = w.x; wi[1] = w.y; wi[2] = w.z;
    f[0] = r.x; f[1] = r.y; f[2] = r.z;
}

float oracle_brdf_pdf(const float wo[3], const float wi[3], const float n[3], float roughness) {
    return brdf_pdf(load3(wo), load3(wi), load3(n), roughness);
}

// ── ReSTIR PT (restir_pt.slang:567-1000; ReSTIRPTPass.cpp:529-812) ────────────
void oracle_restir_pt_initial(const OracleScene* scene, const GpuCameraData* cam, const OracleRestirPtParams* p,
                              const OracleRestirPtImages* img, int threads) {
    const OracleScene& s = *scene;
    const uint32_t W = cam->screen_width, H = cam->screen_height;
    const V3 cp = load3(cam->position);
    const float bias = p->ray_bias;
    parallel_rows(H, threads, [&](uint32_t y) {
        for (uint32_t x = 0; x < W; ++x) {
            const size_t px = (size_t)y * W + x;
            uint32_t seed = make_seed(x, y, p->frame_seed);
            V3 pp, pn; uint32_t pmat;
            if (!pt_surface(s, img->gbuf_pos, img->gbuf_norm, px, pp, pn, pmat)) {
                put4(img->history_curr[0] + 4 * px, v3(0, 0, 0), -1.0f);
                put4(img->history_curr[1] + 4 * px, v3(0, 0, 0), 0.0f);
                pt_store_empty(img->reservoir_curr, px);
                continue;
            }
            memcpy(img->history_curr[0] + 4 * px, img->gbuf_pos + 4 * px, 16);
            memcpy(img->history_curr[1] + 4 * px, img->gbuf_norm + 4 * px, 16);
            const GpuMaterial& pm = s.materials[pmat];
            PtRes selected{v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0), v3(0, 0, 0), 0.0f, 0.0f, 0u, 0.0f};
            float w_sum = 0.0f;
            uint32_t M_count = 0;
            const uint32_t max_b = std::max(p->max_bounces, 1u);
            for (uint32_t c = 0; c < p->num_initial_candidates; ++c) {
                float src_pdf;
                V3 wi0 = sample_primary_dir(img->guiding_fitted, pp, pn, pmat, cp, p->guiding, seed, src_pdf);
                if (src_pdf <= 1e-6f || dot(pn, wi0) <= 0.0f) continue;
                Hit rh = trace_scene<false>(s, pp + pn * bias, wi0, bias, 1e9f);
                if (!rh.hit) continue;
                Surf rc = hit_surface(s, rh);
                V3 rc_n = rc.normal;
                if (dot(rc_n, wi0) > 0.0f) rc_n = -rc_n;
                const GpuMaterial& rm = s.materials[rc.material];
                V3 suffix = load3(rm.emissive);
                V3 rc_wo = -wi0;
                suffix = suffix + pt_sample_lights(s, rc.pos, rc_n, rc_wo, rm, bias, seed);
                V3 cur_pos = rc.pos, cur_n = rc_n, cur_wo = rc_wo;
                const GpuMaterial* cur_mat = &rm;
                V3 path_thp = v3(1, 1, 1);
                for (uint32_t b = 1; b < max_b; ++b) {
                    float u0 = rand_float(seed);   // rand_float2: x then y
                    float u1 = rand_float(seed);
                    V3 wi; float pdf;
                    V3 f = brdf_sample(cur_wo, cur_n, load3(cur_mat->base_color), cur_mat->metallic,
                                       cur_mat->roughness, u0, u1, wi, pdf);
                    if (pdf <= 1e-6f || dot(cur_n, wi) <= 0.0f) break;
                    float cos_at = fmaxs(dot(cur_n, wi), 0.0f);
                    path_thp = path_thp * (f * cos_at / pdf);
                    if (fmaxs(path_thp.x, fmaxs(path_thp.y, path_thp.z)) <= 0.0f) break;
                    Hit hb = trace_scene<false>(s, cur_pos + cur_n * bias, wi, bias, 1e9f);
                    if (!hb.hit) { suffix = suffix + path_thp * sky(wi); break; }
                    Surf hs = hit_surface(s, hb);
                    V3 hn = hs.normal;
                    if (dot(hn, wi) > 0.0f) hn = -hn;
                    const GpuMaterial& hm = s.materials[hs.material];
                    V3 hwo = -wi;
                    suffix = suffix + path_thp * pt_sample_lights(s, hs.pos, hn, hwo, hm, bias, seed);
                    cur_pos = hs.pos; cur_n = hn; cur_mat = &hm; cur_wo = hwo;
                }
                PtRes cand{rc.pos, rc_n, suffix, v3(1, 1, 1), 0.0f, 0.0f, 1u, 1.0f};
                float p_hat = pt_target(pp, pn, pm, cp, cand);
                if (p_hat <= 0.0f) continue;
                V3 delta = rc.pos - pp;
                if (dot(delta, delta) <= 1e-8f) continue;
                float weight = p_hat / fmaxs(src_pdf, 1e-6f);
                w_sum += weight;
                M_count++;
                if (w_sum > 0.0f && rand_float(seed) < weight / w_sum) selected = cand;
            }
            bool stored = false;
            if (M_count > 0 && selected.valid > 0.5f) {
                float p_hat = pt_target(pp, pn, pm, cp, selected);
                if (p_hat > 1e-10f) {
                    selected.M = M_count;
                    selected.w_sum = w_sum;
                    selected.W = w_sum / (float(M_count) * p_hat);
                    pt_store(img->reservoir_curr, px, selected);
                    stored = true;
                }
            }
            if (!stored) pt_store_empty(img->reservoir_curr, px);
        }
    });
}

void oracle_restir_pt_temporal(const OracleScene* scene, const GpuCameraData* cam, const OracleRestirPtParams* p,
                               const OracleRestirPtImages* img, int threads) {
    if (!p->temporal_enable) return;
    const OracleScene& s = *scene;
    const uint32_t W = cam->screen_width, H = cam->screen_height;
    const V3 cp = load3(cam->position);
    const uint32_t m_cap = std::min(std::max(20u * p->num_initial_candidates, 1u), 8192u);
    parallel_rows(H, threads, [&](uint32_t y) {
        for (uint32_t x = 0; x < W; ++x) {
            const size_t px = (size_t)y * W + x;
            V3 pp, pn; uint32_t pmat;
            if (!pt_surface(s, img->gbuf_pos, img->gbuf_norm, px, pp, pn, pmat)) continue;
            const GpuMaterial& pm = s.materials[pmat];
            // reproject_to_prev_pixel (:326-340)
            V4 clip = mul44(cam->prev_view_proj, V4{pp.x, pp.y, pp.z, 1.0f});
            if (clip.w <= 1.0e-6f) continue;
            float nx = clip.x / clip.w, ny = clip.y / clip.w;
            if (fabsf(nx) > 1.0f || fabsf(ny) > 1.0f) continue;
            float fx = (nx * 0.5f + 0.5f) * float(W) - 0.5f;
            float fy = (ny * 0.5f + 0.5f) * float(H) - 0.5f;
            int cx = (int)floorf(fx + 0.5f), cy = (int)floorf(fy + 0.5f);
            if (cx < 0 || cy < 0 || cx >= (int)W || cy >= (int)H) continue;
            // find_reprojected_history_surface (:355-409)
            bool found = false;
            float best = 1e30f;
            size_t hist = 0;
            V3 hpos = v3(0, 0, 0);
            for (int oy = -1; oy <= 1; ++oy)
                for (int ox = -1; ox <= 1; ++ox) {
                    int qx = cx + ox, qy = cy + oy;
                    if (qx < 0 || qy < 0 || qx >= (int)W || qy >= (int)H) continue;
                    size_t j = (size_t)qy * W + qx;
                    const float* h4 = img->history_prev[0] + 4 * j;
                    const float* hn4 = img->history_prev[1] + 4 * j;
                    if (h4[3] < 0.0f) continue;
                    V3 cpos = load3(h4), cn = normalize(load3(hn4));
                    uint32_t cmat = asuint(hn4[3]);
                    // is_reprojected_history_compatible (:342-353)
                    if (pmat != cmat) continue;
                    if (dot(pn, cn) < 0.9f) continue;
                    float view_dist = fmaxs(length(pp - cp), 1.0f);
                    float plane = fabsf(dot(cpos - pp, pn));
                    float dpos = length(cpos - pp);
                    if (!(plane <= 0.01f * view_dist && dpos <= 0.05f * view_dist)) continue;
                    float err = plane * 4.0f + dpos;
                    if (err < best) { best = err; hist = j; hpos = cpos; found = true; }
                }
            if (!found) continue;
            PtRes cur = pt_load(img->reservoir_curr, px);
            PtRes prv = pt_load(img->reservoir_prev, hist);
            if (prv.M == 0 || prv.valid < 0.5f) continue;
            prv.M = std::min(prv.M, m_cap);
            float jac = pt_jacobian(hpos, pp, prv.rc_pos, prv.rc_normal);
            if (jac <= 0.0f) continue;
            if (!pt_visible(s, pp, pn, prv.rc_pos, p->ray_bias)) continue;
            float ph_prev = pt_target(pp, pn, pm, cp, prv);
            float prev_W = fmins(prv.W, 50.0f);
            float contrib = ph_prev * prev_W * float(prv.M) * jac;
            if (contrib <= 0.0f) continue;
            cur.w_sum += contrib;
            uint32_t seed = make_seed(x, y, p->frame_seed + 1u);
            if (cur.w_sum > 0.0f && rand_float(seed) < contrib / cur.w_sum) {
                cur.rc_pos = prv.rc_pos; cur.rc_normal = prv.rc_normal;
                cur.suffix_rad = prv.suffix_rad; cur.prefix_thp = prv.prefix_thp;
                cur.valid = 1.0f;
            }
            uint32_t new_M = cur.M + prv.M;
            if (new_M > m_cap) { cur.w_sum *= float(m_cap) / float(new_M); cur.M = m_cap; }
            else cur.M = new_M;
            if (cur.M > 0 && cur.valid > 0.5f) {
                float ph_y = pt_target(pp, pn, pm, cp, cur);
                cur.W = (ph_y > 1e-10f) ? (cur.w_sum / (float(cur.M) * ph_y)) : 0.0f;
                cur.W = fmins(cur.W, 50.0f);
            }
            pt_store(img->reservoir_curr, px, cur);
        }
    });
}

void oracle_restir_pt_spatial_shade(const OracleScene* scene, const GpuCameraData* cam,
                                    const OracleRestirPtParams* p, const OracleRestirPtImages* img, int threads) {
    const OracleScene& s = *scene;
    const uint32_t W = cam->screen_width, H = cam->screen_height;
    const V3 cp = load3(cam->position);
    parallel_rows(H, threads, [&](uint32_t y) {
        for (uint32_t x = 0; x < W; ++x) {
            const size_t px = (size_t)y * W + x;
            V3 radiance = v3(0, 0, 0);
            if (p->include_direct_lighting != 0 && img->direct) radiance = radiance + load3(img->direct + 4 * px);
            V3 pp, pn; uint32_t pmat;
            if (!pt_surface(s, img->gbuf_pos, img->gbuf_norm, px, pp, pn, pmat)) {
                if (p->include_direct_lighting == 0) {
                    V3 o, d;
                    primary_ray(*cam, x, y, 0.5f, 0.5f, o, d);
                    radiance = radiance + sky(d);
                }
                put4(img->output + 4 * px, radiance, 1.0f);
                continue;
            }
            const GpuMaterial& pm = s.materials[pmat];
            if (any_positive(pm.emissive)) {
                radiance = radiance + load3(pm.emissive);
                put4(img->output + 4 * px, radiance, 1.0f);
                continue;
            }
            PtRes res = pt_load(img->reservoir_curr, px);
            if (p->spatial_enable && p->spatial_num_neighbors > 0 && res.valid > 0.5f) {
                const float base_phase = frac_hlsl(float(pcg_hash(x ^ (y * 65537u))) * 2.3283064365386963e-10f);
                for (uint32_t k = 0; k < p->spatial_num_neighbors; ++k) {
                    float u = (float(k) + 0.5f) / float(p->spatial_num_neighbors);
                    float angle = frac_hlsl(base_phase + 0.61803398875f * float(k)) * kTwoPi;
                    float radius = sqrtf(u) * float(p->spatial_radius);
                    int ox = (int)(radius * rr_cosf(angle)), oy = (int)(radius * rr_sinf(angle));
                    int nx = std::min(std::max((int)x + ox, 0), (int)W - 1);
                    int ny = std::min(std::max((int)y + oy, 0), (int)H - 1);
                    if (nx == (int)x && ny == (int)y) continue;
                    size_t j = (size_t)ny * W + nx;
                    // is_spatial_neighbor_compatible (:411-430)
                    const float* nb4 = img->gbuf_pos + 4 * j;
                    if (nb4[3] < 0.0f) continue;
                    V3 nbp = load3(nb4), nbn = normalize(load3(img->gbuf_norm + 4 * j));
                    if (dot(nbn, pn) < 0.85f) continue;
                    float plane = fabsf(dot(nbp - pp, pn));
                    float dscale = fmaxs(length(pp - cp), 1.0f);
                    if (!(plane <= 0.02f * dscale)) continue;
                    PtRes nbr = pt_load(img->reservoir_curr, j);
                    if (nbr.M == 0 || nbr.valid < 0.5f) continue;
                    float jac = pt_jacobian(nbp, pp, nbr.rc_pos, nbr.rc_normal);
                    if (jac <= 0.0f) continue;
                    float contrib = pt_target(pp, pn, pm, cp, nbr) * nbr.W * float(nbr.M) * jac;
                    if (contrib <= 0.0f) continue;
                    res.w_sum += contrib;
                    res.M += nbr.M;
                    float accept = frac_hlsl(base_phase + 0.754877666f * float(k + 1u));
                    if (res.w_sum > 0.0f && accept < contrib / res.w_sum) {
                        res.rc_pos = nbr.rc_pos; res.rc_normal = nbr.rc_normal;
                        res.suffix_rad = nbr.suffix_rad; res.prefix_thp = nbr.prefix_thp;
                    }
                }
                if (res.M > 0) {
                    float ph_y = pt_target(pp, pn, pm, cp, res);
                    res.W = (ph_y > 1e-10f) ? (res.w_sum / (float(res.M) * ph_y)) : 0.0f;
                }
            }
            if (res.M > 0 && res.W > 0.0f && res.valid > 0.5f) {
                V3 indirect = pt_contribution(pp, pn, pm, cp, res) * res.W;
                if (luminance709(indirect) > 0.0f && pt_visible(s, pp, pn, res.rc_pos, p->ray_bias))
                    radiance = radiance + indirect * p->indirect_strength;
                if (p->guiding.enabled != 0u) {   // splat (:978-994), integer atomics
                    V3 to_rc = res.rc_pos - pp;
                    float d2 = dot(to_rc, to_rc);
                    if (d2 > 1e-8f) {
                        V3 wi = to_rc * rsqrt_hlsl(d2);
                        uint32_t cell = cell_index(pp, pmat, cp, p->guiding);
                        uint32_t* a = reinterpret_cast<uint32_t*>(img->guiding_accum) + (size_t)cell * 4;
                        __atomic_fetch_add(a + 0, (uint32_t)(int32_t)rintf(wi.x * 1048576.0f), __ATOMIC_RELAXED);
                        __atomic_fetch_add(a + 1, (uint32_t)(int32_t)rintf(wi.y * 1048576.0f), __ATOMIC_RELAXED);
                        __atomic_fetch_add(a + 2, (uint32_t)(int32_t)rintf(wi.z * 1048576.0f), __ATOMIC_RELAXED);
                        __atomic_fetch_add(a + 3, 1u, __ATOMIC_RELAXED);
                    }
                }
            }
            put4(img->output + 4 * px, radiance, 1.0f);
        }
    });
}

// ── traversal work on the library's own BVH ───────────────────────────────
// Restatement of the GPU traversal (research_b200/csrc/rr_trace.cuh:
// make_ray, box_pair, trace_step) over the node and triangle arrays copied
// from a scene (rr_scene_copy_bvh), so that its hits and its node / triangle
// counts — the algorithmic work behind the roofline bytes — can be checked
// ray by ray. Node: (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y), (c1 same),
// (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z), (child0, child1, count0, count1),
// child < 0 a leaf starting at triangle ~child.
void oracle_bvh2_trace(const float* nodes, uint32_t num_nodes, const float* tris, const float* origins,
                       const float* dirs, float tmin, float tmax, uint32_t n, int any_hit, float* hits,
                       uint32_t* prims, uint32_t* work, int threads) {
    auto as_i = [](float f) { int32_t i; memcpy(&i, &f, 4); return i; };
    auto as_u = [](float f) { uint32_t i; memcpy(&i, &f, 4); return i; };
    parallel_rows(n, threads, [&](uint32_t i) {
        const RayPre r = ray_pre(load3(origins + 4 * size_t(i)), load3(dirs + 4 * size_t(i)));
        // slab offsets: t(x) = fma(x, inv, a), near planes nearer and far planes
        // farther by m = 2^-22 |o inv|
        float alo[3], ahi[3];
        const float o3[3] = {r.o.x, r.o.y, r.o.z}, inv3[3] = {r.inv.x, r.inv.y, r.inv.z};
        for (int a = 0; a < 3; ++a) {
            const float oi = o3[a] * inv3[a];
            const float m = fabsf(oi) * 2.384185791015625e-7f;
            const float anear = -oi - m, afar = -oi + m;
            alo[a] = inv3[a] >= 0.0f ? anear : afar;
            ahi[a] = inv3[a] >= 0.0f ? afar : anear;
        }
        float best_t = tmax, bu = 0, bv = 0;
        uint32_t best_key = 0xffffffffu, best_inst = 0, best_prim = 0, nn_count = 0, tri_count = 0;
        bool found = false, done = false;
        int node = 0, sp = 0, stack_node[64];
        float stack_t[64];
        uint32_t visits = 0;
        while (!done) {
            if (++visits > num_nodes + 1) break;
            const float* N = nodes + 16 * size_t(node);
            ++nn_count;
            const float tlim = best_t * 1.00001f;
            bool h[2]; float nr[2];
            for (int k = 0; k < 2; ++k) {
                const float* xy = N + 4 * k;                  // (lo.x, hi.x, lo.y, hi.y)
                const float zlo = N[8 + 2 * k], zhi = N[9 + 2 * k];
                const float tx0 = fmaf(xy[0], inv3[0], alo[0]), tx1 = fmaf(xy[1], inv3[0], ahi[0]);
                const float ty0 = fmaf(xy[2], inv3[1], alo[1]), ty1 = fmaf(xy[3], inv3[1], ahi[1]);
                const float tz0 = fmaf(zlo, inv3[2], alo[2]), tz1 = fmaf(zhi, inv3[2], ahi[2]);
                const float nn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
                const float ff = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1)) * 1.000002f;
                h[k] = nn <= fminf(ff, tlim);
                nr[k] = nn;
            }
            const int c[2] = {as_i(N[12]), as_i(N[13])}, cnt[2] = {as_i(N[14]), as_i(N[15])};
            for (int k = 0; k < 2 && !done; ++k) {
                if (!(h[k] && c[k] < 0)) continue;
                const int first = ~c[k];
                for (int t = first; t < first + cnt[k]; ++t) {
                    ++tri_count;
                    const float* T = tris + 12 * size_t(t);
                    float tt, uu, vv;
                    if (intersect_tri(r, v3(T[0], T[1], T[2]), v3(T[3], T[4], T[5]), v3(T[6], T[7], T[8]), tmin,
                                      best_t, tt, uu, vv)) {
                        const uint32_t key = as_u(T[11]);
                        if (any_hit) { best_t = tt; found = true; done = true; break; }
                        if (!found || tt < best_t || (tt == best_t && key < best_key)) {
                            found = true; best_t = tt; bu = uu; bv = vv; best_key = key;
                            best_inst = as_u(T[9]); best_prim = as_u(T[10]);
                        }
                    }
                }
            }
            if (done) break;
            const bool i0 = h[0] && c[0] >= 0 && nr[0] <= best_t;
            const bool i1 = h[1] && c[1] >= 0 && nr[1] <= best_t;
            if (i0 && i1) {
                // closest hit: nearer child first; any hit: farther first
                const bool first0 = any_hit ? nr[0] > nr[1] : nr[0] <= nr[1];
                stack_node[sp] = first0 ? c[1] : c[0];
                stack_t[sp] = first0 ? nr[1] : nr[0];
                ++sp;
                node = first0 ? c[0] : c[1];
            } else if (i0) {
                node = c[0];
            } else if (i1) {
                node = c[1];
            } else {
                bool next = false;
                while (sp > 0) {
                    --sp;
                    if (stack_t[sp] <= best_t) { node = stack_node[sp]; next = true; break; }
                }
                if (!next) done = true;
            }
        }
        float* H = hits + 4 * size_t(i);
        if (found) {
            H[0] = best_t; H[1] = any_hit ? 0.0f : bu; H[2] = any_hit ? 0.0f : bv;
            const uint32_t inst = any_hit ? 0u : best_inst;
            memcpy(&H[3], &inst, 4);
            prims[i] = any_hit ? 0u : best_prim;
        } else {
            H[0] = -1.0f; H[1] = H[2] = 0.0f;
            const uint32_t none = 0xffffffffu;
            memcpy(&H[3], &none, 4);
            prims[i] = none;
        }
        work[2 * size_t(i)] = nn_count;
        work[2 * size_t(i) + 1] = tri_count;
    });
}

// ── traversal work on the library's 4-wide tree ───────────────────────────
// Restatement of trace_step4 (research_b200/csrc/rr_trace.cuh: box_quad,
// trace_step4) over the 4-wide node array copied from a scene
// (rr_scene_copy_bvh4): 8 float4 per node, lo.x, hi.x, lo.y, hi.y, lo.z,
// hi.z of children 0..3, their references (< 0 a leaf at triangle ~ref) and
// triangle counts. Hit leaf children are intersected in slot order; hit
// inner children within the current t are ordered by a five-comparator
// network on (distance, node) (closest hit ascending, any hit by descending
// distance, a swap only on a strictly smaller key), the first is visited
// next and the rest pushed so that they pop in that order.
void oracle_bvh4_trace(const float* nodes4, uint32_t num_nodes4, const float* tris, const float* origins,
                       const float* dirs, float tmin, float tmax, uint32_t n, int any_hit, float* hits,
                       uint32_t* prims, uint32_t* work, int threads) {
    auto as_i = [](float f) { int32_t i; memcpy(&i, &f, 4); return i; };
    auto as_u = [](float f) { uint32_t i; memcpy(&i, &f, 4); return i; };
    parallel_rows(n, threads, [&](uint32_t i) {
        const RayPre r = ray_pre(load3(origins + 4 * size_t(i)), load3(dirs + 4 * size_t(i)));
        float alo[3], ahi[3];
        const float o3[3] = {r.o.x, r.o.y, r.o.z}, inv3[3] = {r.inv.x, r.inv.y, r.inv.z};
        for (int a = 0; a < 3; ++a) {
            const float oi = o3[a] * inv3[a];
            const float m = fabsf(oi) * 2.384185791015625e-7f;
            const float anear = -oi - m, afar = -oi + m;
            alo[a] = inv3[a] >= 0.0f ? anear : afar;
            ahi[a] = inv3[a] >= 0.0f ? afar : anear;
        }
        float best_t = tmax, bu = 0, bv = 0;
        uint32_t best_key = 0xffffffffu, best_inst = 0, best_prim = 0, nn_count = 0, tri_count = 0;
        bool found = false, done = false;
        int node = 0, sp = 0, stack_node[192];
        float stack_t[192];
        uint32_t visits = 0;
        auto pop = [&]() -> bool {
            while (sp > 0) {
                --sp;
                if (stack_t[sp] <= best_t) { node = stack_node[sp]; return true; }
            }
            return false;
        };
        while (!done) {
            if (++visits > num_nodes4 + 1) break;
            const float* N = nodes4 + 32 * size_t(node);
            ++nn_count;
            const float tlim = best_t * 1.00001f;
            bool h[4]; float nr[4];
            for (int k = 0; k < 4; ++k) {
                const float tx0 = fmaf(N[0 + k], inv3[0], alo[0]), tx1 = fmaf(N[4 + k], inv3[0], ahi[0]);
                const float ty0 = fmaf(N[8 + k], inv3[1], alo[1]), ty1 = fmaf(N[12 + k], inv3[1], ahi[1]);
                const float tz0 = fmaf(N[16 + k], inv3[2], alo[2]), tz1 = fmaf(N[20 + k], inv3[2], ahi[2]);
                const float nn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
                const float ff = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1)) * 1.000002f;
                h[k] = nn <= fminf(ff, tlim);
                nr[k] = nn;
            }
            int R[4], K[4];
            for (int k = 0; k < 4; ++k) { R[k] = as_i(N[24 + k]); K[k] = as_i(N[28 + k]); }
            for (int k = 0; k < 4 && !done; ++k) {
                if (!(h[k] && R[k] < 0)) continue;
                const int first = ~R[k];
                for (int t = first; t < first + K[k]; ++t) {
                    ++tri_count;
                    const float* T = tris + 12 * size_t(t);
                    float tt, uu, vv;
                    if (intersect_tri(r, v3(T[0], T[1], T[2]), v3(T[3], T[4], T[5]), v3(T[6], T[7], T[8]), tmin,
                                      best_t, tt, uu, vv)) {
                        const uint32_t key = as_u(T[11]);
                        if (any_hit) { best_t = tt; found = true; done = true; break; }
                        if (!found || tt < best_t || (tt == best_t && key < best_key)) {
                            found = true; best_t = tt; bu = uu; bv = vv; best_key = key;
                            best_inst = as_u(T[9]); best_prim = as_u(T[10]);
                        }
                    }
                }
            }
            if (done) break;
            float key[4];
            int nd[4], m = 0;
            for (int k = 0; k < 4; ++k) {
                const bool in = h[k] && R[k] >= 0 && nr[k] <= best_t;
                m += in ? 1 : 0;
                key[k] = in ? (any_hit ? -nr[k] : nr[k]) : INFINITY;
                nd[k] = R[k];
            }
            auto cswap = [&](int a, int b) {
                if (key[b] < key[a]) { std::swap(key[a], key[b]); std::swap(nd[a], nd[b]); }
            };
            cswap(0, 1); cswap(2, 3); cswap(0, 2); cswap(1, 3); cswap(1, 2);
            if (m == 0) {
                if (!pop()) done = true;
                continue;
            }
            for (int k = 3; k >= 1; --k) {
                if (k < m) {
                    stack_node[sp] = nd[k];
                    stack_t[sp] = any_hit ? -key[k] : key[k];
                    ++sp;
                }
            }
            node = nd[0];
        }
        float* H = hits + 4 * size_t(i);
        if (found) {
            H[0] = best_t; H[1] = any_hit ? 0.0f : bu; H[2] = any_hit ? 0.0f : bv;
            const uint32_t inst = any_hit ? 0u : best_inst;
            memcpy(&H[3], &inst, 4);
            prims[i] = any_hit ? 0u : best_prim;
        } else {
            H[0] = -1.0f; H[1] = H[2] = 0.0f;
            const uint32_t none = 0xffffffffu;
            memcpy(&H[3], &none, 4);
            prims[i] = none;
        }
        work[2 * size_t(i)] = nn_count;
        work[2 * size_t(i) + 1] = tri_count;
    });
}

// ── ReSTIR GI (restir_gi.slang:568-1000; ReSTIRGIPass.cpp:428-650) ────────────
void oracle_restir_gi_initial(const OracleScene* scene, const GpuCameraData* cam, const OracleRestirGiParams* p,
                              const OracleRestirGiImages* img, int threads) {
    const OracleScene& s = *scene;
    const uint32_t W = cam->screen_width, H = cam->screen_height;
    const V3 cp = load3(cam->position);
    const float bias = p->ray_bias;
    parallel_rows(H, threads, [&](uint32_t y) {
        for (uint32_t x = 0; x < W; ++x) {
            const size_t px = (size_t)y * W + x;
            uint32_t seed = make_seed(x, y, p->frame_seed);
            V3 pp, pn; uint32_t pmat;
            if (!pt_surface(s, img->gbuf_pos, img->gbuf_norm, px, pp, pn, pmat)) {
                put4(img->history_curr[0] + 4 * px, v3(0, 0, 0), -1.0f);
                put4(img->history_curr[1] + 4 * px, v3(0, 0, 0), 0.0f);
                gi_store_empty(img->reservoir_curr, px);
                continue;
            }
            memcpy(img->history_curr[0] + 4 * px, img->gbuf_pos + 4 * px, 16);
            memcpy(img->history_curr[1] + 4 * px, img->gbuf_norm + 4 * px, 16);
            const GpuMaterial& pm = s.materials[pmat];
            V3 sel_pos = v3(0, 0, 0), sel_rad = v3(0, 0, 0), sel_nrm = v3(0, 0, 0);
            float w_sum = 0.0f;
            uint32_t M_count = 0;
            for (uint32_t c = 0; c < p->num_initial_candidates; ++c) {
                float u0 = rand_float(seed);   // arguments evaluated left to right
                float u1 = rand_float(seed);
                float pdf_dir;
                V3 local = sample_cosine_hemisphere(u0, u1, pdf_dir);
                V3 T, B;
                build_onb(pn, T, B);
                V3 bounce = tangent_to_world(local, T, B, pn);
                if (dot(pn, bounce) <= 0.0f) continue;
                Hit sh = trace_scene<false>(s, pp + pn * bias, bounce, bias, 1e9f);
                if (!sh.hit) continue;
                Surf sec = hit_surface(s, sh);
                // evaluate_sample_radiance (:539-552)
                V3 wo = -bounce;
                V3 sn = sec.normal;
                if (dot(sn, wo) < 0.0f) sn = -sn;
                const GpuMaterial& sm = s.materials[sec.material];
                V3 rad = load3(sm.emissive);
                rad = rad + pt_sample_lights(s, sec.pos, sn, wo, sm, bias, seed);
                float tgt = gi_target(pp, pn, pm, cp, sec.pos, rad);
                if (tgt <= 0.0f) continue;
                float pdf = gi_primary_pdf(pp, pn, sec.pos);
                if (pdf <= 1e-6f) continue;
                float weight = tgt / pdf;
                w_sum += weight;
                M_count++;
                if (w_sum > 0.0f && rand_float(seed) < weight / w_sum) {
                    sel_pos = sec.pos; sel_rad = rad; sel_nrm = sec.normal;
                }
            }
            bool stored = false;
            if (M_count > 0) {
                float ph_y = gi_target(pp, pn, pm, cp, sel_pos, sel_rad);
                if (ph_y > 1e-10f) {
                    gi_store(img->reservoir_curr, px,
                             GiRes{sel_pos, sel_rad, sel_nrm, w_sum, w_sum / (float(M_count) * ph_y), M_count});
                    stored = true;
                }
            }
            if (!stored) gi_store_empty(img->reservoir_curr, px);
        }
    });
}

void oracle_restir_gi_temporal(const OracleScene* scene, const GpuCameraData* cam, const OracleRestirGiParams* p,
                               const OracleRestirGiImages* img, int threads) {
    if (!p->temporal_enable) return;
    const OracleScene& s = *scene;
    const uint32_t W = cam->screen_width, H = cam->screen_height;
    const V3 cp = load3(cam->position);
    const uint32_t m_cap = std::min(std::max(20u * p->num_initial_candidates, 1u), 8192u);
    parallel_rows(H, threads, [&](uint32_t y) {
        for (uint32_t x = 0; x < W; ++x) {
            const size_t px = (size_t)y * W + x;
            V3 pp, pn; uint32_t pmat;
            if (!pt_surface(s, img->gbuf_pos, img->gbuf_norm, px, pp, pn, pmat)) continue;
            const GpuMaterial& pm = s.materials[pmat];
            size_t hist; V3 hpos;
            if (!gi_find_history(*cam, img->history_prev, pp, pn, pmat, cp, hist, hpos)) continue;
            GiRes cur = gi_load(img->reservoir_curr, px);
            GiRes prv = gi_load(img->reservoir_prev, hist);
            if (prv.M == 0) continue;
            prv.M = std::min(prv.M, m_cap);
            float jac = pt_jacobian(hpos, pp, prv.pos, prv.nrm);
            if (jac <= 0.0f) continue;
            if (!pt_visible(s, pp, pn, prv.pos, p->ray_bias)) continue;
            float ph_prev = gi_target(pp, pn, pm, cp, prv.pos, prv.rad);
            float prev_W = fmins(prv.W, 50.0f);
            float contrib = ph_prev * prev_W * float(prv.M) * jac;
            if (contrib <= 0.0f) continue;
            cur.w_sum += contrib;
            uint32_t seed = make_seed(x, y, p->frame_seed + 1u);
            if (cur.w_sum > 0.0f && rand_float(seed) < contrib / cur.w_sum) {
                cur.pos = prv.pos; cur.rad = prv.rad; cur.nrm = prv.nrm;
            }
            uint32_t new_M = cur.M + prv.M;
            if (new_M > m_cap) { cur.w_sum *= float(m_cap) / float(new_M); cur.M = m_cap; }
            else cur.M = new_M;
            float W_new = 0.0f;
            if (cur.M > 0) {
                float ph_y = gi_target(pp, pn, pm, cp, cur.pos, cur.rad);
                W_new = (ph_y > 1e-10f) ? (cur.w_sum / (float(cur.M) * ph_y)) : 0.0f;
                W_new = fmins(W_new, 50.0f);
            }
            cur.W = W_new;
            gi_store(img->reservoir_curr, px, cur);
        }
    });
}

void oracle_restir_gi_spatial_shade(const OracleScene* scene, const GpuCameraData* cam,
                                    const OracleRestirGiParams* p, const OracleRestirGiImages* img, int threads) {
    const OracleScene& s = *scene;
    const uint32_t W = cam->screen_width, H = cam->screen_height;
    const V3 cp = load3(cam->position);
    parallel_rows(H, threads, [&](uint32_t y) {
        for (uint32_t x = 0; x < W; ++x) {
            const size_t px = (size_t)y * W + x;
            V3 radiance = v3(0, 0, 0);
            if (p->include_direct_lighting != 0 && img->direct) radiance = radiance + load3(img->direct + 4 * px);
            V3 pp, pn; uint32_t pmat;
            if (!pt_surface(s, img->gbuf_pos, img->gbuf_norm, px, pp, pn, pmat)) {
                if (p->include_direct_lighting == 0) {
                    V3 o, d;
                    primary_ray(*cam, x, y, 0.5f, 0.5f, o, d);
                    radiance = radiance + sky(d);
                }
                put4(img->output + 4 * px, radiance, 1.0f);
                continue;
            }
            const GpuMaterial& pm = s.materials[pmat];
            if (any_positive(pm.emissive)) {
                radiance = radiance + load3(pm.emissive);
                put4(img->output + 4 * px, radiance, 1.0f);
                continue;
            }
            GiRes r = gi_load(img->reservoir_curr, px);
            if (p->spatial_enable && p->spatial_num_neighbors > 0) {
                const float base_phase = frac_hlsl(float(pcg_hash(x ^ (y * 65537u))) * 2.3283064365386963e-10f);
                for (uint32_t k = 0; k < p->spatial_num_neighbors; ++k) {
                    float u = (float(k) + 0.5f) / float(p->spatial_num_neighbors);
                    float angle = frac_hlsl(base_phase + 0.61803398875f * float(k)) * kTwoPi;
                    float radius = sqrtf(u) * float(p->spatial_radius);
                    int ox = (int)(radius * rr_cosf(angle)), oy = (int)(radius * rr_sinf(angle));
                    int nx = std::min(std::max((int)x + ox, 0), (int)W - 1);
                    int ny = std::min(std::max((int)y + oy, 0), (int)H - 1);
                    if (nx == (int)x && ny == (int)y) continue;
                    size_t j = (size_t)ny * W + nx;
                    // is_spatial_neighbor_compatible (:435-459)
                    const float* nb4 = img->gbuf_pos + 4 * j;
                    if (nb4[3] < 0.0f) continue;
                    V3 nbp = load3(nb4), nbn = normalize(load3(img->gbuf_norm + 4 * j));
                    if (dot(nbn, pn) < 0.85f) continue;
                    float plane = fabsf(dot(nbp - pp, pn));
                    float dscale = fmaxs(length(pp - cp), 1.0f);
                    if (!(plane <= 0.02f * dscale)) continue;
                    GiRes nb = gi_load(img->reservoir_curr, j);
                    if (nb.M == 0) continue;
                    float jac = pt_jacobian(nbp, pp, nb.pos, nb.nrm);
                    if (jac <= 0.0f) continue;
                    float contrib = gi_target(pp, pn, pm, cp, nb.pos, nb.rad) * nb.W * float(nb.M) * jac;
                    if (contrib <= 0.0f) continue;
                    r.w_sum += contrib;
                    r.M += nb.M;
                    float accept = frac_hlsl(base_phase + 0.754877666f * float(k + 1u));
                    if (r.w_sum > 0.0f && accept < contrib / r.w_sum) {
                        r.pos = nb.pos; r.rad = nb.rad; r.nrm = nb.nrm;
                    }
                }
                if (r.M > 0) {
                    float ph_y = gi_target(pp, pn, pm, cp, r.pos, r.rad);
                    r.W = (ph_y > 1e-10f) ? (r.w_sum / (float(r.M) * ph_y)) : 0.0f;
                }
            }
            if (r.M > 0 && r.W > 0.0f) {
                V3 indirect = gi_indirect(pp, pn, pm, cp, r.pos, r.rad) * r.W;
                if (luminance709(indirect) > 0.0f && pt_visible(s, pp, pn, r.pos, p->ray_bias))
                    radiance = radiance + indirect * p->indirect_strength;
            }
            put4(img->output + 4 * px, radiance, 1.0f);
        }
    });
}

} // extern "C"
