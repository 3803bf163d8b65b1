// pathtracer.cu — the reference path tracer as wavefront stages.
//
// Restates passes/pathtracer_reference/pathtracer.slang:181-265 (one path per
// pixel per frame seed) as four kernels over SoA queues:
//   raygen : make_seed + jittered primary ray (pathtracer.slang:191-205)
//   extend : closest-hit BVH traversal of the ray queue (trace, :45-120)
//   shade  : miss/sky and emissive termination (:213-229), NEE light pick and
//            shadow-ray emission (:124-177), BSDF sample, throughput update,
//            Russian roulette (:236-260); survivors are compacted into the
//            next ray queue with one warp ballot + one atomic per warp
//   shadow : any-hit traversal; unoccluded NEE contributions are added
// The RNG state travels with each ray, so every path consumes random numbers
// in the reference order (primary 2, per bounce NEE 1 -> BSDF 2 -> RR 1).
// Radiance is accumulated into the caller's image in the same order as the
// reference's `radiance +=` statements, which keeps results bit-identical.

#include "rr_wavefront.cuh"
#include "rr_batch.h"
#include "rr_vmf.cuh"

#include <algorithm>
#include <cstring>

namespace rr {
namespace {

// Result of shading one queued ray: the continuation ray and the shadow ray
// (if any) that the kernel compacts into the next queues.
struct ShadeResult {
    bool cont = false, emit_shadow = false;
    uint32_t pid = 0, seed = 0;
    float3 new_o = make_float3(0, 0, 0), wi = make_float3(0, 0, 0), thp = make_float3(0, 0, 0);
    float3 sh_o = make_float3(0, 0, 0), sh_d = make_float3(0, 0, 0), contrib = make_float3(0, 0, 0);
    float sh_tmax = 0.0f;
    float pdf_next = 0.0f;   // RR_PT_FLAG_EMITTERS: the continuation's bounce density
};

// One ray of the shade stage (a = origin|pid, b = direction|seed, c =
// throughput, h = hit) in scene s, radiance accumulated into out.
RR_D void shade_ray(const DevScene& s, float4* __restrict__ out, uint32_t bounce, uint32_t last, const float4 a,
                    const float4 b, const float4 c, const float4 h, ShadeResult& R) {
    R.pid = __float_as_uint(a.w);
    R.seed = __float_as_uint(b.w);
    const float3 ray_dir = f3(b.x, b.y, b.z);
    R.thp = f3(c.x, c.y, c.z);
    const uint32_t inst = __float_as_uint(h.z);
    if (inst == kNoIndex) {
        // Sky / environment (pathtracer.slang:213-219)
        const float3 L = R.thp * sky_radiance(ray_dir);
        float4 o = out[R.pid];
        o.x = o.x + L.x; o.y = o.y + L.y; o.z = o.z + L.z;
        out[R.pid] = o;
    } else {
        const Surface sf = hit_surface(s, inst, __float_as_uint(h.w), h.x, h.y);
        const float4 m0 = __ldg(s.materials + sf.material * 2);
        const float4 m1 = __ldg(s.materials + sf.material * 2 + 1);
        if (m1.x > 0.0f || m1.y > 0.0f || m1.z > 0.0f) {
            // Emissive surfaces terminate (pathtracer.slang:225-229)
            const float3 L = R.thp * f3(m1.x, m1.y, m1.z);
            float4 o = out[R.pid];
            o.x = o.x + L.x; o.y = o.y + L.y; o.z = o.z + L.z;
            out[R.pid] = o;
        } else {
            const float3 wo = -ray_dir;
            float3 n = sf.normal;
            if (dot(n, wo) < 0.0f) n = -n;
            const float3 base_c = f3(m0.x, m0.y, m0.z);
            const float metallic = m0.w, roughness = m1.w;
            // NEE (pathtracer.slang:124-177): pick, shadow ray, contribution
            if (s.num_lights > 0) {
                const uint32_t N = s.num_lights;
                const uint32_t li = uint32_t(rand_float(R.seed) * float(N)) % N;
                const float4 l0 = __ldg(s.lights + li * 3);
                const float4 l1 = __ldg(s.lights + li * 3 + 1);
                const float4 l2 = __ldg(s.lights + li * 3 + 2);
                const bool is_point = __float_as_uint(l0.w) == 0u;
                float3 ldir; float dist, pdf_light;
                if (is_point) {
                    const float3 to = f3(l0.x, l0.y, l0.z) - sf.pos;
                    dist = length(to);
                    ldir = to / dist;
                    pdf_light = dist * dist;
                } else {
                    ldir = normalize(-f3(l1.x, l1.y, l1.z));
                    dist = 1e9f;
                    pdf_light = 1.0f;
                }
                if (dot(ldir, n) > 0.0f) {
                    const float3 brdf_val = brdf_eval(n, wo, ldir, base_c, metallic, roughness);
                    const float n_dot_l = mx(dot(n, ldir), 0.0f);
                    const float den = is_point ? (pdf_light + 1e-6f) : 1.0f;
                    const float3 irr = f3(l2.x * l2.w / den, l2.y * l2.w / den, l2.z * l2.w / den);
                    float mis = 1.0f;
                    if (!is_point) {
                        const float pb = brdf_pdf(wo, ldir, n, roughness);
                        mis = (pdf_light * pdf_light) / (pdf_light * pdf_light + pb * pb + 1e-10f);
                    }
                    float3 Lr = brdf_val * irr;
                    Lr = Lr * n_dot_l;
                    Lr = Lr * mis;
                    Lr = Lr * float(N);
                    R.contrib = R.thp * Lr;
                    R.sh_o = sf.pos + n * 1e-4f;
                    R.sh_d = ldir;
                    R.sh_tmax = dist - 0.01f;
                    R.emit_shadow = true;
                }
            }
            if (!last) {
                const float u0 = rand_float(R.seed);
                const float u1 = rand_float(R.seed);
                float pdf;
                const float3 f = brdf_sample(wo, n, base_c, metallic, roughness, u0, u1, R.wi, pdf);
                if (!(pdf < 1e-6f)) {
                    const float ndwi = mx(dot(n, R.wi), 0.0f);
                    R.thp = R.thp * ((f * ndwi) / pdf);
                    bool alive = true;
                    if (bounce >= 3) {
                        const float survive = mn(mx(R.thp.x, mx(R.thp.y, R.thp.z)), 0.95f);
                        if (rand_float(R.seed) > survive) alive = false;
                        else R.thp = R.thp / survive;
                    }
                    if (alive) { R.cont = true; R.new_o = sf.pos + n * 1e-4f; }
                }
            }
        }
    }
}

// ── RR_PT_FLAG_EMITTERS (no reference counterpart) ──────────────────────
// Next-event estimation over the GpuLights and the scene's emissive
// triangles: per vertex one group (probability 1/2 each when both exist);
// in the emitter group one triangle in proportion to luminance(Le) * area
// (emitter_pick: the scene's alias table) and a point uniform on it, with the
// solid-angle density p_l = P_E (luminance(Le) / total) d^2 / |cos_y|; the
// GpuLight group is the reference's sample_lights with its factor N divided
// by the group's probability. Bounces are weighted by f cos / p_act, the
// density brdf_sample really draws from (rr_vmf.cuh), which the ray carries
// on (c.w, 0 for camera rays) so that an emissive surface it reaches is
// weighted p_act^2 / (p_act^2 + p_l^2) against the emitter sample's
// p_l^2 / (p_l^2 + p_act^2) (power heuristic; at the last vertex, which
// traces no bounce, the emitter sample's weight is 1). Emissive surfaces
// still end the path.
RR_D float lum709(float3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

RR_D float emitter_pdf(float p_group, float lum, float total, float d2, float cos_y) {
    return p_group * (lum / total) * d2 / cos_y;
}

// First k with cdf[k] > target (n - 1 when none is).
RR_D void shade_ray_emitters(const DevScene& s, float4* __restrict__ out, uint32_t bounce, uint32_t last,
                             const float4 a, const float4 b, const float4 c, const float4 h, ShadeResult& R) {
    R.pid = __float_as_uint(a.w);
    R.seed = __float_as_uint(b.w);
    const float3 ray_dir = f3(b.x, b.y, b.z);
    R.thp = f3(c.x, c.y, c.z);
    const float prev_pdf = c.w;
    const uint32_t inst = __float_as_uint(h.z);
    const uint32_t NL = s.num_lights, NE = s.num_emitters;
    const float pe = NE == 0 ? 0.0f : (NL == 0 ? 1.0f : 0.5f);
    if (inst == kNoIndex) {
        const float3 L = R.thp * sky_radiance(ray_dir);
        float4 o = out[R.pid];
        o.x = o.x + L.x; o.y = o.y + L.y; o.z = o.z + L.z;
        out[R.pid] = o;
        return;
    }
    const uint32_t prim = __float_as_uint(h.w);
    const Surface sf = hit_surface(s, inst, prim, h.x, h.y);
    const float4 m0 = __ldg(s.materials + sf.material * 2);
    const float4 m1 = __ldg(s.materials + sf.material * 2 + 1);
    if (m1.x > 0.0f || m1.y > 0.0f || m1.z > 0.0f) {
        const float3 Le = f3(m1.x, m1.y, m1.z);
        float w = 1.0f;
        if (prev_pdf > 0.0f) {
            const float3 ng = hit_geometric_normal(s, inst, prim);
            const float cos_y = fabsf(dot(ng, ray_dir));
            const float3 dd = sf.pos - f3(a.x, a.y, a.z);
            const float pl = cos_y > 0.0f ? emitter_pdf(pe, lum709(Le), s.emit_total, dot(dd, dd), cos_y) : 0.0f;
            const float aa = prev_pdf * prev_pdf;
            w = aa / (aa + pl * pl);
        }
        const float3 L = R.thp * (Le * w);
        float4 o = out[R.pid];
        o.x = o.x + L.x; o.y = o.y + L.y; o.z = o.z + L.z;
        out[R.pid] = o;
        return;
    }
    const float3 wo = -ray_dir;
    float3 n = sf.normal;
    if (dot(n, wo) < 0.0f) n = -n;
    const float3 base_c = f3(m0.x, m0.y, m0.z);
    const float metallic = m0.w, roughness = m1.w;
    if (NL + NE > 0) {
        const bool use_e = NE > 0 && (NL == 0 || rand_float(R.seed) < 0.5f);
        if (use_e) {
            const float u = rand_float(R.seed);
            const float uc = rand_float(R.seed);
            const float u1 = rand_float(R.seed);
            const float u2 = rand_float(R.seed);
            const uint32_t k = emitter_pick(s, u, uc);
            const float4 e0 = __ldg(s.emitters + k * 3), e1 = __ldg(s.emitters + k * 3 + 1);
            const float4 e2 = __ldg(s.emitters + k * 3 + 2);
            const float3 E1 = xyz(e1), E2 = xyz(e2);
            const float3 Le = f3(e0.w, e1.w, e2.w);
            const float su = sqrtf(u1);
            const float b1 = su * (1.0f - u2), b2 = su * u2;
            const float3 y = xyz(e0) + E1 * b1 + E2 * b2;
            const float3 to = y - sf.pos;
            const float d2 = dot(to, to);
            const float dist = sqrtf(d2);
            const float3 l = to / dist;
            const float cos_x = dot(n, l);
            const float3 ny = normalize(cross(E1, E2));
            const float cos_y = fabsf(dot(ny, l));
            if (cos_x > 0.0f && cos_y > 0.0f && d2 > 0.0f) {
                const float pl = emitter_pdf(pe, lum709(Le), s.emit_total, d2, cos_y);
                const float3 f = brdf_eval(n, wo, l, base_c, metallic, roughness);
                const float pb = brdf_sample_pdfs(wo, n, base_c, metallic, roughness, l).actual;
                const float aa = pl * pl;
                // the last vertex traces no bounce that could reach the
                // emitter: its sample carries the whole weight there
                const float wl = last ? 1.0f : aa / (aa + pb * pb);
                float3 cc = f * Le;
                cc = cc * (cos_x * wl / pl);
                R.contrib = R.thp * cc;
                R.sh_o = sf.pos + n * 1e-4f;
                R.sh_d = l;
                R.sh_tmax = dist - 0.01f;
                R.emit_shadow = true;
            }
        } else {
            // sample_lights (pathtracer.slang:124-177), factor N / (1 - P_E)
            const uint32_t li = uint32_t(rand_float(R.seed) * float(NL)) % NL;
            const float4 l0 = __ldg(s.lights + li * 3);
            const float4 l1 = __ldg(s.lights + li * 3 + 1);
            const float4 l2 = __ldg(s.lights + li * 3 + 2);
            const bool is_point = __float_as_uint(l0.w) == 0u;
            float3 ldir; float dist, pdf_light;
            if (is_point) {
                const float3 to = f3(l0.x, l0.y, l0.z) - sf.pos;
                dist = length(to);
                ldir = to / dist;
                pdf_light = dist * dist;
            } else {
                ldir = normalize(-f3(l1.x, l1.y, l1.z));
                dist = 1e9f;
                pdf_light = 1.0f;
            }
            if (dot(ldir, n) > 0.0f) {
                const float3 brdf_val = brdf_eval(n, wo, ldir, base_c, metallic, roughness);
                const float n_dot_l = mx(dot(n, ldir), 0.0f);
                const float den = is_point ? (pdf_light + 1e-6f) : 1.0f;
                const float3 irr = f3(l2.x * l2.w / den, l2.y * l2.w / den, l2.z * l2.w / den);
                float mis = 1.0f;
                if (!is_point) {
                    const float pb = brdf_pdf(wo, ldir, n, roughness);
                    mis = (pdf_light * pdf_light) / (pdf_light * pdf_light + pb * pb + 1e-10f);
                }
                float3 Lr = brdf_val * irr;
                Lr = Lr * n_dot_l;
                Lr = Lr * mis;
                Lr = Lr * (float(NL) / (1.0f - pe));
                R.contrib = R.thp * Lr;
                R.sh_o = sf.pos + n * 1e-4f;
                R.sh_d = ldir;
                R.sh_tmax = dist - 0.01f;
                R.emit_shadow = true;
            }
        }
    }
    if (last) return;
    const float u0 = rand_float(R.seed);
    const float u1 = rand_float(R.seed);
    float pdf;
    const float3 f = brdf_sample(wo, n, base_c, metallic, roughness, u0, u1, R.wi, pdf);
    if (pdf < 1e-6f) return;
    const float pa = brdf_sample_pdfs(wo, n, base_c, metallic, roughness, R.wi).actual;
    if (!(pa > 0.0f)) return;
    const float ndwi = mx(dot(n, R.wi), 0.0f);
    R.thp = R.thp * ((f * ndwi) / pa);
    if (bounce >= 3) {
        const float survive = mn(mx(R.thp.x, mx(R.thp.y, R.thp.z)), 0.95f);
        if (rand_float(R.seed) > survive) return;
        R.thp = R.thp / survive;
    }
    R.pdf_next = pa;
    R.cont = true;
    R.new_o = sf.pos + n * 1e-4f;
}

// Multi: a batch of scenes; a ray's scene index is in c.w, its scene is
// table[index] and its image outs[index]; the index is carried on.
template <bool Multi, bool Emit = false>
__global__ void __launch_bounds__(kBlock, 4) shade_kernel(DevScene s, const DevScene* __restrict__ table,
                                                       float4* const* __restrict__ outs, uint32_t bounce,
                                                       uint32_t last, const float4* __restrict__ qa,
                                                       const float4* __restrict__ qb,
                                                       const float4* __restrict__ qc,
                                                       const float4* __restrict__ hits,
                                                       float4* na, float4* nb, float4* nc,
                                                       float4* sa, float4* sb, float4* sc,
                                                       float4* __restrict__ out,
                                                       const uint32_t* count_ptr,
                                                       uint32_t* next_count, uint32_t* shadow_count) {
    const uint32_t count = *count_ptr;
    const uint32_t warp_first = blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = warp_first; base < count; base += stride) {
        const uint32_t i = base + lane_id();
        ShadeResult R;
        uint32_t sid = 0;
        if (i < count) {
            const float4 a = qa[i], b = qb[i], c = qc[i];
            const float4 h = hits[i];
            if constexpr (Multi) {
                sid = __float_as_uint(c.w);
                shade_ray(table[sid], outs[sid], bounce, last, a, b, c, h, R);
            } else if constexpr (Emit) {
                shade_ray_emitters(s, out, bounce, last, a, b, c, h, R);
            } else {
                shade_ray(s, out, bounce, last, a, b, c, h, R);
            }
        }
        const float tag = Multi ? __uint_as_float(sid) : 0.0f;
        const uint32_t sslot = warp_alloc(R.emit_shadow, shadow_count);
        if (R.emit_shadow) {
            sa[sslot] = make_float4(R.sh_o.x, R.sh_o.y, R.sh_o.z, __uint_as_float(R.pid));
            sb[sslot] = make_float4(R.sh_d.x, R.sh_d.y, R.sh_d.z, R.sh_tmax);
            sc[sslot] = make_float4(R.contrib.x, R.contrib.y, R.contrib.z, tag);
        }
        const uint32_t rslot = warp_alloc(R.cont, next_count);
        if (R.cont) {
            na[rslot] = make_float4(R.new_o.x, R.new_o.y, R.new_o.z, __uint_as_float(R.pid));
            nb[rslot] = make_float4(R.wi.x, R.wi.y, R.wi.z, __uint_as_float(R.seed));
            nc[rslot] = make_float4(R.thp.x, R.thp.y, R.thp.z, Emit ? R.pdf_next : tag);
        }
    }
}

} // namespace
} // namespace rr

using namespace rr;

extern "C" rr_status rr_pathtracer_execute(rr_ctx* ctx, const rr_scene* scene,
                                           const GpuCameraData* cam, const rr_pt_params* p,
                                           float* radiance_out, void* stream_v) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!scene || !cam || !p || !radiance_out)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_pathtracer_execute: null argument");
    const uint32_t W = cam->screen_width, H = cam->screen_height;
    if (W == 0 || H == 0 || p->spp == 0)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_pathtracer_execute: empty image (%ux%u, spp %u)", W, H, p->spp);
    if (p->max_bounces > uint32_t(kMaxBounces))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "max_bounces %u exceeds %d", p->max_bounces, kMaxBounces);
    const uint64_t n64 = uint64_t(W) * H * p->spp;
    if (n64 >= (1ull << 31)) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "too many paths");
    const size_t n = size_t(n64);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    rr_status st = ensure_queues(ctx, n);
    if (st != RR_OK) return st;
    rr_pt_queues& q = ctx->pt;
    uint32_t* C = ctx->counters;
    RR_TRY_CUDA(ctx, cudaMemsetAsync(C, 0, sizeof(uint32_t) * kCounterWords, stream));

    PtLaunch L;
    L.cam = *cam;
    L.frame_seed = p->frame_seed;
    L.spp = p->spp;
    L.width = W; L.height = H;
    L.tiles_x = (W + 7) / 8;
    L.tiles_per_image = L.tiles_x * ((H + 3) / 4);
    {
        const uint64_t threads = uint64_t(L.tiles_per_image) * p->spp * 32;
        const uint32_t blocks = uint32_t((threads + kBlock - 1) / kBlock);
        float4* out = reinterpret_cast<float4*>(radiance_out);
        rr_stage_timer t0(ctx, stream, (p->flags & RR_PT_FLAG_TIME_STAGES) != 0);
        t0.begin(0);
        raygen_kernel<<<blocks, kBlock, 0, stream>>>(L, out, q.ray_a[0], q.ray_b[0], q.ray_c[0], C);
        RR_CHECK_LAUNCH(ctx);
        t0.end(0);
        rr_status st0 = t0.commit();
        if (st0 != RR_OK) return st0;
    }
    const bool count = (p->flags & RR_PT_FLAG_COUNT_TRAVERSAL) != 0;
    const bool timed = (p->flags & RR_PT_FLAG_TIME_STAGES) != 0;
    QueueKernel ext_k = count ? extend_variant<true>(ctx->extend_variant) : extend_variant<false>(ctx->extend_variant);
    ShadowKernel sh_k = count ? shadow_variant<true>(ctx->shadow_variant) : shadow_variant<false>(ctx->shadow_variant);
    const int g_ext = persistent_grid(ctx, reinterpret_cast<const void*>(ext_k));
    const int g_sh = persistent_grid(ctx, reinterpret_cast<const void*>(sh_k));
    const bool emitters = (p->flags & RR_PT_FLAG_EMITTERS) != 0;
    using ShadeKernel = decltype(&shade_kernel<false, false>);
    const ShadeKernel shade_k = emitters ? shade_kernel<false, true> : shade_kernel<false, false>;
    const int g_shade = std::min<int>(persistent_grid(ctx, reinterpret_cast<const void*>(shade_k)),
                                      int((n + kBlock - 1) / kBlock));
    if (count) RR_TRY_CUDA(ctx, cudaMemsetAsync(ctx->work64, 0, sizeof(unsigned long long) * 4, stream));
    const DevScene& S = scene->dev;
    float4* out = reinterpret_cast<float4*>(radiance_out);
    rr_stage_timer timer(ctx, stream, timed);
    // Bounce b's shadow rays only add to the image and read the shadow queue;
    // bounce b+1's extension rays only read the ray queue and write hits. So
    // the shadow launch runs on the side stream next to the next extend
    // launch, and the next shade launch (which writes the image and the
    // shadow queue) waits for it. Stage timing keeps one stream.
    const bool overlap = ctx->overlap_shadow && !timed;
    if (overlap && (st = ensure_side(ctx)) != RR_OK) return st;
    for (uint32_t b = 0; b < p->max_bounces; ++b) {
        const int cur = b & 1, nxt = cur ^ 1;
        uint32_t* cb = C + 4 * b;
        uint32_t* cn = C + 4 * (b + 1);
        timer.begin(1);
        ext_k<<<g_ext, kBlock, 0, stream>>>(S, q.ray_a[cur], q.ray_b[cur], q.hits, cb, cb + 1, ctx->work64);
        RR_CHECK_LAUNCH(ctx);
        timer.end(1);
        if (overlap && b > 0) RR_TRY_CUDA(ctx, cudaStreamWaitEvent(stream, ctx->shadowed[b - 1], 0));
        timer.begin(2);
        shade_k<<<g_shade, kBlock, 0, stream>>>(S, nullptr, nullptr, b, b + 1 == p->max_bounces ? 1u : 0u,
                                                     q.ray_a[cur], q.ray_b[cur], q.ray_c[cur], q.hits,
                                                     q.ray_a[nxt], q.ray_b[nxt], q.ray_c[nxt],
                                                     q.shadow_a, q.shadow_b, q.shadow_c, out,
                                                     cb, cn, cb + 2);
        RR_CHECK_LAUNCH(ctx);
        timer.end(2);
        cudaStream_t sh_stream = stream;
        if (overlap) {
            RR_TRY_CUDA(ctx, cudaEventRecord(ctx->shaded[b], stream));
            RR_TRY_CUDA(ctx, cudaStreamWaitEvent(ctx->side, ctx->shaded[b], 0));
            sh_stream = ctx->side;
        }
        timer.begin(3);
        sh_k<<<g_sh, kBlock, 0, sh_stream>>>(S, q.shadow_a, q.shadow_b, q.shadow_c, out, cb + 2, cb + 3,
                                             ctx->work64 + 2);
        RR_CHECK_LAUNCH(ctx);
        timer.end(3);
        if (overlap) RR_TRY_CUDA(ctx, cudaEventRecord(ctx->shadowed[b], ctx->side));
    }
    if (overlap && p->max_bounces > 0)
        RR_TRY_CUDA(ctx, cudaStreamWaitEvent(stream, ctx->shadowed[p->max_bounces - 1], 0));
    ctx->launches += 1 + 3 * uint64_t(p->max_bounces);
    ctx->last_max_bounces = p->max_bounces;
    ctx->last_counted = count;
    return timer.commit();
}

extern "C" rr_status rr_pathtracer_stats(rr_ctx* ctx, rr_pt_stats* out, int reset) {
    if (!ctx || !out) return RR_ERR_INVALID_ARGUMENT;
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    RR_TRY_CUDA(ctx, cudaDeviceSynchronize());
    uint32_t h[kCounterWords];
    RR_TRY_CUDA(ctx, cudaMemcpy(h, ctx->counters, sizeof(h), cudaMemcpyDeviceToHost));
    std::memset(out, 0, sizeof(*out));
    for (uint32_t b = 0; b < ctx->last_max_bounces; ++b) {
        out->extension_rays += h[4 * b];
        out->shadow_rays += h[4 * b + 2];
    }
    if (ctx->last_counted) {
        unsigned long long w[4];
        RR_TRY_CUDA(ctx, cudaMemcpy(w, ctx->work64, sizeof(w), cudaMemcpyDeviceToHost));
        out->extension_nodes = w[0]; out->extension_tris = w[1];
        out->shadow_nodes = w[2]; out->shadow_tris = w[3];
    }
    rr_status st = rr_stage_timer::collect(ctx);
    if (st != RR_OK) return st;
    out->ms_raygen = ctx->stage_ms[0]; out->ms_extend = ctx->stage_ms[1];
    out->ms_shade = ctx->stage_ms[2]; out->ms_shadow = ctx->stage_ms[3];
    out->launches_extend = ctx->stage_launches[1];
    out->launches_total = ctx->launches;
    if (reset) {
        for (int k = 0; k < 4; ++k) { ctx->stage_ms[k] = 0.0; ctx->stage_launches[k] = 0; }
    }
    return RR_OK;
}

extern "C" rr_status rr_pathtracer_set_overlap(rr_ctx* ctx, int enable) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    ctx->overlap_shadow = enable != 0;
    return RR_OK;
}

extern "C" int rr_pathtracer_variant_width(int v) {
    if (v < 0 || v >= RR_PT_VARIANT_COUNT) return 0;
    return (v == 3 || v == 4 || v == 6) ? 4 : 2;   // the Wide variants of the kernel tables (rr_wavefront.cuh)
}

extern "C" rr_status rr_pathtracer_set_variants(rr_ctx* ctx, int ev, int sv) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (ev < 0 || ev >= RR_PT_VARIANT_COUNT || sv < 0 || sv >= RR_PT_VARIANT_COUNT)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "traversal variant out of range");
    ctx->extend_variant = ev;
    ctx->shadow_variant = sv;
    return RR_OK;
}

extern "C" rr_status rr_pathtracer_tune(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                        const rr_pt_params* p, float* radiance_out, void* stream,
                                        rr_pt_tune_result* out) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!scene || !cam || !p || !radiance_out || !out)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_pathtracer_tune: null argument");
    rr_pt_stats st;
    rr_status s = rr_pathtracer_stats(ctx, &st, 1);  // drop earlier timings
    if (s != RR_OK) return s;
    rr_pt_params q = *p;
    q.flags = RR_PT_FLAG_TIME_STAGES;
    double best_e = 1e30, best_s = 1e30;
    out->best_extend = out->best_shadow = 0;
    for (int v = 0; v < RR_PT_VARIANT_COUNT; ++v) {
        ctx->extend_variant = v;
        ctx->shadow_variant = v;
        // one untimed pass to settle caches and clocks, then one timed pass
        rr_pt_params warm = *p;
        warm.flags = 0;
        if ((s = rr_pathtracer_execute(ctx, scene, cam, &warm, radiance_out, stream)) != RR_OK) return s;
        if ((s = rr_pathtracer_execute(ctx, scene, cam, &q, radiance_out, stream)) != RR_OK) return s;
        if ((s = rr_pathtracer_stats(ctx, &st, 1)) != RR_OK) return s;
        out->extend_ms[v] = st.ms_extend;
        out->shadow_ms[v] = st.ms_shadow;
        if (st.ms_extend < best_e) { best_e = st.ms_extend; out->best_extend = v; }
        if (st.ms_shadow < best_s) { best_s = st.ms_shadow; out->best_shadow = v; }
    }
    ctx->extend_variant = out->best_extend;
    ctx->shadow_variant = out->best_shadow;
    return RR_OK;
}

// ── batches of scenes ──────────────────────────────────────────────────────
namespace {

// Enqueues one batch frame: counter reset, raygen over every scene's tiles,
// then per bounce one extend, one shade and one shadow launch for all scenes.
rr_status enqueue_batch(rr_ctx* ctx, rr_batch* B, uint32_t total_tiles, size_t n, uint32_t max_bounces,
                        uint32_t flags, cudaStream_t stream) {
    using namespace rr;
    rr_pt_queues& q = ctx->pt;
    uint32_t* C = ctx->counters;
    const uint32_t count_scenes = uint32_t(B->scenes.size());
    const BatchEntry* entries = reinterpret_cast<const BatchEntry*>(B->d_call);
    float4* const* outs = reinterpret_cast<float4* const*>(B->d_call + B->entries_bytes);
    const bool count = (flags & RR_PT_FLAG_COUNT_TRAVERSAL) != 0;
    const bool timed = (flags & RR_PT_FLAG_TIME_STAGES) != 0;
    RR_TRY_CUDA(ctx, cudaMemsetAsync(C, 0, sizeof(uint32_t) * kCounterWords, stream));
    {
        const uint64_t threads = uint64_t(total_tiles) * 32;
        rr_stage_timer t0(ctx, stream, timed);
        t0.begin(0);
        raygen_batch_kernel<<<uint32_t((threads + kBlock - 1) / kBlock), kBlock, 0, stream>>>(
            entries, count_scenes, total_tiles, outs, q.ray_a[0], q.ray_b[0], q.ray_c[0], C);
        RR_CHECK_LAUNCH(ctx);
        t0.end(0);
        rr_status st0 = t0.commit();
        if (st0 != RR_OK) return st0;
    }
    BatchQueueKernel ext_k = count ? extend_batch_variant<true>(ctx->extend_variant)
                                   : extend_batch_variant<false>(ctx->extend_variant);
    BatchShadowKernel sh_k = count ? shadow_batch_variant<true>(ctx->shadow_variant)
                                   : shadow_batch_variant<false>(ctx->shadow_variant);
    const int g_ext = persistent_grid(ctx, reinterpret_cast<const void*>(ext_k));
    const int g_sh = persistent_grid(ctx, reinterpret_cast<const void*>(sh_k));
    const int g_shade = std::min<int>(persistent_grid(ctx, reinterpret_cast<const void*>(shade_kernel<true>)),
                                      int((n + kBlock - 1) / kBlock));
    if (count) RR_TRY_CUDA(ctx, cudaMemsetAsync(ctx->work64, 0, sizeof(unsigned long long) * 4, stream));
    rr_stage_timer timer(ctx, stream, timed);
    // shadow rays of bounce b beside the extension rays of bounce b+1, as in
    // rr_pathtracer_execute (stage timing keeps one stream)
    const bool overlap = ctx->overlap_shadow && !timed;
    if (overlap) {
        const rr_status so = ensure_side(ctx);
        if (so != RR_OK) return so;
    }
    for (uint32_t b = 0; b < max_bounces; ++b) {
        const int cur = b & 1, nxt = cur ^ 1;
        uint32_t* cb = C + 4 * b;
        uint32_t* cn = C + 4 * (b + 1);
        timer.begin(1);
        ext_k<<<g_ext, kBlock, 0, stream>>>(B->d_table, q.ray_a[cur], q.ray_b[cur], q.ray_c[cur], q.hits, cb, cb + 1,
                                            ctx->work64);
        RR_CHECK_LAUNCH(ctx);
        timer.end(1);
        if (overlap && b > 0) RR_TRY_CUDA(ctx, cudaStreamWaitEvent(stream, ctx->shadowed[b - 1], 0));
        timer.begin(2);
        shade_kernel<true><<<g_shade, kBlock, 0, stream>>>(DevScene{}, B->d_table, outs, b,
                                                           b + 1 == max_bounces ? 1u : 0u, q.ray_a[cur],
                                                           q.ray_b[cur], q.ray_c[cur], q.hits, q.ray_a[nxt],
                                                           q.ray_b[nxt], q.ray_c[nxt], q.shadow_a, q.shadow_b,
                                                           q.shadow_c, nullptr, cb, cn, cb + 2);
        RR_CHECK_LAUNCH(ctx);
        timer.end(2);
        cudaStream_t sh_stream = stream;
        if (overlap) {
            RR_TRY_CUDA(ctx, cudaEventRecord(ctx->shaded[b], stream));
            RR_TRY_CUDA(ctx, cudaStreamWaitEvent(ctx->side, ctx->shaded[b], 0));
            sh_stream = ctx->side;
        }
        timer.begin(3);
        sh_k<<<g_sh, kBlock, 0, sh_stream>>>(B->d_table, outs, q.shadow_a, q.shadow_b, q.shadow_c, cb + 2, cb + 3,
                                             ctx->work64 + 2);
        RR_CHECK_LAUNCH(ctx);
        timer.end(3);
        if (overlap) RR_TRY_CUDA(ctx, cudaEventRecord(ctx->shadowed[b], ctx->side));
    }
    if (overlap && max_bounces > 0) RR_TRY_CUDA(ctx, cudaStreamWaitEvent(stream, ctx->shadowed[max_bounces - 1], 0));
    return timer.commit();
}

} // namespace

extern "C" rr_status rr_batch_destroy(rr_batch* B) {
    if (!B) return RR_ERR_INVALID_ARGUMENT;
    if (B->ctx) cudaSetDevice(B->ctx->device);
    rr_batch_free_guided(B);
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->cap_stream) cudaStreamDestroy(B->cap_stream);
    for (int k = 0; k < 2; ++k) {
        if (B->staged[k]) cudaEventDestroy(B->staged[k]);
        if (B->h_call[k]) cudaFreeHost(B->h_call[k]);
    }
    cudaFree(B->d_table);
    cudaFree(B->d_call);
    delete B;
    return RR_OK;
}

extern "C" rr_status rr_batch_create(rr_ctx* ctx, const rr_scene* const* scenes, uint32_t count, rr_batch** out) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!scenes || !out || count == 0) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_create: bad argument");
    *out = nullptr;
    for (uint32_t i = 0; i < count; ++i)
        if (!scenes[i] || scenes[i]->ctx != ctx)
            return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_create: scene %u is null or of another context", i);
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    rr_batch* B = new rr_batch;
    B->ctx = ctx;
    B->scenes.assign(scenes, scenes + count);
    auto fail = [&](rr_status s) { rr_batch_destroy(B); return s; };
    std::vector<rr::DevScene> table(count);
    for (uint32_t i = 0; i < count; ++i) table[i] = scenes[i]->dev;
    B->entries_bytes = (sizeof(rr::BatchEntry) * count + 15) & ~size_t(15);
    B->call_bytes = B->entries_bytes + sizeof(void*) * count;
    cudaError_t e;
    if ((e = cudaMalloc(&B->d_table, sizeof(rr::DevScene) * count)) != cudaSuccess ||
        (e = cudaMemcpy(B->d_table, table.data(), sizeof(rr::DevScene) * count, cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMalloc(&B->d_call, B->call_bytes)) != cudaSuccess ||
        (e = cudaStreamCreateWithFlags(&B->cap_stream, cudaStreamNonBlocking)) != cudaSuccess)
        return fail(rr_fail(ctx, e == cudaErrorMemoryAllocation ? RR_ERR_OUT_OF_MEMORY : RR_ERR_CUDA,
                            "rr_batch_create: %s", cudaGetErrorString(e)));
    for (int k = 0; k < 2; ++k) {
        if ((e = cudaMallocHost(&B->h_call[k], B->call_bytes)) != cudaSuccess ||
            (e = cudaEventCreateWithFlags(&B->staged[k], cudaEventDisableTiming)) != cudaSuccess)
            return fail(rr_fail(ctx, RR_ERR_CUDA, "rr_batch_create: %s", cudaGetErrorString(e)));
    }
    *out = B;
    return RR_OK;
}

rr_status rr_batch_stage_call(rr_ctx* ctx, rr_batch* B, const GpuCameraData* cams, const rr_pt_params* p,
                              float* const* radiance_out, cudaStream_t stream, uint32_t* tiles_out,
                              uint64_t* paths_out) {
    using namespace rr;
    const uint32_t count = uint32_t(B->scenes.size());
    // per-call table into this call's staging slot (the copy out of it two calls ago has completed)
    const int k = B->slot;
    RR_TRY_CUDA(ctx, cudaEventSynchronize(B->staged[k]));
    BatchEntry* E = reinterpret_cast<BatchEntry*>(B->h_call[k]);
    float4** O = reinterpret_cast<float4**>(B->h_call[k] + B->entries_bytes);
    uint64_t paths = 0;
    uint32_t tiles = 0;
    for (uint32_t i = 0; i < count; ++i) {
        const GpuCameraData& c = cams[i];
        if (c.screen_width == 0 || c.screen_height == 0 || !radiance_out[i])
            return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_execute: scene %u: empty image or null output", i);
        BatchEntry& e = E[i];
        std::memset(&e, 0, sizeof(e));
        e.L.cam = c;
        e.L.frame_seed = p->frame_seed;
        e.L.spp = p->spp;
        e.L.width = c.screen_width;
        e.L.height = c.screen_height;
        e.L.tiles_x = (c.screen_width + 7) / 8;
        e.L.tiles_per_image = e.L.tiles_x * ((c.screen_height + 3) / 4);
        e.tile_begin = tiles;
        const uint64_t t = uint64_t(e.L.tiles_per_image) * p->spp;
        if (uint64_t(tiles) + t >= (1ull << 26))
            return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_execute: too many tiles");
        tiles += uint32_t(t);
        paths += uint64_t(c.screen_width) * c.screen_height * p->spp;
        O[i] = reinterpret_cast<float4*>(radiance_out[i]);
    }
    if (paths >= (1ull << 31)) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_execute: too many paths");
    rr_status st = ensure_queues(ctx, size_t(paths));
    if (st != RR_OK) return st;
    RR_TRY_CUDA(ctx, cudaMemcpyAsync(B->d_call, B->h_call[k], B->call_bytes, cudaMemcpyHostToDevice, stream));
    RR_TRY_CUDA(ctx, cudaEventRecord(B->staged[k], stream));
    B->slot ^= 1;
    *tiles_out = tiles;
    *paths_out = paths;
    return RR_OK;
}

extern "C" rr_status rr_batch_execute(rr_ctx* ctx, rr_batch* B, const GpuCameraData* cams, const rr_pt_params* p,
                                      float* const* radiance_out, void* stream_v) {
    using namespace rr;
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!B || !cams || !p || !radiance_out) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_execute: null argument");
    if (B->ctx != ctx) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_execute: batch of another context");
    if (p->spp == 0 || p->max_bounces > uint32_t(kMaxBounces))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_execute: bad spp or max_bounces");
    const bool graph = (p->flags & RR_PT_FLAG_GRAPH) != 0;
    if (graph && (p->flags & (RR_PT_FLAG_COUNT_TRAVERSAL | RR_PT_FLAG_TIME_STAGES)))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_execute: counting and timing flags need non-graph runs");
    if (p->flags & RR_PT_FLAG_EMITTERS)
        return rr_fail(ctx, RR_ERR_UNSUPPORTED, "rr_batch_execute: RR_PT_FLAG_EMITTERS is a single-scene mode");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    uint32_t tiles = 0;
    uint64_t paths = 0;
    rr_status st = rr_batch_stage_call(ctx, B, cams, p, radiance_out, stream, &tiles, &paths);
    if (st != RR_OK) return st;
    if (B->mode == RR_BATCH_PER_SCENE && !(p->flags & (RR_PT_FLAG_COUNT_TRAVERSAL | RR_PT_FLAG_TIME_STAGES))) {
        // scene by scene (the staged table above checked the arguments and
        // sized the queues for the whole batch)
        rr_pt_params q = *p;
        q.flags = 0;
        for (size_t i = 0; i < B->scenes.size(); ++i)
            if ((st = rr_pathtracer_execute(ctx, B->scenes[i], &cams[i], &q, radiance_out[i], stream)) != RR_OK)
                return st;
        return RR_OK;
    }
    // the overlap's stream and events exist before any graph capture starts
    if (ctx->overlap_shadow && (st = ensure_side(ctx)) != RR_OK) return st;
    if (graph) {
        rr_batch::Key key;
        key.paths = paths; key.total_tiles = tiles; key.max_bounces = p->max_bounces;
        key.ev = uint32_t(ctx->extend_variant); key.sv = uint32_t(ctx->shadow_variant);
        key.queue = ctx->pt.ray_a[0];
        key.overlap = ctx->overlap_shadow;
        if (!B->exec || key != B->key) {
            if (B->exec) { cudaGraphExecDestroy(B->exec); B->exec = nullptr; }
            RR_TRY_CUDA(ctx, cudaStreamBeginCapture(B->cap_stream, cudaStreamCaptureModeThreadLocal));
            st = enqueue_batch(ctx, B, tiles, size_t(paths), p->max_bounces, 0u, B->cap_stream);
            cudaGraph_t g = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(B->cap_stream, &g);
            if (st != RR_OK) { if (g) cudaGraphDestroy(g); return st; }
            if (ce != cudaSuccess) return rr_fail(ctx, RR_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
            const cudaError_t ie = cudaGraphInstantiate(&B->exec, g, 0);
            cudaGraphDestroy(g);
            if (ie != cudaSuccess) return rr_fail(ctx, RR_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ie));
            B->key = key;
        }
        RR_TRY_CUDA(ctx, cudaGraphLaunch(B->exec, stream));
        st = RR_OK;
    } else {
        st = enqueue_batch(ctx, B, tiles, size_t(paths), p->max_bounces, p->flags, stream);
    }
    ctx->launches += 1 + 3 * uint64_t(p->max_bounces);
    ctx->last_max_bounces = p->max_bounces;
    ctx->last_counted = (p->flags & RR_PT_FLAG_COUNT_TRAVERSAL) != 0;
    return st;
}

extern "C" rr_status rr_batch_tune(rr_ctx* ctx, rr_batch* B, const GpuCameraData* cams, const rr_pt_params* p,
                                   float* const* radiance_out, void* stream, rr_pt_tune_result* out) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!B || !cams || !p || !radiance_out || !out)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_tune: null argument");
    rr_pt_stats st;
    rr_status s;
    if ((s = rr_pathtracer_stats(ctx, &st, 1)) != RR_OK) return s;
    double best_e = 1e300, best_s = 1e300;
    rr_pt_params warm = *p, q = *p;
    warm.flags = 0;
    q.flags = RR_PT_FLAG_TIME_STAGES;
    for (int v = 0; v < RR_PT_VARIANT_COUNT; ++v) {
        ctx->extend_variant = v;
        ctx->shadow_variant = v;
        if ((s = rr_batch_execute(ctx, B, cams, &warm, radiance_out, stream)) != RR_OK) return s;
        if ((s = rr_batch_execute(ctx, B, cams, &q, radiance_out, stream)) != RR_OK) return s;
        if ((s = rr_pathtracer_stats(ctx, &st, 1)) != RR_OK) return s;
        out->extend_ms[v] = st.ms_extend;
        out->shadow_ms[v] = st.ms_shadow;
        if (st.ms_extend < best_e) { best_e = st.ms_extend; out->best_extend = v; }
        if (st.ms_shadow < best_s) { best_s = st.ms_shadow; out->best_shadow = v; }
    }
    ctx->extend_variant = out->best_extend;
    ctx->shadow_variant = out->best_shadow;
    // the batch's form: each timed (after one warm-up call) with the caller's
    // graph flag, three calls each, compared by their medians (a shared GPU
    // makes single calls noisy)
    rr_pt_params m = *p;
    m.flags = p->flags & RR_PT_FLAG_GRAPH;
    cudaStream_t st0 = static_cast<cudaStream_t>(stream);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    RR_TRY_CUDA(ctx, cudaEventCreate(&e0));
    cudaError_t ce = cudaEventCreate(&e1);
    if (ce != cudaSuccess) {
        cudaEventDestroy(e0);
        RR_TRY_CUDA(ctx, ce);
    }
    constexpr int kRepeats = 3;
    float median_ms[2] = {0.0f, 0.0f};
    const int modes[2] = {RR_BATCH_WAVEFRONT, RR_BATCH_PER_SCENE};
    s = RR_OK;
    for (int k = 0; k < 2 && s == RR_OK && ce == cudaSuccess; ++k) {
        B->mode = modes[k];
        if ((s = rr_batch_execute(ctx, B, cams, &m, radiance_out, stream)) != RR_OK) break;
        float ms[kRepeats];
        for (int r = 0; r < kRepeats && s == RR_OK && ce == cudaSuccess; ++r) {
            if ((ce = cudaEventRecord(e0, st0)) != cudaSuccess) break;
            if ((s = rr_batch_execute(ctx, B, cams, &m, radiance_out, stream)) != RR_OK) break;
            if ((ce = cudaEventRecord(e1, st0)) != cudaSuccess) break;
            if ((ce = cudaEventSynchronize(e1)) != cudaSuccess) break;
            ce = cudaEventElapsedTime(&ms[r], e0, e1);
        }
        if (s != RR_OK || ce != cudaSuccess) break;
        std::sort(ms, ms + kRepeats);
        median_ms[k] = ms[kRepeats / 2];
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (s != RR_OK) return s;
    if (ce != cudaSuccess)
        return rr_fail(ctx, RR_ERR_CUDA, "rr_batch_tune: timing the batch forms failed: %s", cudaGetErrorString(ce));
    B->mode = median_ms[1] < median_ms[0] ? RR_BATCH_PER_SCENE : RR_BATCH_WAVEFRONT;
    return RR_OK;
}

extern "C" rr_status rr_batch_set_mode(rr_batch* B, int mode) {
    if (!B || (mode != RR_BATCH_WAVEFRONT && mode != RR_BATCH_PER_SCENE)) return RR_ERR_INVALID_ARGUMENT;
    B->mode = mode;
    return RR_OK;
}

extern "C" rr_status rr_batch_get_mode(const rr_batch* B, int* mode_out) {
    if (!B || !mode_out) return RR_ERR_INVALID_ARGUMENT;
    *mode_out = B->mode;
    return RR_OK;
}
