// restir_di.cu — ReSTIR DI (ReSTIRDIPass.cpp:306-446; kernels in
// passes/restir_di/restir_di.slang). Three per-pixel kernels, 16x8 pixel
// blocks; reservoirs are float4(as_float(sel), w_sum, W, as_float(M)) with
// sel = 0xffffffff meaning empty (restir_di.slang:57-72).

#include "rr_internal.h"

namespace rr {
namespace {

struct DiLaunch {
    GpuCameraData cam;
    uint32_t frame_seed;
    uint32_t num_initial_candidates;
    uint32_t spatial_on;
    uint32_t spatial_num_neighbors;
    uint32_t spatial_radius;
    uint32_t m_cap;
};

// restir_di.slang:152-178 — p_hat = max(n.l, 0) * Rec.709 luminance(irradiance)
RR_D float compute_p_hat(const DevScene& s, uint32_t li, float3 pos, float3 n) {
    if (li >= s.num_lights) return 0.0f;
    const float4 l0 = __ldg(s.lights + li * 3);
    const float4 l1 = __ldg(s.lights + li * 3 + 1);
    const float4 l2 = __ldg(s.lights + li * 3 + 2);
    float3 l, irr;
    if (__float_as_uint(l0.w) == 0u) {
        const float3 to = f3(l0.x, l0.y, l0.z) - pos;
        const float d2 = mx(dot(to, to), 1e-6f);
        l = normalize(to);
        irr = f3(l2.x * l2.w / d2, l2.y * l2.w / d2, l2.z * l2.w / d2);
    } else {
        l = normalize(-f3(l1.x, l1.y, l1.z));
        irr = f3(l2.x, l2.y, l2.z) * l2.w;
    }
    const float ndl = mx(dot(n, l), 0.0f);
    const float lum = 0.2126f * irr.x + 0.7152f * irr.y + 0.0722f * irr.z;
    return ndl * lum;
}

// ── Emitter candidates (RR_DI_FLAG_EMITTERS; no reference counterpart). A
// candidate is a 32-bit RNG state; the light sample it names is decoded
// from it (group, then a GpuLight or an emissive triangle by power and a
// point on it). inv_src = 1 / source density (probability for a GpuLight,
// area density for an emitter point).
RR_D float lum709(float3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

struct DiLightSample {
    bool emitter;
    uint32_t li;
    float3 y, Le, ny;
    float inv_src;
};

RR_D DiLightSample di_decode(const DevScene& s, uint32_t c) {
    uint32_t st = c;
    const uint32_t NL = s.num_lights, NE = s.num_emitters;
    const float pe = NE == 0 ? 0.0f : (NL == 0 ? 1.0f : 0.5f);
    DiLightSample r;
    r.li = 0;
    r.y = r.Le = r.ny = f3(0.0f, 0.0f, 0.0f);
    r.emitter = NE > 0 && (NL == 0 || rand_float(st) < 0.5f);
    if (r.emitter) {
        const float u = rand_float(st);
        const float uc = rand_float(st);
        const float u1 = rand_float(st);
        const float u2 = rand_float(st);
        const uint32_t k = emitter_pick(s, u, uc);
        const float4 e0 = __ldg(s.emitters + k * 3), e1 = __ldg(s.emitters + k * 3 + 1);
        const float4 e2 = __ldg(s.emitters + k * 3 + 2);
        const float3 E1 = xyz(e1), E2 = xyz(e2);
        const float su = sqrtf(u1);
        r.y = xyz(e0) + E1 * (su * (1.0f - u2)) + E2 * (su * u2);
        r.Le = f3(e0.w, e1.w, e2.w);
        r.ny = normalize(cross(E1, E2));
        r.inv_src = s.emit_total / (pe * lum709(r.Le));
    } else {
        r.li = uint32_t(rand_float(st) * float(NL)) % NL;
        r.inv_src = float(NL) / (1.0f - pe);
    }
    return r;
}

RR_D float di_p_hat_emit(const DevScene& s, const DiLightSample& d, float3 pos, float3 n) {
    if (!d.emitter) return compute_p_hat(s, d.li, pos, n);
    const float3 to = d.y - pos;
    const float d2 = mx(dot(to, to), 1e-6f);
    const float3 l = normalize(to);
    const float cos_y = fabsf(dot(d.ny, l));
    const float3 irr = d.Le * (cos_y / d2);
    return mx(dot(n, l), 0.0f) * lum709(irr);
}

// p_hat of selection sel: a GpuLight index, or (Emit) a candidate state.
template <bool Emit>
RR_D float di_p_hat(const DevScene& s, uint32_t sel, float3 pos, float3 n) {
    if constexpr (Emit) return di_p_hat_emit(s, di_decode(s, sel), pos, n);
    else return compute_p_hat(s, sel, pos, n);
}

RR_D bool pixel_of(const GpuCameraData& cam, uint32_t& x, uint32_t& y) {
    x = blockIdx.x * 16 + (threadIdx.x & 15);
    y = blockIdx.y * 8 + (threadIdx.x >> 4);
    return x < cam.screen_width && y < cam.screen_height;
}

// cs_initial (restir_di.slang:186-262). The initial and spatial kernels run
// 10 blocks of 128 threads per SM (48 registers, a few spilled): 251.9
// against 250.8 Mpaths/s for the bench frame with 8 blocks (64 registers),
// 250.6 with 6.
template <bool Emit>
__global__ void __launch_bounds__(128, 10) di_initial_kernel(DevScene s, DiLaunch L, float4* __restrict__ gpos,
                                                         float4* __restrict__ gnrm, float4* __restrict__ res) {
    uint32_t x, y;
    if (!pixel_of(L.cam, x, y)) return;
    const size_t i = size_t(y) * L.cam.screen_width + x;
    uint32_t seed = make_seed(x, y, L.frame_seed);
    const float jx = rand_float(seed);
    const float jy = rand_float(seed);
    const float3 d = primary_dir(L.cam, float(x) + jx, float(y) + jy);
    const float3 o = f3(L.cam.position[0], L.cam.position[1], L.cam.position[2]);
    HitRec h;
    if (!trace<false>(s, make_ray(o, d), 0.001f, 1e9f, h)) {
        gpos[i] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
        gnrm[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        res[i] = make_float4(__uint_as_float(kNoIndex), 0.0f, 0.0f, __uint_as_float(0u));
        return;
    }
    const Surface sf = hit_surface(s, h.inst, h.prim, h.u, h.v);
    float3 n = sf.normal;
    if (dot(n, -d) < 0.0f) n = -n;
    gpos[i] = make_float4(sf.pos.x, sf.pos.y, sf.pos.z, h.t);
    gnrm[i] = make_float4(n.x, n.y, n.z, __uint_as_float(sf.material));
    const uint32_t N = s.num_lights;
    if (Emit ? N + s.num_emitters == 0 : N == 0) {
        res[i] = make_float4(__uint_as_float(kNoIndex), 0.0f, 0.0f, __uint_as_float(0u));
        return;
    }
    uint32_t sel = kNoIndex;
    float w_sum = 0.0f;
    uint32_t M_count = 0;
    for (uint32_t c = 0; c < L.num_initial_candidates; ++c) {
        uint32_t cand;
        float w_i;
        if constexpr (Emit) {
            (void)rand_float(seed);
            cand = seed == kNoIndex ? kNoIndex - 1u : seed;   // never the empty marker
            const DiLightSample ds = di_decode(s, cand);
            w_i = di_p_hat_emit(s, ds, sf.pos, n) * ds.inv_src;
        } else {
            cand = uint32_t(rand_float(seed) * float(N)) % N;
            const float ph = compute_p_hat(s, cand, sf.pos, n);
            w_i = ph * float(N);
        }
        w_sum += w_i;
        M_count++;
        if (w_sum > 0.0f && rand_float(seed) < w_i / w_sum) sel = cand;
    }
    float W_final = 0.0f;
    if (sel != kNoIndex) {
        const float ph_y = di_p_hat<Emit>(s, sel, sf.pos, n);
        W_final = (ph_y > 1e-10f) ? (w_sum / (float(M_count) * ph_y)) : 0.0f;
    }
    res[i] = make_float4(__uint_as_float(sel), w_sum, W_final, __uint_as_float(M_count));
}

// cs_temporal (restir_di.slang:266-335): same-pixel history, M-cap.
template <bool Emit>
__global__ void __launch_bounds__(128) di_temporal_kernel(DevScene s, DiLaunch L, const float4* __restrict__ gpos,
                                                          const float4* __restrict__ gnrm, float4* __restrict__ res,
                                                          const float4* __restrict__ prev) {
    uint32_t x, y;
    if (!pixel_of(L.cam, x, y)) return;
    const size_t i = size_t(y) * L.cam.screen_width + x;
    const float4 gp = gpos[i];
    if (gp.w < 0.0f) return;
    const float3 pos = xyz(gp), n = xyz(gnrm[i]);
    const float4 cr = res[i], pr = prev[i];
    uint32_t curr_sel = __float_as_uint(cr.x);
    float curr_wsum = cr.y;
    uint32_t curr_M = __float_as_uint(cr.w);
    const uint32_t prev_sel = __float_as_uint(pr.x);
    const float prev_W = pr.z;
    uint32_t prev_M = __float_as_uint(pr.w);
    if (prev_sel == kNoIndex || prev_M == 0) return;
    prev_M = min(prev_M, L.m_cap);
    const float ph_prev = di_p_hat<Emit>(s, prev_sel, pos, n);
    const float contrib = ph_prev * prev_W * float(prev_M);
    curr_wsum += contrib;
    const uint32_t new_M = curr_M + prev_M;
    if (new_M > L.m_cap) {
        const float scale = float(L.m_cap) / float(new_M);
        curr_wsum *= scale;
        curr_M = L.m_cap;
    } else {
        curr_M = new_M;
    }
    uint32_t seed = make_seed(x, y, L.frame_seed + 1u);
    if (contrib > 0.0f && rand_float(seed) < contrib / curr_wsum) curr_sel = prev_sel;
    float W_new = 0.0f;
    if (curr_sel != kNoIndex) {
        const float ph_y = di_p_hat<Emit>(s, curr_sel, pos, n);
        W_new = (ph_y > 1e-10f) ? (curr_wsum / (float(curr_M) * ph_y)) : 0.0f;
        W_new = mn(W_new, 1e4f);
    }
    res[i] = make_float4(__uint_as_float(curr_sel), curr_wsum, W_new, __uint_as_float(curr_M));
}

// cs_spatial_shade (restir_di.slang:339-472)
template <bool Emit>
__global__ void __launch_bounds__(128, 10) di_spatial_shade_kernel(DevScene s, DiLaunch L, const float4* __restrict__ gpos,
                                                               const float4* __restrict__ gnrm,
                                                               const float4* __restrict__ res,
                                                               float4* __restrict__ out) {
    uint32_t x, y;
    if (!pixel_of(L.cam, x, y)) return;
    const uint32_t W = L.cam.screen_width, H = L.cam.screen_height;
    const size_t i = size_t(y) * W + x;
    const float4 gp = gpos[i];
    if (gp.w < 0.0f) {
        const float3 dir = primary_dir(L.cam, float(x) + 0.5f, float(y) + 0.5f);
        const float3 c = sky_radiance(dir);
        out[i] = make_float4(c.x, c.y, c.z, 1.0f);
        return;
    }
    const float3 pos = xyz(gp);
    const float4 gn = gnrm[i];
    const float3 n = xyz(gn);
    const uint32_t mat = __float_as_uint(gn.w);
    const float4 m0 = __ldg(s.materials + mat * 2), m1 = __ldg(s.materials + mat * 2 + 1);
    if (m1.x > 0.0f || m1.y > 0.0f || m1.z > 0.0f) {
        out[i] = make_float4(m1.x, m1.y, m1.z, 1.0f);
        return;
    }
    const float4 r = res[i];
    uint32_t r_sel = __float_as_uint(r.x);
    float r_wsum = r.y, r_W = r.z;
    uint32_t r_M = __float_as_uint(r.w);
    const uint32_t N = s.num_lights;
    const uint32_t NA = Emit ? N + s.num_emitters : N;   // lights a reservoir can name
    if (L.spatial_on && L.spatial_num_neighbors > 0 && NA > 0) {
        uint32_t seed = make_seed(x, y, L.frame_seed + 2u);
        for (uint32_t k = 0; k < L.spatial_num_neighbors; ++k) {
            const float angle = rand_float(seed) * 6.28318530717958f;
            const float radius = rand_float(seed) * float(L.spatial_radius);
            const int ox = int(radius * rr_cosf(angle)), oy = int(radius * rr_sinf(angle));
            const int nx = min(max(int(x) + ox, 0), int(W) - 1);
            const int ny = min(max(int(y) + oy, 0), int(H) - 1);
            const size_t j = size_t(ny) * W + nx;
            if (gpos[j].w < 0.0f) continue;
            const float4 nr = res[j];
            const uint32_t nb_sel = __float_as_uint(nr.x);
            const uint32_t nb_M = __float_as_uint(nr.w);
            if (nb_sel == kNoIndex || nb_M == 0) continue;
            const float ph_nb = di_p_hat<Emit>(s, nb_sel, pos, n);
            const float contrib = ph_nb * nr.z * float(nb_M);
            r_wsum += contrib;
            r_M += nb_M;
            if (contrib > 0.0f && rand_float(seed) < contrib / r_wsum) r_sel = nb_sel;
        }
        if (r_sel != kNoIndex) {
            const float ph_y = di_p_hat<Emit>(s, r_sel, pos, n);
            r_W = (ph_y > 1e-10f) ? (r_wsum / (float(r_M) * ph_y)) : 0.0f;
        }
    }
    float3 o = f3(0.0f, 0.0f, 0.0f);
    uint32_t li = r_sel;
    bool gpu_light;
    if constexpr (Emit) {
        gpu_light = false;
        if (r_sel != kNoIndex && NA > 0 && r_W > 0.0f) {
            const DiLightSample ds = di_decode(s, r_sel);
            if (ds.emitter) {
                // a point on an emissive triangle: irradiance Le |cos_y| / d^2
                const float3 to = ds.y - pos;
                const float dist = length(to);
                const float3 l = to / mx(dist, 1e-6f);
                const float dd = mx(dist * dist, 1e-6f);
                const float cos_y = fabsf(dot(ds.ny, l));
                const float3 irr = ds.Le * (cos_y / dd);
                const float ndl = mx(dot(n, l), 0.0f);
                if (ndl > 0.0f) {
                    HitRec h;
                    if (!trace<true>(s, make_ray(pos + n * 1e-4f, l), 0.001f, dist - 0.01f, h)) {
                        const float3 wo = normalize(f3(L.cam.position[0], L.cam.position[1], L.cam.position[2]) - pos);
                        const float3 bv = brdf_eval(n, wo, l, f3(m0.x, m0.y, m0.z), m0.w, m1.w);
                        o = ((bv * irr) * ndl) * r_W;
                    }
                }
            } else {
                li = ds.li;
                gpu_light = N > 0;
            }
        }
    } else {
        // r_sel < N guards the light fetch for reservoirs that were never
        // written by this scene; valid reservoirs always satisfy it.
        gpu_light = r_sel != kNoIndex && r_sel < N && r_W > 0.0f && N > 0;
    }
    if (gpu_light) {
        const float4 l0 = __ldg(s.lights + li * 3);
        const float4 l1 = __ldg(s.lights + li * 3 + 1);
        const float4 l2 = __ldg(s.lights + li * 3 + 2);
        float3 l, irr; float dist;
        if (__float_as_uint(l0.w) == 0u) {
            const float3 to = f3(l0.x, l0.y, l0.z) - pos;
            dist = length(to);
            l = to / mx(dist, 1e-6f);
            const float dd = mx(dist * dist, 1e-6f);
            irr = f3(l2.x * l2.w / dd, l2.y * l2.w / dd, l2.z * l2.w / dd);
        } else {
            l = normalize(-f3(l1.x, l1.y, l1.z));
            dist = 1e9f;
            irr = f3(l2.x, l2.y, l2.z) * l2.w;
        }
        const float ndl = mx(dot(n, l), 0.0f);
        if (ndl > 0.0f) {
            HitRec h;
            if (!trace<true>(s, make_ray(pos + n * 1e-4f, l), 0.001f, dist - 0.01f, h)) {
                const float3 wo = normalize(f3(L.cam.position[0], L.cam.position[1], L.cam.position[2]) - pos);
                const float3 bv = brdf_eval(n, wo, l, f3(m0.x, m0.y, m0.z), m0.w, m1.w);
                o = ((bv * irr) * ndl) * r_W;
            }
        }
    }
    out[i] = make_float4(o.x, o.y, o.z, 1.0f);
}

DiLaunch make_launch(const GpuCameraData* cam, const rr_di_params* p) {
    DiLaunch L;
    L.cam = *cam;
    L.frame_seed = p->frame_seed;
    L.num_initial_candidates = p->num_initial_candidates;
    L.spatial_on = p->spatial_enable;
    L.spatial_num_neighbors = p->spatial_num_neighbors;
    L.spatial_radius = p->spatial_radius;
    // clamp(20u * M, 1u, 8192u) in 32-bit unsigned arithmetic (restir_di.slang:300)
    const uint32_t cap = p->m_cap_factor * p->num_initial_candidates;
    L.m_cap = std::min(std::max(cap, 1u), 8192u);
    return L;
}

dim3 grid_of(const GpuCameraData* cam) { return dim3((cam->screen_width + 15) / 16, (cam->screen_height + 7) / 8); }

rr_status check(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam, const rr_di_params* p) {
    if (!scene || !cam || !p) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR DI: null argument");
    if (p->flags & ~RR_DI_FLAG_EMITTERS) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR DI: unknown flags");
    if (cam->screen_width == 0 || cam->screen_height == 0 || cam->screen_width > 65535u * 16u ||
        cam->screen_height > 65535u * 8u)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR DI: bad image size");
    return RR_OK;
}

} // namespace
} // namespace rr

using namespace rr;

extern "C" rr_status rr_restir_di_initial(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                          const rr_di_params* p, float* gpos, float* gnrm, float* res,
                                          void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    rr_status st = check(ctx, scene, cam, p);
    if (st != RR_OK) return st;
    if (!gpos || !gnrm || !res) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "null buffer");
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    const auto di_initial_kernel_f = (p->flags & RR_DI_FLAG_EMITTERS) ? di_initial_kernel<true> : di_initial_kernel<false>;
    di_initial_kernel_f<<<grid_of(cam), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        scene->dev, make_launch(cam, p), reinterpret_cast<float4*>(gpos), reinterpret_cast<float4*>(gnrm),
        reinterpret_cast<float4*>(res));
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

extern "C" rr_status rr_restir_di_temporal(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                           const rr_di_params* p, const float* gpos, const float* gnrm,
                                           float* res, const float* prev, void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    rr_status st = check(ctx, scene, cam, p);
    if (st != RR_OK) return st;
    if (!gpos || !gnrm || !res || !prev) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "null buffer");
    if (!p->temporal_enable) return RR_OK;  // restir_di.slang:270
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    const auto di_temporal_kernel_f = (p->flags & RR_DI_FLAG_EMITTERS) ? di_temporal_kernel<true> : di_temporal_kernel<false>;
    di_temporal_kernel_f<<<grid_of(cam), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        scene->dev, make_launch(cam, p), reinterpret_cast<const float4*>(gpos),
        reinterpret_cast<const float4*>(gnrm), reinterpret_cast<float4*>(res),
        reinterpret_cast<const float4*>(prev));
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

extern "C" rr_status rr_restir_di_spatial_shade(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                                const rr_di_params* p, const float* gpos, const float* gnrm,
                                                const float* res, float* out, void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    rr_status st = check(ctx, scene, cam, p);
    if (st != RR_OK) return st;
    if (!gpos || !gnrm || !res || !out) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "null buffer");
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    const auto di_spatial_shade_kernel_f = (p->flags & RR_DI_FLAG_EMITTERS) ? di_spatial_shade_kernel<true> : di_spatial_shade_kernel<false>;
    di_spatial_shade_kernel_f<<<grid_of(cam), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        scene->dev, make_launch(cam, p), reinterpret_cast<const float4*>(gpos),
        reinterpret_cast<const float4*>(gnrm), reinterpret_cast<const float4*>(res),
        reinterpret_cast<float4*>(out));
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

extern "C" rr_status rr_restir_di_execute(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                          const rr_di_params* p, float* gpos, float* gnrm, float* res,
                                          const float* prev, float* out, void* stream) {
    rr_status st = rr_restir_di_initial(ctx, scene, cam, p, gpos, gnrm, res, stream);
    if (st != RR_OK) return st;
    st = rr_restir_di_temporal(ctx, scene, cam, p, gpos, gnrm, res, prev, stream);
    if (st != RR_OK) return st;
    return rr_restir_di_spatial_shade(ctx, scene, cam, p, gpos, gnrm, res, out, stream);
}
