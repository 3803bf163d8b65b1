// restir_gi.cu — ReSTIR GI (ReSTIRGIPass.cpp:428-650; kernels in
// passes/restir_gi/restir_gi.slang). Three per-pixel kernels on 16x8 pixel
// blocks, each ray traced inline on the scene BVH:
//   initial      : cs_initial (:568-686) — M cosine-hemisphere candidates from
//                  the primary surface, each a secondary hit whose outgoing
//                  radiance is its emission plus one light sample, resampled
//                  by weighted reservoir sampling (source pdf cos / pi)
//   temporal     : cs_temporal (:688-848) — reprojected history pixel (3x3
//                  search), reconnection Jacobian, visibility, M-cap, W <= 50
//   spatial_shade: cs_spatial_shade (:851-1000) — golden-ratio neighbour
//                  pattern, reconnection, final shading
// The reservoir is three RGBA32F images (restir_gi.slang:3-7):
//   (sample_pos, w_sum), (sample_radiance, W), (sample_normal, asfloat(M)).

#include "rr_reuse.cuh"

namespace rr {
namespace {

struct GiLaunch {
    GpuCameraData cam;
    uint32_t frame_seed, num_candidates, spatial, num_neighbors, radius, include_direct;
    float indirect_strength, ray_bias;
    uint32_t m_cap;
};

struct GiImages {
    const float4* gpos;
    const float4* gnrm;
    const float4* direct;   // may be null
    float4* rc[3];          // current reservoir
    const float4* rp[3];    // previous reservoir
    float4* hc[2];          // current primary history (pos, normal)
    const float4* hp[2];    // previous primary history
    float4* out;
};

struct GiRes {
    float3 pos, rad, nrm;
    float w_sum, W;
    uint32_t M;
};

// unpack_reservoir / pack_reservoir (restir_gi.slang:199-238)
RR_D GiRes load_gi(const float4* const* img, size_t i) {
    const float4 p = img[0][i], r = img[1][i], m = img[2][i];
    GiRes res;
    res.pos = xyz(p); res.w_sum = p.w;
    res.rad = xyz(r); res.W = r.w;
    res.nrm = xyz(m); res.M = __float_as_uint(m.w);
    return res;
}
RR_D void store_gi(float4* const* img, size_t i, const GiRes& r) {
    img[0][i] = make_float4(r.pos.x, r.pos.y, r.pos.z, r.w_sum);
    img[1][i] = make_float4(r.rad.x, r.rad.y, r.rad.z, r.W);
    img[2][i] = make_float4(r.nrm.x, r.nrm.y, r.nrm.z, __uint_as_float(r.M));
}
// write_empty_reservoir (restir_gi.slang:192-197)
RR_D void store_gi_empty(float4* const* img, size_t i) {
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    img[0][i] = z;
    img[1][i] = z;
    img[2][i] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(0u));
}

// evaluate_indirect_radiance (restir_gi.slang:487-508): brdf * radiance * cos
RR_D float3 gi_indirect(float3 pp, float3 pn, const Mat& pm, float3 cp, float3 spos, float3 srad) {
    const float3 to = spos - pp;
    const float d2 = dot(to, to);
    if (d2 <= 1e-8f) return f3(0.0f, 0.0f, 0.0f);
    const float3 wi = to * rsqrt_(d2);
    const float cos_x = mx(dot(pn, wi), 0.0f);
    if (cos_x <= 0.0f) return f3(0.0f, 0.0f, 0.0f);
    const float3 wo = normalize(cp - pp);
    const float3 bv = brdf_eval(pn, wo, wi, pm.base, pm.metallic, pm.roughness);
    return (bv * srad) * cos_x;
}
// compute_target_function (restir_gi.slang:524-537)
RR_D float gi_target(float3 pp, float3 pn, const Mat& pm, float3 cp, float3 spos, float3 srad) {
    return luminance(gi_indirect(pp, pn, pm, cp, spos, srad));
}
// sample_primary_pdf (restir_gi.slang:510-522): the cosine lobe's density
RR_D float gi_source_pdf(float3 pp, float3 pn, float3 spos) {
    const float3 d = spos - pp;
    const float d2 = dot(d, d);
    if (d2 <= 1e-8f) return 0.0f;
    const float3 wi = d * rsqrt_(d2);
    const float cos_x = mx(dot(pn, wi), 0.0f);
    return mx(cos_x * kInvPi, 0.0f);
}

// cs_initial (restir_gi.slang:568-686)
__global__ void __launch_bounds__(128, 8) gi_initial_kernel(DevScene s, GiLaunch L, GiImages I) {
    uint32_t x, y;
    if (!pixel_of(L.cam, x, y)) return;
    const size_t i = size_t(y) * L.cam.screen_width + x;
    uint32_t seed = make_seed(x, y, L.frame_seed);
    float4 p4, n4;
    float3 pp, pn;
    uint32_t pmat;
    if (!load_surface(s, I.gpos, I.gnrm, i, p4, n4, pp, pn, pmat)) {
        I.hc[0][i] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
        I.hc[1][i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        store_gi_empty(I.rc, i);
        return;
    }
    I.hc[0][i] = p4;
    I.hc[1][i] = n4;
    const Mat pm = load_mat(s, pmat);
    const float3 cp = cam_pos(L.cam);
    const float bias = L.ray_bias;
    GiRes sel;
    sel.pos = sel.rad = sel.nrm = f3(0.0f, 0.0f, 0.0f);
    float w_sum = 0.0f;
    uint32_t M_count = 0;
    float3 T, B;
    build_onb(pn, T, B);
    for (uint32_t c = 0; c < L.num_candidates; ++c) {
        const float u0 = rand_float(seed);
        const float u1 = rand_float(seed);
        float pdf_dir;
        const float3 d = tangent_to_world(sample_cosine_hemisphere(u0, u1, pdf_dir), T, B, pn);
        if (dot(pn, d) <= 0.0f) continue;
        HitRec h;
        if (!trace<false>(s, make_ray(pp + pn * bias, d), bias, 1e9f, h)) continue;
        const Surface sec = hit_surface(s, h.inst, h.prim, h.u, h.v);
        // evaluate_sample_radiance (:539-552): normal turned toward wo = -d
        const float3 wo = -d;
        float3 sn = sec.normal;
        if (dot(sn, wo) < 0.0f) sn = -sn;
        const Mat sm = load_mat(s, sec.material);
        const float3 rad = sm.emissive + sample_lights(s, sec.pos, sn, wo, sm, bias, seed);
        const float tgt = gi_target(pp, pn, pm, cp, sec.pos, rad);
        if (tgt <= 0.0f) continue;
        const float pdf = gi_source_pdf(pp, pn, sec.pos);
        if (pdf <= 1e-6f) continue;
        const float weight = tgt / pdf;
        w_sum += weight;
        M_count++;
        if (w_sum > 0.0f && rand_float(seed) < weight / w_sum) {
            sel.pos = sec.pos; sel.rad = rad; sel.nrm = sec.normal;
        }
    }
    if (M_count > 0) {
        const float ph_y = gi_target(pp, pn, pm, cp, sel.pos, sel.rad);
        if (ph_y > 1e-10f) {
            sel.w_sum = w_sum;
            sel.W = w_sum / (float(M_count) * ph_y);
            sel.M = M_count;
            store_gi(I.rc, i, sel);
            return;
        }
    }
    store_gi_empty(I.rc, i);
}

// cs_temporal (restir_gi.slang:688-848)
__global__ void __launch_bounds__(128, 8) gi_temporal_kernel(DevScene s, GiLaunch L, GiImages I) {
    uint32_t x, y;
    if (!pixel_of(L.cam, x, y)) return;
    const size_t i = size_t(y) * L.cam.screen_width + x;
    float4 p4, n4;
    float3 pp, pn;
    uint32_t pmat;
    if (!load_surface(s, I.gpos, I.gnrm, i, p4, n4, pp, pn, pmat)) return;
    const Mat pm = load_mat(s, pmat);
    const float3 cp = cam_pos(L.cam);
    size_t hist;
    float3 hpos;
    if (!find_history(L.cam, I.hp[0], I.hp[1], pp, pn, pmat, cp, hist, hpos)) return;
    GiRes cur = load_gi(I.rc, i);
    GiRes prv = load_gi(I.rp, hist);
    if (prv.M == 0) return;
    prv.M = min(prv.M, L.m_cap);
    const float jac = reconnection_jacobian(hpos, pp, prv.pos, prv.nrm);
    if (jac <= 0.0f) return;
    if (!visible(s, pp, pn, prv.pos, L.ray_bias)) return;
    const float ph_prev = gi_target(pp, pn, pm, cp, prv.pos, prv.rad);
    const float contrib = ((ph_prev * mn(prv.W, 50.0f)) * float(prv.M)) * jac;
    if (contrib <= 0.0f) return;
    cur.w_sum += contrib;
    uint32_t seed = make_seed(x, y, L.frame_seed + 1u);
    if (cur.w_sum > 0.0f && rand_float(seed) < contrib / cur.w_sum) {
        cur.pos = prv.pos; cur.rad = prv.rad; cur.nrm = prv.nrm;
    }
    // M-cap after the selection (:807-818)
    const uint32_t new_M = cur.M + prv.M;
    if (new_M > L.m_cap) {
        cur.w_sum *= float(L.m_cap) / float(new_M);
        cur.M = L.m_cap;
    } else {
        cur.M = new_M;
    }
    float W_new = 0.0f;
    if (cur.M > 0) {
        const float ph_y = gi_target(pp, pn, pm, cp, cur.pos, cur.rad);
        W_new = (ph_y > 1e-10f) ? (cur.w_sum / (float(cur.M) * ph_y)) : 0.0f;
        W_new = mn(W_new, 50.0f);
    }
    cur.W = W_new;
    store_gi(I.rc, i, cur);
}

// cs_spatial_shade (restir_gi.slang:851-1000)
__global__ void __launch_bounds__(128, 8) gi_spatial_shade_kernel(DevScene s, GiLaunch L, GiImages I) {
    uint32_t x, y;
    if (!pixel_of(L.cam, x, y)) return;
    const uint32_t W = L.cam.screen_width, H = L.cam.screen_height;
    const size_t i = size_t(y) * W + x;
    float3 radiance = f3(0.0f, 0.0f, 0.0f);
    if (L.include_direct != 0u && I.direct) radiance = radiance + xyz(I.direct[i]);
    float4 p4, n4;
    float3 pp, pn;
    uint32_t pmat;
    if (!load_surface(s, I.gpos, I.gnrm, i, p4, n4, pp, pn, pmat)) {
        if (L.include_direct == 0u) radiance = radiance + sky_radiance(primary_dir(L.cam, float(x) + 0.5f, float(y) + 0.5f));
        I.out[i] = make_float4(radiance.x, radiance.y, radiance.z, 1.0f);
        return;
    }
    const Mat pm = load_mat(s, pmat);
    if (pm.emissive.x > 0.0f || pm.emissive.y > 0.0f || pm.emissive.z > 0.0f) {
        radiance = radiance + pm.emissive;
        I.out[i] = make_float4(radiance.x, radiance.y, radiance.z, 1.0f);
        return;
    }
    const float3 cp = cam_pos(L.cam);
    GiRes res = load_gi(I.rc, i);
    if (L.spatial != 0u && L.num_neighbors > 0u) {
        const float base_phase = spatial_phase(x, y);
        for (uint32_t k = 0; k < L.num_neighbors; ++k) {
            size_t j;
            if (!spatial_neighbor(base_phase, k, L.num_neighbors, L.radius, x, y, W, H, j)) continue;
            float3 nbp;
            if (!spatial_compatible(I.gpos, I.gnrm, j, pp, pn, cp, nbp)) continue;
            const GiRes nbr = load_gi(I.rc, j);
            if (nbr.M == 0) continue;
            const float jac = reconnection_jacobian(nbp, pp, nbr.pos, nbr.nrm);
            if (jac <= 0.0f) continue;
            const float contrib = ((gi_target(pp, pn, pm, cp, nbr.pos, nbr.rad) * nbr.W) * float(nbr.M)) * jac;
            if (contrib <= 0.0f) continue;
            res.w_sum += contrib;
            res.M += nbr.M;
            const float accept = frac_(base_phase + 0.754877666f * float(k + 1u));
            if (res.w_sum > 0.0f && accept < contrib / res.w_sum) {
                res.pos = nbr.pos; res.rad = nbr.rad; res.nrm = nbr.nrm;
            }
        }
        if (res.M > 0) {
            const float ph_y = gi_target(pp, pn, pm, cp, res.pos, res.rad);
            res.W = (ph_y > 1e-10f) ? (res.w_sum / (float(res.M) * ph_y)) : 0.0f;
        }
    }
    if (res.M > 0 && res.W > 0.0f) {
        const float3 ind = gi_indirect(pp, pn, pm, cp, res.pos, res.rad) * res.W;
        if (luminance(ind) > 0.0f && visible(s, pp, pn, res.pos, L.ray_bias))
            radiance = radiance + ind * L.indirect_strength;
    }
    I.out[i] = make_float4(radiance.x, radiance.y, radiance.z, 1.0f);
}

// History reset (ReSTIRGIPass.cpp:484-530): prev reservoir to zero, prev
// history position to (0, 0, 0, -1), prev history normal to zero.
__global__ void gi_reset_kernel(float4* r0, float4* r1, float4* r2, float4* h0, float4* h1, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    r0[i] = z; r1[i] = z; r2[i] = z;
    h0[i] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
    h1[i] = z;
}

GiLaunch make_launch(const GpuCameraData* cam, const rr_restir_gi_params* p) {
    GiLaunch L;
    L.cam = *cam;
    L.frame_seed = p->frame_seed;
    L.num_candidates = p->num_initial_candidates;
    L.spatial = p->spatial_enable;
    L.num_neighbors = p->spatial_num_neighbors;
    L.radius = p->spatial_radius;
    L.include_direct = p->include_direct_lighting;
    L.indirect_strength = p->indirect_strength;
    L.ray_bias = p->ray_bias;
    // clamp(20u * M, 1u, 8192u) in 32-bit unsigned arithmetic (restir_gi.slang:764)
    L.m_cap = std::min(std::max(20u * p->num_initial_candidates, 1u), 8192u);
    return L;
}

GiImages make_images(const rr_restir_gi_images* b) {
    GiImages I;
    I.gpos = reinterpret_cast<const float4*>(b->gbuf_pos);
    I.gnrm = reinterpret_cast<const float4*>(b->gbuf_norm);
    I.direct = reinterpret_cast<const float4*>(b->direct);
    for (int k = 0; k < 3; ++k) {
        I.rc[k] = reinterpret_cast<float4*>(b->reservoir_curr[k]);
        I.rp[k] = reinterpret_cast<const float4*>(b->reservoir_prev[k]);
    }
    for (int k = 0; k < 2; ++k) {
        I.hc[k] = reinterpret_cast<float4*>(b->history_curr[k]);
        I.hp[k] = reinterpret_cast<const float4*>(b->history_prev[k]);
    }
    I.out = reinterpret_cast<float4*>(b->output);
    return I;
}

dim3 grid_of(const GpuCameraData* cam) { return dim3((cam->screen_width + 15) / 16, (cam->screen_height + 7) / 8); }

enum Stage { kInitial, kTemporal, kSpatial };

rr_status check(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam, const rr_restir_gi_params* p,
                const rr_restir_gi_images* b, Stage st) {
    if (!scene || !cam || !p || !b) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR GI: null argument");
    if (cam->screen_width == 0 || cam->screen_height == 0 || cam->screen_width > 65535u * 16u ||
        cam->screen_height > 65535u * 8u)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR GI: bad image size");
    if (!b->gbuf_pos || !b->gbuf_norm) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR GI: null G-buffer");
    for (int k = 0; k < 3; ++k)
        if (!b->reservoir_curr[k] || (st == kTemporal && !b->reservoir_prev[k]))
            return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR GI: null reservoir image");
    if (st == kInitial && (!b->history_curr[0] || !b->history_curr[1]))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR GI: null history image");
    if (st == kTemporal && (!b->history_prev[0] || !b->history_prev[1]))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR GI: null history image");
    if (st == kSpatial && !b->output) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR GI: null output");
    return RR_OK;
}

} // namespace
} // namespace rr

using namespace rr;

extern "C" rr_status rr_restir_gi_initial(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                          const rr_restir_gi_params* p, const rr_restir_gi_images* b,
                                          void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    rr_status st = check(ctx, scene, cam, p, b, kInitial);
    if (st != RR_OK) return st;
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    gi_initial_kernel<<<grid_of(cam), 128, 0, static_cast<cudaStream_t>(stream)>>>(scene->dev, make_launch(cam, p),
                                                                                  make_images(b));
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

extern "C" rr_status rr_restir_gi_temporal(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                           const rr_restir_gi_params* p, const rr_restir_gi_images* b,
                                           void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    rr_status st = check(ctx, scene, cam, p, b, kTemporal);
    if (st != RR_OK) return st;
    if (!p->temporal_enable) return RR_OK;  // restir_gi.slang:690
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    gi_temporal_kernel<<<grid_of(cam), 128, 0, static_cast<cudaStream_t>(stream)>>>(scene->dev, make_launch(cam, p),
                                                                                   make_images(b));
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

extern "C" rr_status rr_restir_gi_spatial_shade(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                                const rr_restir_gi_params* p, const rr_restir_gi_images* b,
                                                void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    rr_status st = check(ctx, scene, cam, p, b, kSpatial);
    if (st != RR_OK) return st;
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    gi_spatial_shade_kernel<<<grid_of(cam), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        scene->dev, make_launch(cam, p), make_images(b));
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

extern "C" rr_status rr_restir_gi_execute(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                          const rr_restir_gi_params* p, const rr_restir_gi_images* b,
                                          void* stream) {
    rr_status st = rr_restir_gi_initial(ctx, scene, cam, p, b, stream);
    if (st != RR_OK) return st;
    st = rr_restir_gi_temporal(ctx, scene, cam, p, b, stream);
    if (st != RR_OK) return st;
    return rr_restir_gi_spatial_shade(ctx, scene, cam, p, b, stream);
}

extern "C" rr_status rr_restir_gi_reset_history(rr_ctx* ctx, const rr_restir_gi_images* b, uint32_t width,
                                                uint32_t height, void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!b || width == 0 || height == 0) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR GI: bad reset argument");
    for (int k = 0; k < 3; ++k)
        if (!b->reservoir_prev[k]) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR GI: null reservoir image");
    if (!b->history_prev[0] || !b->history_prev[1])
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR GI: null history image");
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t n = size_t(width) * height;
    gi_reset_kernel<<<unsigned((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<float4*>(b->reservoir_prev[0]), reinterpret_cast<float4*>(b->reservoir_prev[1]),
        reinterpret_cast<float4*>(b->reservoir_prev[2]), reinterpret_cast<float4*>(b->history_prev[0]),
        reinterpret_cast<float4*>(b->history_prev[1]), n);
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}
