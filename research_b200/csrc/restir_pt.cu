// restir_pt.cu — ReSTIR PT with the reconnection shift (ReSTIRPTPass.cpp:529-812;
// kernels in passes/restir_pt/restir_pt.slang). Three per-pixel kernels on
// 16x8 pixel blocks, each ray traced inline on the scene BVH:
//   initial      : cs_initial (:567-757) — M candidate paths from the primary
//                  surface (first direction by sample_primary_dir, i.e. the
//                  guiding grid's lobe or a cosine lobe), a reconnection vertex
//                  at the first secondary hit, suffix radiance by NEE and BRDF
//                  sampling, resampled by weighted reservoir sampling
//   temporal     : cs_temporal (:760-857) — reprojected history pixel (3x3
//                  search), reconnection Jacobian, visibility, M-cap
//   spatial_shade: cs_spatial_shade (:860-1000) — golden-ratio neighbour
//                  pattern, reconnection, final shading, guiding splat
// The reservoir is four RGBA32F images (restir_pt.slang:10-25):
//   (rc_pos, w_sum), (rc_normal, asfloat(M)), (suffix_radiance, W),
//   (prefix_throughput, valid).

#include "rr_grid.cuh"
#include "rr_reuse.cuh"

namespace rr {
namespace {

struct PtrLaunch {
    GpuCameraData cam;
    uint32_t frame_seed, num_candidates, max_bounces, temporal, spatial, num_neighbors, radius, include_direct;
    float indirect_strength, ray_bias;
    uint32_t m_cap;
    GridParams grid;
};

struct PtrImages {
    const float4* gpos;
    const float4* gnrm;
    const float4* direct;       // may be null
    float4* rc[4];              // current reservoir
    const float4* rp[4];        // previous reservoir
    float4* hc[2];              // current primary history (pos, normal)
    const float4* hp[2];        // previous primary history
    float4* out;
    uint32_t* accum;            // guiding accumulators (int32 x 4 per cell)
    const float4* fitted;       // guiding lobes (mu, kappa) per cell
};

struct Reservoir {
    float3 rc_pos, rc_normal, suffix_rad, prefix_thp;
    float w_sum, W;
    uint32_t M;
    float valid;
};

RR_D Reservoir load_reservoir(const float4* const* img, size_t i) {
    const float4 p = img[0][i], n = img[1][i], r = img[2][i], e = img[3][i];
    Reservoir res;
    res.rc_pos = xyz(p); res.w_sum = p.w;
    res.rc_normal = xyz(n); res.M = __float_as_uint(n.w);
    res.suffix_rad = xyz(r); res.W = r.w;
    res.prefix_thp = xyz(e); res.valid = e.w;
    return res;
}

RR_D void store_reservoir(float4* const* img, size_t i, const Reservoir& r) {
    img[0][i] = make_float4(r.rc_pos.x, r.rc_pos.y, r.rc_pos.z, r.w_sum);
    img[1][i] = make_float4(r.rc_normal.x, r.rc_normal.y, r.rc_normal.z, __uint_as_float(r.M));
    img[2][i] = make_float4(r.suffix_rad.x, r.suffix_rad.y, r.suffix_rad.z, r.W);
    img[3][i] = make_float4(r.prefix_thp.x, r.prefix_thp.y, r.prefix_thp.z, r.valid);
}

// write_empty_reservoir (restir_pt.slang:223-229)
RR_D void store_empty(float4* const* img, size_t i) {
    img[0][i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    img[1][i] = make_float4(0.0f, 0.0f, 0.0f, __uint_as_float(0u));
    img[2][i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    img[3][i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
}

// evaluate_contribution / target_function (restir_pt.slang:474-503)
RR_D float3 evaluate_contribution(float3 pp, float3 pn, const Mat& pm, float3 cam_pos, const Reservoir& r) {
    const float3 to_rc = r.rc_pos - pp;
    const float dist2 = dot(to_rc, to_rc);
    if (dist2 <= 1e-8f) return f3(0.0f, 0.0f, 0.0f);
    const float3 wi = to_rc * rsqrt_(dist2);
    const float cos_x = mx(dot(pn, wi), 0.0f);
    if (cos_x <= 0.0f) return f3(0.0f, 0.0f, 0.0f);
    const float3 wo = normalize(cam_pos - pp);
    const float3 bv = brdf_eval(pn, wo, wi, pm.base, pm.metallic, pm.roughness);
    return ((bv * cos_x) * r.prefix_thp) * r.suffix_rad;
}
RR_D float target_function(float3 pp, float3 pn, const Mat& pm, float3 cam_pos, const Reservoir& r) {
    return luminance(evaluate_contribution(pp, pn, pm, cam_pos, r));
}

// cs_initial (restir_pt.slang:567-757)
__global__ void __launch_bounds__(128, 8) ptr_initial_kernel(DevScene s, PtrLaunch L, PtrImages I) {
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
        store_empty(I.rc, i);
        return;
    }
    I.hc[0][i] = p4;
    I.hc[1][i] = n4;
    const Mat pm = load_mat(s, pmat);
    const float3 cp = cam_pos(L.cam);
    const float bias = L.ray_bias;
    Reservoir sel;
    sel.rc_pos = sel.rc_normal = sel.suffix_rad = sel.prefix_thp = f3(0.0f, 0.0f, 0.0f);
    sel.w_sum = 0.0f; sel.W = 0.0f; sel.M = 0u; sel.valid = 0.0f;
    float w_sum = 0.0f;
    uint32_t M_count = 0;
    const uint32_t max_b = L.max_bounces > 1u ? L.max_bounces : 1u;
    for (uint32_t c = 0; c < L.num_candidates; ++c) {
        float src_pdf;
        const float3 wi0 = sample_primary_dir(I.fitted, pp, pn, pmat, L.grid, seed, src_pdf);
        if (src_pdf <= 1e-6f || dot(pn, wi0) <= 0.0f) continue;
        HitRec h;
        if (!trace<false>(s, make_ray(pp + pn * bias, wi0), bias, 1e9f, h)) continue;
        const Surface rc = hit_surface(s, h.inst, h.prim, h.u, h.v);
        float3 rc_n = rc.normal;
        if (dot(rc_n, wi0) > 0.0f) rc_n = -rc_n;
        const Mat rc_mat = load_mat(s, rc.material);
        float3 suffix = rc_mat.emissive;
        const float3 rc_wo = -wi0;
        suffix = suffix + sample_lights(s, rc.pos, rc_n, rc_wo, rc_mat, bias, seed);
        float3 cur_pos = rc.pos, cur_n = rc_n, cur_wo = rc_wo;
        Mat cur_mat = rc_mat;
        float3 path_thp = f3(1.0f, 1.0f, 1.0f);
        for (uint32_t b = 1; b < max_b; ++b) {
            const float u0 = rand_float(seed);
            const float u1 = rand_float(seed);
            float3 wi;
            float pdf;
            const float3 f = brdf_sample(cur_wo, cur_n, cur_mat.base, cur_mat.metallic, cur_mat.roughness, u0, u1,
                                         wi, pdf);
            if (pdf <= 1e-6f || dot(cur_n, wi) <= 0.0f) break;
            const float cos_at = mx(dot(cur_n, wi), 0.0f);
            path_thp = path_thp * ((f * cos_at) / pdf);
            if (mx(path_thp.x, mx(path_thp.y, path_thp.z)) <= 0.0f) break;
            HitRec hb;
            if (!trace<false>(s, make_ray(cur_pos + cur_n * bias, wi), bias, 1e9f, hb)) {
                suffix = suffix + path_thp * sky_radiance(wi);
                break;
            }
            const Surface hs = hit_surface(s, hb.inst, hb.prim, hb.u, hb.v);
            float3 hn = hs.normal;
            if (dot(hn, wi) > 0.0f) hn = -hn;
            const Mat hm = load_mat(s, hs.material);
            const float3 hwo = -wi;
            suffix = suffix + path_thp * sample_lights(s, hs.pos, hn, hwo, hm, bias, seed);
            cur_pos = hs.pos; cur_n = hn; cur_mat = hm; cur_wo = hwo;
        }
        Reservoir cand;
        cand.rc_pos = rc.pos; cand.rc_normal = rc_n; cand.suffix_rad = suffix;
        cand.prefix_thp = f3(1.0f, 1.0f, 1.0f);
        cand.M = 1u; cand.W = 0.0f; cand.w_sum = 0.0f; cand.valid = 1.0f;
        const float p_hat = target_function(pp, pn, pm, cp, cand);
        if (p_hat <= 0.0f) continue;
        const float3 delta = rc.pos - pp;
        if (dot(delta, delta) <= 1e-8f) continue;
        const float weight = p_hat / mx(src_pdf, 1e-6f);
        w_sum += weight;
        M_count++;
        if (w_sum > 0.0f && rand_float(seed) < weight / w_sum) sel = cand;
    }
    if (M_count > 0 && sel.valid > 0.5f) {
        const float p_hat = target_function(pp, pn, pm, cp, sel);
        if (p_hat > 1e-10f) {
            sel.M = M_count;
            sel.w_sum = w_sum;
            sel.W = w_sum / (float(M_count) * p_hat);
            store_reservoir(I.rc, i, sel);
            return;
        }
    }
    store_empty(I.rc, i);
}

// cs_temporal (restir_pt.slang:760-857)
__global__ void __launch_bounds__(128, 8) ptr_temporal_kernel(DevScene s, PtrLaunch L, PtrImages I) {
    uint32_t x, y;
    if (!pixel_of(L.cam, x, y)) return;
    const uint32_t W = L.cam.screen_width, H = L.cam.screen_height;
    const size_t i = size_t(y) * W + x;
    float4 p4, n4;
    float3 pp, pn;
    uint32_t pmat;
    if (!load_surface(s, I.gpos, I.gnrm, i, p4, n4, pp, pn, pmat)) return;
    const Mat pm = load_mat(s, pmat);
    const float3 cp = cam_pos(L.cam);
    size_t hist;
    float3 hpos;
    if (!find_history(L.cam, I.hp[0], I.hp[1], pp, pn, pmat, cp, hist, hpos)) return;
    Reservoir cur = load_reservoir(I.rc, i);
    Reservoir prv = load_reservoir(I.rp, hist);
    if (prv.M == 0 || prv.valid < 0.5f) return;
    prv.M = min(prv.M, L.m_cap);
    const float jac = reconnection_jacobian(hpos, pp, prv.rc_pos, prv.rc_normal);
    if (jac <= 0.0f) return;
    if (!visible(s, pp, pn, prv.rc_pos, L.ray_bias)) return;
    const float ph_prev = target_function(pp, pn, pm, cp, prv);
    const float prev_W = mn(prv.W, 50.0f);
    const float contrib = ((ph_prev * prev_W) * float(prv.M)) * jac;
    if (contrib <= 0.0f) return;
    cur.w_sum += contrib;
    uint32_t seed = make_seed(x, y, L.frame_seed + 1u);
    if (cur.w_sum > 0.0f && rand_float(seed) < contrib / cur.w_sum) {
        cur.rc_pos = prv.rc_pos; cur.rc_normal = prv.rc_normal;
        cur.suffix_rad = prv.suffix_rad; cur.prefix_thp = prv.prefix_thp;
        cur.valid = 1.0f;
    }
    const uint32_t new_M = cur.M + prv.M;
    if (new_M > L.m_cap) {
        cur.w_sum *= float(L.m_cap) / float(new_M);
        cur.M = L.m_cap;
    } else {
        cur.M = new_M;
    }
    if (cur.M > 0 && cur.valid > 0.5f) {
        const float ph_y = target_function(pp, pn, pm, cp, cur);
        cur.W = (ph_y > 1e-10f) ? (cur.w_sum / (float(cur.M) * ph_y)) : 0.0f;
        cur.W = mn(cur.W, 50.0f);
    }
    store_reservoir(I.rc, i, cur);
}

// cs_spatial_shade (restir_pt.slang:860-1000)
__global__ void __launch_bounds__(128, 8) ptr_spatial_shade_kernel(DevScene s, PtrLaunch L, PtrImages I) {
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
    Reservoir res = load_reservoir(I.rc, i);
    if (L.spatial != 0u && L.num_neighbors > 0u && res.valid > 0.5f) {
        const float base_phase = spatial_phase(x, y);
        for (uint32_t k = 0; k < L.num_neighbors; ++k) {
            size_t j;
            if (!spatial_neighbor(base_phase, k, L.num_neighbors, L.radius, x, y, W, H, j)) continue;
            float3 nbp;
            if (!spatial_compatible(I.gpos, I.gnrm, j, pp, pn, cp, nbp)) continue;
            const Reservoir nbr = load_reservoir(I.rc, j);
            if (nbr.M == 0 || nbr.valid < 0.5f) continue;
            const float jac = reconnection_jacobian(nbp, pp, nbr.rc_pos, nbr.rc_normal);
            if (jac <= 0.0f) continue;
            const float contrib = ((target_function(pp, pn, pm, cp, nbr) * nbr.W) * float(nbr.M)) * jac;
            if (contrib <= 0.0f) continue;
            res.w_sum += contrib;
            res.M += nbr.M;
            const float accept = frac_(base_phase + 0.754877666f * float(k + 1u));
            if (res.w_sum > 0.0f && accept < contrib / res.w_sum) {
                res.rc_pos = nbr.rc_pos; res.rc_normal = nbr.rc_normal;
                res.suffix_rad = nbr.suffix_rad; res.prefix_thp = nbr.prefix_thp;
            }
        }
        if (res.M > 0) {
            const float ph_y = target_function(pp, pn, pm, cp, res);
            res.W = (ph_y > 1e-10f) ? (res.w_sum / (float(res.M) * ph_y)) : 0.0f;
        }
    }
    if (res.M > 0 && res.W > 0.0f && res.valid > 0.5f) {
        const float3 ind = evaluate_contribution(pp, pn, pm, cp, res) * res.W;
        if (luminance(ind) > 0.0f && visible(s, pp, pn, res.rc_pos, L.ray_bias))
            radiance = radiance + ind * L.indirect_strength;
        if (L.grid.enabled != 0u) {  // splat (:978-994)
            const float3 to_rc = res.rc_pos - pp;
            const float d2 = dot(to_rc, to_rc);
            if (d2 > 1e-8f) splat_dir(I.accum, cell_index(pp, pmat, L.grid), to_rc * rsqrt_(d2));
        }
    }
    I.out[i] = make_float4(radiance.x, radiance.y, radiance.z, 1.0f);
}

__global__ void ptr_reset_kernel(float4* r0, float4* r1, float4* r2, float4* r3, float4* h0, float4* h1, size_t n) {
    const size_t i = size_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    r0[i] = z; r1[i] = z; r2[i] = z; r3[i] = z;
    h0[i] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
    h1[i] = z;
}

PtrLaunch make_launch(const GpuCameraData* cam, const rr_restir_pt_params* p) {
    PtrLaunch L;
    L.cam = *cam;
    L.frame_seed = p->frame_seed;
    L.num_candidates = p->num_initial_candidates;
    L.max_bounces = p->max_bounces;
    L.temporal = p->temporal_enable;
    L.spatial = p->spatial_enable;
    L.num_neighbors = p->spatial_num_neighbors;
    L.radius = p->spatial_radius;
    L.include_direct = p->include_direct_lighting;
    L.indirect_strength = p->indirect_strength;
    L.ray_bias = p->ray_bias;
    // clamp(20u * M, 1u, 8192u) in 32-bit unsigned arithmetic (restir_pt.slang:801)
    L.m_cap = std::min(std::max(20u * p->num_initial_candidates, 1u), 8192u);
    // make_grid_params (restir_pt.slang:505-514): enabled = guiding_enable
    L.grid = to_grid(&p->guiding, cam->position);
    return L;
}

PtrImages make_images(const rr_restir_pt_images* b) {
    PtrImages I;
    I.gpos = reinterpret_cast<const float4*>(b->gbuf_pos);
    I.gnrm = reinterpret_cast<const float4*>(b->gbuf_norm);
    I.direct = reinterpret_cast<const float4*>(b->direct);
    for (int k = 0; k < 4; ++k) {
        I.rc[k] = reinterpret_cast<float4*>(b->reservoir_curr[k]);
        I.rp[k] = reinterpret_cast<const float4*>(b->reservoir_prev[k]);
    }
    for (int k = 0; k < 2; ++k) {
        I.hc[k] = reinterpret_cast<float4*>(b->history_curr[k]);
        I.hp[k] = reinterpret_cast<const float4*>(b->history_prev[k]);
    }
    I.out = reinterpret_cast<float4*>(b->output);
    I.accum = reinterpret_cast<uint32_t*>(b->guiding_accum);
    I.fitted = reinterpret_cast<const float4*>(b->guiding_fitted);
    return I;
}

dim3 grid_of(const GpuCameraData* cam) { return dim3((cam->screen_width + 15) / 16, (cam->screen_height + 7) / 8); }

enum Stage { kInitial, kTemporal, kSpatial };

rr_status check(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam, const rr_restir_pt_params* p,
                const rr_restir_pt_images* b, Stage st) {
    if (!scene || !cam || !p || !b) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR PT: null argument");
    if (cam->screen_width == 0 || cam->screen_height == 0 || cam->screen_width > 65535u * 16u ||
        cam->screen_height > 65535u * 8u)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR PT: bad image size");
    if (!b->gbuf_pos || !b->gbuf_norm) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR PT: null G-buffer");
    for (int k = 0; k < 4; ++k)
        if (!b->reservoir_curr[k] || (st == kTemporal && !b->reservoir_prev[k]))
            return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR PT: null reservoir image");
    if (st == kInitial && (!b->history_curr[0] || !b->history_curr[1]))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR PT: null history image");
    if (st == kTemporal && (!b->history_prev[0] || !b->history_prev[1]))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR PT: null history image");
    if (st == kSpatial && !b->output) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR PT: null output");
    const bool guided = p->guiding.enabled != 0u && (st == kSpatial || p->guiding.alpha > 0.0f);
    if (guided && (p->guiding.cell_count == 0 || (st == kInitial && !b->guiding_fitted) ||
                   (st == kSpatial && !b->guiding_accum)))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR PT: guiding enabled without its grid buffers");
    return RR_OK;
}

} // namespace
} // namespace rr

using namespace rr;

extern "C" rr_status rr_restir_pt_initial(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                          const rr_restir_pt_params* p, const rr_restir_pt_images* b,
                                          void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    rr_status st = check(ctx, scene, cam, p, b, kInitial);
    if (st != RR_OK) return st;
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    ptr_initial_kernel<<<grid_of(cam), 128, 0, static_cast<cudaStream_t>(stream)>>>(scene->dev, make_launch(cam, p),
                                                                                   make_images(b));
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

extern "C" rr_status rr_restir_pt_temporal(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                           const rr_restir_pt_params* p, const rr_restir_pt_images* b,
                                           void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    rr_status st = check(ctx, scene, cam, p, b, kTemporal);
    if (st != RR_OK) return st;
    if (!p->temporal_enable) return RR_OK;  // restir_pt.slang:764
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    ptr_temporal_kernel<<<grid_of(cam), 128, 0, static_cast<cudaStream_t>(stream)>>>(scene->dev, make_launch(cam, p),
                                                                                    make_images(b));
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

extern "C" rr_status rr_restir_pt_spatial_shade(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                                const rr_restir_pt_params* p, const rr_restir_pt_images* b,
                                                void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    rr_status st = check(ctx, scene, cam, p, b, kSpatial);
    if (st != RR_OK) return st;
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    ptr_spatial_shade_kernel<<<grid_of(cam), 128, 0, static_cast<cudaStream_t>(stream)>>>(
        scene->dev, make_launch(cam, p), make_images(b));
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}

extern "C" rr_status rr_restir_pt_execute(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                          const rr_restir_pt_params* p, const rr_restir_pt_images* b,
                                          void* stream) {
    rr_status st = rr_restir_pt_initial(ctx, scene, cam, p, b, stream);
    if (st != RR_OK) return st;
    st = rr_restir_pt_temporal(ctx, scene, cam, p, b, stream);
    if (st != RR_OK) return st;
    st = rr_restir_pt_spatial_shade(ctx, scene, cam, p, b, stream);
    if (st != RR_OK) return st;
    if (p->guiding.enabled == 0u) return RR_OK;
    // cs_fit_guiding after the splats (ReSTIRPTPass.cpp:784-810)
    return rr_guiding_fit(ctx, b->guiding_accum, b->guiding_fitted, &p->guiding, stream);
}

extern "C" rr_status rr_restir_pt_reset_history(rr_ctx* ctx, const rr_restir_pt_images* b, uint32_t width,
                                                uint32_t height, void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!b || width == 0 || height == 0) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR PT: bad reset argument");
    for (int k = 0; k < 4; ++k)
        if (!b->reservoir_prev[k]) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR PT: null reservoir image");
    if (!b->history_prev[0] || !b->history_prev[1])
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR PT: null history image");
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    const size_t n = size_t(width) * height;
    ptr_reset_kernel<<<unsigned((n + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<float4*>(b->reservoir_prev[0]), reinterpret_cast<float4*>(b->reservoir_prev[1]),
        reinterpret_cast<float4*>(b->reservoir_prev[2]), reinterpret_cast<float4*>(b->reservoir_prev[3]),
        reinterpret_cast<float4*>(b->history_prev[0]), reinterpret_cast<float4*>(b->history_prev[1]), n);
    RR_CHECK_LAUNCH(ctx);
    ctx->launches += 1;
    return RR_OK;
}
