// rr_reuse.cuh — device helpers shared by the ReSTIR PT (restir_pt.cu) and
// ReSTIR GI (restir_gi.cu) kernels; restir_pt.slang and restir_gi.slang define
// the same helpers with the same arithmetic (line numbers below are those of
// restir_pt.slang; restir_gi.slang:132-565 has the same functions).
#pragma once

#include "rr_internal.h"

namespace rr {

// HLSL rsqrt, restated as 1 / sqrt (both correctly rounded), as normalize is.
RR_D float rsqrt_(float x) { return 1.0f / sqrtf(x); }
RR_D float frac_(float x) { return x - floorf(x); }
RR_D float luminance(float3 c) { return dot(c, f3(0.2126f, 0.7152f, 0.0722f)); }

// mul(M, float4(v, w)) for a row-major float4x4 given as 16 floats
RR_D float4 mul44(const float* M, float x, float y, float z, float w) {
    return make_float4(M[0] * x + M[1] * y + M[2] * z + M[3] * w, M[4] * x + M[5] * y + M[6] * z + M[7] * w,
                       M[8] * x + M[9] * y + M[10] * z + M[11] * w, M[12] * x + M[13] * y + M[14] * z + M[15] * w);
}

struct Mat {
    float3 base, emissive;
    float metallic, roughness;
};
RR_D Mat load_mat(const DevScene& s, uint32_t m) {
    const float4 m0 = __ldg(s.materials + m * 2), m1 = __ldg(s.materials + m * 2 + 1);
    Mat r;
    r.base = xyz(m0); r.metallic = m0.w; r.emissive = xyz(m1); r.roughness = m1.w;
    return r;
}

// load_surface_from_images (restir_pt.slang:287-305); a material index past
// the scene's materials counts as no surface.
RR_D bool load_surface(const DevScene& s, const float4* pos_img, const float4* nrm_img, size_t i, float4& p4,
                       float4& n4, float3& pos, float3& n, uint32_t& mat) {
    p4 = pos_img[i];
    n4 = nrm_img[i];
    if (p4.w < 0.0f) return false;
    pos = xyz(p4);
    n = normalize(xyz(n4));
    mat = __float_as_uint(n4.w);
    return mat < s.num_materials;
}

// The light sample of sample_lights without its visibility test: the light
// pick (one random number), the shadow ray (origin, direction, t_max; t_min
// is the bias) and the contribution if the light is visible. Returns false
// where sample_lights returns zero before tracing (no lights, light below
// the surface).
RR_D bool sample_light_ray(const DevScene& s, float3 hit_pos, float3 normal, float3 wo, const Mat& m, float bias,
                           uint32_t& seed, float3& origin, float3& dir, float& tmax, float3& contrib) {
    const uint32_t N = s.num_lights;
    if (N == 0) return false;
    const uint32_t li = uint32_t(rand_float(seed) * float(N)) % N;
    const float4 l0 = __ldg(s.lights + li * 3), l1 = __ldg(s.lights + li * 3 + 1), l2 = __ldg(s.lights + li * 3 + 2);
    const bool is_point = __float_as_uint(l0.w) == 0u;
    float3 ldir;
    float dist, pdf_light;
    if (is_point) {
        const float3 to = f3(l0.x, l0.y, l0.z) - hit_pos;
        dist = length(to);
        ldir = to / mx(dist, 1e-6f);
        pdf_light = dist * dist;
    } else {
        ldir = normalize(-f3(l1.x, l1.y, l1.z));
        dist = 1e9f;
        pdf_light = 1.0f;
    }
    if (dot(ldir, normal) <= 0.0f) return false;
    origin = hit_pos + normal * bias;
    dir = ldir;
    tmax = dist - 0.01f;
    const float3 brdf_val = brdf_eval(normal, wo, ldir, m.base, m.metallic, m.roughness);
    const float n_dot_l = mx(dot(normal, ldir), 0.0f);
    const float den = is_point ? (pdf_light + 1e-6f) : 1.0f;
    const float3 irr = f3(l2.x * l2.w / den, l2.y * l2.w / den, l2.z * l2.w / den);
    const float pdf_bsdf = brdf_pdf(wo, ldir, normal, m.roughness);
    const float mis = is_point ? 1.0f : (pdf_light * pdf_light) / (pdf_light * pdf_light + pdf_bsdf * pdf_bsdf + 1e-10f);
    contrib = (((brdf_val * irr) * n_dot_l) * mis) * float(N);
    return true;
}

// sample_lights (restir_pt.slang:172-221): one light picked uniformly,
// shadow ray from hit_pos + normal * ray_bias over [ray_bias, dist - 0.01].
RR_D float3 sample_lights(const DevScene& s, float3 hit_pos, float3 normal, float3 wo, const Mat& m, float bias,
                          uint32_t& seed) {
    float3 o, d, c;
    float tmax;
    if (!sample_light_ray(s, hit_pos, normal, wo, m, bias, seed, o, d, tmax, c)) return f3(0.0f, 0.0f, 0.0f);
    HitRec h;
    if (trace<true>(s, make_ray(o, d), bias, tmax, h)) return f3(0.0f, 0.0f, 0.0f);
    return c;
}

// reconnection_jacobian (restir_pt.slang:437-457)
RR_D float reconnection_jacobian(float3 src, float3 tgt, float3 rc_pos, float3 rc_n) {
    const float3 sd = rc_pos - src, td = rc_pos - tgt;
    const float sd2 = dot(sd, sd), td2 = dot(td, td);
    if (sd2 <= 1e-8f || td2 <= 1e-8f) return 0.0f;
    const float3 sdir = sd * rsqrt_(sd2), tdir = td * rsqrt_(td2);
    const float scos = fabsf(dot(rc_n, -sdir)), tcos = fabsf(dot(rc_n, -tdir));
    if (scos <= 0.05f || tcos <= 0.05f) return 0.0f;
    const float j = (tcos * sd2) / (scos * td2);
    return clampf(j, 0.0f, 3.0f);
}

// trace_visibility (restir_pt.slang:459-469)
RR_D bool visible(const DevScene& s, float3 origin, float3 normal, float3 target, float bias) {
    const float3 delta = target - origin;
    const float dist = length(delta);
    if (dist <= bias) return false;
    const float3 dir = delta / dist;
    HitRec h;
    return !trace<true>(s, make_ray(origin + normal * bias, dir), bias, dist - bias, h);
}

RR_D bool pixel_of(const GpuCameraData& cam, uint32_t& x, uint32_t& y) {
    x = blockIdx.x * 16 + (threadIdx.x & 15);
    y = blockIdx.y * 8 + (threadIdx.x >> 4);
    return x < cam.screen_width && y < cam.screen_height;
}

RR_D float3 cam_pos(const GpuCameraData& c) { return f3(c.position[0], c.position[1], c.position[2]); }

// reproject_to_prev_pixel (restir_pt.slang:326-340)
RR_D bool reproject(const GpuCameraData& cam, float3 wp, int& px, int& py) {
    const float4 clip = mul44(cam.prev_view_proj, wp.x, wp.y, wp.z, 1.0f);
    if (clip.w <= 1.0e-6f) return false;
    const float nx = clip.x / clip.w, ny = clip.y / clip.w;
    if (fabsf(nx) > 1.0f || fabsf(ny) > 1.0f) return false;
    const float fx = (nx * 0.5f + 0.5f) * float(cam.screen_width) - 0.5f;
    const float fy = (ny * 0.5f + 0.5f) * float(cam.screen_height) - 0.5f;
    px = int(floorf(fx + 0.5f));
    py = int(floorf(fy + 0.5f));
    return px >= 0 && py >= 0 && px < int(cam.screen_width) && py < int(cam.screen_height);
}


// find_reprojected_history_surface (restir_pt.slang:355-409): the best
// compatible pixel (is_reprojected_history_compatible, :342-353) of the 3x3
// window around the reprojected position in the previous primary history.
RR_D bool find_history(const GpuCameraData& cam, const float4* __restrict__ hpos_img,
                       const float4* __restrict__ hnrm_img, float3 pp, float3 pn, uint32_t pmat, float3 cp,
                       size_t& hist, float3& hpos) {
    const uint32_t W = cam.screen_width, H = cam.screen_height;
    int cx, cy;
    if (!reproject(cam, pp, cx, cy)) return false;
    bool found = false;
    float best = 1e30f;
    hist = 0;
    hpos = f3(0.0f, 0.0f, 0.0f);
    for (int oy = -1; oy <= 1; ++oy) {
        for (int ox = -1; ox <= 1; ++ox) {
            const int qx = cx + ox, qy = cy + oy;
            if (qx < 0 || qy < 0 || qx >= int(W) || qy >= int(H)) continue;
            const size_t j = size_t(qy) * W + qx;
            const float4 h4 = hpos_img[j];
            if (h4.w < 0.0f) continue;
            const float4 hn4 = hnrm_img[j];
            const float3 cpos = xyz(h4), cn = normalize(xyz(hn4));
            const uint32_t cmat = __float_as_uint(hn4.w);
            if (pmat != cmat) continue;
            if (dot(pn, cn) < 0.9f) continue;
            const float view_dist = mx(length(pp - cp), 1.0f);
            const float plane = fabsf(dot(cpos - pp, pn));
            const float dpos = length(cpos - pp);
            if (!(plane <= 0.01f * view_dist && dpos <= 0.05f * view_dist)) continue;
            const float err = plane * 4.0f + dpos;
            if (err < best) { best = err; hist = j; hpos = cpos; found = true; }
        }
    }
    return found;
}

// The spatial pass's neighbour k (restir_pt.slang:908-919): golden-ratio
// angles from a per-pixel phase, radius sqrt((k + 0.5) / K) R, offsets
// truncated and clamped to the image. Returns false for the pixel itself.
RR_D float spatial_phase(uint32_t x, uint32_t y) {
    return frac_(float(pcg_hash(x ^ (y * 65537u))) * 2.3283064365386963e-10f);
}
RR_D bool spatial_neighbor(float base_phase, uint32_t k, uint32_t K, uint32_t R, uint32_t x, uint32_t y, uint32_t W,
                           uint32_t H, size_t& j) {
    const float u = (float(k) + 0.5f) / float(K);
    const float angle = frac_(base_phase + 0.61803398875f * float(k)) * kTwoPi;
    const float radius = sqrtf(u) * float(R);
    const int ox = int(radius * rr_cosf(angle)), oy = int(radius * rr_sinf(angle));
    const int nx = min(max(int(x) + ox, 0), int(W) - 1);
    const int ny = min(max(int(y) + oy, 0), int(H) - 1);
    if (nx == int(x) && ny == int(y)) return false;
    j = size_t(ny) * W + nx;
    return true;
}

// is_spatial_neighbor_compatible (restir_pt.slang:411-430)
RR_D bool spatial_compatible(const float4* __restrict__ gpos, const float4* __restrict__ gnrm, size_t j, float3 pp,
                             float3 pn, float3 cp, float3& nbp) {
    const float4 nb4 = gpos[j];
    if (nb4.w < 0.0f) return false;
    nbp = xyz(nb4);
    const float3 nbn = normalize(xyz(gnrm[j]));
    if (dot(nbn, pn) < 0.85f) return false;
    const float plane = fabsf(dot(nbp - pp, pn));
    const float dscale = mx(length(pp - cp), 1.0f);
    return plane <= 0.02f * dscale;
}

} // namespace rr
