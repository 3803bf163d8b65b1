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
#include "rr_wave.cuh"

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

// ── wavefront form of cs_initial ───────────────────────────────────────────
// gi_initial_kernel cut at its rays, as the ReSTIR PT initial pass is (steps
// in rr_wave.cuh). A candidate is one segment, so each step takes one
// candidate of every pixel with work: extend (the cosine ray), shade (the
// secondary vertex: its emission, the light sample with its shadow ray
// queued), shadow (the light's contribution or zero added to the vertex's
// radiance), advance (resampling, then the next candidate's direction or the
// reservoir). Random numbers and additions keep the inline order, so the
// results are the same bits; num_candidates steps cover every pixel.
struct GiWave {
    uint4* st;          // (seed, candidate, -, M)
    float4* acc;        // (w_sum, -, -, -)
    float4* spos;       // the candidate's secondary vertex
    float4* snrm;       // its geometric normal as hit_surface returns it
    float4* rad;        // its outgoing radiance: emission + light sample
    float4* selp;       // selected sample: position
    float4* selr;       // radiance
    float4* seln;       // normal
    float4* qa[2];
    float4* qb[2];
    float4* hits;
    float4* sa;
    float4* sb;
    float4* sc;
    uint32_t* ended;
    uint32_t* cnt;
    uint32_t n;
};
constexpr int kGiWaveArrays = 8;

// The pixel's next candidate direction from candidate c on (cosine lobe;
// directions below the surface are skipped as the inline `continue`).
RR_D bool giw_next(const GiLaunch& L, float3 pp, float3 pn, uint32_t& seed, uint32_t& c, float3& o, float3& d) {
    float3 T, B;
    build_onb(pn, T, B);
    for (; c < L.num_candidates; ++c) {
        const float u0 = rand_float(seed);
        const float u1 = rand_float(seed);
        float pdf_dir;
        const float3 dd = tangent_to_world(sample_cosine_hemisphere(u0, u1, pdf_dir), T, B, pn);
        if (dot(pn, dd) <= 0.0f) continue;
        o = pp + pn * L.ray_bias;
        d = dd;
        return true;
    }
    return false;
}

// The end of gi_initial_kernel: the selected sample's reservoir or an empty one.
RR_D void giw_finish(const GiLaunch& L, const GiImages& I, const GiWave& V, size_t i, float3 pp, float3 pn,
                     const Mat& pm, uint32_t M_count, float w_sum) {
    if (M_count > 0) {
        GiRes sel;
        sel.pos = xyz(V.selp[i]); sel.rad = xyz(V.selr[i]); sel.nrm = xyz(V.seln[i]);
        const float ph_y = gi_target(pp, pn, pm, cam_pos(L.cam), sel.pos, sel.rad);
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

__global__ void __launch_bounds__(kBlock) giw_begin_kernel(DevScene s, GiLaunch L, GiImages I, GiWave V) {
    const uint32_t W = L.cam.screen_width;
    const uint32_t warp_first = blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
    for (uint32_t base = warp_first; base < V.n; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + lane_id();
        bool emit = false;
        float3 o = f3(0.0f, 0.0f, 0.0f), d = f3(0.0f, 0.0f, 0.0f);
        if (i < V.n) {
            const uint32_t x = i % W, y = i / W;
            uint32_t seed = make_seed(x, y, L.frame_seed);
            float4 p4, n4;
            float3 pp, pn;
            uint32_t pmat;
            if (!load_surface(s, I.gpos, I.gnrm, i, p4, n4, pp, pn, pmat)) {
                I.hc[0][i] = make_float4(0.0f, 0.0f, 0.0f, -1.0f);
                I.hc[1][i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                store_gi_empty(I.rc, i);
            } else {
                I.hc[0][i] = p4;
                I.hc[1][i] = n4;
                const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                V.selp[i] = z; V.selr[i] = z; V.seln[i] = z;
                uint32_t c = 0;
                emit = giw_next(L, pp, pn, seed, c, o, d);
                if (emit) {
                    V.st[i] = make_uint4(seed, c, 0u, 0u);
                    V.acc[i] = z;
                } else {
                    store_gi_empty(I.rc, i);   // no candidate: M = 0
                }
            }
        }
        const uint32_t slot = warp_alloc(emit, V.cnt);
        if (emit) {
            V.qa[0][slot] = make_float4(o.x, o.y, o.z, __uint_as_float(i));
            V.qb[0][slot] = make_float4(d.x, d.y, d.z, 0.0f);
        }
    }
}

__global__ void __launch_bounds__(kBlock, 4) giw_shade_kernel(DevScene s, GiLaunch L, GiWave V, uint32_t step) {
    const int cur = step & 1;
    uint32_t* c0 = V.cnt + size_t(step) * kWaveWords;
    const uint32_t count = c0[0];
    const float bias = L.ray_bias;
    const uint32_t warp_first = blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
    for (uint32_t base = warp_first; base < count; base += gridDim.x * blockDim.x) {
        const uint32_t q = base + lane_id();
        bool shadow = false, ris = false;
        uint32_t pid = 0;
        float3 so = f3(0.0f, 0.0f, 0.0f), sd = so, sc = so;
        float stmax = 0.0f;
        if (q < count) {
            const float4 a = V.qa[cur][q], b = V.qb[cur][q], h = V.hits[q];
            pid = __float_as_uint(a.w);
            const uint32_t inst = __float_as_uint(h.z);
            if (inst != kNoIndex) {
                // evaluate_sample_radiance (:539-552): normal turned toward wo = -d
                uint4 st = V.st[pid];
                uint32_t seed = st.x;
                const float3 d = xyz(b);
                const Surface sec = hit_surface(s, inst, __float_as_uint(h.w), h.x, h.y);
                const float3 wo = -d;
                float3 sn = sec.normal;
                if (dot(sn, wo) < 0.0f) sn = -sn;
                const Mat sm = load_mat(s, sec.material);
                float3 rad = sm.emissive;
                float3 c;
                shadow = sample_light_ray(s, sec.pos, sn, wo, sm, bias, seed, so, sd, stmax, c);
                if (shadow) sc = c;
                else rad = rad + f3(0.0f, 0.0f, 0.0f);
                V.spos[pid] = make_float4(sec.pos.x, sec.pos.y, sec.pos.z, 0.0f);
                V.snrm[pid] = make_float4(sec.normal.x, sec.normal.y, sec.normal.z, 0.0f);
                V.rad[pid] = make_float4(rad.x, rad.y, rad.z, 0.0f);
                st.x = seed;
                V.st[pid] = st;
                ris = true;
            }
        }
        const uint32_t sslot = warp_alloc(shadow, c0 + 2);
        if (shadow) {
            V.sa[sslot] = make_float4(so.x, so.y, so.z, __uint_as_float(pid));
            V.sb[sslot] = make_float4(sd.x, sd.y, sd.z, stmax);
            V.sc[sslot] = make_float4(sc.x, sc.y, sc.z, 0.0f);
        }
        // every segment ends its candidate (a miss drops it)
        const uint32_t eslot = warp_alloc(q < count, c0 + 4);
        if (q < count) V.ended[eslot] = pid | (ris ? kRis : 0u);
    }
}

__global__ void __launch_bounds__(kBlock) giw_advance_kernel(DevScene s, GiLaunch L, GiImages I, GiWave V,
                                                             uint32_t step) {
    const int nxt = (step & 1) ^ 1;
    uint32_t* c0 = V.cnt + size_t(step) * kWaveWords;
    uint32_t* c1 = c0 + kWaveWords;
    const uint32_t count = c0[4];
    const float3 cp = cam_pos(L.cam);
    const uint32_t warp_first = blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
    for (uint32_t base = warp_first; base < count; base += gridDim.x * blockDim.x) {
        const uint32_t q = base + lane_id();
        bool emit = false;
        uint32_t pid = 0;
        float3 o = f3(0.0f, 0.0f, 0.0f), d = o;
        if (q < count) {
            const uint32_t e = V.ended[q];
            pid = e & ~kRis;
            const uint4 st = V.st[pid];
            uint32_t seed = st.x, c = st.y, M_count = st.w;
            float w_sum = V.acc[pid].x;
            float4 p4, n4;
            float3 pp, pn;
            uint32_t pmat;
            load_surface(s, I.gpos, I.gnrm, pid, p4, n4, pp, pn, pmat);
            const Mat pm = load_mat(s, pmat);
            if (e & kRis) {
                const float3 spos = xyz(V.spos[pid]), rad = xyz(V.rad[pid]);
                const float tgt = gi_target(pp, pn, pm, cp, spos, rad);
                if (!(tgt <= 0.0f)) {
                    const float pdf = gi_source_pdf(pp, pn, spos);
                    if (!(pdf <= 1e-6f)) {
                        const float weight = tgt / pdf;
                        w_sum += weight;
                        M_count++;
                        if (w_sum > 0.0f && rand_float(seed) < weight / w_sum) {
                            V.selp[pid] = make_float4(spos.x, spos.y, spos.z, 0.0f);
                            V.selr[pid] = make_float4(rad.x, rad.y, rad.z, 0.0f);
                            V.seln[pid] = V.snrm[pid];
                        }
                    }
                }
            }
            ++c;
            emit = giw_next(L, pp, pn, seed, c, o, d);
            if (emit) {
                V.st[pid] = make_uint4(seed, c, 0u, M_count);
                V.acc[pid] = make_float4(w_sum, 0.0f, 0.0f, 0.0f);
            } else {
                giw_finish(L, I, V, pid, pp, pn, pm, M_count, w_sum);
            }
        }
        const uint32_t slot = warp_alloc(emit, c1);
        if (emit) {
            V.qa[nxt][slot] = make_float4(o.x, o.y, o.z, __uint_as_float(pid));
            V.qb[nxt][slot] = make_float4(d.x, d.y, d.z, 0.0f);
        }
    }
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

// cs_initial as the wavefront above: one launch to start every pixel, then
// per candidate extend, shade, shadow and advance.
rr_status gi_initial_wavefront(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                               const rr_restir_gi_params* p, const rr_restir_gi_images* b, cudaStream_t stream) {
    const size_t n = size_t(cam->screen_width) * cam->screen_height;
    rr_status st = ensure_queues(ctx, n);
    if (st != RR_OK) return st;
    if (p->num_initial_candidates > (1u << 20))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR GI: too many candidates");
    const uint32_t steps = p->num_initial_candidates;
    float4* a = nullptr;
    uint32_t* cnt = nullptr;
    if ((st = wave_scratch(ctx, n, kGiWaveArrays, steps, stream, &a, &cnt)) != RR_OK) return st;
    GiWave V;
    V.st = reinterpret_cast<uint4*>(a);
    V.acc = a + n; V.spos = a + 2 * n; V.snrm = a + 3 * n; V.rad = a + 4 * n;
    V.selp = a + 5 * n; V.selr = a + 6 * n; V.seln = a + 7 * n;
    rr_pt_queues& q = ctx->pt;
    V.qa[0] = q.ray_a[0]; V.qa[1] = q.ray_a[1];
    V.qb[0] = q.ray_b[0]; V.qb[1] = q.ray_b[1];
    V.hits = q.hits;
    V.sa = q.shadow_a; V.sb = q.shadow_b; V.sc = q.shadow_c;
    V.ended = reinterpret_cast<uint32_t*>(q.ray_c[0]);   // n words fit in n float4
    V.cnt = cnt;
    V.n = uint32_t(n);
    const DevScene& S = scene->dev;
    const GiLaunch L = make_launch(cam, p);
    const GiImages I = make_images(b);
    const int cap = int((n + kBlock - 1) / kBlock);
    const int g_begin = std::min<int>(persistent_grid(ctx, reinterpret_cast<const void*>(giw_begin_kernel)), cap);
    giw_begin_kernel<<<g_begin, kBlock, 0, stream>>>(S, L, I, V);
    RR_CHECK_LAUNCH(ctx);
    const int g_ext = persistent_grid(ctx, reinterpret_cast<const void*>(wave_extend_kernel));
    const int g_sh = persistent_grid(ctx, reinterpret_cast<const void*>(wave_shadow_kernel));
    const int g_shade = std::min<int>(persistent_grid(ctx, reinterpret_cast<const void*>(giw_shade_kernel)), cap);
    const int g_adv = std::min<int>(persistent_grid(ctx, reinterpret_cast<const void*>(giw_advance_kernel)), cap);
    for (uint32_t k = 0; k < steps; ++k) {
        uint32_t* c0 = cnt + size_t(k) * kWaveWords;
        wave_extend_kernel<<<g_ext, kBlock, 0, stream>>>(S, V.qa[k & 1], V.qb[k & 1], V.hits, c0, L.ray_bias);
        RR_CHECK_LAUNCH(ctx);
        giw_shade_kernel<<<g_shade, kBlock, 0, stream>>>(S, L, V, k);
        RR_CHECK_LAUNCH(ctx);
        wave_shadow_kernel<<<g_sh, kBlock, 0, stream>>>(S, V.sa, V.sb, V.sc, V.rad, c0, L.ray_bias);
        RR_CHECK_LAUNCH(ctx);
        giw_advance_kernel<<<g_adv, kBlock, 0, stream>>>(S, L, I, V, k);
        RR_CHECK_LAUNCH(ctx);
    }
    ctx->launches += 1 + 4 * uint64_t(steps);
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
    if (ctx->wave_initial && uint64_t(cam->screen_width) * cam->screen_height < (1ull << 31))
        return gi_initial_wavefront(ctx, scene, cam, p, b, static_cast<cudaStream_t>(stream));
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
