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
#include "rr_wave.cuh"

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

// ── wavefront form of cs_initial ───────────────────────────────────────────
// The same per-pixel computation as ptr_initial_kernel, cut at every ray
// (traversal steps in rr_wave.cuh).
// Each pixel keeps its state in HBM (random-number seed, candidate index,
// segment index, M, w_sum, source pdf, path throughput, suffix radiance, the
// candidate's reconnection vertex, the selected candidate); each step
// advances every pixel with work by one path segment:
//   extend  : closest hit of the step's segment rays (wave_extend_kernel)
//   shade   : the reconnection vertex or a bounce vertex as the inline loop
//             handles it: sky on a miss, the light sample (its shadow ray is
//             queued with the contribution it adds if the light is visible),
//             then the next BSDF direction, or the candidate ends
//   shadow  : any-hit traversal of the step's shadow rays; each adds its
//             contribution (or zero) to its pixel's suffix (wave_shadow_kernel)
//   advance : for every candidate that ended, the resampling step, then the
//             next candidates' first directions (ray into the next step's
//             queue) or, after the last one, the reservoir
// Random numbers are drawn in the inline order (light pick, BSDF pair,
// resampling, next candidate), and the suffix receives the same additions
// in the same order: a light sample's contribution lands in the step's
// shadow stage, before the vertex after it is shaded. Each pixel has at most
// one segment ray and one shadow ray per step, so a pixel takes at most
// num_candidates x max(max_bounces, 1) steps.

struct PtrWave {
    uint4* st;          // (seed, candidate, segment, M)
    float4* acc;        // (w_sum, source pdf, -, -)
    float4* thp;        // path throughput after the segment's vertex
    float4* suf;        // suffix radiance
    float4* rcp;        // the candidate's reconnection vertex
    float4* rcn;        // and its normal
    float4* selp;       // selected candidate: rc_pos, valid
    float4* seln;       // rc_normal
    float4* sels;       // suffix radiance
    float4* qa[2];      // segment rays: (origin, pixel)
    float4* qb[2];      // (direction, -)
    float4* hits;
    float4* sa;         // shadow rays: (origin, pixel)
    float4* sb;         // (direction, t_max)
    float4* sc;         // (contribution, -)
    uint32_t* ended;    // pixel | kRis (the candidate enters resampling)
    uint32_t* cnt;      // kWaveWords per step
    uint32_t n;
};

// The pixel's next candidates from candidate c on: sample_primary_dir until
// one gives a usable direction (the ones that do not are skipped, as the
// inline loop's `continue`). Returns false after the last candidate.
RR_D bool wave_next(const PtrLaunch& L, const PtrImages& I, float3 pp, float3 pn, uint32_t pmat, uint32_t& seed,
                    uint32_t& c, float& src_pdf, float3& o, float3& d) {
    for (; c < L.num_candidates; ++c) {
        const float3 wi0 = sample_primary_dir(I.fitted, pp, pn, pmat, L.grid, seed, src_pdf);
        if (src_pdf <= 1e-6f || dot(pn, wi0) <= 0.0f) continue;
        o = pp + pn * L.ray_bias;
        d = wi0;
        return true;
    }
    return false;
}

// The end of ptr_initial_kernel: the selected candidate's reservoir or an empty one.
RR_D void wave_finish(const PtrLaunch& L, const PtrImages& I, const PtrWave& V, size_t i, float3 pp, float3 pn,
                      const Mat& pm, uint32_t M_count, float w_sum) {
    const float4 sp = V.selp[i];
    if (M_count > 0 && sp.w > 0.5f) {
        Reservoir sel;
        sel.rc_pos = xyz(sp); sel.rc_normal = xyz(V.seln[i]); sel.suffix_rad = xyz(V.sels[i]);
        sel.prefix_thp = f3(1.0f, 1.0f, 1.0f);
        sel.valid = sp.w;
        const float p_hat = target_function(pp, pn, pm, cam_pos(L.cam), sel);
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

__global__ void __launch_bounds__(kBlock) ptrw_begin_kernel(DevScene s, PtrLaunch L, PtrImages I, PtrWave V) {
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
                store_empty(I.rc, i);
            } else {
                I.hc[0][i] = p4;
                I.hc[1][i] = n4;
                V.selp[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                uint32_t c = 0;
                float src_pdf = 0.0f;
                emit = wave_next(L, I, pp, pn, pmat, seed, c, src_pdf, o, d);
                if (emit) {
                    V.st[i] = make_uint4(seed, c, 0u, 0u);
                    V.acc[i] = make_float4(0.0f, src_pdf, 0.0f, 0.0f);
                } else {
                    store_empty(I.rc, i);   // no candidate: M = 0
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

__global__ void __launch_bounds__(kBlock, 4) ptrw_shade_kernel(DevScene s, PtrLaunch L, PtrWave V, uint32_t step) {
    const int cur = step & 1, nxt = cur ^ 1;
    uint32_t* c0 = V.cnt + size_t(step) * kWaveWords;
    uint32_t* c1 = c0 + kWaveWords;
    const uint32_t count = c0[0];
    const uint32_t max_b = L.max_bounces > 1u ? L.max_bounces : 1u;
    const float bias = L.ray_bias;
    const uint32_t warp_first = blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
    for (uint32_t base = warp_first; base < count; base += gridDim.x * blockDim.x) {
        const uint32_t q = base + lane_id();
        bool cont = false, shadow = false, ended = false, ris = false;
        uint32_t pid = 0;
        float3 no = f3(0.0f, 0.0f, 0.0f), nd = no, so = no, sd = no, sc = no;
        float stmax = 0.0f;
        if (q < count) {
            const float4 a = V.qa[cur][q], b = V.qb[cur][q], h = V.hits[q];
            pid = __float_as_uint(a.w);
            const float3 wi = xyz(b);
            uint4 st = V.st[pid];
            uint32_t seed = st.x;
            const uint32_t seg = st.z;
            const uint32_t inst = __float_as_uint(h.z);
            float3 suffix = f3(0.0f, 0.0f, 0.0f), thp = f3(1.0f, 1.0f, 1.0f);
            float3 cur_pos = f3(0.0f, 0.0f, 0.0f), cur_n = cur_pos;
            Mat cur_mat{};
            bool vertex = false;
            if (seg == 0) {
                // the reconnection vertex: a miss drops the candidate
                if (inst == kNoIndex) {
                    ended = true;
                } else {
                    const Surface rc = hit_surface(s, inst, __float_as_uint(h.w), h.x, h.y);
                    float3 rc_n = rc.normal;
                    if (dot(rc_n, wi) > 0.0f) rc_n = -rc_n;
                    const Mat rc_mat = load_mat(s, rc.material);
                    suffix = rc_mat.emissive;
                    const float3 rc_wo = -wi;
                    float3 c;
                    shadow = sample_light_ray(s, rc.pos, rc_n, rc_wo, rc_mat, bias, seed, so, sd, stmax, c);
                    if (shadow) sc = c;
                    else suffix = suffix + f3(0.0f, 0.0f, 0.0f);
                    V.rcp[pid] = make_float4(rc.pos.x, rc.pos.y, rc.pos.z, 0.0f);
                    V.rcn[pid] = make_float4(rc_n.x, rc_n.y, rc_n.z, 0.0f);
                    cur_pos = rc.pos; cur_n = rc_n; cur_mat = rc_mat;
                    vertex = true;
                }
            } else {
                thp = xyz(V.thp[pid]);
                suffix = xyz(V.suf[pid]);
                if (inst == kNoIndex) {
                    suffix = suffix + thp * sky_radiance(wi);
                    ended = ris = true;
                } else {
                    const Surface hs = hit_surface(s, inst, __float_as_uint(h.w), h.x, h.y);
                    float3 hn = hs.normal;
                    if (dot(hn, wi) > 0.0f) hn = -hn;
                    const Mat hm = load_mat(s, hs.material);
                    const float3 hwo = -wi;
                    float3 c;
                    shadow = sample_light_ray(s, hs.pos, hn, hwo, hm, bias, seed, so, sd, stmax, c);
                    if (shadow) sc = thp * c;
                    else suffix = suffix + thp * f3(0.0f, 0.0f, 0.0f);
                    cur_pos = hs.pos; cur_n = hn; cur_mat = hm;
                    vertex = true;
                }
            }
            uint32_t nseg = seg;
            if (vertex) {
                nseg = seg + 1;   // the bounce loop's next index
                if (nseg >= max_b) {
                    ended = ris = true;
                } else {
                    const float u0 = rand_float(seed);
                    const float u1 = rand_float(seed);
                    float3 nwi;
                    float pdf;
                    const float3 f = brdf_sample(-wi, cur_n, cur_mat.base, cur_mat.metallic, cur_mat.roughness, u0,
                                                 u1, nwi, pdf);
                    if (pdf <= 1e-6f || dot(cur_n, nwi) <= 0.0f) {
                        ended = ris = true;
                    } else {
                        const float cos_at = mx(dot(cur_n, nwi), 0.0f);
                        thp = thp * ((f * cos_at) / pdf);
                        if (mx(thp.x, mx(thp.y, thp.z)) <= 0.0f) {
                            ended = ris = true;
                        } else {
                            cont = true;
                            no = cur_pos + cur_n * bias;
                            nd = nwi;
                        }
                    }
                }
                V.thp[pid] = make_float4(thp.x, thp.y, thp.z, 0.0f);
            }
            if (vertex || seg > 0) V.suf[pid] = make_float4(suffix.x, suffix.y, suffix.z, 0.0f);
            st.x = seed;
            st.z = nseg;
            V.st[pid] = st;
        }
        const uint32_t sslot = warp_alloc(shadow, c0 + 2);
        if (shadow) {
            V.sa[sslot] = make_float4(so.x, so.y, so.z, __uint_as_float(pid));
            V.sb[sslot] = make_float4(sd.x, sd.y, sd.z, stmax);
            V.sc[sslot] = make_float4(sc.x, sc.y, sc.z, 0.0f);
        }
        const uint32_t rslot = warp_alloc(cont, c1);
        if (cont) {
            V.qa[nxt][rslot] = make_float4(no.x, no.y, no.z, __uint_as_float(pid));
            V.qb[nxt][rslot] = make_float4(nd.x, nd.y, nd.z, 0.0f);
        }
        const uint32_t eslot = warp_alloc(ended, c0 + 4);
        if (ended) V.ended[eslot] = pid | (ris ? kRis : 0u);
    }
}

__global__ void __launch_bounds__(kBlock) ptrw_advance_kernel(DevScene s, PtrLaunch L, PtrImages I, PtrWave V,
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
            uint4 st = V.st[pid];
            uint32_t seed = st.x, c = st.y, M_count = st.w;
            const float4 acc = V.acc[pid];
            float w_sum = acc.x;
            float src_pdf = acc.y;
            float4 p4, n4;
            float3 pp, pn;
            uint32_t pmat;
            load_surface(s, I.gpos, I.gnrm, pid, p4, n4, pp, pn, pmat);
            const Mat pm = load_mat(s, pmat);
            if (e & kRis) {
                Reservoir cand;
                cand.rc_pos = xyz(V.rcp[pid]); cand.rc_normal = xyz(V.rcn[pid]); cand.suffix_rad = xyz(V.suf[pid]);
                cand.prefix_thp = f3(1.0f, 1.0f, 1.0f);
                cand.M = 1u; cand.W = 0.0f; cand.w_sum = 0.0f; cand.valid = 1.0f;
                const float p_hat = target_function(pp, pn, pm, cp, cand);
                const float3 delta = cand.rc_pos - pp;
                if (!(p_hat <= 0.0f) && !(dot(delta, delta) <= 1e-8f)) {
                    const float weight = p_hat / mx(src_pdf, 1e-6f);
                    w_sum += weight;
                    M_count++;
                    if (w_sum > 0.0f && rand_float(seed) < weight / w_sum) {
                        V.selp[pid] = make_float4(cand.rc_pos.x, cand.rc_pos.y, cand.rc_pos.z, 1.0f);
                        V.seln[pid] = make_float4(cand.rc_normal.x, cand.rc_normal.y, cand.rc_normal.z, 0.0f);
                        V.sels[pid] = make_float4(cand.suffix_rad.x, cand.suffix_rad.y, cand.suffix_rad.z, 0.0f);
                    }
                }
            }
            ++c;
            emit = wave_next(L, I, pp, pn, pmat, seed, c, src_pdf, o, d);
            if (emit) {
                V.st[pid] = make_uint4(seed, c, 0u, M_count);
                V.acc[pid] = make_float4(w_sum, src_pdf, 0.0f, 0.0f);
            } else {
                wave_finish(L, I, V, pid, pp, pn, pm, M_count, w_sum);
            }
        }
        const uint32_t slot = warp_alloc(emit, c1);
        if (emit) {
            V.qa[nxt][slot] = make_float4(o.x, o.y, o.z, __uint_as_float(pid));
            V.qb[nxt][slot] = make_float4(d.x, d.y, d.z, 0.0f);
        }
    }
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

constexpr int kWaveArrays = 9;   // st, acc, thp, suf, rcp, rcn, selp, seln, sels

// cs_initial as the wavefront of steps above: one launch to start every
// pixel, then per step extend, shade, shadow and advance.
rr_status ptr_initial_wavefront(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                const rr_restir_pt_params* p, const rr_restir_pt_images* b, cudaStream_t stream) {
    const size_t n = size_t(cam->screen_width) * cam->screen_height;
    rr_status st = ensure_queues(ctx, n);
    if (st != RR_OK) return st;
    const uint32_t max_b = std::max(p->max_bounces, 1u);
    const uint64_t steps64 = uint64_t(p->num_initial_candidates) * max_b;
    if (steps64 > (1u << 20)) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "ReSTIR PT: too many candidates x bounces");
    const uint32_t steps = uint32_t(steps64);
    float4* a = nullptr;
    uint32_t* cnt = nullptr;
    if ((st = wave_scratch(ctx, n, kWaveArrays, steps, stream, &a, &cnt)) != RR_OK) return st;
    PtrWave V;
    V.st = reinterpret_cast<uint4*>(a);
    V.acc = a + n; V.thp = a + 2 * n; V.suf = a + 3 * n; V.rcp = a + 4 * n; V.rcn = a + 5 * n;
    V.selp = a + 6 * n; V.seln = a + 7 * n; V.sels = a + 8 * n;
    rr_pt_queues& q = ctx->pt;
    V.qa[0] = q.ray_a[0]; V.qa[1] = q.ray_a[1];
    V.qb[0] = q.ray_b[0]; V.qb[1] = q.ray_b[1];
    V.hits = q.hits;
    V.sa = q.shadow_a; V.sb = q.shadow_b; V.sc = q.shadow_c;
    V.ended = reinterpret_cast<uint32_t*>(q.ray_c[0]);   // n words fit in n float4
    V.cnt = cnt;
    V.n = uint32_t(n);
    const DevScene& S = scene->dev;
    const PtrLaunch L = make_launch(cam, p);
    const PtrImages I = make_images(b);
    const int g_begin = std::min<int>(persistent_grid(ctx, reinterpret_cast<const void*>(ptrw_begin_kernel)),
                                      int((n + kBlock - 1) / kBlock));
    ptrw_begin_kernel<<<g_begin, kBlock, 0, stream>>>(S, L, I, V);
    RR_CHECK_LAUNCH(ctx);
    const int g_ext = persistent_grid(ctx, reinterpret_cast<const void*>(wave_extend_kernel));
    const int g_sh = persistent_grid(ctx, reinterpret_cast<const void*>(wave_shadow_kernel));
    const int g_shade = std::min<int>(persistent_grid(ctx, reinterpret_cast<const void*>(ptrw_shade_kernel)),
                                      int((n + kBlock - 1) / kBlock));
    const int g_adv = std::min<int>(persistent_grid(ctx, reinterpret_cast<const void*>(ptrw_advance_kernel)),
                                    int((n + kBlock - 1) / kBlock));
    for (uint32_t k = 0; k < steps; ++k) {
        uint32_t* c0 = cnt + size_t(k) * kWaveWords;
        wave_extend_kernel<<<g_ext, kBlock, 0, stream>>>(S, V.qa[k & 1], V.qb[k & 1], V.hits, c0, L.ray_bias);
        RR_CHECK_LAUNCH(ctx);
        ptrw_shade_kernel<<<g_shade, kBlock, 0, stream>>>(S, L, V, k);
        RR_CHECK_LAUNCH(ctx);
        wave_shadow_kernel<<<g_sh, kBlock, 0, stream>>>(S, V.sa, V.sb, V.sc, V.suf, c0, L.ray_bias);
        RR_CHECK_LAUNCH(ctx);
        ptrw_advance_kernel<<<g_adv, kBlock, 0, stream>>>(S, L, I, V, k);
        RR_CHECK_LAUNCH(ctx);
    }
    ctx->launches += 1 + 4 * uint64_t(steps);
    return RR_OK;
}

} // namespace
} // namespace rr

using namespace rr;

extern "C" rr_status rr_reuse_set_wavefront(rr_ctx* ctx, int enable) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    ctx->wave_initial = enable != 0;
    return RR_OK;
}

extern "C" rr_status rr_restir_pt_initial(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                          const rr_restir_pt_params* p, const rr_restir_pt_images* b,
                                          void* stream) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    rr_status st = check(ctx, scene, cam, p, b, kInitial);
    if (st != RR_OK) return st;
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    if (ctx->wave_initial && uint64_t(cam->screen_width) * cam->screen_height < (1ull << 31))
        return ptr_initial_wavefront(ctx, scene, cam, p, b, static_cast<cudaStream_t>(stream));
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
