// guided.cu — guided wavefront path tracer and the dense vMF-mixture grid guide.
//
// The guided tracer reuses the reference stages (raygen, extend, shadow,
// NEE of pathtracer.slang:124-177, Russian roulette of :252-257) and replaces
// brdf_sample at each bounce by one-sample MIS between a guide mixture and
// brdf_sample. Each vertex that continues records (position, normal, wo,
// sampled wi, sampling pdf, path throughput after the vertex); the next stage
// stores the radiance gathered so far, and the resolve pass turns the final
// radiance into one training sample per vertex with weight
//     w = L_in(wi) / pdf,  L_in = (L_final - L_before) / throughput_after
// (luminances), an unbiased sample of the incident-radiance distribution.
//
// Grid guide: grid_resolution^3 cells over the guide bounds, 8 vMF lobes per
// cell. rr_guide_update sorts the samples by (cell, vertex id) and runs one
// EM iteration per cell: responsibilities under the cell's current mixture,
// sufficient statistics (sum w*gamma, sum w*gamma*omega) summed in FP64 in a
// fixed order (chunks of a cell's samples, one warp each, then the chunks in
// order) with exponential forgetting, then refits weights, mean directions and
// concentrations (Banerjee's closed form, as GuidingGrid.slang:124-131).

#include "rr_wavefront.cuh"
#include "rr_vmf.cuh"
#include "rr_guide.h"
#include "rr_batch.h"

#include "rr_cellsort.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>

namespace rr {
namespace {

RR_D float lum709(float3 c) { return 0.2126f * c.x + 0.7152f * c.y + 0.0722f * c.z; }

struct GuidedLaunch {
    uint32_t bounce, last, paths, lobes;
    float alpha;
    GridView grid;
    const float4* mix;        // MLP mode: per queue slot, kMaxLobes lobes + 2 float4 of weights
    float4* rec0;             // (pos, pdf)
    float4* rec1;             // (wi, throughput luminance after the vertex)
    float4* rec2;             // (normal, radiance luminance gathered before the vertex's continuation)
    float4* rec3;             // (wo, 0)
};

RR_D void load_mixture_grid(const GridView& g, float3 p, VmfMixture& m, bool& valid) {
    const uint32_t cell = grid_cell(g, p);
    float wsum = 0.0f;
    #pragma unroll
    for (int j = 0; j < kMaxLobes; ++j) {
        m.lobe[j] = __ldg(g.lobes + size_t(cell) * kMaxLobes + j);
        m.weight[j] = __ldg(g.weights + size_t(cell) * kMaxLobes + j);
        wsum += m.weight[j];
    }
    valid = wsum > 0.0f;
}

RR_D void load_mixture_slot(const float4* mix, uint32_t slot, VmfMixture& m, bool& valid) {
    const float4* base = mix + size_t(slot) * (kMaxLobes + 2);
    #pragma unroll
    for (int j = 0; j < kMaxLobes; ++j) m.lobe[j] = base[j];
    const float4 w0 = base[kMaxLobes], w1 = base[kMaxLobes + 1];
    m.weight[0] = w0.x; m.weight[1] = w0.y; m.weight[2] = w0.z; m.weight[3] = w0.w;
    m.weight[4] = w1.x; m.weight[5] = w1.y; m.weight[6] = w1.z; m.weight[7] = w1.w;
    float wsum = 0.0f;
    #pragma unroll
    for (int j = 0; j < kMaxLobes; ++j) wsum += m.weight[j];
    valid = wsum > 0.0f;
}

// Surface inputs of the MLP guide for every queued ray that hit a
// non-emissive surface: (pos, 1), (normal toward wo, valid), (wo, 0).
__global__ void __launch_bounds__(kBlock) guided_surface_kernel(DevScene s, const float4* __restrict__ qb,
                                                                const float4* __restrict__ hits,
                                                                float4* __restrict__ surf,
                                                                const uint32_t* count_ptr) {
    const uint32_t count = *count_ptr;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float4 h = hits[i];
        const uint32_t inst = __float_as_uint(h.z);
        float4 a = make_float4(0, 0, 0, 0), b = make_float4(0, 0, 0, 0), c = make_float4(0, 0, 0, 0);
        if (inst != kNoIndex) {
            const Surface sf = hit_surface(s, inst, __float_as_uint(h.w), h.x, h.y);
            const float4 m1 = __ldg(s.materials + sf.material * 2 + 1);
            if (!(m1.x > 0.0f || m1.y > 0.0f || m1.z > 0.0f)) {
                const float4 qd = qb[i];
                const float3 wo = -f3(qd.x, qd.y, qd.z);
                float3 n = sf.normal;
                if (dot(n, wo) < 0.0f) n = -n;
                a = make_float4(sf.pos.x, sf.pos.y, sf.pos.z, 1.0f);
                b = make_float4(n.x, n.y, n.z, 1.0f);
                c = make_float4(wo.x, wo.y, wo.z, 0.0f);
            }
        }
        surf[size_t(i) * 3] = a; surf[size_t(i) * 3 + 1] = b; surf[size_t(i) * 3 + 2] = c;
    }
}

// A scene's guide as the shade stage uses it.
struct GuideRefs {
    GridView grid;
    float4* rec0;
    float4* rec1;
    float4* rec2;
    float4* rec3;
    uint32_t paths;
    float alpha;
};

// Shade stage of the guided tracer (cf. shade_kernel in pathtracer.cu).
// SlotMixture: the mixture of queue entry i is in G.mix at slot i, or
// (Multi) at slot_map[i] (~0: none). Multi: a batch of scenes; a ray's scene
// index is in c.w, its scene is table[index], its image outs[index] and its
// guide gtab[index]; the index is carried on to the next queues.
// Emit: RR_PT_FLAG_EMITTERS (single scene): next-event estimation also over
// the emissive triangles, as shade_ray_emitters in pathtracer.cu, with the
// bounce's density being the guided mixture alpha p_guide + (1 - alpha)
// p_act (no actual/ref factor: the estimator is unbiased for the rendering
// equation), carried on in the ray record's .w for the MIS weight of an
// emissive surface the bounce reaches.
RR_D float emitter_pdf(float p_group, float lum, float total, float d2, float cos_y) {
    return p_group * (lum / total) * d2 / cos_y;
}

template <bool SlotMixture, bool Multi, bool Emit = false>
__global__ void __launch_bounds__(kBlock, 4) guided_shade_kernel(DevScene s0, GuidedLaunch G,
                                                              const DevScene* __restrict__ table,
                                                              float4* const* __restrict__ outs,
                                                              const GuideEntry* __restrict__ gtab,
                                                              const uint32_t* __restrict__ slot_map,
                                                              const float4* __restrict__ qa,
                                                              const float4* __restrict__ qb,
                                                              const float4* __restrict__ qc,
                                                              const float4* __restrict__ hits,
                                                              float4* na, float4* nb, float4* nc,
                                                              float4* sa, float4* sb, float4* sc,
                                                              float4* __restrict__ out0,
                                                              const uint32_t* count_ptr,
                                                              uint32_t* next_count, uint32_t* shadow_count) {
    const uint32_t count = *count_ptr;
    const uint32_t warp_first = blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = warp_first; base < count; base += stride) {
        const uint32_t i = base + lane_id();
        bool cont = false, emit_shadow = false;
        uint32_t pid = 0, seed = 0, sid = 0;
        float3 new_o = f3(0, 0, 0), wi = f3(0, 0, 0), thp = f3(0, 0, 0);
        float3 sh_o = f3(0, 0, 0), sh_d = f3(0, 0, 0), contrib = f3(0, 0, 0);
        float sh_tmax = 0.0f;
        float pdf_next = 0.0f;
        if (i < count) {
            const float4 a = qa[i], b = qb[i], c = qc[i];
            const float4 h = hits[i];
            if constexpr (Multi) sid = __float_as_uint(c.w);
            const DevScene& s = Multi ? table[sid] : s0;
            float4* const out = Multi ? outs[sid] : out0;
            GuideRefs R;
            if constexpr (Multi) {
                const GuideEntry& E = gtab[sid];
                R = GuideRefs{E.grid, E.rec[0], E.rec[1], E.rec[2], E.rec[3], E.paths, E.alpha};
            } else {
                R = GuideRefs{G.grid, G.rec0, G.rec1, G.rec2, G.rec3, G.paths, G.alpha};
            }
            pid = __float_as_uint(a.w);
            seed = __float_as_uint(b.w);
            const float3 ray_dir = f3(b.x, b.y, b.z);
            thp = f3(c.x, c.y, c.z);
            float4 o = out[pid];
            if (G.bounce > 0)  // radiance gathered before the previous vertex's continuation
                reinterpret_cast<float*>(R.rec2 + size_t(G.bounce - 1) * R.paths + pid)[3] = lum709(xyz(o));
            const uint32_t inst = __float_as_uint(h.z);
            if (inst == kNoIndex) {
                const float3 L = thp * sky_radiance(ray_dir);
                o.x = o.x + L.x; o.y = o.y + L.y; o.z = o.z + L.z;
                out[pid] = o;
            } else {
                const Surface sf = hit_surface(s, inst, __float_as_uint(h.w), h.x, h.y);
                const float4 m0 = __ldg(s.materials + sf.material * 2);
                const float4 m1 = __ldg(s.materials + sf.material * 2 + 1);
                if (m1.x > 0.0f || m1.y > 0.0f || m1.z > 0.0f) {
                    float w = 1.0f;
                    if constexpr (Emit) {
                        const float prev_pdf = c.w;
                        if (prev_pdf > 0.0f) {
                            const uint32_t NL = s.num_lights, NE = s.num_emitters;
                            const float pe = NE == 0 ? 0.0f : (NL == 0 ? 1.0f : 0.5f);
                            const float3 ng = hit_geometric_normal(s, inst, __float_as_uint(h.w));
                            const float cos_y = fabsf(dot(ng, ray_dir));
                            const float3 dd = sf.pos - f3(a.x, a.y, a.z);
                            const float pl = cos_y > 0.0f ? emitter_pdf(pe, lum709(f3(m1.x, m1.y, m1.z)), s.emit_total,
                                                                        dot(dd, dd), cos_y)
                                                          : 0.0f;
                            const float aa = prev_pdf * prev_pdf;
                            w = aa / (aa + pl * pl);
                        }
                    }
                    const float3 L = thp * (f3(m1.x, m1.y, m1.z) * w);
                    o.x = o.x + L.x; o.y = o.y + L.y; o.z = o.z + L.z;
                    out[pid] = o;
                } else {
                    const float3 wo = -ray_dir;
                    float3 n = sf.normal;
                    if (dot(n, wo) < 0.0f) n = -n;
                    const float3 base_c = f3(m0.x, m0.y, m0.z);
                    const float metallic = m0.w, roughness = m1.w;
                    VmfMixture mix;
                    bool valid = false;
                    if (!G.last) {
                        if constexpr (SlotMixture) {
                            const uint32_t slot = Multi ? slot_map[i] : i;
                            if (slot != kNoIndex) load_mixture_slot(G.mix, slot, mix, valid);
                        } else {
                            load_mixture_grid(R.grid, sf.pos, mix, valid);
                        }
                    }
                    bool nee_done = false;
                    if constexpr (Emit) {
                        const uint32_t NL = s.num_lights, NE = s.num_emitters;
                        const float pe = NE == 0 ? 0.0f : (NL == 0 ? 1.0f : 0.5f);
                        if (NE > 0 && (NL == 0 || rand_float(seed) < 0.5f)) {
                            nee_done = true;
                            const float u = rand_float(seed);
                            const float uc = rand_float(seed);
                            const float u1 = rand_float(seed);
                            const float u2 = rand_float(seed);
                            const uint32_t k = emitter_pick(s, u, uc);
                            const float4 e0 = __ldg(s.emitters + k * 3), e1 = __ldg(s.emitters + k * 3 + 1);
                            const float4 e2 = __ldg(s.emitters + k * 3 + 2);
                            const float3 E1 = xyz(e1), E2 = xyz(e2);
                            const float3 Le = f3(e0.w, e1.w, e2.w);
                            const float su = sqrtf(u1);
                            const float3 y = xyz(e0) + E1 * (su * (1.0f - u2)) + E2 * (su * u2);
                            const float3 to = y - sf.pos;
                            const float d2 = dot(to, to);
                            const float dist = sqrtf(d2);
                            const float3 l = to / dist;
                            const float cos_x = dot(n, l);
                            const float cos_y = fabsf(dot(normalize(cross(E1, E2)), l));
                            if (cos_x > 0.0f && cos_y > 0.0f && d2 > 0.0f) {
                                const float pl = emitter_pdf(pe, lum709(Le), s.emit_total, d2, cos_y);
                                float wl = 1.0f;   // the last vertex traces no bounce
                                if (!G.last) {
                                    const float alpha = valid ? R.alpha : 0.0f;
                                    const float pg = valid ? mixture_pdf(mix, G.lobes, l) : 0.0f;
                                    const float pb = alpha * pg + (1.0f - alpha) *
                                                     brdf_sample_pdfs(wo, n, base_c, metallic, roughness, l).actual;
                                    const float aa = pl * pl;
                                    wl = aa / (aa + pb * pb);
                                }
                                const float3 f = brdf_eval(n, wo, l, base_c, metallic, roughness);
                                contrib = thp * ((f * Le) * (cos_x * wl / pl));
                                sh_o = sf.pos + n * 1e-4f;
                                sh_d = l;
                                sh_tmax = dist - 0.01f;
                                emit_shadow = true;
                            }
                        }
                    }
                    if (!nee_done && s.num_lights > 0) {  // NEE as the reference (the GpuLight group)
                        const uint32_t N = s.num_lights;
                        const uint32_t li = uint32_t(rand_float(seed) * float(N)) % N;
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
                            float scale = float(N);
                            if constexpr (Emit) {
                                if (s.num_emitters > 0) scale = float(N) / 0.5f;   // the GpuLight group's probability
                            }
                            contrib = thp * ((((brdf_val * irr) * n_dot_l) * mis) * scale);
                            sh_o = sf.pos + n * 1e-4f;
                            sh_d = ldir;
                            sh_tmax = dist - 0.01f;
                            emit_shadow = true;
                        }
                    }
                    if (!G.last) {
                        const float alpha = valid ? R.alpha : 0.0f;
                        const float u_sel = rand_float(seed);
                        const float u0 = rand_float(seed);
                        const float u1 = rand_float(seed);
                        bool rejected = false;
                        if (u_sel < alpha) {
                            const float u2 = rand_float(seed);
                            wi = mixture_sample(mix, G.lobes, u0, u1, u2);
                        } else {
                            // brdf_sample rejects a VNDF direction below the
                            // surface by returning f = 0 (and wi = +y): the
                            // sample carries nothing, so the path ends here.
                            float pdf_b;
                            const float3 fb = brdf_sample(wo, n, base_c, metallic, roughness, u0, u1, wi, pdf_b);
                            rejected = fb.x == 0.0f && fb.y == 0.0f && fb.z == 0.0f;
                        }
                        const float cos_i = dot(n, wi);
                        float pdf = 0.0f, ratio = 0.0f;
                        if (cos_i > 0.0f && !rejected) {
                            const BrdfPdfs pb = brdf_sample_pdfs(wo, n, base_c, metallic, roughness, wi);
                            const float pg = valid ? mixture_pdf(mix, G.lobes, wi) : 0.0f;
                            pdf = alpha * pg + (1.0f - alpha) * pb.actual;
                            ratio = Emit ? 1.0f : pb.actual / pb.ref;
                        }
                        if (pdf > 1e-6f) {
                            const float3 f = brdf_eval(n, wo, wi, base_c, metallic, roughness);
                            thp = thp * ((f * cos_i) * (ratio / pdf));
                            bool alive = true;
                            if (G.bounce >= 3) {
                                const float survive = mn(mx(thp.x, mx(thp.y, thp.z)), 0.95f);
                                if (rand_float(seed) > survive) alive = false;
                                else thp = thp / survive;
                            }
                            if (alive) {
                                cont = true;
                                pdf_next = pdf;
                                new_o = sf.pos + n * 1e-4f;
                                const size_t r = size_t(G.bounce) * R.paths + pid;
                                R.rec0[r] = make_float4(sf.pos.x, sf.pos.y, sf.pos.z, pdf);
                                R.rec1[r] = make_float4(wi.x, wi.y, wi.z, lum709(thp));
                                R.rec2[r] = make_float4(n.x, n.y, n.z, __int_as_float(-1));
                                R.rec3[r] = make_float4(wo.x, wo.y, wo.z, 0.0f);
                            }
                        }
                    }
                }
            }
        }
        const float tag = Multi ? __uint_as_float(sid) : 0.0f;
        const uint32_t sslot = warp_alloc(emit_shadow, shadow_count);
        if (emit_shadow) {
            sa[sslot] = make_float4(sh_o.x, sh_o.y, sh_o.z, __uint_as_float(pid));
            sb[sslot] = make_float4(sh_d.x, sh_d.y, sh_d.z, sh_tmax);
            sc[sslot] = make_float4(contrib.x, contrib.y, contrib.z, tag);
        }
        const uint32_t rslot = warp_alloc(cont, next_count);
        if (cont) {
            na[rslot] = make_float4(new_o.x, new_o.y, new_o.z, __uint_as_float(pid));
            nb[rslot] = make_float4(wi.x, wi.y, wi.z, __uint_as_float(seed));
            nc[rslot] = make_float4(thp.x, thp.y, thp.z, Emit ? pdf_next : tag);
        }
    }
}

// One training sample per recorded vertex whose continuation was traced:
// record r (bounce r / paths, path r % paths) gives a sample when its
// continuation brought back positive radiance.
__device__ __forceinline__ bool resolve_record(const float4* __restrict__ out, const float4* __restrict__ rec0,
                                               const float4* __restrict__ rec1, const float4* __restrict__ rec2,
                                               const float4* __restrict__ rec3, uint32_t paths, uint32_t r,
                                               float4& s0, float4& s1, float4& s2, float4& s3) {
    const float4 c = rec2[r];
    const float before = c.w;
    if (!(before >= 0.0f)) return false;   // NaN (never filled) fails this test
    const float4 a = rec0[r], b = rec1[r];
    const uint32_t pid = r % paths;
    const float final_l = lum709(xyz(out[pid]));
    const float lin = mx(final_l - before, 0.0f) / mx(b.w, 1e-20f);
    const float w = lin / a.w;
    if (!(w > 0.0f && w < 3.0e38f)) return false;
    s0 = make_float4(a.x, a.y, a.z, w);
    s1 = make_float4(b.x, b.y, b.z, __uint_as_float(r));
    s2 = make_float4(c.x, c.y, c.z, 0.0f);
    const float4 d = rec3[r];
    s3 = make_float4(d.x, d.y, d.z, 0.0f);
    return true;
}

// The samples are compacted in record order, without a shared counter: tile
// t of kResolveTile records counts its samples (resolve_count_kernel), an
// exclusive scan turns the counts into the tiles' first slots, and
// resolve_write_kernel writes each tile's samples from there, round by round
// (kResolveItems rounds of kBlock consecutive records; within a round, warp
// by warp and lane by lane). The sample order, and so everything trained
// from it, does not depend on timing.
constexpr uint32_t kResolveItems = 8;
constexpr uint32_t kResolveTile = kBlock * kResolveItems;

__global__ void __launch_bounds__(kBlock) resolve_count_kernel(const float4* __restrict__ out,
                                                               const float4* __restrict__ rec0,
                                                               const float4* __restrict__ rec1,
                                                               const float4* __restrict__ rec2,
                                                               const float4* __restrict__ rec3, uint32_t paths,
                                                               uint32_t total, uint32_t* __restrict__ tile_count) {
    __shared__ uint32_t red[kBlock / 32];
    uint32_t n = 0;
    #pragma unroll 2
    for (uint32_t k = 0; k < kResolveItems; ++k) {
        const uint32_t r = blockIdx.x * kResolveTile + k * kBlock + threadIdx.x;
        float4 s0, s1, s2, s3;
        if (r < total && resolve_record(out, rec0, rec1, rec2, rec3, paths, r, s0, s1, s2, s3)) ++n;
    }
    #pragma unroll
    for (int off = 16; off > 0; off >>= 1) n += __shfl_xor_sync(kFull, n, off);
    if (lane_id() == 0) red[threadIdx.x >> 5] = n;
    __syncthreads();
    if (threadIdx.x == 0) {
        uint32_t t = 0;
        for (int w = 0; w < kBlock / 32; ++w) t += red[w];
        tile_count[blockIdx.x] = t;
    }
}

__global__ void __launch_bounds__(kBlock) resolve_write_kernel(const float4* __restrict__ out,
                                                               const float4* __restrict__ rec0,
                                                               const float4* __restrict__ rec1,
                                                               const float4* __restrict__ rec2,
                                                               const float4* __restrict__ rec3, uint32_t paths,
                                                               uint32_t total, const uint32_t* __restrict__ tile_first,
                                                               GuideSamples S) {
    __shared__ uint32_t wcount[kBlock / 32];
    const uint32_t w = threadIdx.x >> 5;
    uint32_t base = tile_first[blockIdx.x];
    for (uint32_t k = 0; k < kResolveItems; ++k) {
        const uint32_t r = blockIdx.x * kResolveTile + k * kBlock + threadIdx.x;
        float4 s0, s1, s2, s3;
        const bool emit = r < total && resolve_record(out, rec0, rec1, rec2, rec3, paths, r, s0, s1, s2, s3);
        const uint32_t bal = __ballot_sync(kFull, emit);
        if (lane_id() == 0) wcount[w] = __popc(bal);
        __syncthreads();
        uint32_t before = 0, all = 0;
        for (uint32_t v = 0; v < kBlock / 32; ++v) {
            const uint32_t c = wcount[v];
            before += v < w ? c : 0u;
            all += c;
        }
        const uint32_t slot = base + before + __popc(bal & ((1u << lane_id()) - 1u));
        if (emit && slot < S.capacity) {
            S.s0[slot] = s0; S.s1[slot] = s1; S.s2[slot] = s2; S.s3[slot] = s3;
        }
        base += all;
        __syncthreads();
    }
    // the last tile knows the total
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == 0) S.count[0] = base;
}

// ── guided batches ─────────────────────────────────────────────────────────
// Warp-aggregated slot allocation per scene: the lanes that want a slot and
// share a scene index take consecutive slots from one atomic on that scene's
// counter. Returns the lane's offset (counter value before the lane).
__device__ __forceinline__ uint32_t warp_alloc_keyed(bool want, uint32_t key, uint32_t* counters) {
    const uint32_t peers = __match_any_sync(kFull, want ? key : kNoIndex);
    const uint32_t leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (want && lane_id() == leader) base = atomicAdd(counters + key, __popc(peers));
    base = __shfl_sync(kFull, base, leader);
    return base + __popc(peers & ((1u << lane_id()) - 1u));
}

// MLP guides in a batch: the surface inputs of every queued ray that hit a
// non-emissive surface go to its scene's group of slots (group_base[scene]
// onwards; a scene has at most as many queued rays as paths), and slot_map
// records the slot of each queue entry (~0 for none). The grouped forward
// then runs each group through its scene's network.
__global__ void __launch_bounds__(kBlock) guided_surface_batch_kernel(const DevScene* __restrict__ table,
                                                                      const float4* __restrict__ qb,
                                                                      const float4* __restrict__ qc,
                                                                      const float4* __restrict__ hits,
                                                                      const uint32_t* __restrict__ group_base,
                                                                      uint32_t* group_count, float4* __restrict__ surf,
                                                                      uint32_t* __restrict__ slot_map,
                                                                      const uint32_t* count_ptr) {
    const uint32_t count = *count_ptr;
    const uint32_t warp_first = blockIdx.x * blockDim.x + (threadIdx.x & ~31u);
    for (uint32_t base = warp_first; base < count; base += gridDim.x * blockDim.x) {
        const uint32_t i = base + lane_id();
        bool want = false;
        uint32_t sid = 0;
        float4 a = make_float4(0, 0, 0, 0), b = make_float4(0, 0, 0, 0), c = make_float4(0, 0, 0, 0);
        if (i < count) {
            const float4 h = hits[i];
            sid = __float_as_uint(qc[i].w);
            const uint32_t inst = __float_as_uint(h.z);
            if (inst != kNoIndex) {
                const DevScene& s = table[sid];
                const Surface sf = hit_surface(s, inst, __float_as_uint(h.w), h.x, h.y);
                const float4 m1 = __ldg(s.materials + sf.material * 2 + 1);
                if (!(m1.x > 0.0f || m1.y > 0.0f || m1.z > 0.0f)) {
                    const float4 qd = qb[i];
                    const float3 wo = -f3(qd.x, qd.y, qd.z);
                    float3 n = sf.normal;
                    if (dot(n, wo) < 0.0f) n = -n;
                    a = make_float4(sf.pos.x, sf.pos.y, sf.pos.z, 1.0f);
                    b = make_float4(n.x, n.y, n.z, 1.0f);
                    c = make_float4(wo.x, wo.y, wo.z, 0.0f);
                    want = true;
                }
            }
        }
        const uint32_t off = warp_alloc_keyed(want, sid, group_count);
        if (i < count) {
            uint32_t slot = kNoIndex;
            if (want) {
                slot = group_base[sid] + off;
                surf[size_t(slot) * 3] = a; surf[size_t(slot) * 3 + 1] = b; surf[size_t(slot) * 3 + 2] = c;
            }
            slot_map[i] = slot;
        }
    }
}

// The resolve over the records of every scene of a batch: record k of the
// batch is record k - rec_prefix[g] of scene g (the last g with
// rec_prefix[g] <= k); samples go to that scene's guide through its
// counter, in an order that depends on timing (the single-scene resolve
// above compacts in record order).
__global__ void __launch_bounds__(kBlock) resolve_batch_kernel(const GuideEntry* __restrict__ gtab,
                                                               float4* const* __restrict__ outs,
                                                               const unsigned long long* __restrict__ rec_prefix,
                                                               uint32_t scenes) {
    const unsigned long long total = rec_prefix[scenes];
    for (unsigned long long k = (unsigned long long)(blockIdx.x) * blockDim.x + (threadIdx.x & ~31u); k < total;
         k += (unsigned long long)(gridDim.x) * blockDim.x) {
        const unsigned long long rg = k + lane_id();
        bool emit = false;
        uint32_t sid = 0, r = 0;
        float4 s0, s1, s2, s3;
        if (rg < total) {
            uint32_t lo = 0, hi = scenes - 1;
            while (lo < hi) {
                const uint32_t mid = (lo + hi + 1) >> 1;
                if (rec_prefix[mid] <= rg) lo = mid; else hi = mid - 1;
            }
            sid = lo;
            r = uint32_t(rg - rec_prefix[sid]);
            const GuideEntry& E = gtab[sid];
            const float4 c = E.rec[2][r];
            const float before = c.w;
            if (before >= 0.0f) {  // NaN (never filled) fails this test
                const float4 a = E.rec[0][r], b = E.rec[1][r];
                const uint32_t pid = r % E.paths;
                const float final_l = lum709(xyz(outs[sid][pid]));
                const float lin = mx(final_l - before, 0.0f) / mx(b.w, 1e-20f);
                const float w = lin / a.w;
                if (w > 0.0f && w < 3.0e38f) {
                    emit = true;
                    s0 = make_float4(a.x, a.y, a.z, w);
                    s1 = make_float4(b.x, b.y, b.z, __uint_as_float(r));
                    s2 = make_float4(c.x, c.y, c.z, 0.0f);
                    const float4 d = E.rec[3][r];
                    s3 = make_float4(d.x, d.y, d.z, 0.0f);
                }
            }
        }
        // per-scene aggregation onto that scene's sample counter
        const uint32_t peers = __match_any_sync(kFull, emit ? sid : kNoIndex);
        const uint32_t leader = __ffs(peers) - 1;
        uint32_t base = 0;
        if (emit && lane_id() == leader) base = atomicAdd(gtab[sid].S.count, __popc(peers));
        base = __shfl_sync(kFull, base, leader);
        const uint32_t slot = base + __popc(peers & ((1u << lane_id()) - 1u));
        if (emit) {
            const GuideSamples& S = gtab[sid].S;
            if (slot < S.capacity) {
                S.s0[slot] = s0; S.s1[slot] = s1; S.s2[slot] = s2; S.s3[slot] = s3;
            }
        }
    }
}

// ── grid guide update ──────────────────────────────────────────────────────
// Sample i's cell (the sort key) and index (the sorted value).
__global__ void __launch_bounds__(256) grid_keys_kernel(GridView g, GuideSamples S, uint32_t n, uint32_t* keys,
                                                        uint32_t* vals) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    keys[i] = grid_cell(g, xyz(S.s0[i]));
    vals[i] = i;
}

// Each cell's range [start, end) in the cell-sorted sample order.
__global__ void __launch_bounds__(256) grid_ranges_kernel(const uint32_t* keys, uint32_t n, uint32_t* start,
                                                          uint32_t* end) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t c = keys[i];
    if (i == 0 || keys[i - 1] != c) start[c] = i;
    if (i + 1 == n || keys[i + 1] != c) end[c] = i + 1;
}

// The EM update is one batch E-step per frame: every sample's responsibilities
// are taken under the mixture its cell held at the start of the update, so a
// cell's new sufficient statistics are a plain FP64 sum over its samples.
// That sum runs in parallel and in a fixed order: each cell's sorted sample
// range is cut into chunks of kEmChunk samples, one warp sums a chunk (lane l
// takes samples l, l+32, ... and the warp reduces with a fixed xor butterfly,
// lane 0's result being kept), and the per-cell M-step adds its chunks in
// chunk order. Run to run the fitted guide is bit-identical.
constexpr uint32_t kEmChunk = 1024;
constexpr int kEmStats = kMaxLobes * 4;   // (s0, s1.xyz) per lobe

// The mixture a cell enters the update with: its fitted lobes, or, for a cell
// never fitted, 8 lobes of kappa 2 on the cube diagonals with equal weights.
RR_D void cell_mixture(const float4* __restrict__ lobes, const float* __restrict__ weights, uint32_t cell,
                       VmfMixture& m) {
    float wsum = 0.0f;
    for (int j = 0; j < kMaxLobes; ++j) {
        m.lobe[j] = lobes[size_t(cell) * kMaxLobes + j];
        m.weight[j] = weights[size_t(cell) * kMaxLobes + j];
        wsum += m.weight[j];
    }
    if (!(wsum > 0.0f)) {
        for (int j = 0; j < kMaxLobes; ++j) {
            const float k = 0.57735026918962576f;
            m.lobe[j] = make_float4((j & 1) ? k : -k, (j & 2) ? k : -k, (j & 4) ? k : -k, 2.0f);
            m.weight[j] = 1.0f / kMaxLobes;
        }
    }
}

__global__ void __launch_bounds__(256) grid_chunk_count_kernel(const uint32_t* __restrict__ start,
                                                               const uint32_t* __restrict__ end, uint32_t cells,
                                                               uint32_t* __restrict__ cnt) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < cells) cnt[c] = (end[c] - start[c] + kEmChunk - 1) / kEmChunk;
}

__global__ void __launch_bounds__(256) grid_chunk_map_kernel(const uint32_t* __restrict__ cnt,
                                                             const uint32_t* __restrict__ off, uint32_t cells,
                                                             uint32_t* __restrict__ chunk_cell) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= cells) return;
    for (uint32_t q = 0; q < cnt[c]; ++q) chunk_cell[off[c] + q] = c;
}

// One warp per chunk; launched with an upper bound of warps, the ones past
// the scanned chunk total return at once.
__global__ void __launch_bounds__(128) grid_chunk_kernel(GridView g, GuideSamples S,
                                                         const uint32_t* __restrict__ order,
                                                         const uint32_t* __restrict__ start,
                                                         const uint32_t* __restrict__ end,
                                                         const uint32_t* __restrict__ cnt,
                                                         const uint32_t* __restrict__ off,
                                                         const uint32_t* __restrict__ chunk_cell,
                                                         double* __restrict__ partial) {
    const uint32_t chunk = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t total = off[g.cells - 1] + cnt[g.cells - 1];
    if (chunk >= total) return;   // whole warps
    const uint32_t cell = chunk_cell[chunk];
    const uint32_t b = start[cell] + (chunk - off[cell]) * kEmChunk;
    const uint32_t e = min(end[cell], b + kEmChunk);
    VmfMixture m;
    cell_mixture(g.lobes, g.weights, cell, m);
    double s0[kMaxLobes], s1x[kMaxLobes], s1y[kMaxLobes], s1z[kMaxLobes];
    for (int j = 0; j < kMaxLobes; ++j) s0[j] = s1x[j] = s1y[j] = s1z[j] = 0.0;
    for (uint32_t k = b + lane; k < e; k += 32) {
        const uint32_t si = order[k];
        const float4 a = S.s0[si];
        const float4 d = S.s1[si];
        const float3 om = f3(d.x, d.y, d.z);
        float gam[kMaxLobes];
        float gsum = 0.0f;
        for (int j = 0; j < kMaxLobes; ++j) {
            gam[j] = m.weight[j] > 0.0f ? m.weight[j] * vmf_pdf(xyz(m.lobe[j]), m.lobe[j].w, om) : 0.0f;
            gsum += gam[j];
        }
        if (!(gsum > 0.0f)) continue;
        const double w = double(a.w);
        for (int j = 0; j < kMaxLobes; ++j) {
            const double r = w * double(gam[j] / gsum);
            s0[j] += r;
            s1x[j] += r * double(om.x);
            s1y[j] += r * double(om.y);
            s1z[j] += r * double(om.z);
        }
    }
    for (int j = 0; j < kMaxLobes; ++j) {
        for (int o = 16; o > 0; o >>= 1) {
            s0[j] += __shfl_xor_sync(0xffffffffu, s0[j], o);
            s1x[j] += __shfl_xor_sync(0xffffffffu, s1x[j], o);
            s1y[j] += __shfl_xor_sync(0xffffffffu, s1y[j], o);
            s1z[j] += __shfl_xor_sync(0xffffffffu, s1z[j], o);
        }
    }
    if (lane == 0) {
        double* out = partial + size_t(chunk) * kEmStats;
        for (int j = 0; j < kMaxLobes; ++j) {
            out[j * 4 + 0] = s0[j]; out[j * 4 + 1] = s1x[j]; out[j * 4 + 2] = s1y[j]; out[j * 4 + 3] = s1z[j];
        }
    }
}

// Per cell: decayed statistics + the cell's chunk sums in chunk order, then
// the M-step (Banerjee kappa, lobe weights = normalised s0).
__global__ void __launch_bounds__(128) grid_em_kernel(GridView g, const uint32_t* __restrict__ cnt,
                                                      const uint32_t* __restrict__ off,
                                                      const double* __restrict__ partial, double* __restrict__ stats,
                                                      float4* lobes, float* weights, float decay,
                                                      uint32_t* valid_cells) {
    const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= g.cells) return;
    const uint32_t nq = cnt[cell];
    if (nq == 0) {  // no new samples: the mixture is kept as it is
        float w = 0.0f;
        for (int j = 0; j < kMaxLobes; ++j) w += weights[size_t(cell) * kMaxLobes + j];
        if (w > 0.0f) atomicAdd(valid_cells, 1u);
        return;
    }
    VmfMixture m;
    cell_mixture(lobes, weights, cell, m);
    double s0[kMaxLobes], s1x[kMaxLobes], s1y[kMaxLobes], s1z[kMaxLobes];
    double* st = stats + size_t(cell) * kEmStats;
    for (int j = 0; j < kMaxLobes; ++j) {
        s0[j] = double(decay) * st[j * 4 + 0];
        s1x[j] = double(decay) * st[j * 4 + 1];
        s1y[j] = double(decay) * st[j * 4 + 2];
        s1z[j] = double(decay) * st[j * 4 + 3];
    }
    for (uint32_t q = 0; q < nq; ++q) {
        const double* p = partial + size_t(off[cell] + q) * kEmStats;
        for (int j = 0; j < kMaxLobes; ++j) {
            s0[j] += p[j * 4 + 0]; s1x[j] += p[j * 4 + 1]; s1y[j] += p[j * 4 + 2]; s1z[j] += p[j * 4 + 3];
        }
    }
    double tot = 0.0;
    for (int j = 0; j < kMaxLobes; ++j) tot += s0[j];
    for (int j = 0; j < kMaxLobes; ++j) {
        st[j * 4 + 0] = s0[j]; st[j * 4 + 1] = s1x[j]; st[j * 4 + 2] = s1y[j]; st[j * 4 + 3] = s1z[j];
        float4 lobe = m.lobe[j];
        float wj = 0.0f;
        if (tot > 0.0 && s0[j] > 0.0) {
            const double len = sqrt(s1x[j] * s1x[j] + s1y[j] * s1y[j] + s1z[j] * s1z[j]);
            double r = len / s0[j];
            r = r < 1e-4 ? 1e-4 : (r > 0.9999 ? 0.9999 : r);
            double kappa = r * (3.0 - r * r) / (1.0 - r * r);
            kappa = kappa < 0.5 ? 0.5 : (kappa > 512.0 ? 512.0 : kappa);
            if (len > 1e-12) lobe = make_float4(float(s1x[j] / len), float(s1y[j] / len), float(s1z[j] / len), float(kappa));
            wj = float(s0[j] / tot);
        }
        lobes[size_t(cell) * kMaxLobes + j] = lobe;
        weights[size_t(cell) * kMaxLobes + j] = wj;
    }
    if (tot > 0.0) atomicAdd(valid_cells, 1u);
}

} // namespace
} // namespace rr

using namespace rr;

// ── host side ──────────────────────────────────────────────────────────────
static rr_status guide_alloc(rr_ctx* ctx, rr_guide* g, void** p, size_t bytes) {
    RR_TRY_CUDA(ctx, cudaMalloc(p, bytes));
    g->allocations.push_back(*p);
    return RR_OK;
}

extern "C" rr_status rr_guide_create(rr_ctx* ctx, const rr_guide_desc* d, rr_guide** out) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!d || !out) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_guide_create: null argument");
    *out = nullptr;
    if (d->kind != RR_GUIDE_GRID && d->kind != RR_GUIDE_MLP)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_guide_create: unknown guide kind %u", d->kind);
    if (d->kind == RR_GUIDE_GRID && (d->grid_resolution == 0 || d->grid_resolution > 256))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "grid_resolution must be 1..256");
    for (int a = 0; a < 3; ++a)
        if (!(d->bounds_max[a] > d->bounds_min[a])) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "empty guide bounds");
    if (d->max_samples == 0 || !(d->alpha >= 0.0f && d->alpha <= 1.0f))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_guide_create: bad max_samples or alpha");
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    rr_guide* g = new rr_guide;
    g->ctx = ctx;
    g->desc = *d;
    rr_status st;
    auto fail = [&](rr_status s) { rr_guide_destroy(g); return s; };
    const uint32_t cap = d->max_samples;
    g->samples.capacity = cap;
    for (int k = 0; k < 4; ++k) {
        void* p;
        if ((st = guide_alloc(ctx, g, &p, size_t(cap) * sizeof(float4))) != RR_OK) return fail(st);
        (&g->samples.s0)[k] = static_cast<float4*>(p);
    }
    {
        void* p;
        if ((st = guide_alloc(ctx, g, &p, sizeof(uint32_t) * 4)) != RR_OK) return fail(st);
        g->samples.count = static_cast<uint32_t*>(p);
        cudaMemset(p, 0, sizeof(uint32_t) * 4);
        const cudaError_t e = cudaMallocHost(&p, sizeof(uint32_t) * 4);
        if (e != cudaSuccess) return fail(rr_fail(ctx, RR_ERR_OUT_OF_MEMORY, "rr_guide_create: %s", cudaGetErrorString(e)));
        g->count_host = static_cast<uint32_t*>(p);
    }
    if (d->kind == RR_GUIDE_GRID) {
        const uint32_t R = d->grid_resolution;
        const size_t cells = size_t(R) * R * R;
        GridView& v = g->grid;
        v.res = R;
        v.cells = uint32_t(cells);
        v.bmin = make_float3(d->bounds_min[0], d->bounds_min[1], d->bounds_min[2]);
        v.scale = make_float3(float(R) / (d->bounds_max[0] - d->bounds_min[0]),
                              float(R) / (d->bounds_max[1] - d->bounds_min[1]),
                              float(R) / (d->bounds_max[2] - d->bounds_min[2]));
        void* p;
        if ((st = guide_alloc(ctx, g, &p, cells * kMaxLobes * sizeof(float4))) != RR_OK) return fail(st);
        v.lobes = static_cast<float4*>(p);
        if ((st = guide_alloc(ctx, g, &p, cells * kMaxLobes * sizeof(float))) != RR_OK) return fail(st);
        v.weights = static_cast<float*>(p);
        if ((st = guide_alloc(ctx, g, &p, cells * kMaxLobes * 4 * sizeof(double))) != RR_OK) return fail(st);
        g->stats64 = static_cast<double*>(p);
        if ((st = guide_alloc(ctx, g, &p, cells * sizeof(uint32_t))) != RR_OK) return fail(st);
        g->cell_start = static_cast<uint32_t*>(p);
        if ((st = guide_alloc(ctx, g, &p, cells * sizeof(uint32_t))) != RR_OK) return fail(st);
        g->cell_end = static_cast<uint32_t*>(p);
        if ((st = guide_alloc(ctx, g, &p, size_t(cap) * 8)) != RR_OK) return fail(st);
        g->keys_in = static_cast<unsigned long long*>(p);
        if ((st = guide_alloc(ctx, g, &p, size_t(cap) * 8)) != RR_OK) return fail(st);
        g->keys_out = static_cast<unsigned long long*>(p);
        if ((st = guide_alloc(ctx, g, &p, size_t(cap) * 4)) != RR_OK) return fail(st);
        g->vals_in = static_cast<uint32_t*>(p);
        if ((st = guide_alloc(ctx, g, &p, size_t(cap) * 4)) != RR_OK) return fail(st);
        g->vals_out = static_cast<uint32_t*>(p);
        // EM chunks: at most one partial chunk per non-empty cell plus cap / kEmChunk full ones
        g->chunk_capacity = cells + cap / kEmChunk + 1;
        if ((st = guide_alloc(ctx, g, &p, cells * sizeof(uint32_t))) != RR_OK) return fail(st);
        g->chunk_cnt = static_cast<uint32_t*>(p);
        if ((st = guide_alloc(ctx, g, &p, cells * sizeof(uint32_t))) != RR_OK) return fail(st);
        g->chunk_off = static_cast<uint32_t*>(p);
        if ((st = guide_alloc(ctx, g, &p, g->chunk_capacity * sizeof(uint32_t))) != RR_OK) return fail(st);
        g->chunk_cell = static_cast<uint32_t*>(p);
        if ((st = guide_alloc(ctx, g, &p, g->chunk_capacity * kEmStats * sizeof(double))) != RR_OK) return fail(st);
        g->chunk_partial = static_cast<double*>(p);
        // the cell sort's per-(digit, tile) counts
        const size_t hist = size_t(kSortBins) * ((cap + kSortTile - 1) / kSortTile);
        if ((st = guide_alloc(ctx, g, &p, hist * sizeof(uint32_t))) != RR_OK) return fail(st);
        g->sort_tmp = p;
        g->sort_tmp_bytes = hist * sizeof(uint32_t);
        if (std::max<size_t>(hist, cells) > size_t(kScanChunk) * kScanThreads) return fail(RR_ERR_UNSUPPORTED);
        const size_t sums = std::max<size_t>(hist, cells) / kScanChunk + 1;
        if ((st = guide_alloc(ctx, g, &p, sums * sizeof(uint32_t))) != RR_OK) return fail(st);
        g->scan_sums = static_cast<uint32_t*>(p);
        g->key_bits = 1;
        while ((size_t(1) << g->key_bits) < cells) ++g->key_bits;
    } else {
        if ((st = rr_mlp_guide_init(ctx, g)) != RR_OK) return fail(st);
    }
    if ((st = rr_guide_reset(ctx, g, nullptr)) != RR_OK) return fail(st);
    RR_TRY_CUDA(ctx, cudaDeviceSynchronize());
    *out = g;
    return RR_OK;
}

extern "C" rr_status rr_guide_destroy(rr_guide* g) {
    if (!g) return RR_ERR_INVALID_ARGUMENT;
    if (g->ctx) cudaSetDevice(g->ctx->device);
    for (void* p : g->allocations) cudaFree(p);
    if (g->count_host) cudaFreeHost(g->count_host);
    if (g->ev0) cudaEventDestroy(g->ev0);
    if (g->ev1) cudaEventDestroy(g->ev1);
    delete g;
    return RR_OK;
}

extern "C" rr_status rr_guide_reset(rr_ctx* ctx, rr_guide* g, void* stream_v) {
    if (!ctx || !g) return RR_ERR_INVALID_ARGUMENT;
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    RR_TRY_CUDA(ctx, cudaMemsetAsync(g->samples.count, 0, sizeof(uint32_t) * 4, stream));
    if (g->desc.kind == RR_GUIDE_GRID) {
        const size_t cells = g->grid.cells;
        RR_TRY_CUDA(ctx, cudaMemsetAsync(g->grid.lobes, 0, cells * kMaxLobes * sizeof(float4), stream));
        RR_TRY_CUDA(ctx, cudaMemsetAsync(g->grid.weights, 0, cells * kMaxLobes * sizeof(float), stream));
        RR_TRY_CUDA(ctx, cudaMemsetAsync(g->stats64, 0, cells * kMaxLobes * 4 * sizeof(double), stream));
    } else {
        rr_status st = rr_mlp_guide_reset(ctx, g, stream);
        if (st != RR_OK) return st;
    }
    g->stats = rr_guide_stats{};
    return RR_OK;
}

static rr_status ensure_records(rr_ctx* ctx, rr_guide* g, size_t paths, uint32_t bounces) {
    const size_t need = paths * bounces;
    if (g->rec_capacity >= need) return RR_OK;
    for (int k = 0; k < 4; ++k) { cudaFree(g->rec[k]); g->rec[k] = nullptr; }
    cudaFree(g->resolve_first);
    cudaFree(g->resolve_sums);
    g->resolve_first = g->resolve_sums = nullptr;
    g->rec_capacity = 0;
    if (need >= (size_t(1) << 32))
        return rr_fail(ctx, RR_ERR_UNSUPPORTED, "guided execute: paths x bounces must be below 2^32");
    for (int k = 0; k < 4; ++k) RR_TRY_CUDA(ctx, cudaMalloc(&g->rec[k], need * sizeof(float4)));
    // the resolve's per-tile counts / first slots and its scan's chunk sums
    const size_t tiles = (need + kResolveTile - 1) / kResolveTile + 1;
    RR_TRY_CUDA(ctx, cudaMalloc(&g->resolve_first, tiles * sizeof(uint32_t)));
    RR_TRY_CUDA(ctx, cudaMalloc(&g->resolve_sums, (tiles / kScanChunk + 2) * sizeof(uint32_t)));
    g->rec_capacity = need;
    return RR_OK;
}

extern "C" rr_status rr_guided_pathtracer_execute(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* cam,
                                                  const rr_pt_params* p, rr_guide* g, float* radiance_out,
                                                  void* stream_v) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!scene || !cam || !p || !g || !radiance_out)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_guided_pathtracer_execute: null argument");
    const uint32_t W = cam->screen_width, H = cam->screen_height;
    if (W == 0 || H == 0 || p->spp == 0 || p->max_bounces == 0 || p->max_bounces > uint32_t(kMaxBounces))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_guided_pathtracer_execute: bad size or bounces");
    const uint64_t n64 = uint64_t(W) * H * p->spp;
    if (n64 >= (1ull << 31) || n64 * p->max_bounces >= (1ull << 32))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_guided_pathtracer_execute: too many paths");
    const size_t n = size_t(n64);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    rr_status st = ensure_queues(ctx, n);
    if (st != RR_OK) return st;
    if ((st = ensure_records(ctx, g, n, p->max_bounces)) != RR_OK) return st;
    const bool mlp = g->desc.kind == RR_GUIDE_MLP;
    if (mlp && (st = rr_mlp_guide_ensure(ctx, g, n)) != RR_OK) return st;
    rr_pt_queues& q = ctx->pt;
    uint32_t* C = ctx->counters;
    RR_TRY_CUDA(ctx, cudaMemsetAsync(C, 0, sizeof(uint32_t) * kCounterWords, stream));
    RR_TRY_CUDA(ctx, cudaMemsetAsync(g->samples.count, 0, sizeof(uint32_t) * 4, stream));
    // unfilled records read as NaN and are skipped by the resolve pass
    RR_TRY_CUDA(ctx, cudaMemsetAsync(g->rec[2], 0xff, n * p->max_bounces * sizeof(float4), stream));

    PtLaunch L;
    L.cam = *cam;
    L.frame_seed = p->frame_seed;
    L.spp = p->spp;
    L.width = W; L.height = H;
    L.tiles_x = (W + 7) / 8;
    L.tiles_per_image = L.tiles_x * ((H + 3) / 4);
    float4* out = reinterpret_cast<float4*>(radiance_out);
    {
        const uint64_t threads = uint64_t(L.tiles_per_image) * p->spp * 32;
        raygen_kernel<<<uint32_t((threads + kBlock - 1) / kBlock), kBlock, 0, stream>>>(L, out, q.ray_a[0], q.ray_b[0],
                                                                                       q.ray_c[0], C);
        RR_CHECK_LAUNCH(ctx);
    }
    QueueKernel ext_k = extend_variant<false>(ctx->extend_variant);
    ShadowKernel sh_k = shadow_variant<false>(ctx->shadow_variant);
    const int g_ext = persistent_grid(ctx, reinterpret_cast<const void*>(ext_k));
    const int g_sh = persistent_grid(ctx, reinterpret_cast<const void*>(sh_k));
    const bool emitters = (p->flags & RR_PT_FLAG_EMITTERS) != 0;
    auto shade_k = mlp ? (emitters ? guided_shade_kernel<true, false, true> : guided_shade_kernel<true, false, false>)
                       : (emitters ? guided_shade_kernel<false, false, true> : guided_shade_kernel<false, false, false>);
    const int g_shade = std::min<int>(persistent_grid(ctx, reinterpret_cast<const void*>(shade_k)),
                                      int((n + kBlock - 1) / kBlock));
    GuidedLaunch G;
    G.paths = uint32_t(n);
    G.lobes = kMaxLobes;
    G.alpha = g->desc.alpha;
    G.grid = g->grid;
    G.mix = mlp ? g->mlp_mix : nullptr;
    G.rec0 = g->rec[0]; G.rec1 = g->rec[1]; G.rec2 = g->rec[2]; G.rec3 = g->rec[3];
    const DevScene& S = scene->dev;
    uint64_t launches = 1;
    // shadow rays of bounce b beside bounce b+1's extension rays (and MLP
    // inference), as in rr_pathtracer_execute; the next shade stage, which
    // reads and writes the image, waits for them
    const bool overlap = ctx->overlap_shadow;
    if (overlap && (st = ensure_side(ctx)) != RR_OK) return st;
    for (uint32_t b = 0; b < p->max_bounces; ++b) {
        const int cur = b & 1, nxt = cur ^ 1;
        uint32_t* cb = C + 4 * b;
        uint32_t* cn = C + 4 * (b + 1);
        G.bounce = b;
        G.last = b + 1 == p->max_bounces ? 1u : 0u;
        ext_k<<<g_ext, kBlock, 0, stream>>>(S, q.ray_a[cur], q.ray_b[cur], q.hits, cb, cb + 1, ctx->work64);
        RR_CHECK_LAUNCH(ctx);
        if (mlp && !G.last) {
            guided_surface_kernel<<<g_shade, kBlock, 0, stream>>>(S, q.ray_b[cur], q.hits, g->mlp_surf, cb);
            RR_CHECK_LAUNCH(ctx);
            if ((st = rr_mlp_guide_infer(ctx, g, cb, uint32_t(n), stream)) != RR_OK) return st;
            launches += 1 + g->mlp_infer_launches;
        }
        if (overlap && b > 0) RR_TRY_CUDA(ctx, cudaStreamWaitEvent(stream, ctx->shadowed[b - 1], 0));
        shade_k<<<g_shade, kBlock, 0, stream>>>(S, G, nullptr, nullptr, nullptr, nullptr, q.ray_a[cur], q.ray_b[cur],
                                                q.ray_c[cur], q.hits,
                                                q.ray_a[nxt], q.ray_b[nxt], q.ray_c[nxt], q.shadow_a, q.shadow_b,
                                                q.shadow_c, out, cb, cn, cb + 2);
        RR_CHECK_LAUNCH(ctx);
        cudaStream_t sh_stream = stream;
        if (overlap) {
            RR_TRY_CUDA(ctx, cudaEventRecord(ctx->shaded[b], stream));
            RR_TRY_CUDA(ctx, cudaStreamWaitEvent(ctx->side, ctx->shaded[b], 0));
            sh_stream = ctx->side;
        }
        sh_k<<<g_sh, kBlock, 0, sh_stream>>>(S, q.shadow_a, q.shadow_b, q.shadow_c, out, cb + 2, cb + 3,
                                             ctx->work64 + 2);
        RR_CHECK_LAUNCH(ctx);
        if (overlap) RR_TRY_CUDA(ctx, cudaEventRecord(ctx->shadowed[b], ctx->side));
        launches += 3;
    }
    if (overlap) RR_TRY_CUDA(ctx, cudaStreamWaitEvent(stream, ctx->shadowed[p->max_bounces - 1], 0));
    const uint32_t total = p->max_bounces > 1 ? uint32_t(n * (p->max_bounces - 1)) : 0u;
    if (total > 0) {
        const uint32_t tiles = (total + kResolveTile - 1) / kResolveTile;
        resolve_count_kernel<<<tiles, kBlock, 0, stream>>>(out, g->rec[0], g->rec[1], g->rec[2], g->rec[3],
                                                          uint32_t(n), total, g->resolve_first);
        RR_CHECK_LAUNCH(ctx);
        scan_exclusive(g->resolve_first, g->resolve_first, tiles, g->resolve_sums, stream);
        resolve_write_kernel<<<tiles, kBlock, 0, stream>>>(out, g->rec[0], g->rec[1], g->rec[2], g->rec[3],
                                                          uint32_t(n), total, g->resolve_first, g->samples);
        RR_CHECK_LAUNCH(ctx);
        launches += 5;
    }
    ctx->launches += launches;
    ctx->last_max_bounces = p->max_bounces;
    ctx->last_counted = false;
    g->frame_paths = uint32_t(n);
    return RR_OK;
}

// One update of guide g from the n samples its last execute recorded.
static rr_status guide_update_n(rr_ctx* ctx, rr_guide* g, uint32_t n, cudaStream_t stream) {
    if (!g->ev0) { RR_TRY_CUDA(ctx, cudaEventCreate(&g->ev0)); RR_TRY_CUDA(ctx, cudaEventCreate(&g->ev1)); }
    g->stats.samples_recorded = n;
    n = std::min(n, g->samples.capacity);
    RR_TRY_CUDA(ctx, cudaEventRecord(g->ev0, stream));
    if (g->desc.kind == RR_GUIDE_GRID) {
        GridView& v = g->grid;
        RR_TRY_CUDA(ctx, cudaMemsetAsync(g->cell_start, 0, size_t(v.cells) * 4, stream));
        RR_TRY_CUDA(ctx, cudaMemsetAsync(g->cell_end, 0, size_t(v.cells) * 4, stream));
        RR_TRY_CUDA(ctx, cudaMemsetAsync(g->samples.count + 1, 0, sizeof(uint32_t), stream));
        if (n > 0) {
            uint32_t* kin = reinterpret_cast<uint32_t*>(g->keys_in);
            uint32_t* kout = reinterpret_cast<uint32_t*>(g->keys_out);
            uint32_t* vin = g->vals_in;
            uint32_t* vout = g->vals_out;
            grid_keys_kernel<<<(n + 255) / 256, 256, 0, stream>>>(v, g->samples, n, kin, vin);
            RR_CHECK_LAUNCH(ctx);
            const uint32_t tiles = (n + kSortTile - 1) / kSortTile;
            uint32_t* hist = static_cast<uint32_t*>(g->sort_tmp);
            for (int shift = 0; shift < g->key_bits; shift += 8) {
                sort_hist_kernel<<<tiles, kSortThreads, 0, stream>>>(kin, n, shift, tiles, hist);
                scan_exclusive(hist, hist, uint32_t(kSortBins) * tiles, g->scan_sums, stream);
                sort_scatter_kernel<<<tiles, kSortThreads, 0, stream>>>(kin, vin, kout, vout, n, shift, tiles, hist);
                RR_CHECK_LAUNCH(ctx);
                std::swap(kin, kout);
                std::swap(vin, vout);
                ctx->launches += 5;
            }
            g->sorted_vals = vin;   // after the last pass's swap, the sorted arrays are the "in" pair
            grid_ranges_kernel<<<(n + 255) / 256, 256, 0, stream>>>(kin, n, g->cell_start, g->cell_end);
            RR_CHECK_LAUNCH(ctx);
        }
        const uint32_t cb = (v.cells + 255) / 256;
        grid_chunk_count_kernel<<<cb, 256, 0, stream>>>(g->cell_start, g->cell_end, v.cells, g->chunk_cnt);
        RR_CHECK_LAUNCH(ctx);
        scan_exclusive(g->chunk_cnt, g->chunk_off, v.cells, g->scan_sums, stream);
        RR_CHECK_LAUNCH(ctx);
        grid_chunk_map_kernel<<<cb, 256, 0, stream>>>(g->chunk_cnt, g->chunk_off, v.cells, g->chunk_cell);
        RR_CHECK_LAUNCH(ctx);
        if (n > 0) {
            const size_t warps = std::min<size_t>(v.cells, n) + n / kEmChunk + 1;
            grid_chunk_kernel<<<unsigned((warps * 32 + 127) / 128), 128, 0, stream>>>(
                v, g->samples, g->sorted_vals, g->cell_start, g->cell_end, g->chunk_cnt, g->chunk_off, g->chunk_cell,
                g->chunk_partial);
            RR_CHECK_LAUNCH(ctx);
        }
        grid_em_kernel<<<(v.cells + 127) / 128, 128, 0, stream>>>(v, g->chunk_cnt, g->chunk_off, g->chunk_partial,
                                                                   g->stats64, v.lobes, v.weights, g->desc.decay,
                                                                   g->samples.count + 1);
        RR_CHECK_LAUNCH(ctx);
        ctx->launches += n > 0 ? 9 : 6;   // besides the sort passes counted above
    } else {
        rr_status st = rr_mlp_guide_train(ctx, g, n, stream);
        if (st != RR_OK) return st;
    }
    RR_TRY_CUDA(ctx, cudaEventRecord(g->ev1, stream));
    g->stats.samples_used = n;
    g->stats.updates += 1;
    g->pending_stats = true;
    return RR_OK;
}

extern "C" rr_status rr_guide_update(rr_ctx* ctx, rr_guide* g, void* stream_v) {
    return rr_guides_update(ctx, &g, 1, stream_v);
}

extern "C" rr_status rr_guides_update(rr_ctx* ctx, rr_guide* const* guides, uint32_t count, void* stream_v) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!guides) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_guides_update: null argument");
    for (uint32_t i = 0; i < count; ++i)
        if (!guides[i] || guides[i]->ctx != ctx)
            return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_guides_update: guide %u is null or of another context", i);
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    // the sample counts decide the launch sizes: read them back (one small
    // copy per guide into its pinned word, one wait for all)
    for (uint32_t i = 0; i < count; ++i)
        RR_TRY_CUDA(ctx, cudaMemcpyAsync(guides[i]->count_host, guides[i]->samples.count, sizeof(uint32_t),
                                         cudaMemcpyDeviceToHost, stream));
    RR_TRY_CUDA(ctx, cudaStreamSynchronize(stream));
    std::vector<uint32_t> n(count);
    for (uint32_t i = 0; i < count; ++i) n[i] = guides[i]->count_host[0];
    for (uint32_t i = 0; i < count; ++i) {
        const rr_status st = guide_update_n(ctx, guides[i], n[i], stream);
        if (st != RR_OK) return st;
    }
    return RR_OK;
}

extern "C" rr_status rr_guide_get_stats(rr_ctx* ctx, const rr_guide* gc, rr_guide_stats* out) {
    if (!ctx || !gc || !out) return RR_ERR_INVALID_ARGUMENT;
    rr_guide* g = const_cast<rr_guide*>(gc);
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    if (g->pending_stats) {
        RR_TRY_CUDA(ctx, cudaEventSynchronize(g->ev1));
        float ms = 0.0f;
        RR_TRY_CUDA(ctx, cudaEventElapsedTime(&ms, g->ev0, g->ev1));
        g->stats.ms_update = ms;
        uint32_t c[4];
        RR_TRY_CUDA(ctx, cudaMemcpy(c, g->samples.count, sizeof(c), cudaMemcpyDeviceToHost));
        if (g->desc.kind == RR_GUIDE_GRID) g->stats.cells_valid = c[1];
        else g->stats.last_loss = rr_mlp_guide_last_loss(g);
        g->pending_stats = false;
    }
    *out = g->stats;
    return RR_OK;
}

namespace rr {
namespace {
__global__ void __launch_bounds__(256) grid_eval_kernel(GridView g, const float4* __restrict__ surf,
                                                        float4* __restrict__ mix, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t cell = grid_cell(g, xyz(surf[size_t(i) * 3]));
    float4* m = mix + size_t(i) * (kMaxLobes + 2);
    float w[kMaxLobes];
    for (int j = 0; j < kMaxLobes; ++j) {
        m[j] = g.lobes[size_t(cell) * kMaxLobes + j];
        w[j] = g.weights[size_t(cell) * kMaxLobes + j];
    }
    m[kMaxLobes] = make_float4(w[0], w[1], w[2], w[3]);
    m[kMaxLobes + 1] = make_float4(w[4], w[5], w[6], w[7]);
}
__global__ void set_count_kernel(uint32_t* c, uint32_t n) { *c = n; }
} // namespace
} // namespace rr

extern "C" rr_status rr_guide_eval(rr_ctx* ctx, rr_guide* g, const float* surf, uint32_t count, float* mix_out,
                                   void* stream_v) {
    if (!ctx || !g) return RR_ERR_INVALID_ARGUMENT;
    if (count == 0) return RR_OK;
    if (!surf || !mix_out) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_guide_eval: null buffer");
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    if (g->desc.kind == RR_GUIDE_GRID) {
        grid_eval_kernel<<<(count + 255) / 256, 256, 0, stream>>>(g->grid, reinterpret_cast<const float4*>(surf),
                                                                  reinterpret_cast<float4*>(mix_out), count);
        RR_CHECK_LAUNCH(ctx);
        ctx->launches += 1;
        return RR_OK;
    }
    set_count_kernel<<<1, 1, 0, stream>>>(g->samples.count + 2, count);
    RR_CHECK_LAUNCH(ctx);
    return rr_mlp_guide_eval(ctx, g, reinterpret_cast<const float4*>(surf), reinterpret_cast<float4*>(mix_out),
                             g->samples.count + 2, count, stream);
}

namespace rr {
namespace {
__global__ void __launch_bounds__(256) set_samples_kernel(const float4* __restrict__ src, GuideSamples S, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i == 0) S.count[0] = n;
    if (i >= n) return;
    S.s0[i] = src[size_t(i) * 4]; S.s1[i] = src[size_t(i) * 4 + 1];
    S.s2[i] = src[size_t(i) * 4 + 2]; S.s3[i] = src[size_t(i) * 4 + 3];
}
} // namespace
} // namespace rr

extern "C" rr_status rr_guide_set_samples(rr_ctx* ctx, rr_guide* g, const float* samples, uint32_t count,
                                          void* stream_v) {
    if (!ctx || !g) return RR_ERR_INVALID_ARGUMENT;
    if ((count && !samples) || count > g->samples.capacity)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_guide_set_samples: null buffer or count above capacity");
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    set_samples_kernel<<<std::max(1u, (count + 255) / 256), 256, 0, static_cast<cudaStream_t>(stream_v)>>>(
        reinterpret_cast<const float4*>(samples), g->samples, count);
    RR_CHECK_LAUNCH(ctx);
    return RR_OK;
}

// ── guided batches ─────────────────────────────────────────────────────────
// Per-call guide table in d_gcall (staged through h_gcall like the batch's
// own table): GuideEntry[count] | MlpView[count] | u64 rec_prefix[count + 1]
// (first record of each scene in the batch's record index space) |
// u32 group_base[count] (first mixture slot of each scene: prefix of paths).
static size_t align16(size_t x) { return (x + 15) & ~size_t(15); }

void rr_batch_free_guided(rr_batch* B) {
    if (B->gexec) cudaGraphExecDestroy(B->gexec);
    B->gexec = nullptr;
    for (int k = 0; k < 2; ++k) {
        if (B->gstaged[k]) cudaEventDestroy(B->gstaged[k]);
        if (B->h_gcall[k]) cudaFreeHost(B->h_gcall[k]);
        B->gstaged[k] = nullptr;
        B->h_gcall[k] = nullptr;
    }
    cudaFree(B->d_gcall); cudaFree(B->surf); cudaFree(B->mix); cudaFree(B->slot_map);
    cudaFree(B->group_count); cudaFree(B->tile_prefix);
    B->d_gcall = nullptr; B->surf = nullptr; B->mix = nullptr; B->slot_map = nullptr;
    B->group_count = nullptr; B->tile_prefix = nullptr;
    B->slots = 0;
}

static rr_status ensure_batch_guided(rr_ctx* ctx, rr_batch* B, size_t slots, bool mlp) {
    const size_t count = B->scenes.size();
    if (!B->d_gcall) {
        B->gcall_bytes = align16(sizeof(GuideEntry) * count) + align16(sizeof(MlpView) * count) +
                         align16(sizeof(unsigned long long) * (count + 1)) + align16(sizeof(uint32_t) * count);
        RR_TRY_CUDA(ctx, cudaMalloc(&B->d_gcall, B->gcall_bytes));
        RR_TRY_CUDA(ctx, cudaMalloc(&B->group_count, sizeof(uint32_t) * count));
        RR_TRY_CUDA(ctx, cudaMalloc(&B->tile_prefix, sizeof(uint32_t) * (count + 1)));
        for (int k = 0; k < 2; ++k) {
            RR_TRY_CUDA(ctx, cudaMallocHost(&B->h_gcall[k], B->gcall_bytes));
            RR_TRY_CUDA(ctx, cudaEventCreateWithFlags(&B->gstaged[k], cudaEventDisableTiming));
        }
    }
    if (mlp && B->slots < slots) {
        cudaFree(B->surf); cudaFree(B->mix); cudaFree(B->slot_map);
        B->surf = nullptr; B->mix = nullptr; B->slot_map = nullptr;
        B->slots = 0;
        RR_TRY_CUDA(ctx, cudaMalloc(&B->surf, slots * 3 * sizeof(float4)));
        RR_TRY_CUDA(ctx, cudaMalloc(&B->mix, slots * (kMaxLobes + 2) * sizeof(float4)));
        RR_TRY_CUDA(ctx, cudaMalloc(&B->slot_map, slots * sizeof(uint32_t)));
        B->slots = slots;
    }
    return RR_OK;
}

// Enqueues one guided batch frame; returns the kernels launched.
static rr_status enqueue_guided_batch(rr_ctx* ctx, rr_batch* B, rr_guide* const* guides, const size_t* paths_of,
                                      uint32_t tiles, size_t paths, uint32_t max_bounces, bool mlp,
                                      cudaStream_t stream, uint64_t* launches_out) {
    const uint32_t count = uint32_t(B->scenes.size());
    rr_pt_queues& q = ctx->pt;
    uint32_t* C = ctx->counters;
    const BatchEntry* entries = reinterpret_cast<const BatchEntry*>(B->d_call);
    float4* const* outs = reinterpret_cast<float4* const*>(B->d_call + B->entries_bytes);
    const GuideEntry* gtab = reinterpret_cast<const GuideEntry*>(B->d_gcall);
    const size_t o_nets = align16(sizeof(GuideEntry) * count);
    const size_t o_prefix = o_nets + align16(sizeof(MlpView) * count);
    const size_t o_base = o_prefix + align16(sizeof(unsigned long long) * (count + 1));
    const MlpView* nets = reinterpret_cast<const MlpView*>(B->d_gcall + o_nets);
    const unsigned long long* rec_prefix = reinterpret_cast<const unsigned long long*>(B->d_gcall + o_prefix);
    const uint32_t* group_base = reinterpret_cast<const uint32_t*>(B->d_gcall + o_base);
    uint64_t launches = 0;
    RR_TRY_CUDA(ctx, cudaMemsetAsync(C, 0, sizeof(uint32_t) * kCounterWords, stream));
    for (uint32_t i = 0; i < count; ++i) {
        rr_guide* g = guides[i];
        RR_TRY_CUDA(ctx, cudaMemsetAsync(g->samples.count, 0, sizeof(uint32_t) * 4, stream));
        // unfilled records read as NaN and are skipped by the resolve pass
        RR_TRY_CUDA(ctx, cudaMemsetAsync(g->rec[2], 0xff, paths_of[i] * max_bounces * sizeof(float4), stream));
    }
    {
        const uint64_t threads = uint64_t(tiles) * 32;
        raygen_batch_kernel<<<uint32_t((threads + kBlock - 1) / kBlock), kBlock, 0, stream>>>(
            entries, count, tiles, outs, q.ray_a[0], q.ray_b[0], q.ray_c[0], C);
        RR_CHECK_LAUNCH(ctx);
        launches += 1;
    }
    BatchQueueKernel ext_k = extend_batch_variant<false>(ctx->extend_variant);
    BatchShadowKernel sh_k = shadow_batch_variant<false>(ctx->shadow_variant);
    const int g_ext = persistent_grid(ctx, reinterpret_cast<const void*>(ext_k));
    const int g_sh = persistent_grid(ctx, reinterpret_cast<const void*>(sh_k));
    auto shade_k = mlp ? guided_shade_kernel<true, true> : guided_shade_kernel<false, true>;
    const int g_shade = std::min<int>(persistent_grid(ctx, reinterpret_cast<const void*>(shade_k)),
                                      int((paths + kBlock - 1) / kBlock));
    GuidedLaunch G{};
    G.lobes = kMaxLobes;
    G.mix = mlp ? B->mix : nullptr;
    // shadow rays of bounce b beside bounce b+1's extension rays (and MLP
    // inference), as in rr_pathtracer_execute; the next shade stage waits
    const bool overlap = ctx->overlap_shadow;
    if (overlap) {
        const rr_status so = ensure_side(ctx);
        if (so != RR_OK) return so;
    }
    for (uint32_t b = 0; b < max_bounces; ++b) {
        const int cur = b & 1, nxt = cur ^ 1;
        uint32_t* cb = C + 4 * b;
        uint32_t* cn = C + 4 * (b + 1);
        G.bounce = b;
        G.last = b + 1 == max_bounces ? 1u : 0u;
        ext_k<<<g_ext, kBlock, 0, stream>>>(B->d_table, q.ray_a[cur], q.ray_b[cur], q.ray_c[cur], q.hits, cb, cb + 1,
                                            ctx->work64);
        RR_CHECK_LAUNCH(ctx);
        if (mlp && !G.last) {
            RR_TRY_CUDA(ctx, cudaMemsetAsync(B->group_count, 0, sizeof(uint32_t) * count, stream));
            guided_surface_batch_kernel<<<g_shade, kBlock, 0, stream>>>(B->d_table, q.ray_b[cur], q.ray_c[cur], q.hits,
                                                                        group_base, B->group_count, B->surf,
                                                                        B->slot_map, cb);
            RR_CHECK_LAUNCH(ctx);
            const rr_status st = rr_mlp_guide_infer_grouped(ctx, nets, count, B->surf, B->mix, group_base,
                                                            B->group_count, B->tile_prefix, stream);
            if (st != RR_OK) return st;
            launches += 3;
        }
        if (overlap && b > 0) RR_TRY_CUDA(ctx, cudaStreamWaitEvent(stream, ctx->shadowed[b - 1], 0));
        shade_k<<<g_shade, kBlock, 0, stream>>>(DevScene{}, G, B->d_table, outs, gtab, B->slot_map, q.ray_a[cur],
                                                q.ray_b[cur], q.ray_c[cur], q.hits, q.ray_a[nxt], q.ray_b[nxt],
                                                q.ray_c[nxt], q.shadow_a, q.shadow_b, q.shadow_c, nullptr, cb, cn,
                                                cb + 2);
        RR_CHECK_LAUNCH(ctx);
        cudaStream_t sh_stream = stream;
        if (overlap) {
            RR_TRY_CUDA(ctx, cudaEventRecord(ctx->shaded[b], stream));
            RR_TRY_CUDA(ctx, cudaStreamWaitEvent(ctx->side, ctx->shaded[b], 0));
            sh_stream = ctx->side;
        }
        sh_k<<<g_sh, kBlock, 0, sh_stream>>>(B->d_table, outs, q.shadow_a, q.shadow_b, q.shadow_c, cb + 2, cb + 3,
                                             ctx->work64 + 2);
        RR_CHECK_LAUNCH(ctx);
        if (overlap) RR_TRY_CUDA(ctx, cudaEventRecord(ctx->shadowed[b], ctx->side));
        launches += 3;
    }
    if (overlap) RR_TRY_CUDA(ctx, cudaStreamWaitEvent(stream, ctx->shadowed[max_bounces - 1], 0));
    if (max_bounces > 1) {
        resolve_batch_kernel<<<std::max(1, ctx->sm_count * 8), kBlock, 0, stream>>>(gtab, outs, rec_prefix, count);
        RR_CHECK_LAUNCH(ctx);
        launches += 1;
    }
    *launches_out = launches;
    return RR_OK;
}

extern "C" rr_status rr_batch_execute_guided(rr_ctx* ctx, rr_batch* B, const GpuCameraData* cams,
                                             const rr_pt_params* p, rr_guide* const* guides,
                                             float* const* radiance_out, void* stream_v) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    if (!B || !cams || !p || !guides || !radiance_out)
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_execute_guided: null argument");
    if (B->ctx != ctx) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_execute_guided: batch of another context");
    if (p->spp == 0 || p->max_bounces == 0 || p->max_bounces > uint32_t(kMaxBounces))
        return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_execute_guided: bad spp or max_bounces");
    if (p->flags & RR_PT_FLAG_EMITTERS)
        return rr_fail(ctx, RR_ERR_UNSUPPORTED, "rr_batch_execute_guided: RR_PT_FLAG_EMITTERS is a single-scene mode");
    const uint32_t count = uint32_t(B->scenes.size());
    for (uint32_t i = 0; i < count; ++i)
        if (!guides[i] || guides[i]->ctx != ctx)
            return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_execute_guided: guide %u is null or of another context",
                           i);
    const uint32_t kind = guides[0]->desc.kind;
    for (uint32_t i = 1; i < count; ++i)
        if (guides[i]->desc.kind != kind)
            return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_execute_guided: guides of different kinds");
    {
        std::vector<const rr_guide*> sorted(guides, guides + count);
        std::sort(sorted.begin(), sorted.end());
        if (std::adjacent_find(sorted.begin(), sorted.end()) != sorted.end())
            return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_execute_guided: a guide appears twice");
    }
    std::vector<size_t> paths_of(count);
    for (uint32_t i = 0; i < count; ++i) {
        const uint64_t n = uint64_t(cams[i].screen_width) * cams[i].screen_height * p->spp;
        if (n * p->max_bounces >= (1ull << 32))
            return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "rr_batch_execute_guided: scene %u: too many paths", i);
        paths_of[i] = size_t(n);
    }
    cudaStream_t stream = static_cast<cudaStream_t>(stream_v);
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    uint32_t tiles = 0;
    uint64_t paths = 0;
    rr_status st = rr_batch_stage_call(ctx, B, cams, p, radiance_out, stream, &tiles, &paths);
    if (st != RR_OK) return st;
    // the overlap's stream and events exist before any graph capture starts
    if (ctx->overlap_shadow && (st = ensure_side(ctx)) != RR_OK) return st;
    const bool mlp = kind == RR_GUIDE_MLP;
    if ((st = ensure_batch_guided(ctx, B, size_t(paths), mlp)) != RR_OK) return st;
    for (uint32_t i = 0; i < count; ++i)
        if ((st = ensure_records(ctx, guides[i], paths_of[i], p->max_bounces)) != RR_OK) return st;
    // this call's guide table
    const int k = B->gslot;
    RR_TRY_CUDA(ctx, cudaEventSynchronize(B->gstaged[k]));
    unsigned char* h = B->h_gcall[k];
    GuideEntry* ge = reinterpret_cast<GuideEntry*>(h);
    MlpView* nv = reinterpret_cast<MlpView*>(h + align16(sizeof(GuideEntry) * count));
    unsigned long long* rp = reinterpret_cast<unsigned long long*>(
        h + align16(sizeof(GuideEntry) * count) + align16(sizeof(MlpView) * count));
    uint32_t* gb = reinterpret_cast<uint32_t*>(reinterpret_cast<unsigned char*>(rp) +
                                               align16(sizeof(unsigned long long) * (count + 1)));
    unsigned long long racc = 0;
    uint32_t sacc = 0;
    for (uint32_t i = 0; i < count; ++i) {
        rr_guide* g = guides[i];
        std::memset(&ge[i], 0, sizeof(GuideEntry));
        ge[i].grid = g->grid;
        for (int r = 0; r < 4; ++r) ge[i].rec[r] = g->rec[r];
        ge[i].S = g->samples;
        ge[i].paths = uint32_t(paths_of[i]);
        ge[i].alpha = g->desc.alpha;
        std::memset(&nv[i], 0, sizeof(MlpView));
        if (mlp) nv[i] = rr_mlp_guide_view(g);
        rp[i] = racc;
        racc += (unsigned long long)(paths_of[i]) * (p->max_bounces - 1);
        gb[i] = sacc;
        sacc += uint32_t(paths_of[i]);
    }
    rp[count] = racc;
    RR_TRY_CUDA(ctx, cudaMemcpyAsync(B->d_gcall, h, B->gcall_bytes, cudaMemcpyHostToDevice, stream));
    RR_TRY_CUDA(ctx, cudaEventRecord(B->gstaged[k], stream));
    B->gslot ^= 1;

    uint64_t launches = 0;
    if (p->flags & RR_PT_FLAG_GRAPH) {
        // the graph holds the queue, record and sample pointers and the launch sizes
        std::vector<const void*> key = {reinterpret_cast<const void*>(uintptr_t(paths)),
                                        reinterpret_cast<const void*>(uintptr_t(tiles)),
                                        reinterpret_cast<const void*>(uintptr_t(p->max_bounces)),
                                        reinterpret_cast<const void*>(uintptr_t(ctx->extend_variant)),
                                        reinterpret_cast<const void*>(uintptr_t(ctx->shadow_variant)),
                                        reinterpret_cast<const void*>(uintptr_t(ctx->overlap_shadow)),
                                        ctx->pt.ray_a[0], B->surf};
        for (uint32_t i = 0; i < count; ++i) {
            key.push_back(guides[i]);
            key.push_back(guides[i]->rec[2]);
            key.push_back(guides[i]->samples.count);
            key.push_back(reinterpret_cast<const void*>(uintptr_t(paths_of[i])));
        }
        if (!B->gexec || key != B->gkey) {
            if (B->gexec) { cudaGraphExecDestroy(B->gexec); B->gexec = nullptr; }
            RR_TRY_CUDA(ctx, cudaStreamBeginCapture(B->cap_stream, cudaStreamCaptureModeThreadLocal));
            st = enqueue_guided_batch(ctx, B, guides, paths_of.data(), tiles, size_t(paths), p->max_bounces, mlp,
                                      B->cap_stream, &launches);
            cudaGraph_t gr = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(B->cap_stream, &gr);
            if (st != RR_OK) { if (gr) cudaGraphDestroy(gr); return st; }
            if (ce != cudaSuccess) return rr_fail(ctx, RR_ERR_CUDA, "graph capture: %s", cudaGetErrorString(ce));
            const cudaError_t ie = cudaGraphInstantiate(&B->gexec, gr, 0);
            cudaGraphDestroy(gr);
            if (ie != cudaSuccess) return rr_fail(ctx, RR_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(ie));
            B->gkey = key;
        } else {
            launches = 1 + 3 * uint64_t(p->max_bounces) + (mlp ? 3 * uint64_t(p->max_bounces - 1) : 0) +
                       (p->max_bounces > 1 ? 1 : 0);
        }
        RR_TRY_CUDA(ctx, cudaGraphLaunch(B->gexec, stream));
    } else {
        st = enqueue_guided_batch(ctx, B, guides, paths_of.data(), tiles, size_t(paths), p->max_bounces, mlp, stream,
                                  &launches);
        if (st != RR_OK) return st;
    }
    ctx->launches += launches;
    ctx->last_max_bounces = p->max_bounces;
    ctx->last_counted = false;
    for (uint32_t i = 0; i < count; ++i) guides[i]->frame_paths = uint32_t(paths_of[i]);
    return RR_OK;
}
