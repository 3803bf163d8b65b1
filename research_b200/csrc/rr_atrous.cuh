// rr_atrous.cuh — one output pixel of the A-trous filter (atrous.slang:41-106:
// 5x5 B3 taps (1,4,6,4,1)/16 per axis at the pass's stride, clamped to the
// image, skipping G-buffer misses, weighted by exp(-|dp|^2/sp^2) *
// exp(-max(0, 1-n.n')/sn^2) * exp(-dl^2/sl^2)), shared by every A-trous
// kernel of the library so that they all run one tap loop.
#pragma once

#include "rr_dev.cuh"

namespace rr {

RR_D float luminance601(float3 c) { return dot(c, f3(0.299f, 0.587f, 0.114f)); }
RR_D float kernel_weight(int o) { return (o == 2 || o == -2) ? 1.0f : ((o == 1 || o == -1) ? 4.0f : 6.0f); }

// The weight of tap (tx, ty) of a centre pixel (position cp, unit normal cn,
// luminance cl) on a neighbour (sp, sn, srad). Every factor is the same bits
// with the two pixels swapped and (tx, ty) negated: (-d).(-d) = d.d,
// dot(a, b) = dot(b, a) term by term, (-l)^2 = l^2, and the B3 weights are
// symmetric; atrous_pair_weights_kernel relies on it.
RR_D float tap_weight(int tx, int ty, float3 cp, float3 cn, float cl, float3 sp, float3 sn, float3 srad, float sp2,
                      float sn2, float sl2) {
    const float base_w = (kernel_weight(tx) * kernel_weight(ty)) / 256.0f;
    const float3 pd = sp - cp;
    const float pos_w = rr_expf(-dot(pd, pd) / sp2);
    const float nd = mx(0.0f, 1.0f - dot(cn, sn));
    const float normal_w = rr_expf(-nd / sn2);
    const float ld = luminance601(srad) - cl;
    const float luma_w = rr_expf(-(ld * ld) / sl2);
    return base_w * pos_w * normal_w * luma_w;
}

// One output pixel of atrous.slang:cs_main (atrous.slang:41-106) at stride
// `stride`, reading the three images through `f` (global memory or a tile
// in shared memory: the same values, so the same bits either way).
template <class Fetch>
RR_D float4 atrous_pixel(const Fetch& f, int x, int y, int W, int H, int stride, float sp2, float sn2, float sl2) {
    const float4 cpos = f.pos(x, y);
    const float4 crad = f.rad(x, y);
    if (cpos.w < 0.0f) return crad;
    const float3 cn = xyz(f.nrm(x, y));
    const float cl = luminance601(xyz(crad));
    float3 filtered = f3(0.0f, 0.0f, 0.0f);
    float wsum = 0.0f;
    #pragma unroll
    for (int ty = -2; ty <= 2; ++ty) {
        const int sy = min(max(y + ty * stride, 0), H - 1);
        #pragma unroll
        for (int tx = -2; tx <= 2; ++tx) {
            const int sx = min(max(x + tx * stride, 0), W - 1);
            // the tap's values are read before its miss test (the address is
            // in the image), so the taps' loads can be in flight together
            const float4 spos = f.pos(sx, sy);
            const float3 srad = xyz(f.rad(sx, sy));
            const float3 sn = xyz(f.nrm(sx, sy));
            if (spos.w < 0.0f) continue;
            const float w = tap_weight(tx, ty, xyz(cpos), cn, cl, xyz(spos), sn, srad, sp2, sn2, sl2);
            filtered = filtered + srad * w;
            wsum += w;
        }
    }
    const float3 o = wsum > 0.0f ? filtered / wsum : xyz(crad);
    return make_float4(o.x, o.y, o.z, crad.w);
}

// The images in global memory (read-only path).
struct GlobalFetch {
    const float4* __restrict__ rad_g;
    const float4* __restrict__ pos_g;
    const float4* __restrict__ nrm_g;
    int W;
    RR_D float4 rad(int x, int y) const { return __ldg(rad_g + size_t(y) * W + x); }
    RR_D float4 pos(int x, int y) const { return __ldg(pos_g + size_t(y) * W + x); }
    RR_D float4 nrm(int x, int y) const { return __ldg(nrm_g + size_t(y) * W + x); }
};

} // namespace rr
