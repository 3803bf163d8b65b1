// rr_wave.cuh — the traversal steps shared by the wavefront forms of the
// reuse passes' initial candidates (ReSTIR PT and ReSTIR GI cs_initial).
//
// Each step of such a pass traces one queue of segment rays, (origin, pixel)
// and (direction, -), to their closest hit from t = tmin, and one queue of
// shadow rays, (origin, pixel), (direction, t_max) and (contribution, -),
// whose contributions are added to their pixel's radiance sum when the light
// is visible (zero otherwise, as the inline light sample returns). A pixel
// has at most one ray in each queue per step. Per step the counters hold
// kWaveWords words: segment rays, their cursor, shadow rays, their cursor,
// candidates that ended.
#pragma once

#include "rr_wavefront.cuh"

namespace rr {
namespace {

constexpr int kWaveWords = 8;
constexpr uint32_t kRis = 0x80000000u;   // ended-candidate flag: it enters resampling

__global__ void __launch_bounds__(kBlock, 4) wave_extend_kernel(DevScene s, const float4* __restrict__ qa,
                                                                const float4* __restrict__ qb,
                                                                float4* __restrict__ hits, uint32_t* c0,
                                                                float tmin) {
    traverse_queue<false, false, false>(
        s, nullptr, c0[0], c0 + 1, nullptr,
        [&](uint32_t i, Ray& r, float& tmax) -> uint32_t {
            r = make_ray(xyz(qa[i]), xyz(qb[i]));
            tmax = 1e9f;
            return 0u;
        },
        [&](uint32_t i, bool found, const HitRec& h) {
            hits[i] = found ? make_float4(h.u, h.v, __uint_as_float(h.inst), __uint_as_float(h.prim))
                            : make_float4(0.0f, 0.0f, __uint_as_float(kNoIndex), __uint_as_float(kNoIndex));
        },
        tmin);
}

__global__ void __launch_bounds__(kBlock, 5) wave_shadow_kernel(DevScene s, const float4* __restrict__ sa,
                                                                const float4* __restrict__ sb,
                                                                const float4* __restrict__ sc, float4* sum,
                                                                uint32_t* c0, float tmin) {
    traverse_queue<true, false, false>(
        s, nullptr, c0[2], c0 + 3, nullptr,
        [&](uint32_t i, Ray& r, float& tmax) -> uint32_t {
            const float4 b = sb[i];
            r = make_ray(xyz(sa[i]), xyz(b));
            tmax = b.w;
            return 0u;
        },
        [&](uint32_t i, bool found, const HitRec&) {
            const uint32_t pid = __float_as_uint(sa[i].w);
            const float3 add = found ? f3(0.0f, 0.0f, 0.0f) : xyz(sc[i]);
            const float3 v = xyz(sum[pid]) + add;
            sum[pid] = make_float4(v.x, v.y, v.z, 0.0f);
        },
        tmin);
}

// The context's wavefront scratch: `arrays` float4 per pixel of state and the
// counters of `steps` steps (plus one for the rays the last step emits),
// zeroed on `stream`. One pass uses it at a time (calls on one context are
// stream-ordered, as for the path tracer's queues).
rr_status wave_scratch(rr_ctx* ctx, size_t n, int arrays, uint32_t steps, cudaStream_t stream, float4** state,
                       uint32_t** counters) {
    const size_t need = n * size_t(arrays);
    if (ctx->wave_state_len < need) {
        cudaFree(ctx->wave_state);
        ctx->wave_state = nullptr;
        ctx->wave_state_len = 0;
        RR_TRY_CUDA(ctx, cudaMalloc(&ctx->wave_state, need * sizeof(float4)));
        ctx->wave_state_len = need;
    }
    const size_t words = size_t(steps + 1) * kWaveWords;
    if (ctx->wave_counter_words < words) {
        cudaFree(ctx->wave_counters);
        ctx->wave_counters = nullptr;
        ctx->wave_counter_words = 0;
        RR_TRY_CUDA(ctx, cudaMalloc(&ctx->wave_counters, words * sizeof(uint32_t)));
        ctx->wave_counter_words = words;
    }
    RR_TRY_CUDA(ctx, cudaMemsetAsync(ctx->wave_counters, 0, words * sizeof(uint32_t), stream));
    *state = ctx->wave_state;
    *counters = ctx->wave_counters;
    return RR_OK;
}

} // namespace
} // namespace rr
