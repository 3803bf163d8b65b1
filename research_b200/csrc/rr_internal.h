// rr_internal.h — library-private state behind the rr_cuda.h handles.
#pragma once

#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "rr_cuda.h"
#include "rr_trace.cuh"

struct rr_ctx;
rr_status rr_fail(rr_ctx* ctx, rr_status st, const char* fmt, ...);

// Wavefront queues of the path tracer, grown on demand. Ray queue entries
// are three float4 (origin, path id), (direction, rng seed), (throughput);
// shadow entries are (origin, path id), (direction, t_max), (contribution).
struct rr_pt_queues {
    size_t capacity = 0;
    float4* ray_a[2] = {nullptr, nullptr};
    float4* ray_b[2] = {nullptr, nullptr};
    float4* ray_c[2] = {nullptr, nullptr};
    float4* hits = nullptr;      // (u, v, instance, primitive)
    float4* shadow_a = nullptr;
    float4* shadow_b = nullptr;
    float4* shadow_c = nullptr;
};

// Device counters: per bounce b, [4b+0] rays in queue b, [4b+1] ray work
// cursor, [4b+2] shadow rays emitted at bounce b, [4b+3] shadow work cursor.
constexpr int kMaxBounces = 64;
constexpr int kCounterWords = 4 * (kMaxBounces + 1);

struct rr_stage_event {
    int stage;
    cudaEvent_t start, stop;
};

struct rr_ctx {
    int device = 0;
    int sm_count = 148;
    std::string last_error;
    rr_pt_queues pt;
    uint32_t* counters = nullptr;          // kCounterWords
    unsigned long long* work64 = nullptr;  // traversal work: ext nodes, ext tris, shadow nodes, shadow tris
    uint32_t last_max_bounces = 0;
    int extend_variant = 0;                // traversal schedule/occupancy variant (rr_pathtracer_tune)
    int shadow_variant = 0;
    bool last_counted = false;
    uint64_t launches = 0;                 // kernels issued by this context
    double stage_ms[4] = {0, 0, 0, 0};     // raygen, extend, shade, shadow
    uint64_t stage_launches[4] = {0, 0, 0, 0};
    std::vector<rr_stage_event> pending;   // recorded, not yet read back
    std::vector<cudaEvent_t> event_pool;
    double* mse_partial = nullptr;         // rr_image_mse block partials
    float4* atrous_nrm = nullptr;          // A-trous: the G-buffer normals, normalized once per call
    size_t atrous_nrm_px = 0;
    float* atrous_wt = nullptr;            // A-trous: the forward tap weights of every pixel (12 planes)
    size_t atrous_wt_floats = 0;
    bool atrous_tma = true;                // strides 1, 2, 4 through TMA-staged tiles
    int* atrous_error = nullptr;           // host-mapped word, set when a tile's copies missed the bounded wait
    int* atrous_error_dev = nullptr;       // its device address
    uint32_t atrous_wait_tries = 1u << 22; // tries of that bounded wait
    size_t queue_limit = 0;                // most ray-queue entries the context may hold (0: no limit)
    // The path tracer traces bounce b's shadow rays on a second stream while
    // bounce b+1's extension rays run on the caller's (fork after shade b,
    // join before shade b+1); created on first use.
    bool overlap_shadow = true;
    cudaStream_t side = nullptr;
    cudaEvent_t shaded[kMaxBounces] = {};
    cudaEvent_t shadowed[kMaxBounces] = {};
    // ReSTIR PT / GI initial passes in wavefront form (default) or one thread
    // per pixel: the wavefront's per-pixel state and per-step counters
    bool wave_initial = true;
    float4* wave_state = nullptr;
    size_t wave_state_len = 0;             // float4
    uint32_t* wave_counters = nullptr;
    size_t wave_counter_words = 0;
};

// Records a CUDA event pair around stage launches on the caller's stream;
// elapsed times are read back lazily by rr_pathtracer_stats.
struct rr_stage_timer {
    rr_ctx* ctx;
    cudaStream_t stream;
    bool on;
    cudaEvent_t cur_start = nullptr;
    cudaError_t err = cudaSuccess;
    rr_stage_timer(rr_ctx* c, cudaStream_t s, bool enabled) : ctx(c), stream(s), on(enabled) {}
    cudaEvent_t get() {
        if (!ctx->event_pool.empty()) { cudaEvent_t e = ctx->event_pool.back(); ctx->event_pool.pop_back(); return e; }
        cudaEvent_t e = nullptr;
        cudaError_t r = cudaEventCreate(&e);
        if (r != cudaSuccess) err = r;
        return e;
    }
    void begin(int) {
        if (!on) return;
        cur_start = get();
        if (cur_start) { cudaError_t r = cudaEventRecord(cur_start, stream); if (r != cudaSuccess) err = r; }
    }
    void end(int stage) {
        if (!on || !cur_start) return;
        cudaEvent_t e = get();
        if (!e) return;
        cudaError_t r = cudaEventRecord(e, stream);
        if (r != cudaSuccess) err = r;
        ctx->pending.push_back({stage, cur_start, e});
        cur_start = nullptr;
    }
    rr_status commit() {
        if (err != cudaSuccess) return rr_fail(ctx, RR_ERR_CUDA, "stage timer: %s", cudaGetErrorString(err));
        return RR_OK;
    }
    static rr_status collect(rr_ctx* c) {
        for (const rr_stage_event& ev : c->pending) {
            float ms = 0.0f;
            cudaError_t r = cudaEventElapsedTime(&ms, ev.start, ev.stop);
            if (r != cudaSuccess) return rr_fail(c, RR_ERR_CUDA, "cudaEventElapsedTime: %s", cudaGetErrorString(r));
            c->stage_ms[ev.stage] += ms;
            c->stage_launches[ev.stage] += 1;
            c->event_pool.push_back(ev.start);
            c->event_pool.push_back(ev.stop);
        }
        c->pending.clear();
        return RR_OK;
    }
};

struct rr_scene {
    rr_ctx* ctx = nullptr;
    rr::DevScene dev{};
    std::vector<void*> allocations;
    rr_scene_stats stats{};
};


#define RR_TRY_CUDA(ctx, expr)                                                              \
    do {                                                                                    \
        cudaError_t rr_e_ = (expr);                                                         \
        if (rr_e_ != cudaSuccess)                                                           \
            return rr_fail((ctx), rr_e_ == cudaErrorMemoryAllocation ? RR_ERR_OUT_OF_MEMORY \
                                                                     : RR_ERR_CUDA,         \
                           "%s failed: %s (%s:%d)", #expr, cudaGetErrorString(rr_e_),      \
                           __FILE__, __LINE__);                                             \
    } while (0)

#define RR_CHECK_LAUNCH(ctx) RR_TRY_CUDA(ctx, cudaGetLastError())

#include "rr_bvh.h"
