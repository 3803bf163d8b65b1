// rr_wavefront.cuh — wavefront stages shared by the reference and the guided
// path tracers: ray generation, queue traversal (closest hit / any hit) with
// its schedule and occupancy variants, and queue allocation.
#pragma once

#include "rr_internal.h"

namespace rr {
namespace {

constexpr int kBlock = 256;
constexpr uint32_t kFull = 0xffffffffu;

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Warp-aggregated slot allocation: returns this lane's slot when `want`.
__device__ __forceinline__ uint32_t warp_alloc(bool want, uint32_t* counter) {
    const uint32_t mask = __ballot_sync(kFull, want);
    uint32_t base = 0;
    if (lane_id() == 0 && mask) base = atomicAdd(counter, __popc(mask));
    base = __shfl_sync(kFull, base, 0);
    return base + __popc(mask & ((1u << lane_id()) - 1u));
}

struct PtLaunch {
    GpuCameraData cam;
    uint32_t frame_seed;
    uint32_t spp;
    uint32_t width, height;
    uint32_t tiles_x, tiles_per_image;
};

// One warp per 8x4 pixel tile so that primary rays of a warp are coherent.
__global__ void __launch_bounds__(kBlock) raygen_kernel(PtLaunch L, float4* __restrict__ out,
                                                        float4* qa, float4* qb, float4* qc,
                                                        uint32_t* counters) {
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t tile = gtid >> 5;
    const uint32_t lane = lane_id();
    const uint32_t total_tiles = L.tiles_per_image * L.spp;
    bool active = tile < total_tiles;
    uint32_t s = 0, px = 0, py = 0;
    if (active) {
        s = tile / L.tiles_per_image;
        const uint32_t t = tile % L.tiles_per_image;
        px = (t % L.tiles_x) * 8 + (lane & 7);
        py = (t / L.tiles_x) * 4 + (lane >> 3);
        active = px < L.width && py < L.height;
    }
    if (__all_sync(kFull, tile >= total_tiles)) return;
    const uint32_t slot = warp_alloc(active, &counters[0]);
    if (!active) return;
    const uint32_t pid = (s * L.height + py) * L.width + px;
    uint32_t seed = make_seed(px, py, L.frame_seed + s);
    const float jx = rand_float(seed);
    const float jy = rand_float(seed);
    const float3 dir = primary_dir(L.cam, float(px) + jx, float(py) + jy);
    out[pid] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    qa[slot] = make_float4(L.cam.position[0], L.cam.position[1], L.cam.position[2], __uint_as_float(pid));
    qb[slot] = make_float4(dir.x, dir.y, dir.z, __uint_as_float(seed));
    qc[slot] = make_float4(1.0f, 1.0f, 1.0f, 0.0f);
}

// Adds per-thread traversal work to two 64-bit counters, one atomic per warp.
__device__ __forceinline__ void flush_work(const TraceWork& w, unsigned long long* out) {
    unsigned long long n = w.nodes, t = w.tris;
    #pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        n += __shfl_down_sync(kFull, n, o);
        t += __shfl_down_sync(kFull, t, o);
    }
    if (lane_id() == 0 && (n | t)) { atomicAdd(out, n); atomicAdd(out + 1, t); }
}

// Queue traversal: each warp takes 32 consecutive queue entries (neighbouring
// paths after compaction, hence coherent rays) and traces them to the end,
// then takes the next 32 (the grid is persistent). MinBlocks is the
// occupancy target handed to the register allocator.
// `Finish(i, found, hit)` consumes a finished ray; `Load(i, ray, tmax)` makes
// one and returns its scene index. Multi: a batch of scenes, each ray traced
// in the scene `table[index]` (the lane binds that scene's node and triangle
// arrays when it loads the ray); otherwise every ray is traced in `s`. Rays
// start at t = tmin (the path tracer's 0.001).
template <int SmemS, int N> struct QueueStackOf { using type = SplitStack<SmemS, kBlock, N>; };
template <int N> struct QueueStackOf<0, N> { using type = LocalStackN<N>; };

// SmemS > 0: the bottom SmemS stack entries of every thread in shared memory.
// Wide: the 4-wide tree (trace_step4).
template <bool AnyHit, bool Count, bool Multi, bool Postpone = false, int SmemS = 0, bool Wide = false, class Load,
          class Finish>
__device__ __forceinline__ void traverse_queue(const DevScene& s, const DevScene* __restrict__ table, uint32_t count,
                                               uint32_t* cursor, unsigned long long* work_out, Load load,
                                               Finish finish, float tmin = 0.001f) {
    TraceWork tw;
    static_assert(!(Wide && Postpone), "postponed leaves are a binary-tree schedule");
    typename QueueStackOf<SmemS, Wide ? kStackSize4 : kStackSize>::type stack;   // (node, near distance) entries
    if constexpr (SmemS > 0) {
        __shared__ int2 stack_smem[SmemS * kBlock];
        stack.col = stack_smem + threadIdx.x;
    }
    DevScene ls{};           // Multi: the current ray's scene (traversal fields)
    auto bind = [&](uint32_t sid) {
        if constexpr (Multi) {
            ls.nodes = table[sid].nodes;
            ls.tris = table[sid].tris;
            ls.num_nodes = table[sid].num_nodes;
            ls.nodes4 = table[sid].nodes4;
            ls.num_nodes4 = table[sid].num_nodes4;
        }
    };
    auto step = [&](const Ray& r, HitRec& h, TravState& st) -> bool {
        const DevScene& sc = Multi ? ls : s;
        if constexpr (Wide) return trace_step4<AnyHit, Count>(sc, r, tmin, h, st, stack, &tw);
        else return trace_step<AnyHit, Count, Postpone>(sc, r, tmin, h, st, stack, &tw);
    };
    while (true) {
        uint32_t base = 0;
        if (lane_id() == 0) base = atomicAdd(cursor, 32u);
        base = __shfl_sync(kFull, base, 0);
        if (base >= count) break;
        const uint32_t i = base + lane_id();
        if (i < count) {
            Ray r; float tmax;
            bind(load(i, r, tmax));
            HitRec h; TravState st;
            trav_begin(st, h, tmax);
            while (!step(r, h, st)) {}
            finish(i, st.found, h);
        }
    }
    if (Count) flush_work(tw, work_out);
}

template <bool Count, int MinBlocks, bool Postpone = false, int SmemS = 0, bool Wide = false>
__global__ void __launch_bounds__(kBlock, MinBlocks) extend_kernel(DevScene s, const float4* __restrict__ qa,
                                                                   const float4* __restrict__ qb,
                                                                   float4* __restrict__ hits,
                                                                   const uint32_t* count_ptr, uint32_t* cursor,
                                                                   unsigned long long* work_out) {
    traverse_queue<false, Count, false, Postpone, SmemS, Wide>(
        s, nullptr, *count_ptr, cursor, work_out,
        [&](uint32_t i, Ray& r, float& tmax) -> uint32_t {
            const float4 a = qa[i], b = qb[i];
            r = make_ray(f3(a.x, a.y, a.z), f3(b.x, b.y, b.z));
            tmax = 1e9f;
            return 0u;
        },
        [&](uint32_t i, bool found, const HitRec& h) {
            hits[i] = found ? make_float4(h.u, h.v, __uint_as_float(h.inst), __uint_as_float(h.prim))
                            : make_float4(0.0f, 0.0f, __uint_as_float(kNoIndex), __uint_as_float(kNoIndex));
        });
}

// Any-hit shadow rays; unoccluded NEE contributions are added to the image.
template <bool Count, int MinBlocks, bool Postpone = false, int SmemS = 0, bool Wide = false>
__global__ void __launch_bounds__(kBlock, MinBlocks) shadow_kernel(DevScene s, const float4* __restrict__ sa,
                                                                   const float4* __restrict__ sb,
                                                                   const float4* __restrict__ sc,
                                                                   float4* __restrict__ out,
                                                                   const uint32_t* count_ptr, uint32_t* cursor,
                                                                   unsigned long long* work_out) {
    traverse_queue<true, Count, false, Postpone, SmemS, Wide>(
        s, nullptr, *count_ptr, cursor, work_out,
        [&](uint32_t i, Ray& r, float& tmax) -> uint32_t {
            const float4 a = sa[i], b = sb[i];
            r = make_ray(f3(a.x, a.y, a.z), f3(b.x, b.y, b.z));
            tmax = b.w;
            return 0u;
        },
        [&](uint32_t i, bool found, const HitRec&) {
            if (!found) {
                const float4 c = sc[i];
                const uint32_t pid = __float_as_uint(sa[i].w);
                float4 o = out[pid];
                o.x = o.x + c.x; o.y = o.y + c.y; o.z = o.z + c.z;
                out[pid] = o;
            }
        });
}

// ── batches of scenes (no reference counterpart: the reference renders one
// scene per pass execute). Queue entries carry their scene index in the
// .w of the throughput (rays) and contribution (shadow rays) records.
struct BatchEntry {
    PtLaunch L;            // the scene's camera, frame seed, spp and image size
    uint32_t tile_begin;   // first raygen tile of the scene in the batch
    uint32_t _pad[3];
};

// raygen_kernel over all scenes of a batch: the global tile index picks the
// scene (binary search over tile_begin), the rest is raygen_kernel's.
__global__ void __launch_bounds__(kBlock) raygen_batch_kernel(const BatchEntry* __restrict__ E, uint32_t n_scenes,
                                                              uint32_t total_tiles, float4* const* __restrict__ outs,
                                                              float4* qa, float4* qb, float4* qc,
                                                              uint32_t* counters) {
    const uint32_t gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const uint32_t tile = gtid >> 5;
    const uint32_t lane = lane_id();
    bool active = tile < total_tiles;
    uint32_t sid = 0, s = 0, px = 0, py = 0;
    if (active) {
        uint32_t lo = 0, hi = n_scenes - 1;
        while (lo < hi) {
            const uint32_t mid = (lo + hi + 1) >> 1;
            if (E[mid].tile_begin <= tile) lo = mid; else hi = mid - 1;
        }
        sid = lo;
        const PtLaunch& L = E[sid].L;
        const uint32_t local = tile - E[sid].tile_begin;
        s = local / L.tiles_per_image;
        const uint32_t t = local % L.tiles_per_image;
        px = (t % L.tiles_x) * 8 + (lane & 7);
        py = (t / L.tiles_x) * 4 + (lane >> 3);
        active = s < L.spp && px < L.width && py < L.height;
    }
    if (__all_sync(kFull, tile >= total_tiles)) return;
    const uint32_t slot = warp_alloc(active, &counters[0]);
    if (!active) return;
    const PtLaunch& L = E[sid].L;
    const uint32_t pid = (s * L.height + py) * L.width + px;
    uint32_t seed = make_seed(px, py, L.frame_seed + s);
    const float jx = rand_float(seed);
    const float jy = rand_float(seed);
    const float3 dir = primary_dir(L.cam, float(px) + jx, float(py) + jy);
    outs[sid][pid] = make_float4(0.0f, 0.0f, 0.0f, 1.0f);
    qa[slot] = make_float4(L.cam.position[0], L.cam.position[1], L.cam.position[2], __uint_as_float(pid));
    qb[slot] = make_float4(dir.x, dir.y, dir.z, __uint_as_float(seed));
    qc[slot] = make_float4(1.0f, 1.0f, 1.0f, __uint_as_float(sid));
}

template <bool Count, int MinBlocks, bool Postpone = false, int SmemS = 0, bool Wide = false>
__global__ void __launch_bounds__(kBlock, MinBlocks) extend_batch_kernel(const DevScene* __restrict__ table,
                                                                         const float4* __restrict__ qa,
                                                                         const float4* __restrict__ qb,
                                                                         const float4* __restrict__ qc,
                                                                         float4* __restrict__ hits,
                                                                         const uint32_t* count_ptr, uint32_t* cursor,
                                                                         unsigned long long* work_out) {
    const DevScene none{};
    traverse_queue<false, Count, true, Postpone, SmemS, Wide>(
        none, table, *count_ptr, cursor, work_out,
        [&](uint32_t i, Ray& r, float& tmax) -> uint32_t {
            const float4 a = qa[i], b = qb[i];
            r = make_ray(f3(a.x, a.y, a.z), f3(b.x, b.y, b.z));
            tmax = 1e9f;
            return __float_as_uint(qc[i].w);
        },
        [&](uint32_t i, bool found, const HitRec& h) {
            hits[i] = found ? make_float4(h.u, h.v, __uint_as_float(h.inst), __uint_as_float(h.prim))
                            : make_float4(0.0f, 0.0f, __uint_as_float(kNoIndex), __uint_as_float(kNoIndex));
        });
}

template <bool Count, int MinBlocks, bool Postpone = false, int SmemS = 0, bool Wide = false>
__global__ void __launch_bounds__(kBlock, MinBlocks) shadow_batch_kernel(const DevScene* __restrict__ table,
                                                                         float4* const* __restrict__ outs,
                                                                         const float4* __restrict__ sa,
                                                                         const float4* __restrict__ sb,
                                                                         const float4* __restrict__ sc,
                                                                         const uint32_t* count_ptr, uint32_t* cursor,
                                                                         unsigned long long* work_out) {
    const DevScene none{};
    traverse_queue<true, Count, true, Postpone, SmemS, Wide>(
        none, table, *count_ptr, cursor, work_out,
        [&](uint32_t i, Ray& r, float& tmax) -> uint32_t {
            const float4 a = sa[i], b = sb[i];
            r = make_ray(f3(a.x, a.y, a.z), f3(b.x, b.y, b.z));
            tmax = b.w;
            return __float_as_uint(sc[i].w);
        },
        [&](uint32_t i, bool found, const HitRec&) {
            if (!found) {
                const float4 c = sc[i];
                const uint32_t pid = __float_as_uint(sa[i].w);
                float4* out = outs[__float_as_uint(c.w)];
                float4 o = out[pid];
                o.x = o.x + c.x; o.y = o.y + c.y; o.z = o.z + c.z;
                out[pid] = o;
            }
        });
}

using BatchQueueKernel = void (*)(const DevScene*, const float4*, const float4*, const float4*, float4*,
                                  const uint32_t*, uint32_t*, unsigned long long*);
using BatchShadowKernel = void (*)(const DevScene*, float4* const*, const float4*, const float4*, const float4*,
                                   const uint32_t*, uint32_t*, unsigned long long*);
// Variant 0 of the batch extend kernel asks for 4 blocks per SM: left free,
// the per-ray scene binding takes it to 68 registers (3 blocks of 256 per
// SM), where the single-scene kernel settles at 64 (4 blocks).
template <bool Count>
BatchQueueKernel extend_batch_variant(int v) {
    switch (v) {
    case 1: return extend_batch_kernel<Count, 5>;
    case 2: return extend_batch_kernel<Count, 1, false, 8>;
    case 3: return extend_batch_kernel<Count, 1, false, 0, true>;
    case 4: return extend_batch_kernel<Count, 1, false, 8, true>;
    case 5: return extend_batch_kernel<Count, 5, false, 8>;
    case 6: return extend_batch_kernel<Count, 3, false, 8, true>;
    case 7: return extend_batch_kernel<Count, 4, true>;
    default: return extend_batch_kernel<Count, 4>;
    }
}
template <bool Count>
BatchShadowKernel shadow_batch_variant(int v) {
    switch (v) {
    case 1: return shadow_batch_kernel<Count, 5>;
    case 2: return shadow_batch_kernel<Count, 1, false, 8>;
    case 3: return shadow_batch_kernel<Count, 1, false, 0, true>;
    case 4: return shadow_batch_kernel<Count, 1, false, 8, true>;
    case 5: return shadow_batch_kernel<Count, 5, false, 8>;
    case 6: return shadow_batch_kernel<Count, 3, false, 8, true>;
    case 7: return shadow_batch_kernel<Count, 4, true>;
    default: return shadow_batch_kernel<Count, 1>;
    }
}

// Traversal kernel variants: schedule x occupancy target x stack placement.
using QueueKernel = void (*)(DevScene, const float4*, const float4*, float4*, const uint32_t*, uint32_t*,
                             unsigned long long*);
using ShadowKernel = void (*)(DevScene, const float4*, const float4*, const float4*, float4*, const uint32_t*,
                              uint32_t*, unsigned long long*);
template <bool Count>
QueueKernel extend_variant(int v) {
    switch (v) {
    case 1: return extend_kernel<Count, 5>;
    case 2: return extend_kernel<Count, 1, false, 8>;
    case 3: return extend_kernel<Count, 1, false, 0, true>;
    case 4: return extend_kernel<Count, 1, false, 8, true>;
    case 5: return extend_kernel<Count, 5, false, 8>;
    case 6: return extend_kernel<Count, 3, false, 8, true>;
    case 7: return extend_kernel<Count, 4, true>;
    default: return extend_kernel<Count, 1>;
    }
}
template <bool Count>
ShadowKernel shadow_variant(int v) {
    switch (v) {
    case 1: return shadow_kernel<Count, 5>;
    case 2: return shadow_kernel<Count, 1, false, 8>;
    case 3: return shadow_kernel<Count, 1, false, 0, true>;
    case 4: return shadow_kernel<Count, 1, false, 8, true>;
    case 5: return shadow_kernel<Count, 5, false, 8>;
    case 6: return shadow_kernel<Count, 3, false, 8, true>;
    case 7: return shadow_kernel<Count, 4, true>;
    default: return shadow_kernel<Count, 1>;
    }
}

int persistent_grid(const rr_ctx* ctx, const void* kernel) {
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBlock, 0);
    return ctx->sm_count * (per_sm > 0 ? per_sm : 1);
}

// The second stream and the fork/join events of the shadow overlap.
rr_status ensure_side(rr_ctx* ctx) {
    if (ctx->side) return RR_OK;
    for (int b = 0; b < kMaxBounces; ++b) {
        RR_TRY_CUDA(ctx, cudaEventCreateWithFlags(&ctx->shaded[b], cudaEventDisableTiming));
        RR_TRY_CUDA(ctx, cudaEventCreateWithFlags(&ctx->shadowed[b], cudaEventDisableTiming));
    }
    RR_TRY_CUDA(ctx, cudaStreamCreateWithFlags(&ctx->side, cudaStreamNonBlocking));
    return RR_OK;
}

rr_status ensure_queues(rr_ctx* ctx, size_t n) {
    rr_pt_queues& q = ctx->pt;
    if (ctx->queue_limit && n > ctx->queue_limit)
        return rr_fail(ctx, RR_ERR_QUEUE_OVERFLOW,
                       "the call needs %zu ray-queue entries; the context's queue limit is %zu "
                       "(rr_ctx_set_queue_limit)", n, ctx->queue_limit);
    if (q.capacity >= n) return RR_OK;
    for (int i = 0; i < 2; ++i) { cudaFree(q.ray_a[i]); cudaFree(q.ray_b[i]); cudaFree(q.ray_c[i]); }
    cudaFree(q.hits); cudaFree(q.shadow_a); cudaFree(q.shadow_b); cudaFree(q.shadow_c);
    q = rr_pt_queues();
    const size_t bytes = n * sizeof(float4);
    for (int i = 0; i < 2; ++i) {
        RR_TRY_CUDA(ctx, cudaMalloc(&q.ray_a[i], bytes));
        RR_TRY_CUDA(ctx, cudaMalloc(&q.ray_b[i], bytes));
        RR_TRY_CUDA(ctx, cudaMalloc(&q.ray_c[i], bytes));
    }
    RR_TRY_CUDA(ctx, cudaMalloc(&q.hits, bytes));
    RR_TRY_CUDA(ctx, cudaMalloc(&q.shadow_a, bytes));
    RR_TRY_CUDA(ctx, cudaMalloc(&q.shadow_b, bytes));
    RR_TRY_CUDA(ctx, cudaMalloc(&q.shadow_c, bytes));
    q.capacity = n;
    return RR_OK;
}

} // namespace
} // namespace rr
