// rr_guide.h — library-private state of a path-guiding guide (rr_guide).
#pragma once

#include "rr_internal.h"

#include <cuda_bf16.h>

namespace rr {

// Dense grid of vMF mixtures: cells = res^3 over [bmin, bmin + res/scale].
struct GridView {
    uint32_t res = 0;
    uint32_t cells = 0;
    float3 bmin{0, 0, 0};
    float3 scale{0, 0, 0};       // cells per world unit, per axis
    float4* lobes = nullptr;     // cells * 8: (mu.xyz, kappa)
    float* weights = nullptr;    // cells * 8
};

__device__ __forceinline__ uint32_t grid_cell(const GridView& g, float3 p) {
    const int r = int(g.res) - 1;
    int cx = int(floorf((p.x - g.bmin.x) * g.scale.x));
    int cy = int(floorf((p.y - g.bmin.y) * g.scale.y));
    int cz = int(floorf((p.z - g.bmin.z) * g.scale.z));
    cx = cx < 0 ? 0 : (cx > r ? r : cx);
    cy = cy < 0 ? 0 : (cy > r ? r : cy);
    cz = cz < 0 ? 0 : (cz > r ? r : cz);
    return (uint32_t(cz) * g.res + uint32_t(cy)) * g.res + uint32_t(cx);
}

// Training samples: s0 = (pos, weight), s1 = (wi, vertex id), s2 = (normal),
// s3 = (wo). count[0] = samples appended, count[1] = valid cells (grid).
struct GuideSamples {
    float4* s0 = nullptr;
    float4* s1 = nullptr;
    float4* s2 = nullptr;
    float4* s3 = nullptr;
    uint32_t* count = nullptr;
    uint32_t capacity = 0;
};

// One MLP guide's network as its kernels read it: BF16 weights, FP32 master
// parameters (the forward takes the biases from them), the bounds of the
// position encoding and the guide's error flag (set when a tensor-core wait
// gave up).
struct MlpView {
    const __nv_bfloat16* w16;
    const float* params;
    float3 bmin, inv_ext;
    int* error;
};

// One scene of a guided batch: its guide's grid (grid guides), vertex
// records and training samples, its paths per bounce and alpha.
struct GuideEntry {
    GridView grid;
    float4* rec[4];
    GuideSamples S;
    uint32_t paths;
    float alpha;
};

} // namespace rr

struct rr_mlp_state;

struct rr_guide {
    rr_ctx* ctx = nullptr;
    rr_guide_desc desc{};
    std::vector<void*> allocations;
    rr::GuideSamples samples;
    uint32_t* count_host = nullptr;   // pinned: the sample count read back by an update
    float4* rec[4] = {nullptr, nullptr, nullptr, nullptr};
    size_t rec_capacity = 0;
    uint32_t* resolve_first = nullptr;  // per resolve tile: its sample count, then its first slot
    uint32_t* resolve_sums = nullptr;   // chunk sums of the resolve's scan
    uint32_t frame_paths = 0;
    // grid
    rr::GridView grid;
    double* stats64 = nullptr;
    uint32_t* cell_start = nullptr;
    uint32_t* cell_end = nullptr;
    unsigned long long* keys_in = nullptr;
    unsigned long long* keys_out = nullptr;
    uint32_t* vals_in = nullptr;
    uint32_t* vals_out = nullptr;
    void* sort_tmp = nullptr;       // the cell sort's per-(digit, tile) counts (rr_cellsort.cuh)
    size_t sort_tmp_bytes = 0;
    int key_bits = 32;              // sorted key bits: the cell index's
    uint32_t* sorted_vals = nullptr;  // vals_in or vals_out: the cell-sorted sample indices of the last update
    uint32_t* scan_sums = nullptr;    // chunk sums of the scans (rr_cellsort.cuh)
    uint32_t* chunk_cnt = nullptr;  // per cell: EM chunks of its samples
    uint32_t* chunk_off = nullptr;  // per cell: exclusive scan of chunk_cnt
    uint32_t* chunk_cell = nullptr; // per chunk: its cell
    double* chunk_partial = nullptr;// per chunk: 8 x (s0, s1.xyz) FP64 sums
    size_t chunk_capacity = 0;
    // MLP
    rr_mlp_state* mlp = nullptr;
    float4* mlp_surf = nullptr;   // per queue slot: (pos, 1), (normal, valid), (wo, 0)
    float4* mlp_mix = nullptr;    // per queue slot: 8 lobes + 2 float4 of weights
    size_t mlp_slots = 0;
    uint64_t mlp_infer_launches = 0;
    // statistics
    rr_guide_stats stats{};
    bool pending_stats = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ~rr_guide();
};

// MLP guide (mlp_guide.cu)
rr_status rr_mlp_guide_init(rr_ctx* ctx, rr_guide* g);
rr_status rr_mlp_guide_reset(rr_ctx* ctx, rr_guide* g, cudaStream_t stream);
rr_status rr_mlp_guide_ensure(rr_ctx* ctx, rr_guide* g, size_t slots);
rr_status rr_mlp_guide_infer(rr_ctx* ctx, rr_guide* g, const uint32_t* count_dev, uint32_t max_count,
                             cudaStream_t stream);
rr_status rr_mlp_guide_train(rr_ctx* ctx, rr_guide* g, uint32_t n, cudaStream_t stream);
double rr_mlp_guide_last_loss(rr_guide* g);
rr::MlpView rr_mlp_guide_view(rr_guide* g);
// Grouped inference over the scenes of a guided batch: group g's queries
// are surf/mix slots [group_base[g], group_base[g] + group_count[g]) and run
// through network nets[g] (device array); tile_prefix (groups + 1 words) is
// scratch for the per-group tile ranges. All counts are read on the device.
rr_status rr_mlp_guide_infer_grouped(rr_ctx* ctx, const rr::MlpView* nets, uint32_t groups, const float4* surf,
                                     float4* mix, const uint32_t* group_base, const uint32_t* group_count,
                                     uint32_t* tile_prefix, cudaStream_t stream);
rr_status rr_mlp_guide_eval(rr_ctx* ctx, rr_guide* g, const float4* surf, float4* mix, const uint32_t* count_dev,
                            uint32_t count, cudaStream_t stream);
