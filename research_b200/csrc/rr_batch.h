// rr_batch.h — library-private state of a batch of scenes (rr_batch), shared
// by the reference tracer's batch (pathtracer.cu) and the guided batch
// (guided.cu).
#pragma once

#include "rr_internal.h"

#include <vector>

namespace rr {
struct DevScene;
}

struct rr_batch {
    rr_ctx* ctx = nullptr;
    std::vector<const rr_scene*> scenes;
    rr::DevScene* d_table = nullptr;       // per scene, uploaded once
    unsigned char* d_call = nullptr;       // per call: BatchEntry[count], then float4*[count]
    unsigned char* h_call[2] = {nullptr, nullptr};  // pinned staging of d_call, alternating
    cudaEvent_t staged[2] = {nullptr, nullptr};     // the copy out of h_call[k] has completed
    int slot = 0;
    int mode = RR_BATCH_WAVEFRONT;         // rr_batch_set_mode / rr_batch_tune
    size_t entries_bytes = 0, call_bytes = 0;
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    struct Key {
        uint64_t paths = 0;
        uint32_t total_tiles = 0, max_bounces = 0, ev = 0, sv = 0;
        const void* queue = nullptr;
        bool overlap = false;
        bool operator!=(const Key& o) const {
            return paths != o.paths || total_tiles != o.total_tiles || max_bounces != o.max_bounces || ev != o.ev ||
                   sv != o.sv || queue != o.queue || overlap != o.overlap;
        }
    } key;

    // guided batches (rr_batch_execute_guided): a per-call table of the
    // scenes' guides, staged like d_call, and the grouped-inference buffers
    // of MLP guides (one slot per queue entry of the whole batch)
    unsigned char* d_gcall = nullptr;
    unsigned char* h_gcall[2] = {nullptr, nullptr};
    cudaEvent_t gstaged[2] = {nullptr, nullptr};
    int gslot = 0;
    size_t gcall_bytes = 0;
    float4* surf = nullptr;                // per slot: (pos, 1), (normal, 1), (wo, 0)
    float4* mix = nullptr;                 // per slot: 8 lobes + 2 float4 of weights
    uint32_t* slot_map = nullptr;          // per queue entry: its mixture slot or ~0
    uint32_t* group_count = nullptr;       // per scene: slots taken this bounce
    uint32_t* tile_prefix = nullptr;       // per scene + 1: first 128-row inference tile
    size_t slots = 0;
    cudaGraphExec_t gexec = nullptr;
    std::vector<const void*> gkey;         // what the guided graph was captured with
};

// Stages one call's per-scene table (cameras, frame seed, spp, tile ranges,
// output pointers) into the batch's device table on `stream`; returns the
// batch's raygen tiles and paths.
rr_status rr_batch_stage_call(rr_ctx* ctx, rr_batch* B, const GpuCameraData* cams, const rr_pt_params* p,
                              float* const* radiance_out, cudaStream_t stream, uint32_t* tiles_out,
                              uint64_t* paths_out);
// Frees what rr_batch_execute_guided allocated (guided.cu).
void rr_batch_free_guided(rr_batch* B);
