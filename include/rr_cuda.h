/*
 * rr_cuda.h — C ABI of the B200 light-transport library (librr_cuda.so).
 *
 * Drop-in boundary for the reference renderer's hot passes. Each entry point
 * replaces one pass's `execute` (or one compute dispatch inside it) of the
 * reference's rr::render::RenderPass contract (src/render/RenderPass.h:11-48);
 * the parameter structs carry the same fields as the reference push-constant
 * blocks minus the bindless heap indices, which become typed pointers here.
 *
 * Conventions
 *  - Every function returns rr_status; no exception crosses this boundary
 *    (the reference throws std::runtime_error from initialize(); here the
 *    caller gets RR_ERR_* and rr_last_error() text instead).
 *  - Image buffers are caller-owned DEVICE memory, row-major RGBA32F
 *    (4 floats per pixel), exactly like the reference's storage images.
 *  - `stream` is a cudaStream_t (NULL = legacy default stream). Execute calls
 *    only enqueue work; they do not synchronise.
 *  - The library owns the scene (geometry, BVH) and the wavefront queues.
 *    Calls that use a context's queues (the path tracers, batches, the
 *    ReSTIR PT / GI initial passes) must follow one another on one stream;
 *    ReSTIR DI, accumulate and A-trous use none and may run beside them on
 *    another stream.
 *  - Camera data is passed by host pointer (GpuCameraData, 304 bytes,
 *    GpuScene.h:80-98) and reaches the kernels as a launch parameter.
 */
#ifndef RR_CUDA_H
#define RR_CUDA_H

#include <stddef.h>
#include <stdint.h>
#include "rr_layouts.h"

#ifdef __cplusplus
extern "C" {
#endif

#define RR_ABI_VERSION 1u

typedef enum rr_status {
    RR_OK = 0,
    RR_ERR_INVALID_ARGUMENT = 1,
    RR_ERR_CUDA = 2,
    RR_ERR_OUT_OF_MEMORY = 3,
    RR_ERR_NOT_INITIALIZED = 4,
    RR_ERR_QUEUE_OVERFLOW = 5,
    RR_ERR_TIMEOUT = 6,
    RR_ERR_UNSUPPORTED = 7
} rr_status;

typedef struct rr_ctx rr_ctx;
typedef struct rr_scene rr_scene;

/* ── context ─────────────────────────────────────────────────────────────
 * Replaces the per-pass initialize(Device&, SlangSession&, BindlessRegistry&,
 * Extent2D) plumbing (e.g. PathTracerPass.h:28-31): binds a CUDA device. */
uint32_t    rr_abi_version(void);
const char* rr_status_string(rr_status status);
rr_status   rr_ctx_create(int device_ordinal, rr_ctx** out_ctx);
rr_status   rr_ctx_destroy(rr_ctx* ctx);
/* Copies the last error message of this context (NUL-terminated). */
rr_status   rr_last_error(const rr_ctx* ctx, char* buf, size_t buf_size);
/* Caps the wavefront ray queues the context may allocate at `max_entries`
 * entries (one entry per path in flight; 0 = no cap, the default). A call
 * whose paths need more (width x height x spp for the path tracers, width x
 * height for the reuse passes' wavefront steps) returns
 * RR_ERR_QUEUE_OVERFLOW before launching anything. No counterpart in the
 * reference, whose passes size their images at initialize(). */
rr_status   rr_ctx_set_queue_limit(rr_ctx* ctx, uint64_t max_entries);

/* ── scene ───────────────────────────────────────────────────────────────
 * Replaces Scene::upload (Scene.cpp:255-515): copies the flat GpuScene
 * arrays to the device and builds the acceleration structure (a binned-SAH
 * BVH2 over world-space triangles instead of the driver BLAS/TLAS of
 * Scene.cpp:449-507). Host arrays; the call is synchronous. */
typedef struct rr_scene_desc {
    const GpuVertex*   vertices;   uint32_t vertex_count;
    const uint32_t*    indices;    uint32_t index_count;
    const GpuMesh*     meshes;     uint32_t mesh_count;
    const GpuMaterial* materials;  uint32_t material_count;
    const GpuInstance* instances;  uint32_t instance_count;
    const GpuLight*    lights;     uint32_t light_count;
} rr_scene_desc;

typedef struct rr_scene_stats {
    uint32_t triangle_count;
    uint32_t bvh_node_count;      /* GPU nodes (each holds two child boxes) */
    uint32_t bvh_max_depth;
    uint32_t light_count;
    double   build_ms;            /* host BVH build */
    double   upload_ms;
    uint64_t device_bytes;
    uint32_t bvh4_node_count;     /* nodes of the same tree laid out 4-wide (four child boxes each) */
    uint32_t _pad;
} rr_scene_stats;

rr_status rr_scene_create(rr_ctx* ctx, const rr_scene_desc* desc, rr_scene** out_scene);
rr_status rr_scene_destroy(rr_scene* scene);
rr_status rr_scene_get_stats(const rr_scene* scene, rr_scene_stats* out);

/* ── reference path tracer: PathTracerPass::execute
 * (PathTracerPass.cpp:170-224, kernel pathtracer.slang:181-265).
 * PathTracerPushConstants (PathTracerPass.cpp:15-32) -> frame_seed,
 * max_bounces; num_lights/num_instances come from the scene. `spp` > 1
 * renders the consecutive frame seeds frame_seed .. frame_seed+spp-1 in one
 * call (identical to spp reference frames); radiance_out holds spp images of
 * screen_width x screen_height RGBA32F, image k for seed frame_seed+k. */
typedef struct rr_pt_params {
    uint32_t frame_seed;
    uint32_t max_bounces;
    uint32_t spp;
    uint32_t flags;               /* RR_PT_FLAG_* */
} rr_pt_params;

/* Count BVH nodes visited and triangles tested (slower; for roofline bytes). */
#define RR_PT_FLAG_COUNT_TRAVERSAL 1u
/* Record CUDA events around every stage kernel on `stream`. */
#define RR_PT_FLAG_TIME_STAGES 2u

rr_status rr_pathtracer_execute(rr_ctx* ctx, const rr_scene* scene,
                                const GpuCameraData* camera, const rr_pt_params* params,
                                float* radiance_out, void* stream);

/* Statistics of this context's path tracer (synchronises the device):
 * ray counts of the last execute, traversal work of the last execute run
 * with RR_PT_FLAG_COUNT_TRAVERSAL, and stage times summed over all executes
 * run with RR_PT_FLAG_TIME_STAGES since the last reset. */
typedef struct rr_pt_stats {
    uint64_t extension_rays;
    uint64_t shadow_rays;
    uint64_t extension_nodes;     /* BVH nodes visited (each = 64 bytes) */
    uint64_t extension_tris;      /* triangles tested */
    uint64_t shadow_nodes;
    uint64_t shadow_tris;
    double   ms_raygen;
    double   ms_extend;
    double   ms_shade;
    double   ms_shadow;
    uint64_t launches_extend;     /* timed launches per stage */
    uint64_t launches_total;      /* kernel launches issued by this context */
} rr_pt_stats;

rr_status rr_pathtracer_stats(rr_ctx* ctx, rr_pt_stats* out, int reset_times);

/* Traversal kernel variants (no reference counterpart; the reference uses
 * hardware ray queries): variant = tree x stack x occupancy target; every
 * warp traces 32 consecutive queue entries to completion.
 *   0: binary tree, stack in local memory, the compiler's register count
 *      (default);
 *   1: as 0 with a register budget for 5 blocks of 256 threads per SM;
 *   2: as 0 with the bottom 8 stack entries in shared memory;
 *   5: as 2 with a budget for 5 blocks;
 *   3, 4, 6: the 4-wide tree (rr_pathtracer_variant_width), stack in local
 *      memory / bottom 8 entries in shared memory / as 4 with a budget for 3
 *      blocks;
 *   7: binary tree with leaves postponed until every lane of the warp holds
 *      one, budget for 4 blocks.
 * Results are identical for every variant; only speed differs. */
#define RR_PT_VARIANT_COUNT 8
rr_status rr_pathtracer_set_variants(rr_ctx* ctx, int extend_variant, int shadow_variant);

/* Shadow overlap (default on): the path tracers (rr_pathtracer_execute,
 * rr_guided_pathtracer_execute, rr_batch_execute, rr_batch_execute_guided)
 * trace bounce b's shadow rays on a second stream of the context while
 * bounce b+1's extension rays run on the caller's stream; the next shade
 * stage waits for both, and the call's work is joined back into the caller's
 * stream before it returns (so CUDA-graph capture of the caller's stream
 * still works). Results are identical either way. Calls with
 * RR_PT_FLAG_TIME_STAGES run on one stream, so that each stage is timed
 * alone. */
rr_status rr_pathtracer_set_overlap(rr_ctx* ctx, int enable);

/* Autotuner: renders the given frame once per variant with stage timing,
 * keeps the fastest extension and shadow variants on this context and
 * reports every measured time (ms per frame). Synchronises the device. */
typedef struct rr_pt_tune_result {
    double extend_ms[RR_PT_VARIANT_COUNT];
    double shadow_ms[RR_PT_VARIANT_COUNT];
    int    best_extend;
    int    best_shadow;
} rr_pt_tune_result;

rr_status rr_pathtracer_tune(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* camera,
                             const rr_pt_params* params, float* radiance_out, void* stream,
                             rr_pt_tune_result* out);

/* ── batches of scenes (no reference counterpart: the reference renders one
 * scene per PathTracerPass::execute). A batch renders many scenes, each with
 * its own camera and image size, in one set of wavefront launches (raygen,
 * then per bounce one extend, one shade and one shadow launch for all
 * scenes). Every scene's images are bit-identical to rr_pathtracer_execute
 * of that scene with the same camera and params. The scenes must outlive
 * the batch. */
typedef struct rr_batch rr_batch;
rr_status rr_batch_create(rr_ctx* ctx, const rr_scene* const* scenes, uint32_t count, rr_batch** out);
rr_status rr_batch_destroy(rr_batch* batch);

/* Capture the batch's launches in a CUDA graph (on the first call with a
 * given configuration) and replay it; the per-call cameras, frame seed and
 * output pointers travel in a small table copied before the replay. */
#define RR_PT_FLAG_GRAPH 4u
/* Emitter sampling (no reference counterpart; the reference's NEE samples
 * only its point and directional GpuLights, pathtracer.slang:124-177, and
 * reaches emissive triangles only by BSDF sampling, :225-229). For
 * rr_pathtracer_execute: next-event estimation picks, per vertex, the
 * GpuLights (as the reference picks among them) or the scene's emissive
 * triangles (each with probability 1/2 when both exist); an emissive
 * triangle is picked in proportion to luminance(emission) x area and a
 * point uniform on it, with its area-measure density turned into solid
 * angle; BSDF bounces are weighted by the density brdf_sample actually
 * draws from, and an emissive surface reached by a bounce is weighted
 * against the emitter sample by the power heuristic. The default (flag
 * clear) is the reference's estimator, bit for bit. Also for
 * rr_guided_pathtracer_execute, where the bounce density in the weights is
 * the guided mixture's. Not for batches (RR_ERR_UNSUPPORTED). */
#define RR_PT_FLAG_EMITTERS 8u

/* cameras[i] and radiance_out[i] (spp images of cameras[i]'s size, device
 * memory) for scene i; params are shared by all scenes (frame_seed,
 * max_bounces, spp, flags: RR_PT_FLAG_COUNT_TRAVERSAL and
 * RR_PT_FLAG_TIME_STAGES as for rr_pathtracer_execute, or RR_PT_FLAG_GRAPH).
 * Host memory of the arguments may be reused as soon as the call returns. */
rr_status rr_batch_execute(rr_ctx* ctx, rr_batch* batch, const GpuCameraData* cameras,
                           const rr_pt_params* params, float* const* radiance_out, void* stream);

/* rr_pathtracer_tune for a batch: times every traversal variant on the
 * batch, keeps the fastest on the context (graphs are recaptured), then
 * times the batch's two forms with those variants and keeps the faster on
 * the batch (rr_batch_get_mode). */
rr_status rr_batch_tune(rr_ctx* ctx, rr_batch* batch, const GpuCameraData* cameras,
                        const rr_pt_params* params, float* const* radiance_out, void* stream,
                        rr_pt_tune_result* out);

/* The batch's form: RR_BATCH_WAVEFRONT (default) renders all scenes in one
 * set of wavefront launches (graph-replayable); RR_BATCH_PER_SCENE renders
 * them one rr_pathtracer_execute after another (launched directly, also with
 * RR_PT_FLAG_GRAPH), which is faster when every scene alone fills the GPU:
 * the scenes' many short launch tails are then filled by the shadow overlap.
 * Both give the same images; calls with RR_PT_FLAG_COUNT_TRAVERSAL or
 * RR_PT_FLAG_TIME_STAGES use the wavefront form. */
#define RR_BATCH_WAVEFRONT 0
#define RR_BATCH_PER_SCENE 1
rr_status rr_batch_set_mode(rr_batch* batch, int mode);
rr_status rr_batch_get_mode(const rr_batch* batch, int* mode_out);

/* ── accumulate: AccumulatePass::execute (AccumulatePass.cpp:167-218,
 * kernel accumulate.slang:21-46). AccumulatePushConstants minus indices.
 * Folds `image_count` consecutive radiance images into `accumulated` in
 * order, as image_count reference frames would (the first with the given
 * camera_moved flag). oracle_sum (nullable, double[4*W*H]) keeps the FP64
 * per-pixel sum of every folded image (reset together with the FP32 mean),
 * the judge buffer for RMSE; it is the only FP64 state of the path.
 * width * height must be below 2^30 (RR_ERR_INVALID_ARGUMENT otherwise). */
typedef struct rr_acc_params {
    uint32_t width;
    uint32_t height;
    uint32_t camera_moved;
    uint32_t accumulated_spp;     /* spp BEFORE this call */
} rr_acc_params;

rr_status rr_accumulate_execute(rr_ctx* ctx, const float* radiance, uint32_t image_count,
                                float* accumulated, double* oracle_sum,
                                const rr_acc_params* params, void* stream);

/* ── ReSTIR DI: ReSTIRDIPass::execute (ReSTIRDIPass.cpp:306-446; kernels
 * restir_di.slang cs_initial :186-262, cs_temporal :266-335,
 * cs_spatial_shade :339-472). ReSTIRDIPushConstants (ReSTIRDIPass.cpp:18-45)
 * minus indices. m_cap_factor is 20 in the reference (restir_di.slang:300).
 * gbuf_pos/gbuf_norm/reservoir_curr/reservoir_prev/output: W x H RGBA32F. */
typedef struct rr_di_params {
    uint32_t frame_seed;
    uint32_t num_initial_candidates;
    uint32_t temporal_enable;
    uint32_t spatial_enable;
    uint32_t spatial_num_neighbors;
    uint32_t spatial_radius;
    uint32_t m_cap_factor;
    uint32_t flags;               /* RR_DI_FLAG_* */
} rr_di_params;

/* Emitter candidates (no reference counterpart; the reference's candidates
 * are its GpuLights only, restir_di.slang:229-247). A candidate is the pixel
 * RNG's next 32-bit state, stored as the reservoir's selection; the light
 * sample it names is decoded from that state wherever the reservoir is
 * reused: the group (GpuLights or the scene's emissive triangles, 1/2 each
 * when both exist), then a GpuLight picked as the reference picks one, or an
 * emissive triangle picked in proportion to luminance(emission) x area and a
 * point uniform on it. RIS weights use each sample's own source density; an
 * emitter point's target is max(n.l, 0) luminance(Le |cos_y| / d^2) and its
 * shading irradiance Le |cos_y| / d^2. Same reservoir layout and buffers. */
#define RR_DI_FLAG_EMITTERS 1u

rr_status rr_restir_di_initial(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* camera,
                               const rr_di_params* params, float* gbuf_pos, float* gbuf_norm,
                               float* reservoir_curr, void* stream);
rr_status rr_restir_di_temporal(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* camera,
                                const rr_di_params* params, const float* gbuf_pos,
                                const float* gbuf_norm, float* reservoir_curr,
                                const float* reservoir_prev, void* stream);
rr_status rr_restir_di_spatial_shade(rr_ctx* ctx, const rr_scene* scene,
                                     const GpuCameraData* camera, const rr_di_params* params,
                                     const float* gbuf_pos, const float* gbuf_norm,
                                     const float* reservoir_curr, float* output, void* stream);
/* The three dispatches in order (one ReSTIRDIPass::execute). */
rr_status rr_restir_di_execute(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* camera,
                               const rr_di_params* params, float* gbuf_pos, float* gbuf_norm,
                               float* reservoir_curr, const float* reservoir_prev,
                               float* output, void* stream);

/* ── A-trous denoiser: AtrousPass (AtrousPass.cpp:243-306, kernel
 * atrous.slang:41-106). rr_atrous_iteration is one cs_main dispatch with
 * AtrousPushConstants (AtrousPass.cpp:18-34); rr_atrous_execute runs
 * `iterations` (clamped to 1..7) ping-ponging ping0/ping1 with stride 1<<i
 * and reports which buffer holds the result ((iterations-1) & 1). */
typedef struct rr_atrous_params {
    uint32_t width;
    uint32_t height;
    uint32_t iterations;          /* execute: count; iteration: index */
    uint32_t stride;              /* iteration only */
    float    sigma_position;
    float    sigma_normal;
    float    sigma_luminance;
    uint32_t _pad;
} rr_atrous_params;

rr_status rr_atrous_iteration(rr_ctx* ctx, const float* input, const float* gbuf_pos,
                              const float* gbuf_norm, float* output,
                              const rr_atrous_params* params, void* stream);
rr_status rr_atrous_execute(rr_ctx* ctx, const float* input, const float* gbuf_pos,
                            const float* gbuf_norm, float* ping0, float* ping1,
                            const rr_atrous_params* params, uint32_t* out_slot, void* stream);

/* Strides 1, 2 and 4 run a kernel whose blocks first copy their halo tile
 * of the three images into shared memory with TMA tensor copies (default
 * on; the same bits as the direct-load kernel, which strides 8 and up use).
 * A block whose copies miss the kernel's bounded wait (wait_tries tries,
 * default 2^22) sets a host-mapped flag, waits once more (bounded) for its
 * copies, and filters its pixels from global memory instead: the output is
 * still complete and the same bits. The next rr_atrous_iteration or
 * rr_atrous_execute call on the context then returns RR_ERR_TIMEOUT without
 * doing its work (the message says so) and clears the flag; calling again
 * proceeds. rr_atrous_tma_error synchronizes the device, reports the flag
 * and clears it. rr_atrous_set_tma_wait_tries sets the tries (0 makes every
 * block give up at once, which exercises that path: the copies still land
 * before the block leaves). */
rr_status rr_atrous_set_tma(rr_ctx* ctx, int enable);
rr_status rr_atrous_tma_error(rr_ctx* ctx, int* error_out);
rr_status rr_atrous_set_tma_wait_tries(rr_ctx* ctx, uint32_t tries);

/* No counterpart in the reference: an A-trous entry point that allocates
 * nothing, for callers that cannot allocate device memory (an engine that
 * only lends the library buffers from its own fixed budget, a host that
 * forbids cudaMalloc while it renders frames). It needs no rr_ctx and gives
 * the same result as rr_atrous_execute, written to `output`. Its one
 * intermediate image lives in a fixed array in the library's device memory
 * (RR_ATROUS_STATIC_MAX_PIXELS RGBA32F pixels, 36 MiB, held on every GPU
 * that loads the library until the process exits). Images with more pixels
 * return RR_ERR_UNSUPPORTED; null buffers, a width above 65535 x 16 or a
 * height above 65535 x 8, or an output that overlaps the input or either
 * G-buffer image return RR_ERR_INVALID_ARGUMENT. The first call in each CUDA
 * context of a device looks up the array's device address (with that device
 * current) and should come before any stream capture; the address is cached
 * with the context's unique id, so a call after cudaDeviceReset (a new
 * context) looks it up again instead of using a stale address. A failed
 * launch returns RR_ERR_CUDA; errors left by earlier, unrelated work are not
 * reported or cleared. All calls share the array: calls whose kernels
 * overlap on the GPU race on it. */
#define RR_ATROUS_STATIC_MAX_PIXELS (2048u * 1152u)
rr_status rr_atrous_execute_static(const float* input, const float* gbuf_pos,
                                   const float* gbuf_norm, float* output,
                                   const rr_atrous_params* params, void* stream);

/* ── vMF path-guiding grid (GuidingGrid.slang; host side
 * ReSTIRPTPass.cpp:311-341, 602-611, 784-810; params ReSTIRPTPass.h:93-100).
 * accum: int32[4*cell_count] fixed-point sums (x, y, z, count);
 * fitted: float[4*cell_count] (mu.xyz, kappa). Points are float4 arrays. */
typedef struct rr_guiding_params {
    float    base_cell_size;      /* 0.10 */
    float    distance_slope;      /* 0.02 */
    uint32_t cell_count;          /* 1 << 20 */
    uint32_t enabled;
    uint32_t min_samples;         /* 8 */
    float    kappa_max;           /* 512 */
    float    alpha;               /* 0.5, P(guided sample) */
    uint32_t _pad;
} rr_guiding_params;

/* guiding_splat at the call site restir_pt.slang:982-994: one direction per
 * point into the cell of (pos, bsdf_id). */
rr_status rr_guiding_splat(rr_ctx* ctx, int32_t* accum, const float* pos, const float* dir,
                           const uint32_t* bsdf_id, uint32_t count, const float camera_pos[3],
                           const rr_guiding_params* params, void* stream);
/* cs_fit_guiding (restir_pt.slang:1005-1015): fit every cell, reset accum. */
rr_status rr_guiding_fit(rr_ctx* ctx, int32_t* accum, float* fitted,
                         const rr_guiding_params* params, void* stream);
/* sample_primary_dir (restir_pt.slang:520-563) at `count` points; seeds are
 * advanced in place; wi_out float4, pdf_out float. */
rr_status rr_guiding_sample(rr_ctx* ctx, const float* fitted, const float* pos,
                            const float* normal, const uint32_t* bsdf_id, uint32_t* seeds,
                            uint32_t count, const float camera_pos[3],
                            const rr_guiding_params* params, float* wi_out, float* pdf_out,
                            void* stream);
/* Host-side grid reset of ReSTIRPTPass.cpp:602-611 (zero accum and fitted). */
rr_status rr_guiding_reset(rr_ctx* ctx, int32_t* accum, float* fitted,
                           const rr_guiding_params* params, void* stream);

/* ── ReSTIR PT: ReSTIRPTPass::execute (ReSTIRPTPass.cpp:529-812; kernels in
 * passes/restir_pt/restir_pt.slang) ──────────────────────────────────────
 * rr_restir_pt_params holds the ReSTIRPTPushConstants fields
 * (ReSTIRPTPass.cpp:34-83) other than the bindless indices; the guiding
 * fields are an rr_guiding_params (guiding_enable -> enabled, guiding_alpha ->
 * alpha). Reference defaults (ReSTIRPTPass.h:86-100) in comments. */
typedef struct rr_restir_pt_params {
    uint32_t frame_seed;               /* frame_count_++ */
    uint32_t num_initial_candidates;   /* 8 */
    uint32_t max_bounces;              /* 4 */
    uint32_t temporal_enable;          /* 1 */
    uint32_t spatial_enable;           /* 1 */
    uint32_t spatial_num_neighbors;    /* 4 */
    uint32_t spatial_radius;           /* 12 */
    uint32_t include_direct_lighting;  /* 1 */
    float    indirect_strength;        /* 1.0 */
    float    ray_bias;                 /* 1e-3 */
    uint32_t _pad[2];
    rr_guiding_params guiding;         /* enabled 1, alpha 0.5, 0.10 / 0.02, 1 << 20 cells, 8, 512 */
} rr_restir_pt_params;

/* The pass's images, every one width x height RGBA32F (float4 per pixel),
 * device memory owned by the caller. The reservoir is four images
 * (restir_pt.slang:10-25): [0] (rc_pos, w_sum), [1] (rc_normal, asfloat(M)),
 * [2] (suffix radiance, W), [3] (prefix throughput, valid); the primary
 * history is (position, t) and (normal, asfloat(material)). "curr" and "prev"
 * swap after every frame, as ReSTIRPTPass::execute flips reservoir_flip_. */
typedef struct rr_restir_pt_images {
    const float* gbuf_pos;        /* ReSTIR DI's G-buffer (restir_di.slang:212-223) */
    const float* gbuf_norm;
    const float* direct;          /* direct lighting to add (the DI output) or NULL */
    float*       reservoir_curr[4];
    float*       reservoir_prev[4];
    float*       history_curr[2];
    float*       history_prev[2];
    float*       output;
    int32_t*     guiding_accum;   /* guiding.cell_count x int32 x 4 */
    float*       guiding_fitted;  /* guiding.cell_count x float x 4 */
} rr_restir_pt_images;

/* cs_initial (restir_pt.slang:567-757). By default run as a wavefront: the
 * per-pixel candidate loop is cut at every ray, each pixel's state kept in
 * device memory, and every step traces one path segment (and its light
 * sample's shadow ray) of every pixel that has one, through the queue
 * traversal kernels; the results are those of one thread per pixel running
 * the loop, bit for bit. */
rr_status rr_restir_pt_initial(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* camera,
                               const rr_restir_pt_params* params, const rr_restir_pt_images* images,
                               void* stream);
/* 1 (default): rr_restir_pt_initial and rr_restir_gi_initial run as
 * wavefronts; 0: one thread per pixel runs the whole candidate loop. Both
 * forms give the same bits. */
rr_status rr_reuse_set_wavefront(rr_ctx* ctx, int enable);
/* cs_temporal (restir_pt.slang:760-857); returns at once when temporal_enable is 0. */
rr_status rr_restir_pt_temporal(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* camera,
                                const rr_restir_pt_params* params, const rr_restir_pt_images* images,
                                void* stream);
/* cs_spatial_shade (restir_pt.slang:860-1000), including the guiding splat. */
rr_status rr_restir_pt_spatial_shade(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* camera,
                                     const rr_restir_pt_params* params,
                                     const rr_restir_pt_images* images, void* stream);
/* The dispatches of one ReSTIRPTPass::execute in order: initial, temporal,
 * spatial shade, and cs_fit_guiding when guiding is enabled. The caller swaps
 * curr and prev afterwards. */
rr_status rr_restir_pt_execute(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* camera,
                               const rr_restir_pt_params* params, const rr_restir_pt_images* images,
                               void* stream);
/* History reset (ReSTIRPTPass.cpp:616-652, consume_history_dirty): the prev
 * reservoir images to zero, the prev history position to (0, 0, 0, -1) and
 * normal to zero. */
rr_status rr_restir_pt_reset_history(rr_ctx* ctx, const rr_restir_pt_images* images, uint32_t width,
                                     uint32_t height, void* stream);

/* ── ReSTIR GI: ReSTIRGIPass::execute (ReSTIRGIPass.cpp:428-650; kernels in
 * passes/restir_gi/restir_gi.slang) ──────────────────────────────────────
 * rr_restir_gi_params holds the ReSTIRGIPushConstants fields
 * (restir_gi.slang:18-55) other than the bindless indices. Reference
 * defaults (ReSTIRGIPass.h:67-74) in comments. */
typedef struct rr_restir_gi_params {
    uint32_t frame_seed;               /* frame_count_++ */
    uint32_t num_initial_candidates;   /* 8 */
    uint32_t temporal_enable;          /* 1 */
    uint32_t spatial_enable;           /* 1 */
    uint32_t spatial_num_neighbors;    /* 4 */
    uint32_t spatial_radius;           /* 12 */
    uint32_t include_direct_lighting;  /* 1 */
    float    indirect_strength;        /* 1.0 */
    float    ray_bias;                 /* 1e-3 */
    uint32_t _pad[3];
} rr_restir_gi_params;

/* The pass's images, every one width x height RGBA32F, device memory owned
 * by the caller. The reservoir is three images (restir_gi.slang:3-7):
 * [0] (sample_pos, w_sum), [1] (sample_radiance, W), [2] (sample_normal,
 * asfloat(M)); the primary history is (position, t) and (normal,
 * asfloat(material)). "curr" and "prev" swap after every frame, as
 * ReSTIRGIPass::execute flips reservoir_flip_. */
typedef struct rr_restir_gi_images {
    const float* gbuf_pos;        /* ReSTIR DI's G-buffer (restir_di.slang:212-223) */
    const float* gbuf_norm;
    const float* direct;          /* direct lighting to add (the DI output) or NULL */
    float*       reservoir_curr[3];
    float*       reservoir_prev[3];
    float*       history_curr[2];
    float*       history_prev[2];
    float*       output;
} rr_restir_gi_images;

/* cs_initial (restir_gi.slang:568-686): writes reservoir_curr and history_curr.
 * By default run as a wavefront (one candidate of every pixel per step; see
 * rr_reuse_set_wavefront), bit-identical to one thread per pixel. */
rr_status rr_restir_gi_initial(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* camera,
                               const rr_restir_gi_params* params, const rr_restir_gi_images* images,
                               void* stream);
/* cs_temporal (restir_gi.slang:688-848); returns at once when temporal_enable is 0. */
rr_status rr_restir_gi_temporal(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* camera,
                                const rr_restir_gi_params* params, const rr_restir_gi_images* images,
                                void* stream);
/* cs_spatial_shade (restir_gi.slang:851-1000). */
rr_status rr_restir_gi_spatial_shade(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* camera,
                                     const rr_restir_gi_params* params,
                                     const rr_restir_gi_images* images, void* stream);
/* The three dispatches of one ReSTIRGIPass::execute in order; the caller
 * swaps curr and prev afterwards. */
rr_status rr_restir_gi_execute(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* camera,
                               const rr_restir_gi_params* params, const rr_restir_gi_images* images,
                               void* stream);
/* History reset (ReSTIRGIPass.cpp:484-530, consume_history_dirty): the prev
 * reservoir images to zero, the prev history position to (0, 0, 0, -1) and
 * normal to zero. */
rr_status rr_restir_gi_reset_history(rr_ctx* ctx, const rr_restir_gi_images* images, uint32_t width,
                                     uint32_t height, void* stream);

/* ── guided path tracing (no reference counterpart beyond the hash grid
 * above: the reference guides only ReSTIR PT's primary bounce with one vMF
 * lobe per hashed cell, restir_pt.slang:520-563). A guide predicts a mixture
 * of up to 8 vMF lobes at every path vertex; the guided tracer draws each
 * bounce by one-sample MIS between the guide (probability alpha where the
 * guide has a lobe) and brdf_sample, with pdf = alpha p_guide + (1-alpha)
 * p_bsdf, so the estimator stays unbiased for any guide. It records, per
 * vertex, the sampled direction and the radiance that came back along it;
 * rr_guide_update trains the guide on those samples:
 *   RR_GUIDE_GRID: dense grid_resolution^3 cells over bounds_min..max, 8
 *     lobes per cell, stepwise EM whose sufficient statistics are FP64 sums
 *     reduced in a fixed order (deterministic);
 *   RR_GUIDE_MLP: a BF16 multilayer perceptron (position frequency encoding,
 *     normal, view direction -> 8 lobes) run on the tensor cores, trained
 *     with Adam on mlp_batch samples per update. */
typedef struct rr_guide rr_guide;

#define RR_GUIDE_GRID 0u
#define RR_GUIDE_MLP 1u

typedef struct rr_guide_desc {
    uint32_t kind;
    uint32_t grid_resolution;      /* cells per axis (64) */
    float    alpha;                /* P(sample the guide) at a guided vertex (0.5) */
    float    decay;                /* weight of earlier statistics per update (grid) */
    float    bounds_min[3];
    float    bounds_max[3];
    uint32_t max_samples;          /* training samples kept per frame */
    uint32_t mlp_batch;            /* samples per Adam step (1 << 18) */
    float    learning_rate;        /* Adam (1e-2) */
    uint32_t seed;
} rr_guide_desc;

typedef struct rr_guide_stats {
    uint64_t samples_recorded;     /* by the last guided execute */
    uint64_t samples_used;         /* by the last update */
    uint32_t cells_valid;          /* grid: cells with a fitted mixture */
    uint32_t updates;
    double   last_loss;            /* MLP: weighted NLL of the last step */
    double   ms_update;            /* device time of the last update */
} rr_guide_stats;

rr_status rr_guide_create(rr_ctx* ctx, const rr_guide_desc* desc, rr_guide** out);
rr_status rr_guide_destroy(rr_guide* guide);
rr_status rr_guide_reset(rr_ctx* ctx, rr_guide* guide, void* stream);
rr_status rr_guide_update(rr_ctx* ctx, rr_guide* guide, void* stream);
rr_status rr_guide_get_stats(rr_ctx* ctx, const rr_guide* guide, rr_guide_stats* out);
/* Same contract as rr_pathtracer_execute (spp images out); guide may not be
 * NULL. Training samples of this call replace the previous call's. */
/* Evaluates the guide at `count` surface points: surf holds 3 float4 per
 * point, (position, 1), (normal, 1 = valid), (view direction wo, 0); mix_out
 * receives 10 float4 per point: 8 lobes (mu.xyz, kappa) and the 8 lobe
 * weights (weights all zero where the guide has no mixture). */
rr_status rr_guide_eval(rr_ctx* ctx, rr_guide* guide, const float* surf, uint32_t count, float* mix_out,
                        void* stream);
/* MLP guides: host copies of the FP32 master parameters and of the last
 * gradient (loss-scaled by 1024), and an optional host overwrite of the
 * parameters (params_in). count must equal the parameter count (20784:
 * per layer W[out][in] then b[out], layers 80->64->64->64->64->48).
 * error_flag receives 1 if a tensor-core wait ever gave up. */
/* Replaces the training samples a guided execute recorded by caller-made
 * ones (device array, 16 floats per sample: position, weight; direction wi,
 * unique id as uint bits; normal, 0; view direction wo, 0), e.g. to train a
 * guide from another integrator. count <= max_samples. */
rr_status rr_guide_set_samples(rr_ctx* ctx, rr_guide* guide, const float* samples, uint32_t count,
                               void* stream);
#define RR_MLP_PARAM_COUNT 20784u
rr_status rr_guide_mlp_params(rr_ctx* ctx, rr_guide* guide, float* params_out, float* grad_out,
                              float* params_in, uint32_t count, int* error_flag);
rr_status rr_guided_pathtracer_execute(rr_ctx* ctx, const rr_scene* scene, const GpuCameraData* camera,
                                       const rr_pt_params* params, rr_guide* guide,
                                       float* radiance_out, void* stream);

/* Guided batches: rr_batch_execute with one guide per scene (guides[i] for
 * scene i; all of one kind, none twice). Each scene's image, and the training
 * samples recorded into its guide (as a set), are those of
 * rr_guided_pathtracer_execute of that scene alone with the same guide,
 * camera and params. MLP guides run grouped: at every bounce the queries are
 * gathered per scene and one tensor-core launch runs each group through its
 * own scene's network. flags: RR_PT_FLAG_GRAPH captures the frame in a CUDA
 * graph on first use and replays it after; the counting and timing flags are
 * ignored. */
rr_status rr_batch_execute_guided(rr_ctx* ctx, rr_batch* batch, const GpuCameraData* cameras,
                                  const rr_pt_params* params, rr_guide* const* guides,
                                  float* const* radiance_out, void* stream);
/* rr_guide_update of `count` guides, with one host wait for all of their
 * sample counts (rr_guide_update is this call with one guide). */
rr_status rr_guides_update(rr_ctx* ctx, rr_guide* const* guides, uint32_t count, void* stream);

/* ── output formats: tonemap, PNG and the crop MSE ──────────────────────
 * rr_tonemap_execute: exposure, ACES filmic approximation, clamp, gamma
 * 1/2.2, 8-bit RGBA (Application.cpp:853-866; tonemap.slang:40-69).
 * rr_image_mse: FP64 mean squared error over the RGB channels of the window
 * [x0, x0+w) x [y0, y0+h) of two W x H RGBA32F images, written to a device
 * double (Application::compute_mse, Application.cpp:892-949). Fixed
 * reduction order: deterministic. */
rr_status rr_tonemap_execute(rr_ctx* ctx, const float* hdr, uint32_t width, uint32_t height,
                             float exposure, uint8_t* rgba8_out, void* stream);
rr_status rr_image_mse(rr_ctx* ctx, const float* a, const float* b, uint32_t width, uint32_t height,
                       uint32_t x0, uint32_t y0, uint32_t w, uint32_t h, double* mse_out_dev,
                       void* stream);

/* ── ray queries (checking and tooling) ─────────────────────────────────
 * Closest hit for `count` rays: origins/dirs float4, hits float4
 * (t, u, v, as_float(instance)) and prims uint32; instance 0xffffffff = miss. */
rr_status rr_trace_closest(rr_ctx* ctx, const rr_scene* scene, const float* origins,
                           const float* dirs, float tmin, float tmax, uint32_t count,
                           float* hits, uint32_t* prims, void* stream);
/* The same query with the traversal's work counters. flags: bit 0
 * (RR_TRACE_ANY_HIT) selects the shadow-ray (first hit) form, bit 1
 * (RR_TRACE_WIDE) the 4-wide tree; work receives per ray (BVH nodes
 * visited, triangles tested), the counts behind RR_PT_FLAG_COUNT_TRAVERSAL. */
#define RR_TRACE_ANY_HIT 1
#define RR_TRACE_WIDE 2
rr_status rr_trace_counted(rr_ctx* ctx, const rr_scene* scene, const float* origins,
                           const float* dirs, float tmin, float tmax, uint32_t count, int flags,
                           float* hits, uint32_t* prims, uint32_t* work, void* stream);
/* Host copies of the scene's BVH (rr_scene_stats.bvh_node_count nodes of
 * 16 floats, layout in rr_trace.cuh) and triangle records (triangle_count
 * records of 12 floats). Synchronous. */
rr_status rr_scene_copy_bvh(rr_ctx* ctx, const rr_scene* scene, float* nodes_out, float* tris_out);
/* Host copy of the 4-wide layout of the same tree (rr_scene_stats.
 * bvh4_node_count nodes of 32 floats, layout in rr_trace.cuh). Synchronous. */
rr_status rr_scene_copy_bvh4(rr_ctx* ctx, const rr_scene* scene, float* nodes4_out);
/* Width of the tree a traversal variant walks: 2 or 4 (0 for a variant out
 * of range). A node of the 4-wide tree is 128 bytes, of the binary one 64. */
int rr_pathtracer_variant_width(int variant);
/* Bounded-wait self-test of the tensor-core kernels' mbarrier waits: one
 * block waits (at most `limit` tries, 1..2^22) on a barrier that nothing
 * arrives on and on one that received its arrival. completed_out[0] = 1 if
 * the first wait completed (0: it gave up, as it must), completed_out[1] =
 * 1 if the second completed. The kernel returns normally either way. */
rr_status rr_tc_wait_selftest(rr_ctx* ctx, uint32_t limit, int* completed_out);

#ifdef __cplusplus
}
#endif
#endif /* RR_CUDA_H */
