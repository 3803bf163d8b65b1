/*
 * rr_oracle.h — CPU checker for the light-transport path (TEST INFRASTRUCTURE).
 *
 * This library is the oracle: a scalar C++ restatement of the reference's
 * Slang kernels, used only by tests/, the smoke check and the CPU-baseline leg
 * of bench.py. It is never linked into, loaded by or called from the product
 * library. Every function cites the reference file:line it restates
 * (paths are relative to the reference project root).
 *
 * Parity status: the reference cannot be built or run as shipped (Vulkan 1.4
 * ray query + Slang + a Windows toolchain; no graphics stack exists on either
 * machine), and it ships no tests, golden images or known-answer vectors.
 * Its shader text is pinned instead: oracle/make_ref.py rewrites the
 * reference's .slang files mechanically into C++ (oracle/_ref/), and
 * tests/test_ref_text.py requires this restatement to give the same bits as
 * that text for the RNG, the BRDF, the guiding grid, the path tracer,
 * accumulate, ReSTIR DI, A-trous, ReSTIR PT and ReSTIR GI. Unpinned: the
 * hardware ray/triangle intersection (no source; this file's watertight test
 * decides hits), the driver's sin/cos/exp/log (rr_detmath.h on both sides)
 * and glm's camera math (absent; restated in closed form).
 *
 * Arithmetic is IEEE-754 binary32 in the expression order of the Slang source,
 * compiled with -ffp-contract=off; sin/cos/exp/log come from rr_detmath.h.
 */
#ifndef RR_ORACLE_H
#define RR_ORACLE_H

#include <stdint.h>
#include <stddef.h>
#include "rr_layouts.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleScene OracleScene;

/* ── RNG (Common.slang:18-28, Sampling.slang:11-30) ─────────────────────── */
uint32_t oracle_pcg_hash(uint32_t seed);
uint32_t oracle_make_seed(uint32_t px, uint32_t py, uint32_t frame_index);
float    oracle_rand_float(uint32_t* seed);

/* ── elementary functions used by the path (for checking rr_detmath.h) ─── */
void oracle_detmath_eval(int which, const float* x, float* y, size_t n);

/* ── Scene + ray queries ────────────────────────────────────────────────── */
/* use_bvh = 0: brute force over every triangle (small scenes).
 * use_bvh = 1: the oracle's own median-split BVH (independent of the product
 * builder); both return the same closest hit. */
OracleScene* oracle_scene_create(const GpuVertex* vertices, uint32_t vertex_count,
                                 const uint32_t* indices, uint32_t index_count,
                                 const GpuMesh* meshes, uint32_t mesh_count,
                                 const GpuMaterial* materials, uint32_t material_count,
                                 const GpuInstance* instances, uint32_t instance_count,
                                 const GpuLight* lights, uint32_t light_count,
                                 int use_bvh);
void oracle_scene_destroy(OracleScene* scene);
uint32_t oracle_scene_triangle_count(const OracleScene* scene);

/* Closest hit in [tmin, tmax]; returns 1 on hit and fills t, barycentrics
 * (weights of v1, v2) and (instance, mesh-local primitive). */
int oracle_trace(const OracleScene* scene, const float origin[3], const float dir[3],
                 float tmin, float tmax, float* t, float* bu, float* bv,
                 uint32_t* inst, uint32_t* prim);

/* Batched closest-hit queries; hits[i] = {t, u, v, as_float(inst)} and
 * prim[i] = primitive, inst = 0xffffffff on miss. */
void oracle_trace_batch(const OracleScene* scene, const float* origins /*n*4*/,
                        const float* dirs /*n*4*/, float tmin, float tmax, size_t n,
                        float* hits /*n*4*/, uint32_t* prims, int threads);

/* Primary-ray generation of pathtracer.slang:192-205 for one pixel. */
void oracle_primary_ray(const GpuCameraData* cam, uint32_t px, uint32_t py,
                        uint32_t frame_seed, float origin[3], float dir[3],
                        uint32_t* seed_out);

/* ── Reference path tracer (pathtracer.slang:181-265) ───────────────────── */
/* Renders the region [x0, x0+w) x [y0, y0+h) of the camera's image for
 * frame seeds frame_seed .. frame_seed+spp-1; out is spp images of w*h RGBA.
 * stats (nullable) receives {extension rays, shadow rays}. */
void oracle_pathtrace(const OracleScene* scene, const GpuCameraData* cam,
                      uint32_t frame_seed, uint32_t max_bounces, uint32_t spp,
                      uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                      float* out, int threads, uint64_t* stats);
/* The same with flags: ORACLE_PT_EMITTERS selects the emitter-sampling mode
 * (no reference counterpart; the library's RR_PT_FLAG_EMITTERS): NEE over the
 * GpuLights and the emissive triangles (power-proportional pick, uniform
 * point, area-measure density), bounces weighted by brdf_sample's actual
 * density, emissive hits weighted by the power heuristic. */
#define ORACLE_PT_EMITTERS 8u
void oracle_pathtrace_ex(const OracleScene* scene, const GpuCameraData* cam,
                         uint32_t frame_seed, uint32_t max_bounces, uint32_t spp,
                         uint32_t x0, uint32_t y0, uint32_t w, uint32_t h,
                         float* out, int threads, uint64_t* stats, uint32_t flags);
/* The emitter table: count, total power, and (if out is non-null) the
 * 12-float records followed by nothing else; cdf_out (nullable) receives
 * the prefix sums. */
uint32_t oracle_emitters(const OracleScene* scene, float* records_out, float* prob_out, uint32_t* alias_out,
                         float* total_out);

/* ── Accumulate (accumulate.slang:21-46) ────────────────────────────────── */
void oracle_accumulate(const float* radiance, float* accumulated, size_t pixels,
                       uint32_t camera_moved, uint32_t accumulated_spp);

/* ── ReSTIR DI (restir_di.slang) ────────────────────────────────────────── */
typedef struct OracleDIParams {
    uint32_t frame_seed;
    uint32_t num_initial_candidates;
    uint32_t temporal_enable;
    uint32_t spatial_enable;
    uint32_t spatial_num_neighbors;
    uint32_t spatial_radius;
    uint32_t m_cap_factor; /* 20 in the reference (restir_di.slang:300) */
    uint32_t flags;        /* ORACLE_DI_EMITTERS: candidates also from the emissive triangles */
} OracleDIParams;
/* Emitter candidates (no reference counterpart; the library's
 * RR_DI_FLAG_EMITTERS): a candidate is the pixel RNG's next state, and the
 * light sample it names (group, then a GpuLight, or an emissive triangle and
 * a point on it, as the emitter-sampling path tracer picks them) is decoded
 * from that state wherever the reservoir is reused. */
#define ORACLE_DI_EMITTERS 1u

void oracle_restir_di_initial(const OracleScene* scene, const GpuCameraData* cam,
                              const OracleDIParams* p, float* gbuf_pos, float* gbuf_norm,
                              float* reservoir_curr, int threads);
void oracle_restir_di_temporal(const OracleScene* scene, const GpuCameraData* cam,
                               const OracleDIParams* p, const float* gbuf_pos,
                               const float* gbuf_norm, float* reservoir_curr,
                               const float* reservoir_prev, int threads);
void oracle_restir_di_spatial_shade(const OracleScene* scene, const GpuCameraData* cam,
                                    const OracleDIParams* p, const float* gbuf_pos,
                                    const float* gbuf_norm, const float* reservoir_curr,
                                    float* output, int threads);

/* ── A-trous (atrous.slang:41-106) ──────────────────────────────────────── */
/* One tap's weight (the loop of oracle_atrous_iteration): centre position,
 * unit normal and luminance, neighbour position, unit normal and radiance,
 * tap offset, squared sigmas. */
float oracle_atrous_tap_weight(const float cp[3], const float cn[3], float cl, const float sp[3], const float sn[3],
                               const float srad[3], int tx, int ty, float sp2, float sn2, float sl2);
void oracle_atrous_iteration(const float* input, const float* gbuf_pos,
                             const float* gbuf_norm, float* output,
                             uint32_t width, uint32_t height, uint32_t stride,
                             float sigma_position, float sigma_normal,
                             float sigma_luminance, int threads);

/* ── vMF guiding grid (GuidingGrid.slang) ───────────────────────────────── */
typedef struct OracleGuidingParams {
    float    base_cell_size;
    float    distance_slope;
    uint32_t cell_count;
    uint32_t enabled;
    uint32_t min_samples;
    float    kappa_max;
    float    alpha;
    uint32_t _pad;
} OracleGuidingParams;

uint32_t oracle_guiding_cell_index(const float pos[3], uint32_t bsdf_id,
                                   const float cam_pos[3], const OracleGuidingParams* gp);
void oracle_guiding_splat(int32_t* accum, const float* pos /*n*4*/, const float* dir /*n*4*/,
                          const uint32_t* bsdf, size_t n, const float cam_pos[3],
                          const OracleGuidingParams* gp);
void oracle_guiding_fit(int32_t* accum, float* fitted, const OracleGuidingParams* gp);
/* sample_primary_dir (restir_pt.slang:520-563) for n surface points. */
void oracle_guiding_sample(const float* fitted, const float* pos /*n*4*/,
                           const float* normal /*n*4*/, const uint32_t* bsdf,
                           uint32_t* seeds, size_t n, const float cam_pos[3],
                           const OracleGuidingParams* gp, float* wi_out /*n*4*/,
                           float* pdf_out);
float oracle_vmf_pdf(const float mu[3], float kappa, const float dir[3]);

/* ── ReSTIR PT (restir_pt.slang:567-1000) ───────────────────────────────── */
typedef struct OracleRestirPtParams {
    uint32_t frame_seed;
    uint32_t num_initial_candidates;
    uint32_t max_bounces;
    uint32_t temporal_enable;
    uint32_t spatial_enable;
    uint32_t spatial_num_neighbors;
    uint32_t spatial_radius;
    uint32_t include_direct_lighting;
    float    indirect_strength;
    float    ray_bias;
    uint32_t _pad[2];
    OracleGuidingParams guiding;
} OracleRestirPtParams;

/* Images: width x height x 4 floats each (reservoir [0..3], history [0..1]). */
typedef struct OracleRestirPtImages {
    const float* gbuf_pos;
    const float* gbuf_norm;
    const float* direct;          /* or NULL */
    float*       reservoir_curr[4];
    float*       reservoir_prev[4];
    float*       history_curr[2];
    float*       history_prev[2];
    float*       output;
    int32_t*     guiding_accum;
    float*       guiding_fitted;
} OracleRestirPtImages;

void oracle_restir_pt_initial(const OracleScene* scene, const GpuCameraData* cam,
                              const OracleRestirPtParams* p, const OracleRestirPtImages* img, int threads);
void oracle_restir_pt_temporal(const OracleScene* scene, const GpuCameraData* cam,
                               const OracleRestirPtParams* p, const OracleRestirPtImages* img, int threads);
void oracle_restir_pt_spatial_shade(const OracleScene* scene, const GpuCameraData* cam,
                                    const OracleRestirPtParams* p, const OracleRestirPtImages* img,
                                    int threads);

/* The library's BVH2 traversal restated over its node / triangle arrays
 * (rr_scene_copy_bvh): hits as rr_trace_counted, work = (nodes, tris) per ray. */
void oracle_bvh2_trace(const float* nodes, uint32_t num_nodes, const float* tris, const float* origins,
                       const float* dirs, float tmin, float tmax, uint32_t n, int any_hit, float* hits,
                       uint32_t* prims, uint32_t* work, int threads);
void oracle_bvh4_trace(const float* nodes4, uint32_t num_nodes4, const float* tris, const float* origins,
                       const float* dirs, float tmin, float tmax, uint32_t n, int any_hit, float* hits,
                       uint32_t* prims, uint32_t* work, int threads);

/* ── ReSTIR GI (restir_gi.slang:568-1000) ───────────────────────────────── */
typedef struct OracleRestirGiParams {
    uint32_t frame_seed;
    uint32_t num_initial_candidates;
    uint32_t temporal_enable;
    uint32_t spatial_enable;
    uint32_t spatial_num_neighbors;
    uint32_t spatial_radius;
    uint32_t include_direct_lighting;
    float    indirect_strength;
    float    ray_bias;
    uint32_t _pad[3];
} OracleRestirGiParams;

/* Images: width x height x 4 floats each (reservoir [0..2], history [0..1]). */
typedef struct OracleRestirGiImages {
    const float* gbuf_pos;
    const float* gbuf_norm;
    const float* direct;          /* or NULL */
    float*       reservoir_curr[3];
    float*       reservoir_prev[3];
    float*       history_curr[2];
    float*       history_prev[2];
    float*       output;
} OracleRestirGiImages;

void oracle_restir_gi_initial(const OracleScene* scene, const GpuCameraData* cam,
                              const OracleRestirGiParams* p, const OracleRestirGiImages* img, int threads);
void oracle_restir_gi_temporal(const OracleScene* scene, const GpuCameraData* cam,
                               const OracleRestirGiParams* p, const OracleRestirGiImages* img, int threads);
void oracle_restir_gi_spatial_shade(const OracleScene* scene, const GpuCameraData* cam,
                                    const OracleRestirGiParams* p, const OracleRestirGiImages* img,
                                    int threads);

/* ── BRDF (BRDF.slang) for direct checks ────────────────────────────────── */
void oracle_brdf_eval(const float n[3], const float wo[3], const float wi[3],
                      const float base[3], float metallic, float roughness, float out[3]);
void oracle_brdf_sample(const float wo[3], const float n[3], const float base[3],
                        float metallic, float roughness, float u0, float u1,
                        float wi[3], float* pdf, float f[3]);
float oracle_brdf_pdf(const float wo[3], const float wi[3], const float n[3], float roughness);

#ifdef __cplusplus
}
#endif
#endif /* RR_ORACLE_H */
