// slang_ref_harness.cpp — runs the reference's own shader text (rewritten to
// C++ by oracle/make_ref.py into oracle/_ref/slang_ref_gen.h) on the CPU
// (TEST INFRASTRUCTURE ONLY; built into oracle/_ref/librr_slangref.so by
// oracle/Makefile, target `ref`).
//
// Each entry point mirrors one function of the hand-written oracle
// (rr_oracle.h), with the same arguments, so that the tests can check the
// restatement against the reference's text on the same inputs: it binds the
// scene arrays and images to the heap slots, fills the pass's push-constant
// block as the reference's host pass does, and dispatches the pass's compute
// entry point once per pixel (rows spread over threads; a dispatch's pixels
// are independent in the reference too). Ray queries go to the oracle's
// closest-hit intersector (oracle_trace), the stand-in for the reference's
// hardware BLAS/TLAS traversal.

#include "slang_ref_gen.h"

#include "rr_oracle.h"

#include <algorithm>
#include <thread>
#include <vector>

namespace slang {
ByteAddressBuffer gScene[16];
RWByteAddressBuffer gSceneRW[16];
RWTexture2D gStorageImages[32];
Texture2D gTextures[32];
RaytracingAccelerationStructure gTLAS[1];
} // namespace slang

using namespace slang;

namespace {

// scene heap slots
enum : uint { kCam = 0, kVtx = 1, kIdx = 2, kMesh = 3, kMat = 4, kInst = 5, kLight = 6 };

bool oracle_closest_hit(const void* scene, const float o[3], const float d[3], float tmin, float tmax, float* t,
                        float* u, float* v, uint* inst, uint* prim) {
    return oracle_trace(static_cast<const OracleScene*>(scene), o, d, tmin, tmax, t, u, v, inst, prim) != 0;
}

struct SrefScene {
    const OracleScene* tracer = nullptr;
    std::vector<GpuVertex> vertices;
    std::vector<uint32_t> indices;
    std::vector<GpuMesh> meshes;
    std::vector<GpuMaterial> materials;
    std::vector<GpuInstance> instances;
    std::vector<GpuLight> lights;
};

template <class T> void bind_buffer(uint slot, const std::vector<T>& v) {
    gScene[slot].data = reinterpret_cast<const unsigned char*>(v.data());
    gScene[slot].size = v.size() * sizeof(T);
}

void bind_scene(const SrefScene* s, const GpuCameraData* cam) {
    gScene[kCam].data = reinterpret_cast<const unsigned char*>(cam);
    gScene[kCam].size = sizeof(GpuCameraData);
    bind_buffer(kVtx, s->vertices);
    bind_buffer(kIdx, s->indices);
    bind_buffer(kMesh, s->meshes);
    bind_buffer(kMat, s->materials);
    bind_buffer(kInst, s->instances);
    bind_buffer(kLight, s->lights);
    gTLAS[0].scene = s->tracer;
    gTLAS[0].closest_hit = oracle_closest_hit;
}

void bind_image(uint slot, float* data, uint W, uint H) {
    gStorageImages[slot].data = reinterpret_cast<float4*>(data);
    gStorageImages[slot].width = W;
    gStorageImages[slot].height = H;
    gStorageImages[slot].ox = 0;
    gStorageImages[slot].oy = 0;
}

// Runs fn(x, y) for every pixel of [x0, x0+w) x [y0, y0+h), rows over threads.
template <class F> void dispatch(uint x0, uint y0, uint w, uint h, int threads, F fn) {
    const int nt = std::max(1, std::min<int>(threads, int(h)));
    std::vector<std::thread> pool;
    for (int t = 0; t < nt; ++t)
        pool.emplace_back([=] {
            for (uint y = y0 + uint(t); y < y0 + h; y += uint(nt))
                for (uint x = x0; x < x0 + w; ++x) fn(x, y);
        });
    for (auto& th : pool) th.join();
}

float3 f3(const float* p) { return float3(p[0], p[1], p[2]); }
void put3(float* o, const float3& v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }

} // namespace

static_assert(sizeof(ref_pt::GpuCameraData) == sizeof(GpuCameraData), "camera layout");
static_assert(sizeof(ref_pt::GpuInstance) == sizeof(GpuInstance) && sizeof(ref_pt::GpuMaterial) == sizeof(GpuMaterial),
              "scene layouts");
static_assert(sizeof(ref_pt::GpuLight) == sizeof(GpuLight) && sizeof(ref_pt::GpuVertex) == sizeof(GpuVertex) &&
                  sizeof(ref_pt::GpuMesh) == sizeof(GpuMesh),
              "scene layouts");

extern "C" {

// ── shared includes (Common, Sampling, BRDF, GuidingGrid) ──────────────────
uint32_t sref_pcg_hash(uint32_t x) { return ref_inc::pcg_hash(x); }
uint32_t sref_make_seed(uint32_t px, uint32_t py, uint32_t frame) { return ref_inc::make_seed(uint2(px, py), frame); }
float sref_rand_float(uint32_t* seed) {
    uint s = *seed;
    const float r = ref_inc::rand_float(s);
    *seed = s;
    return r;
}

void sref_brdf_eval(const float n[3], const float wo[3], const float wi[3], const float base[3], float metallic,
                    float roughness, float out[3]) {
    put3(out, ref_inc::brdf_eval(f3(n), f3(wo), f3(wi), f3(base), metallic, roughness));
}

void sref_brdf_sample(const float wo[3], const float n[3], const float base[3], float metallic, float roughness,
                      float u0, float u1, float wi[3], float* pdf, float f[3]) {
    float3 w;
    float p = 0.0f;
    put3(f, ref_inc::brdf_sample(f3(wo), f3(n), f3(base), metallic, roughness, float2(u0, u1), w, p));
    put3(wi, w);
    *pdf = p;
}

float sref_brdf_pdf(const float wo[3], const float wi[3], const float n[3], float roughness) {
    return ref_inc::brdf_pdf(f3(wo), f3(wi), f3(n), roughness);
}

void sref_sample_cosine_hemisphere(float u0, float u1, float out[3], float* pdf) {
    float p = 0.0f;
    put3(out, ref_inc::sample_cosine_hemisphere(u0, u1, p));
    *pdf = p;
}

void sref_build_onb(const float n[3], float T[3], float B[3]) {
    float3 t, b;
    ref_inc::build_onb(f3(n), t, b);
    put3(T, t);
    put3(B, b);
}

void sref_vmf_sample(const float mu[3], float kappa, float u0, float u1, float dir[3], float* pdf) {
    float p = 0.0f;
    put3(dir, ref_inc::vmf_sample(f3(mu), kappa, float2(u0, u1), p));
    *pdf = p;
}

float sref_vmf_pdf(const float mu[3], float kappa, const float dir[3]) {
    return ref_inc::vmf_pdf(f3(mu), kappa, f3(dir));
}

uint32_t sref_guiding_cell_index(const float pos[3], uint32_t bsdf_id, const float cam_pos[3],
                                 const OracleGuidingParams* gp) {
    ref_inc::GuidingGridParams p;
    p.base_cell_size = gp->base_cell_size;
    p.distance_slope = gp->distance_slope;
    p.cell_count = gp->cell_count;
    p.enabled = gp->enabled;
    return ref_inc::guiding_cell_index(f3(pos), bsdf_id, f3(cam_pos), p);
}

// guiding_splat of direction i into its cell (cell index from
// guiding_cell_index of pos i), then nothing else: the accumulator as the
// reference's splat stage leaves it.
void sref_guiding_splat(int32_t* accum, const float* pos, const float* dir, const uint32_t* bsdf, size_t n,
                        const float cam_pos[3], const OracleGuidingParams* gp) {
    gSceneRW[0].data = reinterpret_cast<unsigned char*>(accum);
    gSceneRW[0].size = size_t(gp->cell_count) * 16u;
    for (size_t i = 0; i < n; ++i) {
        const uint cell = sref_guiding_cell_index(pos + 4 * i, bsdf[i], cam_pos, gp);
        ref_inc::guiding_splat(0u, cell, f3(dir + 4 * i));
    }
}

void sref_guiding_fit(int32_t* accum, float* fitted, const OracleGuidingParams* gp) {
    gSceneRW[0].data = reinterpret_cast<unsigned char*>(accum);
    gSceneRW[0].size = size_t(gp->cell_count) * 16u;
    gSceneRW[1].data = reinterpret_cast<unsigned char*>(fitted);
    gSceneRW[1].size = size_t(gp->cell_count) * 16u;
    for (uint c = 0; c < gp->cell_count; ++c) ref_inc::guiding_fit_cell(0u, 1u, c, gp->min_samples, gp->kappa_max);
}

// ── scenes ──────────────────────────────────────────────────────────────────
void* sref_scene_create(const OracleScene* tracer, const GpuVertex* v, uint32_t nv, const uint32_t* idx,
                        uint32_t ni, const GpuMesh* m, uint32_t nm, const GpuMaterial* mat, uint32_t nmat,
                        const GpuInstance* inst, uint32_t ninst, const GpuLight* l, uint32_t nl) {
    auto* s = new SrefScene;
    s->tracer = tracer;
    s->vertices.assign(v, v + nv);
    s->indices.assign(idx, idx + ni);
    s->meshes.assign(m, m + nm);
    s->materials.assign(mat, mat + nmat);
    s->instances.assign(inst, inst + ninst);
    if (nl) s->lights.assign(l, l + nl);
    return s;
}

void sref_scene_destroy(void* s) { delete static_cast<SrefScene*>(s); }

// ── pathtracer.slang:cs_main, PathTracerPass::execute (PathTracerPass.cpp:170-224)
void sref_pathtrace(const void* sv, const GpuCameraData* cam, uint32_t frame_seed, uint32_t max_bounces,
                    uint32_t spp, uint32_t x0, uint32_t y0, uint32_t w, uint32_t h, float* out, int threads) {
    const auto* s = static_cast<const SrefScene*>(sv);
    bind_scene(s, cam);
    using namespace ref_pt;
    pc = PushConstants{};
    pc.camera_buf_idx = kCam;
    pc.tlas_idx = 0;
    pc.radiance_img_idx = 0;
    pc.vertex_buf_idx = kVtx;
    pc.index_buf_idx = kIdx;
    pc.mesh_buf_idx = kMesh;
    pc.material_buf_idx = kMat;
    pc.instance_buf_idx = kInst;
    pc.light_buf_idx = kLight;
    pc.num_instances = uint(s->instances.size());
    pc.num_lights = uint(s->lights.size());
    pc.max_bounces = max_bounces;
    for (uint32_t k = 0; k < spp; ++k) {
        pc.frame_seed = frame_seed + k;
        // the region's image, addressed at full-image pixel coordinates
        bind_image(0, out + size_t(k) * w * h * 4, w, h);
        gStorageImages[0].ox = x0;
        gStorageImages[0].oy = y0;
        dispatch(x0, y0, w, h, threads, [](uint x, uint y) { cs_main(uint3(x, y, 0u)); });
    }
}

// ── accumulate.slang:cs_main (AccumulatePass.cpp:167-218)
void sref_accumulate(const float* radiance, float* accumulated, uint32_t W, uint32_t H, uint32_t camera_moved,
                     uint32_t accumulated_spp) {
    using namespace ref_acc;
    bind_image(0, const_cast<float*>(radiance), W, H);
    bind_image(1, accumulated, W, H);
    pc = PushConstants{};
    pc.radiance_idx = 0;
    pc.accumulated_idx = 1;
    pc.screen_width = W;
    pc.screen_height = H;
    pc.camera_moved = camera_moved;
    pc.accumulated_spp = accumulated_spp;
    dispatch(0, 0, W, H, 1, [](uint x, uint y) { cs_main(uint3(x, y, 0u)); });
}

// ── restir_di.slang (ReSTIRDIPass::execute, ReSTIRDIPass.cpp:306-446)
// stage 0 = cs_initial, 1 = cs_temporal, 2 = cs_spatial_shade
void sref_restir_di(int stage, const void* sv, const GpuCameraData* cam, const OracleDIParams* p, float* gbuf_pos,
                    float* gbuf_norm, float* res_curr, float* res_prev, float* output, int threads) {
    const auto* s = static_cast<const SrefScene*>(sv);
    bind_scene(s, cam);
    const uint W = cam->screen_width, H = cam->screen_height;
    bind_image(0, gbuf_pos, W, H);
    bind_image(1, gbuf_norm, W, H);
    bind_image(2, res_curr, W, H);
    bind_image(3, res_prev, W, H);
    bind_image(4, output, W, H);
    using namespace ref_di;
    pc = PushConstants{};
    pc.camera_buf_idx = kCam;
    pc.tlas_idx = 0;
    pc.vertex_buf_idx = kVtx;
    pc.index_buf_idx = kIdx;
    pc.mesh_buf_idx = kMesh;
    pc.material_buf_idx = kMat;
    pc.instance_buf_idx = kInst;
    pc.light_buf_idx = kLight;
    pc.num_instances = uint(s->instances.size());
    pc.num_lights = uint(s->lights.size());
    pc.frame_seed = p->frame_seed;
    pc.gbuf_pos_idx = 0;
    pc.gbuf_norm_idx = 1;
    pc.reservoir_curr_idx = 2;
    pc.reservoir_prev_idx = 3;
    pc.output_idx = 4;
    pc.num_initial_candidates = p->num_initial_candidates;
    pc.temporal_enable = p->temporal_enable;
    pc.spatial_enable = p->spatial_enable;
    pc.spatial_num_neighbors = p->spatial_num_neighbors;
    pc.spatial_radius = p->spatial_radius;
    if (stage == 0) dispatch(0, 0, W, H, threads, [](uint x, uint y) { cs_initial(uint3(x, y, 0u)); });
    else if (stage == 1) dispatch(0, 0, W, H, threads, [](uint x, uint y) { cs_temporal(uint3(x, y, 0u)); });
    else dispatch(0, 0, W, H, threads, [](uint x, uint y) { cs_spatial_shade(uint3(x, y, 0u)); });
}

// ── atrous.slang:cs_main, one iteration (AtrousPass.cpp:269-302)
void sref_atrous_iteration(const float* input, const float* gbuf_pos, const float* gbuf_norm, float* output,
                           uint32_t W, uint32_t H, uint32_t stride, float sp, float sn, float sl, int threads) {
    using namespace ref_atrous;
    gTextures[0].data = reinterpret_cast<const float4*>(input);
    gTextures[0].width = W;
    gTextures[0].height = H;
    bind_image(0, output, W, H);
    bind_image(1, const_cast<float*>(gbuf_pos), W, H);
    bind_image(2, const_cast<float*>(gbuf_norm), W, H);
    pc = PushConstants{};
    pc.input_idx = 0;
    pc.output_idx = 0;
    pc.gbuf_pos_idx = 1;
    pc.gbuf_norm_idx = 2;
    pc.screen_width = W;
    pc.screen_height = H;
    pc.stride = stride;
    pc.sigma_position = sp;
    pc.sigma_normal = sn;
    pc.sigma_luminance = sl;
    dispatch(0, 0, W, H, threads, [](uint x, uint y) { cs_main(uint3(x, y, 0u)); });
}

// ── restir_pt.slang (ReSTIRPTPass::execute, ReSTIRPTPass.cpp:529-812)
// stage 0 = cs_initial, 1 = cs_temporal, 2 = cs_spatial_shade, 3 = cs_fit_guiding
void sref_restir_pt(int stage, const void* sv, const GpuCameraData* cam, const OracleRestirPtParams* p,
                    const OracleRestirPtImages* img, int threads) {
    const auto* s = static_cast<const SrefScene*>(sv);
    bind_scene(s, cam);
    const uint W = cam->screen_width, H = cam->screen_height;
    bind_image(0, const_cast<float*>(img->gbuf_pos), W, H);
    bind_image(1, const_cast<float*>(img->gbuf_norm), W, H);
    for (int k = 0; k < 4; ++k) {
        bind_image(2 + k, img->reservoir_curr[k], W, H);
        bind_image(6 + k, img->reservoir_prev[k], W, H);
    }
    bind_image(10, img->history_curr[0], W, H);
    bind_image(11, img->history_curr[1], W, H);
    bind_image(12, img->history_prev[0], W, H);
    bind_image(13, img->history_prev[1], W, H);
    bind_image(14, img->output, W, H);
    if (img->direct) {
        gTextures[0].data = reinterpret_cast<const float4*>(img->direct);
        gTextures[0].width = W;
        gTextures[0].height = H;
    }
    gSceneRW[0].data = reinterpret_cast<unsigned char*>(img->guiding_accum);
    gSceneRW[0].size = size_t(p->guiding.cell_count) * 16u;
    gSceneRW[1].data = reinterpret_cast<unsigned char*>(img->guiding_fitted);
    gSceneRW[1].size = size_t(p->guiding.cell_count) * 16u;
    using namespace ref_rpt;
    pc = PushConstants{};
    pc.camera_buf_idx = kCam;
    pc.tlas_idx = 0;
    pc.vertex_buf_idx = kVtx;
    pc.index_buf_idx = kIdx;
    pc.mesh_buf_idx = kMesh;
    pc.material_buf_idx = kMat;
    pc.instance_buf_idx = kInst;
    pc.light_buf_idx = kLight;
    pc.num_instances = uint(s->instances.size());
    pc.num_lights = uint(s->lights.size());
    pc.frame_seed = p->frame_seed;
    pc.gbuf_pos_idx = 0;
    pc.gbuf_norm_idx = 1;
    pc.direct_input_idx = img->direct ? 0u : 0xffffffffu;
    pc.reservoir_curr_pos_idx = 2;
    pc.reservoir_curr_nrm_idx = 3;
    pc.reservoir_curr_rad_idx = 4;
    pc.reservoir_curr_pre_idx = 5;
    pc.reservoir_prev_pos_idx = 6;
    pc.reservoir_prev_nrm_idx = 7;
    pc.reservoir_prev_rad_idx = 8;
    pc.reservoir_prev_pre_idx = 9;
    pc.history_curr_pos_idx = 10;
    pc.history_curr_norm_idx = 11;
    pc.history_prev_pos_idx = 12;
    pc.history_prev_norm_idx = 13;
    pc.output_idx = 14;
    pc.num_initial_candidates = p->num_initial_candidates;
    pc.max_bounces = p->max_bounces;
    pc.temporal_enable = p->temporal_enable;
    pc.spatial_enable = p->spatial_enable;
    pc.spatial_num_neighbors = p->spatial_num_neighbors;
    pc.spatial_radius = p->spatial_radius;
    pc.include_direct_lighting = p->include_direct_lighting;
    pc.indirect_strength = p->indirect_strength;
    pc.ray_bias = p->ray_bias;
    pc.guiding_accum_idx = 0;
    pc.guiding_fitted_idx = 1;
    pc.guiding_enable = p->guiding.enabled;
    pc.guiding_alpha = p->guiding.alpha;
    pc.grid_base_cell_size = p->guiding.base_cell_size;
    pc.grid_distance_slope = p->guiding.distance_slope;
    pc.grid_cell_count = p->guiding.cell_count;
    pc.grid_min_samples = p->guiding.min_samples;
    pc.grid_kappa_max = p->guiding.kappa_max;
    if (stage == 0) dispatch(0, 0, W, H, threads, [](uint x, uint y) { cs_initial(uint3(x, y, 0u)); });
    else if (stage == 1) dispatch(0, 0, W, H, threads, [](uint x, uint y) { cs_temporal(uint3(x, y, 0u)); });
    else if (stage == 2) dispatch(0, 0, W, H, threads, [](uint x, uint y) { cs_spatial_shade(uint3(x, y, 0u)); });
    else
        for (uint c = 0; c < p->guiding.cell_count; ++c) cs_fit_guiding(uint3(c, 0u, 0u));
}

// ── restir_gi.slang (ReSTIRGIPass::execute, ReSTIRGIPass.cpp:428-650)
// stage 0 = cs_initial, 1 = cs_temporal, 2 = cs_spatial_shade
void sref_restir_gi(int stage, const void* sv, const GpuCameraData* cam, const OracleRestirGiParams* p,
                    const OracleRestirGiImages* img, int threads) {
    const auto* s = static_cast<const SrefScene*>(sv);
    bind_scene(s, cam);
    const uint W = cam->screen_width, H = cam->screen_height;
    bind_image(0, const_cast<float*>(img->gbuf_pos), W, H);
    bind_image(1, const_cast<float*>(img->gbuf_norm), W, H);
    for (int k = 0; k < 3; ++k) {
        bind_image(2 + k, img->reservoir_curr[k], W, H);
        bind_image(5 + k, img->reservoir_prev[k], W, H);
    }
    bind_image(8, img->history_curr[0], W, H);
    bind_image(9, img->history_curr[1], W, H);
    bind_image(10, img->history_prev[0], W, H);
    bind_image(11, img->history_prev[1], W, H);
    bind_image(12, img->output, W, H);
    if (img->direct) {
        gTextures[0].data = reinterpret_cast<const float4*>(img->direct);
        gTextures[0].width = W;
        gTextures[0].height = H;
    }
    using namespace ref_rgi;
    pc = PushConstants{};
    pc.camera_buf_idx = kCam;
    pc.tlas_idx = 0;
    pc.vertex_buf_idx = kVtx;
    pc.index_buf_idx = kIdx;
    pc.mesh_buf_idx = kMesh;
    pc.material_buf_idx = kMat;
    pc.instance_buf_idx = kInst;
    pc.light_buf_idx = kLight;
    pc.num_instances = uint(s->instances.size());
    pc.num_lights = uint(s->lights.size());
    pc.frame_seed = p->frame_seed;
    pc.gbuf_pos_idx = 0;
    pc.gbuf_norm_idx = 1;
    pc.direct_input_idx = img->direct ? 0u : 0xffffffffu;
    pc.reservoir_curr_pos_idx = 2;
    pc.reservoir_curr_rad_idx = 3;
    pc.reservoir_curr_meta_idx = 4;
    pc.reservoir_prev_pos_idx = 5;
    pc.reservoir_prev_rad_idx = 6;
    pc.reservoir_prev_meta_idx = 7;
    pc.history_curr_pos_idx = 8;
    pc.history_curr_norm_idx = 9;
    pc.history_prev_pos_idx = 10;
    pc.history_prev_norm_idx = 11;
    pc.output_idx = 12;
    pc.num_initial_candidates = p->num_initial_candidates;
    pc.temporal_enable = p->temporal_enable;
    pc.spatial_enable = p->spatial_enable;
    pc.spatial_num_neighbors = p->spatial_num_neighbors;
    pc.spatial_radius = p->spatial_radius;
    pc.include_direct_lighting = p->include_direct_lighting;
    pc.indirect_strength = p->indirect_strength;
    pc.ray_bias = p->ray_bias;
    if (stage == 0) dispatch(0, 0, W, H, threads, [](uint x, uint y) { cs_initial(uint3(x, y, 0u)); });
    else if (stage == 1) dispatch(0, 0, W, H, threads, [](uint x, uint y) { cs_temporal(uint3(x, y, 0u)); });
    else dispatch(0, 0, W, H, threads, [](uint x, uint y) { cs_spatial_shade(uint3(x, y, 0u)); });
}

} // extern "C"
