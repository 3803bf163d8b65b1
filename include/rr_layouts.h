/*
 * rr_layouts.h — GPU scene data layouts shared by the host, the CUDA kernels
 * and the CPU checker.
 *
 * Byte-for-byte mirrors of the reference's scalar-block-layout structs in
 * src/scene/GpuScene.h:17-98 (Slang mirror: assets/shaders/include/
 * GpuScene.slang:7-80). Matrices are row-major float4x4 (Scene.cpp:87-90,
 * 562-566: glm column-major is transposed on upload), and `mul(M, v)` means
 * out[r] = sum_c M[r*4+c] * v[c].
 *
 * Note: the reference's GpuMaterial comment says 80 bytes but its
 * static_assert says 72 (GpuScene.h:39 vs :54); 72 is the layout.
 */
#ifndef RR_LAYOUTS_H
#define RR_LAYOUTS_H

#include <stdint.h>

#ifdef __cplusplus
#define RR_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define RR_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif

/* GpuScene.h:17-24 — one vertex, 48 bytes. */
typedef struct GpuVertex {
    float pos[3];
    float normal[3];
    float uv[2];
    float tangent[4];
} GpuVertex;
RR_STATIC_ASSERT(sizeof(GpuVertex) == 48, "GpuVertex must be 48 bytes");

/* GpuScene.h:28-37 — one mesh, 32 bytes. index_byte_offset is in bytes. */
typedef struct GpuMesh {
    uint32_t vertex_base;
    uint32_t vertex_count;
    uint32_t index_byte_offset;
    uint32_t index_count;
    uint32_t material_index;
    uint32_t _pad[3];
} GpuMesh;
RR_STATIC_ASSERT(sizeof(GpuMesh) == 32, "GpuMesh must be 32 bytes");

/* GpuScene.h:40-54 — one metallic-roughness material, 72 bytes. */
typedef struct GpuMaterial {
    float    base_color[4];
    float    metallic;
    float    roughness;
    float    emissive[3];
    float    ior;
    uint32_t albedo_tex_idx;
    uint32_t normal_tex_idx;
    uint32_t metallic_roughness_tex_idx;
    uint32_t emissive_tex_idx;
    uint32_t sampler_idx;
    uint32_t _pad[3];
} GpuMaterial;
RR_STATIC_ASSERT(sizeof(GpuMaterial) == 72, "GpuMaterial must be 72 bytes");

/* GpuScene.h:57-63 — one instance (row-major transform + mesh), 80 bytes. */
typedef struct GpuInstance {
    float    transform[16];
    uint32_t mesh_index;
    uint32_t _pad[3];
} GpuInstance;
RR_STATIC_ASSERT(sizeof(GpuInstance) == 80, "GpuInstance must be 80 bytes");

/* GpuScene.h:67-76 — one light, 48 bytes. type 0 = point, anything else is
 * treated as directional by the shaders (pathtracer.slang:138-151). */
typedef struct GpuLight {
    float    position[3];
    uint32_t type;
    float    direction[3];
    float    radius;
    float    emission[3];
    float    intensity;
} GpuLight;
RR_STATIC_ASSERT(sizeof(GpuLight) == 48, "GpuLight must be 48 bytes");

/* GpuScene.h:80-98 — per-frame camera block, 304 bytes. */
typedef struct GpuCameraData {
    float    view[16];
    float    inv_view[16];
    float    inv_proj[16];
    float    prev_view_proj[16];
    float    position[3];
    float    near_plane;
    float    direction[3];
    float    far_plane;
    uint32_t frame_index;
    uint32_t screen_width;
    uint32_t screen_height;
    uint32_t _pad;
} GpuCameraData;
RR_STATIC_ASSERT(sizeof(GpuCameraData) == 304, "GpuCameraData must be 304 bytes");

#undef RR_STATIC_ASSERT
#endif /* RR_LAYOUTS_H */
