/*
 * rr_host.h — host-side scene and camera helpers of librr_cuda.so.
 *
 * These run on the CPU and need no GPU. They replace the reference's scene
 * factories and camera math so a caller can produce the flat GpuScene arrays
 * (rr_scene_desc) and the per-frame GpuCameraData block:
 *   - rr_host_scene_cornell: Scene::build_cornell_box (Scene.cpp:144-251)
 *   - rr_host_scene_procedural / _instanced: seeded synthetic scenes of the
 *     benchmark configurations (no reference counterpart)
 *   - rr_host_scene_gltf: GltfLoader::load (GltfLoader.cpp:79-365) plus the
 *     CPU side of Scene::upload (Scene.cpp:255-345)
 *   - rr_camera_*: Camera::look_at / forward / rebuild_matrices
 *     (Camera.cpp:27-36, 120-145) and Scene::update_camera (Scene.cpp:554-585)
 */
#ifndef RR_HOST_H
#define RR_HOST_H

#include <stddef.h>
#include <stdint.h>
#include "rr_cuda.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct rr_host_scene rr_host_scene;

/* variant 0: the reference Cornell box exactly (ceiling quad emissive
 *            (15,15,15) plus a point light (15,15,12) at (0,0.9,0));
 * variant 1: same geometry with the quad's radiance set to (17,12,4). */
rr_status rr_host_scene_cornell(int variant, rr_host_scene** out);

/* Seeded procedural scene: an open-fronted room of four value-noise
 * heightfield grids (floor 256^2..512^2 vertices, three walls 128^2..256^2)
 * spanning [-box_half, box_half], filled with displaced icospheres
 * (subdivision 3..5, uniform scale [0.05, 2] * box_half / 20) until at least
 * target_triangles; GGX materials with roughness U[0.05,1], metallic
 * Bernoulli(0.3), base colour U[0.05,0.95]^3; emissive_triangles single
 * emitting triangles with log-uniform radiance [0.1, 100], each also
 * registered as a point light at its centroid (emission = radiance,
 * intensity = area), mirroring the reference Cornell box, whose emitter has
 * both an emissive quad and a point light. flags: RR_SCENE_NO_EMITTER_LIGHTS
 * leaves those point lights out (the same geometry and materials), for the
 * emitter-sampling mode (RR_PT_FLAG_EMITTERS), which samples the emissive
 * triangles themselves. */
#define RR_SCENE_NO_EMITTER_LIGHTS 1u
typedef struct rr_procedural_params {
    uint64_t seed;
    uint32_t target_triangles;
    uint32_t emissive_triangles;
    float    box_half;
    uint32_t flags;
} rr_procedural_params;
rr_status rr_host_scene_procedural(const rr_procedural_params* p, rr_host_scene** out);

/* Seeded instanced scene: base_meshes meshes of tris_per_mesh triangles,
 * instance_count instances under random affine transforms (rotation,
 * uniform scale [0.2, 3], translation in a [-box_half, box_half]^3 box) and
 * emissive_triangles emitters (+ point lights as above; flags as above). */
typedef struct rr_instanced_params {
    uint64_t seed;
    uint32_t base_meshes;
    uint32_t tris_per_mesh;       /* rounded to an even grid */
    uint32_t instance_count;
    uint32_t emissive_triangles;
    float    box_half;
    uint32_t flags;
} rr_instanced_params;
rr_status rr_host_scene_instanced(const rr_instanced_params* p, rr_host_scene** out);

/* Load a glTF 2.0 file (.gltf with embedded base64 or external buffers, or
 * binary .glb) as GltfLoader::load does: every TRIANGLES primitive becomes a
 * mesh, the default scene's node tree gives one instance per primitive
 * (world = parent * local; node.matrix read as GltfLoader.cpp:36-42 reads
 * it, else T * R * S), materials from the metallic-roughness factors with
 * the glTF defaults, no lights. Textures are not decoded (the path never
 * samples them; Scene::upload binds none). On failure returns
 * RR_ERR_INVALID_ARGUMENT and writes the reason to err (if given); malformed
 * or out-of-range data is an error, never read. */
rr_status rr_host_scene_gltf(const char* path, rr_host_scene** out, char* err, size_t err_size);

/* Pointers stay valid until rr_host_scene_destroy. */
rr_status rr_host_scene_desc(const rr_host_scene* s, rr_scene_desc* out);
rr_status rr_host_scene_destroy(rr_host_scene* s);

/* Camera (Camera.h:55-63 defaults: fov 45, near 0.01, far 1000,
 * position (0,0,3), yaw -90, pitch 0). */
typedef struct rr_camera_desc {
    float    position[3];
    float    yaw_deg;
    float    pitch_deg;
    float    fov_y_deg;
    float    near_plane;
    float    far_plane;
    uint32_t width;
    uint32_t height;
    uint32_t frame_index;
    uint32_t _pad;
} rr_camera_desc;

rr_status rr_camera_default(uint32_t width, uint32_t height, rr_camera_desc* out);
/* Camera::look_at: yaw/pitch from the view direction (up is ignored). */
rr_status rr_camera_look_at(rr_camera_desc* cam, const float eye[3], const float center[3]);
/* rebuild_matrices + update_camera. prev_view_proj is taken from `prev`
 * (its view/proj) when given, else from this camera. */
rr_status rr_camera_build(const rr_camera_desc* cam, const rr_camera_desc* prev, GpuCameraData* out);

#ifdef __cplusplus
}
#endif
#endif /* RR_HOST_H */
