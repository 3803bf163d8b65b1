"""ctypes binding of librr_cuda.so (include/rr_cuda.h, include/rr_host.h).

Device buffers are passed as raw pointers (e.g. ``tensor.data_ptr()`` of a
CUDA torch tensor); streams as ``torch.cuda.current_stream().cuda_stream``.
The library must have been built (``python -m research_b200.build``); there
is no fallback: a missing library raises immediately.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

LIB_PATH = Path(__file__).resolve().parent / "lib" / "librr_cuda.so"

# ── GpuScene.h layouts as numpy dtypes (include/rr_layouts.h) ─────────────
VERTEX = np.dtype([("pos", "<f4", 3), ("normal", "<f4", 3), ("uv", "<f4", 2), ("tangent", "<f4", 4)])
MESH = np.dtype([("vertex_base", "<u4"), ("vertex_count", "<u4"), ("index_byte_offset", "<u4"),
                 ("index_count", "<u4"), ("material_index", "<u4"), ("_pad", "<u4", 3)])
MATERIAL = np.dtype([("base_color", "<f4", 4), ("metallic", "<f4"), ("roughness", "<f4"), ("emissive", "<f4", 3),
                     ("ior", "<f4"), ("albedo_tex_idx", "<u4"), ("normal_tex_idx", "<u4"),
                     ("metallic_roughness_tex_idx", "<u4"), ("emissive_tex_idx", "<u4"), ("sampler_idx", "<u4"),
                     ("_pad", "<u4", 3)])
INSTANCE = np.dtype([("transform", "<f4", 16), ("mesh_index", "<u4"), ("_pad", "<u4", 3)])
LIGHT = np.dtype([("position", "<f4", 3), ("type", "<u4"), ("direction", "<f4", 3), ("radius", "<f4"),
                  ("emission", "<f4", 3), ("intensity", "<f4")])
assert VERTEX.itemsize == 48 and MESH.itemsize == 32 and MATERIAL.itemsize == 72
assert INSTANCE.itemsize == 80 and LIGHT.itemsize == 48

RR_STATUS = {0: "RR_OK", 1: "RR_ERR_INVALID_ARGUMENT", 2: "RR_ERR_CUDA", 3: "RR_ERR_OUT_OF_MEMORY",
             4: "RR_ERR_NOT_INITIALIZED", 5: "RR_ERR_QUEUE_OVERFLOW", 6: "RR_ERR_TIMEOUT", 7: "RR_ERR_UNSUPPORTED"}


class GpuCameraData(C.Structure):
    _fields_ = [("view", C.c_float * 16), ("inv_view", C.c_float * 16), ("inv_proj", C.c_float * 16),
                ("prev_view_proj", C.c_float * 16), ("position", C.c_float * 3), ("near_plane", C.c_float),
                ("direction", C.c_float * 3), ("far_plane", C.c_float), ("frame_index", C.c_uint32),
                ("screen_width", C.c_uint32), ("screen_height", C.c_uint32), ("_pad", C.c_uint32)]


class SceneDesc(C.Structure):
    _fields_ = [("vertices", C.c_void_p), ("vertex_count", C.c_uint32), ("indices", C.c_void_p),
                ("index_count", C.c_uint32), ("meshes", C.c_void_p), ("mesh_count", C.c_uint32),
                ("materials", C.c_void_p), ("material_count", C.c_uint32), ("instances", C.c_void_p),
                ("instance_count", C.c_uint32), ("lights", C.c_void_p), ("light_count", C.c_uint32)]


class SceneStats(C.Structure):
    _fields_ = [("triangle_count", C.c_uint32), ("bvh_node_count", C.c_uint32), ("bvh_max_depth", C.c_uint32),
                ("light_count", C.c_uint32), ("build_ms", C.c_double), ("upload_ms", C.c_double),
                ("device_bytes", C.c_uint64), ("bvh4_node_count", C.c_uint32), ("_pad", C.c_uint32)]


class PtStats(C.Structure):
    _fields_ = [("extension_rays", C.c_uint64), ("shadow_rays", C.c_uint64), ("extension_nodes", C.c_uint64),
                ("extension_tris", C.c_uint64), ("shadow_nodes", C.c_uint64), ("shadow_tris", C.c_uint64),
                ("ms_raygen", C.c_double), ("ms_extend", C.c_double), ("ms_shade", C.c_double),
                ("ms_shadow", C.c_double), ("launches_extend", C.c_uint64), ("launches_total", C.c_uint64)]


class PtTuneResult(C.Structure):
    _fields_ = [("extend_ms", C.c_double * 8), ("shadow_ms", C.c_double * 8), ("best_extend", C.c_int),
                ("best_shadow", C.c_int)]


PT_FLAG_COUNT_TRAVERSAL = 1
PT_FLAG_TIME_STAGES = 2
PT_FLAG_GRAPH = 4
PT_FLAG_EMITTERS = 8
PT_VARIANT_COUNT = 8
TRACE_ANY_HIT, TRACE_WIDE = 1, 2   # rr_trace_counted flags
BATCH_WAVEFRONT = 0
BATCH_PER_SCENE = 1


class PtParams(C.Structure):
    _fields_ = [("frame_seed", C.c_uint32), ("max_bounces", C.c_uint32), ("spp", C.c_uint32), ("flags", C.c_uint32)]


class AccParams(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("camera_moved", C.c_uint32),
                ("accumulated_spp", C.c_uint32)]


class DIParams(C.Structure):
    _fields_ = [("frame_seed", C.c_uint32), ("num_initial_candidates", C.c_uint32), ("temporal_enable", C.c_uint32),
                ("spatial_enable", C.c_uint32), ("spatial_num_neighbors", C.c_uint32), ("spatial_radius", C.c_uint32),
                ("m_cap_factor", C.c_uint32), ("flags", C.c_uint32)]


DI_FLAG_EMITTERS = 1


class AtrousParams(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("iterations", C.c_uint32), ("stride", C.c_uint32),
                ("sigma_position", C.c_float), ("sigma_normal", C.c_float), ("sigma_luminance", C.c_float),
                ("_pad", C.c_uint32)]


class GuidingParams(C.Structure):
    _fields_ = [("base_cell_size", C.c_float), ("distance_slope", C.c_float), ("cell_count", C.c_uint32),
                ("enabled", C.c_uint32), ("min_samples", C.c_uint32), ("kappa_max", C.c_float), ("alpha", C.c_float),
                ("_pad", C.c_uint32)]


class PtReuseParams(C.Structure):
    """rr_restir_pt_params (ReSTIRPTPushConstants minus the bindless indices)."""
    _fields_ = [("frame_seed", C.c_uint32), ("num_initial_candidates", C.c_uint32), ("max_bounces", C.c_uint32),
                ("temporal_enable", C.c_uint32), ("spatial_enable", C.c_uint32),
                ("spatial_num_neighbors", C.c_uint32), ("spatial_radius", C.c_uint32),
                ("include_direct_lighting", C.c_uint32), ("indirect_strength", C.c_float), ("ray_bias", C.c_float),
                ("_pad", C.c_uint32 * 2), ("guiding", GuidingParams)]


class PtReuseImages(C.Structure):
    """rr_restir_pt_images: device pointers (float4 per pixel)."""
    _fields_ = [("gbuf_pos", C.c_void_p), ("gbuf_norm", C.c_void_p), ("direct", C.c_void_p),
                ("reservoir_curr", C.c_void_p * 4), ("reservoir_prev", C.c_void_p * 4),
                ("history_curr", C.c_void_p * 2), ("history_prev", C.c_void_p * 2), ("output", C.c_void_p),
                ("guiding_accum", C.c_void_p), ("guiding_fitted", C.c_void_p)]


def pt_reuse_params(frame_seed=0, candidates=8, max_bounces=4, temporal=1, spatial=1, neighbors=4, radius=12,
                    include_direct=1, indirect_strength=1.0, ray_bias=1e-3, guiding=1, alpha=0.5,
                    cell_count=1 << 20, min_samples=8, kappa_max=512.0) -> "PtReuseParams":
    """Reference defaults of ReSTIRPTPass.h:86-100."""
    g = GuidingParams(0.10, 0.02, cell_count, guiding, min_samples, kappa_max, alpha, 0)
    return PtReuseParams(frame_seed, candidates, max_bounces, temporal, spatial, neighbors, radius, include_direct,
                         indirect_strength, ray_bias, (C.c_uint32 * 2)(0, 0), g)


class GiReuseParams(C.Structure):
    """rr_restir_gi_params (ReSTIRGIPushConstants minus the bindless indices)."""
    _fields_ = [("frame_seed", C.c_uint32), ("num_initial_candidates", C.c_uint32), ("temporal_enable", C.c_uint32),
                ("spatial_enable", C.c_uint32), ("spatial_num_neighbors", C.c_uint32), ("spatial_radius", C.c_uint32),
                ("include_direct_lighting", C.c_uint32), ("indirect_strength", C.c_float), ("ray_bias", C.c_float),
                ("_pad", C.c_uint32 * 3)]


class GiReuseImages(C.Structure):
    """rr_restir_gi_images: device pointers (float4 per pixel)."""
    _fields_ = [("gbuf_pos", C.c_void_p), ("gbuf_norm", C.c_void_p), ("direct", C.c_void_p),
                ("reservoir_curr", C.c_void_p * 3), ("reservoir_prev", C.c_void_p * 3),
                ("history_curr", C.c_void_p * 2), ("history_prev", C.c_void_p * 2), ("output", C.c_void_p)]


def gi_reuse_params(frame_seed=0, candidates=8, temporal=1, spatial=1, neighbors=4, radius=12, include_direct=1,
                    indirect_strength=1.0, ray_bias=1e-3) -> "GiReuseParams":
    """Reference defaults of ReSTIRGIPass.h:67-74."""
    return GiReuseParams(frame_seed, candidates, temporal, spatial, neighbors, radius, include_direct,
                         indirect_strength, ray_bias, (C.c_uint32 * 3)(0, 0, 0))


class GuideDesc(C.Structure):
    _fields_ = [("kind", C.c_uint32), ("grid_resolution", C.c_uint32), ("alpha", C.c_float), ("decay", C.c_float),
                ("bounds_min", C.c_float * 3), ("bounds_max", C.c_float * 3), ("max_samples", C.c_uint32),
                ("mlp_batch", C.c_uint32), ("learning_rate", C.c_float), ("seed", C.c_uint32)]


class GuideStats(C.Structure):
    _fields_ = [("samples_recorded", C.c_uint64), ("samples_used", C.c_uint64), ("cells_valid", C.c_uint32),
                ("updates", C.c_uint32), ("last_loss", C.c_double), ("ms_update", C.c_double)]


GUIDE_GRID = 0
GUIDE_MLP = 1
MLP_PARAM_COUNT = 20784


class ProceduralParams(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("target_triangles", C.c_uint32), ("emissive_triangles", C.c_uint32),
                ("box_half", C.c_float), ("flags", C.c_uint32)]


SCENE_NO_EMITTER_LIGHTS = 1


class InstancedParams(C.Structure):
    _fields_ = [("seed", C.c_uint64), ("base_meshes", C.c_uint32), ("tris_per_mesh", C.c_uint32),
                ("instance_count", C.c_uint32), ("emissive_triangles", C.c_uint32), ("box_half", C.c_float),
                ("flags", C.c_uint32)]


class CameraDesc(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("yaw_deg", C.c_float), ("pitch_deg", C.c_float),
                ("fov_y_deg", C.c_float), ("near_plane", C.c_float), ("far_plane", C.c_float),
                ("width", C.c_uint32), ("height", C.c_uint32), ("frame_index", C.c_uint32), ("_pad", C.c_uint32)]


assert C.sizeof(GpuCameraData) == 304

P, U32, F32, I = C.c_void_p, C.c_uint32, C.c_float, C.c_int
_SIGNATURES = {
    "rr_abi_version": (U32, []),
    "rr_status_string": (C.c_char_p, [I]),
    "rr_ctx_create": (I, [I, C.POINTER(P)]),
    "rr_ctx_destroy": (I, [P]),
    "rr_last_error": (I, [P, C.c_char_p, C.c_size_t]),
    "rr_ctx_set_queue_limit": (I, [P, C.c_uint64]),
    "rr_scene_create": (I, [P, C.POINTER(SceneDesc), C.POINTER(P)]),
    "rr_scene_destroy": (I, [P]),
    "rr_scene_get_stats": (I, [P, C.POINTER(SceneStats)]),
    "rr_pathtracer_execute": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(PtParams), P, P]),
    "rr_pathtracer_stats": (I, [P, C.POINTER(PtStats), I]),
    "rr_pathtracer_set_variants": (I, [P, I, I]),
    "rr_pathtracer_set_overlap": (I, [P, I]),
    "rr_reuse_set_wavefront": (I, [P, I]),
    "rr_atrous_set_tma": (I, [P, I]),
    "rr_atrous_tma_error": (I, [P, C.POINTER(C.c_int)]),
    "rr_atrous_set_tma_wait_tries": (I, [P, U32]),
    "rr_pathtracer_tune": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(PtParams), P, P, C.POINTER(PtTuneResult)]),
    "rr_accumulate_execute": (I, [P, P, U32, P, P, C.POINTER(AccParams), P]),
    "rr_restir_di_initial": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(DIParams), P, P, P, P]),
    "rr_restir_di_temporal": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(DIParams), P, P, P, P, P]),
    "rr_restir_di_spatial_shade": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(DIParams), P, P, P, P, P]),
    "rr_restir_di_execute": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(DIParams), P, P, P, P, P, P]),
    "rr_atrous_iteration": (I, [P, P, P, P, P, C.POINTER(AtrousParams), P]),
    "rr_atrous_execute": (I, [P, P, P, P, P, P, C.POINTER(AtrousParams), C.POINTER(U32), P]),
    "rr_atrous_execute_static": (I, [P, P, P, P, C.POINTER(AtrousParams), P]),
    "rr_guiding_splat": (I, [P, P, P, P, P, U32, C.POINTER(F32), C.POINTER(GuidingParams), P]),
    "rr_guiding_fit": (I, [P, P, P, C.POINTER(GuidingParams), P]),
    "rr_guiding_sample": (I, [P, P, P, P, P, P, U32, C.POINTER(F32), C.POINTER(GuidingParams), P, P, P]),
    "rr_guiding_reset": (I, [P, P, P, C.POINTER(GuidingParams), P]),
    "rr_batch_create": (I, [P, C.POINTER(P), U32, C.POINTER(P)]),
    "rr_batch_destroy": (I, [P]),
    "rr_batch_set_mode": (I, [P, I]),
    "rr_batch_get_mode": (I, [P, C.POINTER(I)]),
    "rr_batch_execute": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(PtParams), C.POINTER(P), P]),
    "rr_batch_tune": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(PtParams), C.POINTER(P), P,
                          C.POINTER(PtTuneResult)]),
    "rr_restir_pt_initial": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(PtReuseParams), C.POINTER(PtReuseImages), P]),
    "rr_restir_pt_temporal": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(PtReuseParams), C.POINTER(PtReuseImages), P]),
    "rr_restir_pt_spatial_shade": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(PtReuseParams),
                                       C.POINTER(PtReuseImages), P]),
    "rr_restir_pt_execute": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(PtReuseParams), C.POINTER(PtReuseImages), P]),
    "rr_restir_pt_reset_history": (I, [P, C.POINTER(PtReuseImages), U32, U32, P]),
    "rr_restir_gi_initial": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(GiReuseParams), C.POINTER(GiReuseImages), P]),
    "rr_restir_gi_temporal": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(GiReuseParams), C.POINTER(GiReuseImages), P]),
    "rr_restir_gi_spatial_shade": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(GiReuseParams),
                                       C.POINTER(GiReuseImages), P]),
    "rr_restir_gi_execute": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(GiReuseParams), C.POINTER(GiReuseImages), P]),
    "rr_restir_gi_reset_history": (I, [P, C.POINTER(GiReuseImages), U32, U32, P]),
    "rr_trace_closest": (I, [P, P, P, P, F32, F32, U32, P, P, P]),
    "rr_tonemap_execute": (I, [P, P, U32, U32, F32, P, P]),
    "rr_guide_create": (I, [P, C.POINTER(GuideDesc), C.POINTER(P)]),
    "rr_guide_destroy": (I, [P]),
    "rr_guide_reset": (I, [P, P, P]),
    "rr_guide_update": (I, [P, P, P]),
    "rr_guides_update": (I, [P, C.POINTER(P), U32, P]),
    "rr_batch_execute_guided": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(PtParams), C.POINTER(P), C.POINTER(P),
                                    P]),
    "rr_guide_get_stats": (I, [P, P, C.POINTER(GuideStats)]),
    "rr_guide_eval": (I, [P, P, P, U32, P, P]),
    "rr_guide_set_samples": (I, [P, P, P, U32, P]),
    "rr_guide_mlp_params": (I, [P, P, P, P, P, U32, C.POINTER(I)]),
    "rr_guided_pathtracer_execute": (I, [P, P, C.POINTER(GpuCameraData), C.POINTER(PtParams), P, P, P]),
    "rr_image_mse": (I, [P, P, P, U32, U32, U32, U32, U32, U32, P, P]),
    "rr_host_scene_cornell": (I, [I, C.POINTER(P)]),
    "rr_host_scene_procedural": (I, [C.POINTER(ProceduralParams), C.POINTER(P)]),
    "rr_host_scene_instanced": (I, [C.POINTER(InstancedParams), C.POINTER(P)]),
    "rr_trace_counted": (I, [P, P, P, P, C.c_float, C.c_float, U32, I, P, P, P, P]),
    "rr_scene_copy_bvh": (I, [P, P, P, P]),
    "rr_scene_copy_bvh4": (I, [P, P, P]),
    "rr_pathtracer_variant_width": (I, [I]),
    "rr_tc_wait_selftest": (I, [P, U32, P]),
    "rr_host_scene_gltf": (I, [C.c_char_p, C.POINTER(P), C.c_char_p, C.c_size_t]),
    "rr_host_scene_desc": (I, [P, C.POINTER(SceneDesc)]),
    "rr_host_scene_destroy": (I, [P]),
    "rr_camera_default": (I, [U32, U32, C.POINTER(CameraDesc)]),
    "rr_camera_look_at": (I, [C.POINTER(CameraDesc), C.POINTER(F32), C.POINTER(F32)]),
    "rr_camera_build": (I, [C.POINTER(CameraDesc), C.POINTER(CameraDesc), C.POINTER(GpuCameraData)]),
}
EXPORTED = tuple(_SIGNATURES)

_lib = None


class RRError(RuntimeError):
    def __init__(self, status: int, message: str = ""):
        self.status = status
        super().__init__(f"{RR_STATUS.get(status, status)}: {message}")


def lib() -> C.CDLL:
    """Load librr_cuda.so (raises if it has not been built)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RRError(4, f"{LIB_PATH} is missing; run `python -m research_b200.build`")
        _lib = bind(C.CDLL(str(LIB_PATH)), _SIGNATURES)
    return _lib


# The host-side scene factories and camera helpers (include/rr_host.h minus
# the glTF loader): the functions another library built from the same
# generator source also exports.
HOST_FUNCTIONS = ("rr_host_scene_cornell", "rr_host_scene_procedural", "rr_host_scene_instanced",
                  "rr_host_scene_desc", "rr_host_scene_destroy", "rr_camera_default", "rr_camera_look_at",
                  "rr_camera_build")


def bind(L: C.CDLL, names) -> C.CDLL:
    """Sets the ctypes signatures of `names` (rr_cuda.h / rr_host.h functions) on `L`."""
    for name in names:
        res, args = _SIGNATURES[name]
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    return L


def _f3(v) -> C.Array:
    return (C.c_float * 3)(*[float(x) for x in v])


def ptr(t) -> int:
    """Raw address of a torch tensor / numpy array / int / None."""
    if t is None:
        return None
    if isinstance(t, int):
        return t
    if hasattr(t, "data_ptr"):
        return t.data_ptr()
    if isinstance(t, np.ndarray):
        return t.ctypes.data
    raise TypeError(type(t))


# ── host scenes and cameras (no GPU needed) ────────────────────────────────
class HostScene:
    """Flat GpuScene arrays produced by the library's scene factories. `L`
    selects the library that runs the factory (default librr_cuda.so)."""

    def __init__(self, handle, L=None):
        self._L = L if L is not None else lib()
        self._h = handle
        d = SceneDesc()
        _check(None, self._L.rr_host_scene_desc(handle, C.byref(d)))
        self.arrays = {
            "vertices": _view(d.vertices, d.vertex_count, VERTEX),
            "indices": _view(d.indices, d.index_count, np.dtype("<u4")),
            "meshes": _view(d.meshes, d.mesh_count, MESH),
            "materials": _view(d.materials, d.material_count, MATERIAL),
            "instances": _view(d.instances, d.instance_count, INSTANCE),
            "lights": _view(d.lights, d.light_count, LIGHT),
        }

    @staticmethod
    def cornell(variant: int = 0, L=None) -> "HostScene":
        L = L if L is not None else lib()
        h = P()
        _check(None, L.rr_host_scene_cornell(variant, C.byref(h)))
        return HostScene(h, L)

    @staticmethod
    def procedural(seed=0x5EED0002, target_triangles=1_000_000, emissive_triangles=4096, box_half=20.0, L=None,
                   flags=0):
        """flags: SCENE_NO_EMITTER_LIGHTS leaves out the emitters' point lights."""
        L = L if L is not None else lib()
        h = P()
        p = ProceduralParams(seed, target_triangles, emissive_triangles, box_half, flags)
        _check(None, L.rr_host_scene_procedural(C.byref(p), C.byref(h)))
        return HostScene(h, L)

    @staticmethod
    def instanced(seed=0x5EED0005, base_meshes=16, tris_per_mesh=2500, instance_count=4096,
                  emissive_triangles=16384, box_half=250.0, L=None, flags=0):
        L = L if L is not None else lib()
        h = P()
        p = InstancedParams(seed, base_meshes, tris_per_mesh, instance_count, emissive_triangles, box_half, flags)
        _check(None, L.rr_host_scene_instanced(C.byref(p), C.byref(h)))
        return HostScene(h, L)

    @staticmethod
    def gltf(path) -> "HostScene":
        """GltfLoader::load of a .gltf / .glb file (RRError with the reason on failure)."""
        h = P()
        err = C.create_string_buffer(1024)
        st = lib().rr_host_scene_gltf(os.fsencode(str(path)), C.byref(h), err, len(err))
        if st != 0:
            raise RRError(st, err.value.decode(errors="replace"))
        return HostScene(h)

    def triangle_count(self) -> int:
        m = self.arrays["meshes"]
        inst = self.arrays["instances"]
        return int((m["index_count"][inst["mesh_index"]] // 3).sum())

    def close(self):
        if self._h:
            self._L.rr_host_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _view(addr, count, dtype) -> np.ndarray:
    if not addr or count == 0:
        return np.zeros(0, dtype=dtype)
    buf = (C.c_char * (count * dtype.itemsize)).from_address(addr)
    return np.frombuffer(buf, dtype=dtype, count=count).copy()


def scene_desc(arrays) -> tuple[SceneDesc, list]:
    """rr_scene_desc over numpy arrays (keeps them alive in the returned list)."""
    keep = [np.ascontiguousarray(arrays[k]) for k in
            ("vertices", "indices", "meshes", "materials", "instances", "lights")]
    v, i, m, mt, ins, l = keep
    d = SceneDesc(v.ctypes.data, len(v), i.ctypes.data, len(i), m.ctypes.data, len(m), mt.ctypes.data, len(mt),
                  ins.ctypes.data, len(ins), l.ctypes.data if len(l) else None, len(l))
    return d, keep


def camera_desc(width: int, height: int, eye=None, center=None, frame_index=0, L=None) -> CameraDesc:
    L = L if L is not None else lib()
    c = CameraDesc()
    _check(None, L.rr_camera_default(width, height, C.byref(c)))
    if eye is not None and center is not None:
        _check(None, L.rr_camera_look_at(C.byref(c), _f3(eye), _f3(center)))
    c.frame_index = frame_index
    return c


def camera_data(desc: CameraDesc, prev: CameraDesc | None = None, L=None) -> GpuCameraData:
    L = L if L is not None else lib()
    out = GpuCameraData()
    _check(None, L.rr_camera_build(C.byref(desc), C.byref(prev) if prev is not None else None, C.byref(out)))
    return out


def _check(ctx, status: int):
    if status != 0:
        msg = ""
        if ctx is not None and ctx._h:
            buf = C.create_string_buffer(1024)
            lib().rr_last_error(ctx._h, buf, 1024)
            msg = buf.value.decode(errors="replace")
        raise RRError(status, msg)


# ── device context and scene ────────────────────────────────────────────────
class Context:
    def __init__(self, device: int = 0):
        self._h = P()
        st = lib().rr_ctx_create(device, C.byref(self._h))
        if st != 0:
            raise RRError(st, f"rr_ctx_create(device={device})")

    def check(self, status: int):
        _check(self, status)

    def last_error(self) -> str:
        buf = C.create_string_buffer(1024)
        lib().rr_last_error(self._h, buf, 1024)
        return buf.value.decode(errors="replace")

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().rr_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many scenes rendered by one set of wavefront launches (rr_batch_*)."""

    def __init__(self, ctx: "Context", scenes):
        self.ctx = ctx
        self.scenes = list(scenes)
        arr = (P * len(self.scenes))(*[sc.handle for sc in self.scenes])
        self._h = P()
        ctx.check(lib().rr_batch_create(ctx.handle, arr, len(self.scenes), C.byref(self._h)))

    def execute(self, cameras, params, outputs, stream):
        cams = (GpuCameraData * len(cameras))(*cameras)
        outs = (P * len(outputs))(*outputs)
        self.ctx.check(lib().rr_batch_execute(self.ctx.handle, self._h, cams, C.byref(params), outs, stream))

    def execute_guided(self, cameras, params, guides, outputs, stream):
        """rr_batch_execute_guided: guides[i] (rr_guide handles) guides scene i."""
        cams = (GpuCameraData * len(cameras))(*cameras)
        gs = (P * len(guides))(*guides)
        outs = (P * len(outputs))(*outputs)
        self.ctx.check(lib().rr_batch_execute_guided(self.ctx.handle, self._h, cams, C.byref(params), gs, outs,
                                                     stream))

    @property
    def mode(self) -> int:
        """BATCH_WAVEFRONT or BATCH_PER_SCENE (rr_batch_get_mode; set by tune)."""
        m = C.c_int()
        self.ctx.check(lib().rr_batch_get_mode(self._h, C.byref(m)))
        return m.value

    def set_mode(self, mode: int):
        self.ctx.check(lib().rr_batch_set_mode(self._h, mode))

    def tune(self, cameras, params, outputs, stream) -> "PtTuneResult":
        cams = (GpuCameraData * len(cameras))(*cameras)
        outs = (P * len(outputs))(*outputs)
        r = PtTuneResult()
        self.ctx.check(lib().rr_batch_tune(self.ctx.handle, self._h, cams, C.byref(params), outs, stream,
                                           C.byref(r)))
        return r

    def close(self):
        if self._h:
            lib().rr_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Scene:
    """Device scene + BVH (rr_scene_create)."""

    def __init__(self, ctx: Context, arrays):
        self.ctx = ctx
        self._h = P()
        d, keep = scene_desc(arrays)
        ctx.check(lib().rr_scene_create(ctx.handle, C.byref(d), C.byref(self._h)))
        self.num_lights = len(keep[5])

    @property
    def handle(self):
        return self._h

    def stats(self) -> SceneStats:
        s = SceneStats()
        self.ctx.check(lib().rr_scene_get_stats(self._h, C.byref(s)))
        return s

    def close(self):
        if self._h:
            lib().rr_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
