"""Python wrapper of the CPU checker (oracle/librr_oracle.so).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, never by the product package. Every function
restates a reference Slang kernel; see rr_oracle.h for citations.
"""
from __future__ import annotations

import ctypes as C
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "librr_oracle.so"

P, U32, F32, I = C.c_void_p, C.c_uint32, C.c_float, C.c_int


class DIParams(C.Structure):
    _fields_ = [("frame_seed", U32), ("num_initial_candidates", U32), ("temporal_enable", U32),
                ("spatial_enable", U32), ("spatial_num_neighbors", U32), ("spatial_radius", U32),
                ("m_cap_factor", U32), ("flags", U32)]


DI_EMITTERS = 1   # ORACLE_DI_EMITTERS = RR_DI_FLAG_EMITTERS


class GuidingParams(C.Structure):
    _fields_ = [("base_cell_size", F32), ("distance_slope", F32), ("cell_count", U32), ("enabled", U32),
                ("min_samples", U32), ("kappa_max", F32), ("alpha", F32), ("_pad", U32)]


class PtReuseParams(C.Structure):
    """OracleRestirPtParams (ReSTIRPTPushConstants minus the bindless indices)."""
    _fields_ = [("frame_seed", U32), ("num_initial_candidates", U32), ("max_bounces", U32),
                ("temporal_enable", U32), ("spatial_enable", U32), ("spatial_num_neighbors", U32),
                ("spatial_radius", U32), ("include_direct_lighting", U32), ("indirect_strength", F32),
                ("ray_bias", F32), ("_pad", U32 * 2), ("guiding", GuidingParams)]


class PtReuseImages(C.Structure):
    _fields_ = [("gbuf_pos", P), ("gbuf_norm", P), ("direct", P), ("reservoir_curr", P * 4),
                ("reservoir_prev", P * 4), ("history_curr", P * 2), ("history_prev", P * 2), ("output", P),
                ("guiding_accum", P), ("guiding_fitted", P)]


class GiReuseParams(C.Structure):
    """OracleRestirGiParams (ReSTIRGIPushConstants minus the bindless indices)."""
    _fields_ = [("frame_seed", U32), ("num_initial_candidates", U32), ("temporal_enable", U32),
                ("spatial_enable", U32), ("spatial_num_neighbors", U32), ("spatial_radius", U32),
                ("include_direct_lighting", U32), ("indirect_strength", F32), ("ray_bias", F32), ("_pad", U32 * 3)]


class GiReuseImages(C.Structure):
    _fields_ = [("gbuf_pos", P), ("gbuf_norm", P), ("direct", P), ("reservoir_curr", P * 3),
                ("reservoir_prev", P * 3), ("history_curr", P * 2), ("history_prev", P * 2), ("output", P)]


_SIG = {
    "oracle_pcg_hash": (U32, [U32]),
    "oracle_make_seed": (U32, [U32, U32, U32]),
    "oracle_rand_float": (F32, [C.POINTER(U32)]),
    "oracle_detmath_eval": (None, [I, P, P, C.c_size_t]),
    "oracle_scene_create": (P, [P, U32, P, U32, P, U32, P, U32, P, U32, P, U32, I]),
    "oracle_scene_destroy": (None, [P]),
    "oracle_scene_triangle_count": (U32, [P]),
    "oracle_trace_batch": (None, [P, P, P, F32, F32, C.c_size_t, P, P, I]),
    "oracle_primary_ray": (None, [P, U32, U32, U32, P, P, C.POINTER(U32)]),
    "oracle_pathtrace": (None, [P, P, U32, U32, U32, U32, U32, U32, U32, P, I, P]),
    "oracle_pathtrace_ex": (None, [P, P, U32, U32, U32, U32, U32, U32, U32, P, I, P, U32]),
    "oracle_emitters": (U32, [P, P, P, P, P]),
    "oracle_accumulate": (None, [P, P, C.c_size_t, U32, U32]),
    "oracle_restir_di_initial": (None, [P, P, C.POINTER(DIParams), P, P, P, I]),
    "oracle_restir_di_temporal": (None, [P, P, C.POINTER(DIParams), P, P, P, P, I]),
    "oracle_restir_di_spatial_shade": (None, [P, P, C.POINTER(DIParams), P, P, P, P, I]),
    "oracle_atrous_iteration": (None, [P, P, P, P, U32, U32, U32, F32, F32, F32, I]),
    "oracle_atrous_tap_weight": (F32, [P, P, F32, P, P, P, I, I, F32, F32, F32]),
    "oracle_guiding_cell_index": (U32, [P, U32, P, C.POINTER(GuidingParams)]),
    "oracle_guiding_splat": (None, [P, P, P, P, C.c_size_t, P, C.POINTER(GuidingParams)]),
    "oracle_guiding_fit": (None, [P, P, C.POINTER(GuidingParams)]),
    "oracle_guiding_sample": (None, [P, P, P, P, P, C.c_size_t, P, C.POINTER(GuidingParams), P, P]),
    "oracle_vmf_pdf": (F32, [P, F32, P]),
    "oracle_brdf_eval": (None, [P, P, P, P, F32, F32, P]),
    "oracle_brdf_sample": (None, [P, P, P, F32, F32, F32, F32, P, P, P]),
    "oracle_brdf_pdf": (F32, [P, P, P, F32]),
    "oracle_restir_pt_initial": (None, [P, P, C.POINTER(PtReuseParams), C.POINTER(PtReuseImages), I]),
    "oracle_restir_pt_temporal": (None, [P, P, C.POINTER(PtReuseParams), C.POINTER(PtReuseImages), I]),
    "oracle_restir_pt_spatial_shade": (None, [P, P, C.POINTER(PtReuseParams), C.POINTER(PtReuseImages), I]),
    "oracle_bvh2_trace": (None, [P, U32, P, P, P, F32, F32, U32, I, P, P, P, I]),
    "oracle_bvh4_trace": (None, [P, U32, P, P, P, F32, F32, U32, I, P, P, P, I]),
    "oracle_restir_gi_initial": (None, [P, P, C.POINTER(GiReuseParams), C.POINTER(GiReuseImages), I]),
    "oracle_restir_gi_temporal": (None, [P, P, C.POINTER(GiReuseParams), C.POINTER(GiReuseImages), I]),
    "oracle_restir_gi_spatial_shade": (None, [P, P, C.POINTER(GiReuseParams), C.POINTER(GiReuseImages), I]),
}

_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} missing; run `make -C oracle`")
        L = C.CDLL(str(LIB_PATH))
        for k, (r, a) in _SIG.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


INPUTS_PATH = HERE / "librr_inputs.so"
_inputs = None


def inputs_lib() -> C.CDLL:
    """The seeded synthetic inputs (scene factories and camera blocks of
    include/rr_host.h), built by oracle/Makefile from the same generator
    source as the product library but without any CUDA code, so that a CPU
    run builds its scene and camera without loading the CUDA library. Use it
    as `rr.HostScene.procedural(..., L=inputs_lib())` and
    `rr.camera_data(rr.camera_desc(..., L=inputs_lib()), L=inputs_lib())`
    (research_b200.rr only supplies the ctypes layouts here)."""
    global _inputs
    if _inputs is None:
        if not INPUTS_PATH.exists():
            raise RuntimeError(f"{INPUTS_PATH} missing; run `make -C oracle`")
        from research_b200 import rr as _rr
        _inputs = _rr.bind(C.CDLL(str(INPUTS_PATH)), _rr.HOST_FUNCTIONS)
    return _inputs


def threads() -> int:
    return max(1, len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1))


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"], "array must be C-contiguous"
    return a.ctypes.data


def _cam_ptr(cam):
    return C.addressof(cam)


def pcg_hash(x: int) -> int:
    return lib().oracle_pcg_hash(x & 0xFFFFFFFF)


def make_seed(px: int, py: int, frame: int) -> int:
    return lib().oracle_make_seed(px, py, frame & 0xFFFFFFFF)


def rand_floats(seed: int, n: int) -> tuple[list[float], int]:
    s = C.c_uint32(seed)
    out = [lib().oracle_rand_float(C.byref(s)) for _ in range(n)]
    return out, s.value


def detmath(which: str, x: np.ndarray) -> np.ndarray:
    x = np.ascontiguousarray(x, dtype=np.float32)
    y = np.empty_like(x)
    lib().oracle_detmath_eval({"sin": 0, "cos": 1, "exp": 2, "log": 3}[which], _p(x), _p(y), x.size)
    return y


class OracleScene:
    def __init__(self, arrays, use_bvh: bool | None = None):
        self._keep = [np.ascontiguousarray(arrays[k]) for k in
                      ("vertices", "indices", "meshes", "materials", "instances", "lights")]
        v, i, m, mt, ins, l = self._keep
        ntri = int((m["index_count"][ins["mesh_index"]] // 3).sum())
        if use_bvh is None:
            use_bvh = ntri > 64
        self._h = lib().oracle_scene_create(_p(v), len(v), _p(i), len(i), _p(m), len(m), _p(mt), len(mt),
                                            _p(ins), len(ins), _p(l) if len(l) else None, len(l), int(use_bvh))
        self.num_lights = len(l)

    @property
    def handle(self):
        return self._h

    def triangle_count(self) -> int:
        return lib().oracle_scene_triangle_count(self._h)

    def trace(self, origins: np.ndarray, dirs: np.ndarray, tmin=0.001, tmax=1e9, nthreads=None):
        o = np.ascontiguousarray(origins, dtype=np.float32).reshape(-1, 4)
        d = np.ascontiguousarray(dirs, dtype=np.float32).reshape(-1, 4)
        hits = np.empty((len(o), 4), np.float32)
        prims = np.empty(len(o), np.uint32)
        lib().oracle_trace_batch(self._h, _p(o), _p(d), tmin, tmax, len(o), _p(hits), _p(prims),
                                 nthreads or threads())
        return hits, prims

    def close(self):
        if self._h:
            lib().oracle_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def primary_ray(cam, px, py, frame_seed):
    o = np.empty(3, np.float32)
    d = np.empty(3, np.float32)
    s = C.c_uint32(0)
    lib().oracle_primary_ray(_cam_ptr(cam), px, py, frame_seed, _p(o), _p(d), C.byref(s))
    return o, d, s.value


PT_EMITTERS = 8   # ORACLE_PT_EMITTERS = RR_PT_FLAG_EMITTERS


def pathtrace(scene: OracleScene, cam, frame_seed: int, max_bounces: int, spp: int = 1, region=None,
              nthreads=None, flags: int = 0):
    """Returns (images[spp, h, w, 4], (extension_rays, shadow_rays)).
    flags=PT_EMITTERS: the emitter-sampling mode."""
    W, H = cam.screen_width, cam.screen_height
    x0, y0, w, h = region if region is not None else (0, 0, W, H)
    out = np.zeros((spp, h, w, 4), np.float32)
    stats = np.zeros(2, np.uint64)
    lib().oracle_pathtrace_ex(scene.handle, _cam_ptr(cam), frame_seed, max_bounces, spp, x0, y0, w, h, _p(out),
                              nthreads or threads(), _p(stats), flags)
    return out, (int(stats[0]), int(stats[1]))


def emitters(scene: OracleScene):
    """The emitter table: (records[n, 12], alias probabilities[n], aliases[n],
    total power)."""
    n = lib().oracle_emitters(scene.handle, None, None, None, None)
    rec = np.zeros((n, 12), np.float32)
    prob = np.zeros(n, np.float32)
    alias = np.zeros(n, np.uint32)
    tot = np.zeros(1, np.float32)
    lib().oracle_emitters(scene.handle, _p(rec) if n else None, _p(prob) if n else None, _p(alias) if n else None,
                          _p(tot))
    return rec, prob, alias, float(tot[0])


def accumulate(radiance: np.ndarray, acc: np.ndarray, camera_moved: int, spp: int) -> None:
    lib().oracle_accumulate(_p(radiance), _p(acc), radiance.size // 4, camera_moved, spp)


def di_params(frame_seed, m=16, temporal=1, spatial=1, k=4, radius=15, m_cap_factor=20, flags=0):
    """flags=DI_EMITTERS: candidates also from the emissive triangles."""
    return DIParams(frame_seed, m, temporal, spatial, k, radius, m_cap_factor, flags)


def restir_di_initial(scene, cam, p, gpos, gnrm, res, nthreads=None):
    lib().oracle_restir_di_initial(scene.handle, _cam_ptr(cam), C.byref(p), _p(gpos), _p(gnrm), _p(res),
                                   nthreads or threads())


def restir_di_temporal(scene, cam, p, gpos, gnrm, res, prev, nthreads=None):
    lib().oracle_restir_di_temporal(scene.handle, _cam_ptr(cam), C.byref(p), _p(gpos), _p(gnrm), _p(res),
                                    _p(prev), nthreads or threads())


def restir_di_spatial_shade(scene, cam, p, gpos, gnrm, res, out, nthreads=None):
    lib().oracle_restir_di_spatial_shade(scene.handle, _cam_ptr(cam), C.byref(p), _p(gpos), _p(gnrm), _p(res),
                                         _p(out), nthreads or threads())


def pt_reuse_params(frame_seed=0, candidates=8, max_bounces=4, temporal=1, spatial=1, neighbors=4, radius=12,
                    include_direct=1, indirect_strength=1.0, ray_bias=1e-3, gp=None):
    """ReSTIRPTPass.h:86-100 defaults; gp = guiding_params(...)."""
    return PtReuseParams(frame_seed, candidates, max_bounces, temporal, spatial, neighbors, radius, include_direct,
                         indirect_strength, ray_bias, (U32 * 2)(0, 0), gp if gp is not None else guiding_params())


def pt_reuse_images(img: dict) -> PtReuseImages:
    """img: gbuf_pos, gbuf_norm, direct (or None), res_curr[4], res_prev[4], hist_curr[2], hist_prev[2], output,
    accum, fitted — C-contiguous float32 (H, W, 4) images, int32 / float32 (cells, 4) grids."""
    def ptr(a):
        return None if a is None else _p(a)
    return PtReuseImages(ptr(img["gbuf_pos"]), ptr(img["gbuf_norm"]), ptr(img.get("direct")),
                         (P * 4)(*[ptr(a) for a in img["res_curr"]]), (P * 4)(*[ptr(a) for a in img["res_prev"]]),
                         (P * 2)(*[ptr(a) for a in img["hist_curr"]]), (P * 2)(*[ptr(a) for a in img["hist_prev"]]),
                         ptr(img["output"]), ptr(img["accum"]), ptr(img["fitted"]))


def restir_pt_initial(scene, cam, p, img, nthreads=None):
    lib().oracle_restir_pt_initial(scene.handle, _cam_ptr(cam), C.byref(p), C.byref(pt_reuse_images(img)),
                                   nthreads or threads())


def restir_pt_temporal(scene, cam, p, img, nthreads=None):
    lib().oracle_restir_pt_temporal(scene.handle, _cam_ptr(cam), C.byref(p), C.byref(pt_reuse_images(img)),
                                    nthreads or threads())


def restir_pt_spatial_shade(scene, cam, p, img, nthreads=None):
    lib().oracle_restir_pt_spatial_shade(scene.handle, _cam_ptr(cam), C.byref(p), C.byref(pt_reuse_images(img)),
                                         nthreads or threads())


def bvh2_trace(nodes, tris, origins, dirs, tmin, tmax, any_hit, nthreads=None):
    """The library's BVH traversal restated on the CPU over its exported arrays:
    returns (hits (n, 4) float32, prims (n,) uint32, work (n, 2) uint32)."""
    n = len(origins)
    hits = np.zeros((n, 4), np.float32)
    prims = np.zeros(n, np.uint32)
    work = np.zeros((n, 2), np.uint32)
    lib().oracle_bvh2_trace(_p(nodes), len(nodes), _p(tris), _p(origins), _p(dirs), tmin, tmax, n, int(any_hit),
                            _p(hits), _p(prims), _p(work), nthreads or threads())
    return hits, prims, work


def bvh4_trace(nodes4, tris, origins, dirs, tmin, tmax, any_hit, nthreads=None):
    """bvh2_trace over the library's 4-wide layout of the same tree (nodes4:
    (n, 32) float32 from rr_scene_copy_bvh4)."""
    n = len(origins)
    hits = np.zeros((n, 4), np.float32)
    prims = np.zeros(n, np.uint32)
    work = np.zeros((n, 2), np.uint32)
    lib().oracle_bvh4_trace(_p(nodes4), len(nodes4), _p(tris), _p(origins), _p(dirs), tmin, tmax, n, int(any_hit),
                            _p(hits), _p(prims), _p(work), nthreads or threads())
    return hits, prims, work


def gi_reuse_params(frame_seed=0, candidates=8, temporal=1, spatial=1, neighbors=4, radius=12, include_direct=1,
                    indirect_strength=1.0, ray_bias=1e-3):
    """ReSTIRGIPass.h:67-74 defaults."""
    return GiReuseParams(frame_seed, candidates, temporal, spatial, neighbors, radius, include_direct,
                         indirect_strength, ray_bias, (U32 * 3)(0, 0, 0))


def gi_reuse_images(img: dict) -> GiReuseImages:
    """img: gbuf_pos, gbuf_norm, direct (or None), res_curr[3], res_prev[3], hist_curr[2], hist_prev[2], output —
    C-contiguous float32 (H, W, 4) images."""
    def ptr(a):
        return None if a is None else _p(a)
    return GiReuseImages(ptr(img["gbuf_pos"]), ptr(img["gbuf_norm"]), ptr(img.get("direct")),
                         (P * 3)(*[ptr(a) for a in img["res_curr"]]), (P * 3)(*[ptr(a) for a in img["res_prev"]]),
                         (P * 2)(*[ptr(a) for a in img["hist_curr"]]), (P * 2)(*[ptr(a) for a in img["hist_prev"]]),
                         ptr(img["output"]))


def restir_gi_initial(scene, cam, p, img, nthreads=None):
    lib().oracle_restir_gi_initial(scene.handle, _cam_ptr(cam), C.byref(p), C.byref(gi_reuse_images(img)),
                                   nthreads or threads())


def restir_gi_temporal(scene, cam, p, img, nthreads=None):
    lib().oracle_restir_gi_temporal(scene.handle, _cam_ptr(cam), C.byref(p), C.byref(gi_reuse_images(img)),
                                    nthreads or threads())


def restir_gi_spatial_shade(scene, cam, p, img, nthreads=None):
    lib().oracle_restir_gi_spatial_shade(scene.handle, _cam_ptr(cam), C.byref(p), C.byref(gi_reuse_images(img)),
                                         nthreads or threads())


def atrous_iteration(inp, gpos, gnrm, out, stride, sp=0.25, sn=0.20, sl=1.0, nthreads=None):
    H, W = inp.shape[0], inp.shape[1]
    lib().oracle_atrous_iteration(_p(inp), _p(gpos), _p(gnrm), _p(out), W, H, stride, sp, sn, sl,
                                  nthreads or threads())


def atrous(inp, gpos, gnrm, iterations=5, sp=0.25, sn=0.20, sl=1.0):
    """AtrousPass::execute semantics (clamp 1..7, stride 1<<i); returns the result."""
    it = min(max(iterations, 1), 7)
    ping = [np.empty_like(inp), np.empty_like(inp)]
    read = inp
    for i in range(it):
        atrous_iteration(read, gpos, gnrm, ping[i & 1], 1 << i, sp, sn, sl)
        read = ping[i & 1]
    return read


def guiding_params(cell_count=1 << 20, enabled=1, min_samples=8, kappa_max=512.0, alpha=0.5,
                   base_cell_size=0.10, distance_slope=0.02):
    return GuidingParams(base_cell_size, distance_slope, cell_count, enabled, min_samples, kappa_max, alpha, 0)


def guiding_cell_index(pos, bsdf, cam_pos, gp) -> int:
    p = np.ascontiguousarray(pos, np.float32)
    c = np.ascontiguousarray(cam_pos, np.float32)
    return lib().oracle_guiding_cell_index(_p(p), bsdf, _p(c), C.byref(gp))


def guiding_splat(accum, pos, dirs, bsdf, cam_pos, gp):
    c = np.ascontiguousarray(cam_pos, np.float32)
    lib().oracle_guiding_splat(_p(accum), _p(pos), _p(dirs), _p(bsdf), len(bsdf), _p(c), C.byref(gp))


def guiding_fit(accum, fitted, gp):
    lib().oracle_guiding_fit(_p(accum), _p(fitted), C.byref(gp))


def guiding_sample(fitted, pos, nrm, bsdf, seeds, cam_pos, gp):
    c = np.ascontiguousarray(cam_pos, np.float32)
    wi = np.empty((len(bsdf), 4), np.float32)
    pdf = np.empty(len(bsdf), np.float32)
    lib().oracle_guiding_sample(_p(fitted), _p(pos), _p(nrm), _p(bsdf), _p(seeds), len(bsdf), _p(c),
                                C.byref(gp), _p(wi), _p(pdf))
    return wi, pdf


def vmf_pdf(mu, kappa, d) -> float:
    m = np.ascontiguousarray(mu, np.float32)
    dd = np.ascontiguousarray(d, np.float32)
    return lib().oracle_vmf_pdf(_p(m), kappa, _p(dd))


def brdf_eval(n, wo, wi, base, metallic, roughness):
    a = [np.ascontiguousarray(x, np.float32) for x in (n, wo, wi, base)]
    out = np.empty(3, np.float32)
    lib().oracle_brdf_eval(*[_p(x) for x in a], metallic, roughness, _p(out))
    return out


def brdf_sample(wo, n, base, metallic, roughness, u0, u1):
    a = [np.ascontiguousarray(x, np.float32) for x in (wo, n, base)]
    wi = np.empty(3, np.float32)
    f = np.empty(3, np.float32)
    pdf = C.c_float(0)
    lib().oracle_brdf_sample(*[_p(x) for x in a], metallic, roughness, u0, u1, _p(wi), C.byref(pdf), _p(f))
    return wi, pdf.value, f


def brdf_pdf(wo, wi, n, roughness) -> float:
    a = [np.ascontiguousarray(x, np.float32) for x in (wo, wi, n)]
    return lib().oracle_brdf_pdf(*[_p(x) for x in a], roughness)
