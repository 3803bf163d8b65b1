"""Python wrapper of oracle/_ref/librr_slangref.so: the reference's own shader
text, rewritten mechanically to C++ (oracle/make_ref.py) and run on the CPU.

TEST INFRASTRUCTURE ONLY (imported by tests/). The library is built from the
reference checkout (`make -C oracle ref`) and exists only where that checkout
does; `available()` says whether it could be built. Each function mirrors the
hand-written oracle's function of the same name (oracle/oracle.py), so the
tests can require both to give the same bits on the same inputs.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

import oracle as O

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "_ref" / "librr_slangref.so"
REFERENCE = Path("/root/reference")

P, U32, F32, I = C.c_void_p, C.c_uint32, C.c_float, C.c_int
_SIG = {
    "sref_pcg_hash": (U32, [U32]),
    "sref_make_seed": (U32, [U32, U32, U32]),
    "sref_rand_float": (F32, [C.POINTER(U32)]),
    "sref_brdf_eval": (None, [P, P, P, P, F32, F32, P]),
    "sref_brdf_sample": (None, [P, P, P, F32, F32, F32, F32, P, P, P]),
    "sref_brdf_pdf": (F32, [P, P, P, F32]),
    "sref_sample_cosine_hemisphere": (None, [F32, F32, P, P]),
    "sref_build_onb": (None, [P, P, P]),
    "sref_vmf_sample": (None, [P, F32, F32, F32, P, P]),
    "sref_vmf_pdf": (F32, [P, F32, P]),
    "sref_guiding_cell_index": (U32, [P, U32, P, C.POINTER(O.GuidingParams)]),
    "sref_guiding_splat": (None, [P, P, P, P, C.c_size_t, P, C.POINTER(O.GuidingParams)]),
    "sref_guiding_fit": (None, [P, P, C.POINTER(O.GuidingParams)]),
    "sref_scene_create": (P, [P, P, U32, P, U32, P, U32, P, U32, P, U32, P, U32]),
    "sref_scene_destroy": (None, [P]),
    "sref_pathtrace": (None, [P, P, U32, U32, U32, U32, U32, U32, U32, P, I]),
    "sref_accumulate": (None, [P, P, U32, U32, U32, U32]),
    "sref_restir_di": (None, [I, P, P, C.POINTER(O.DIParams), P, P, P, P, P, I]),
    "sref_atrous_iteration": (None, [P, P, P, P, U32, U32, U32, F32, F32, F32, I]),
    "sref_restir_pt": (None, [I, P, P, C.POINTER(O.PtReuseParams), C.POINTER(O.PtReuseImages), I]),
    "sref_restir_gi": (None, [I, P, P, C.POINTER(O.GiReuseParams), C.POINTER(O.GiReuseImages), I]),
}
_lib = None


def build() -> bool:
    """Builds the library when the reference checkout is present."""
    if REFERENCE.is_dir():
        r = subprocess.run(["make", "-s", "-C", str(HERE), "ref", f"REFERENCE={REFERENCE}"], capture_output=True,
                           text=True)
        if r.returncode != 0:
            raise RuntimeError(f"make -C oracle ref failed:\n{r.stdout}\n{r.stderr}")
    return LIB_PATH.exists()


def available() -> bool:
    try:
        return build()
    except RuntimeError:
        raise


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        O.lib()   # librr_oracle.so first: the intersector this library links against
        L = C.CDLL(str(LIB_PATH))
        for k, (r, a) in _SIG.items():
            f = getattr(L, k)
            f.restype = r
            f.argtypes = a
        _lib = L
    return _lib


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data


def _f3(v):
    return np.ascontiguousarray(v, np.float32)


class RefScene:
    """The scene arrays in the reference's heap layout, traced by the oracle
    scene `tracer` (the stand-in for the reference's hardware BLAS/TLAS)."""

    def __init__(self, arrays, tracer: O.OracleScene):
        self.tracer = tracer
        keep = [np.ascontiguousarray(arrays[k]) for k in
                ("vertices", "indices", "meshes", "materials", "instances", "lights")]
        v, i, m, mt, ins, l = keep
        self._h = lib().sref_scene_create(tracer.handle, _p(v), len(v), _p(i), len(i), _p(m), len(m), _p(mt),
                                          len(mt), _p(ins), len(ins), _p(l) if len(l) else None, len(l))

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            lib().sref_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def pcg_hash(x: int) -> int:
    return lib().sref_pcg_hash(x & 0xFFFFFFFF)


def make_seed(px: int, py: int, frame: int) -> int:
    return lib().sref_make_seed(px, py, frame & 0xFFFFFFFF)


def rand_float(seed: int) -> tuple[float, int]:
    s = C.c_uint32(seed)
    r = lib().sref_rand_float(C.byref(s))
    return r, s.value


def brdf_eval(n, wo, wi, base, metallic, roughness):
    out = np.zeros(3, np.float32)
    lib().sref_brdf_eval(_p(_f3(n)), _p(_f3(wo)), _p(_f3(wi)), _p(_f3(base)), metallic, roughness, _p(out))
    return out


def brdf_sample(wo, n, base, metallic, roughness, u0, u1):
    wi, f = np.zeros(3, np.float32), np.zeros(3, np.float32)
    pdf = np.zeros(1, np.float32)
    lib().sref_brdf_sample(_p(_f3(wo)), _p(_f3(n)), _p(_f3(base)), metallic, roughness, u0, u1, _p(wi), _p(pdf),
                           _p(f))
    return wi, float(pdf[0]), f


def brdf_pdf(wo, wi, n, roughness):
    return lib().sref_brdf_pdf(_p(_f3(wo)), _p(_f3(wi)), _p(_f3(n)), roughness)


def sample_cosine_hemisphere(u0, u1):
    out, pdf = np.zeros(3, np.float32), np.zeros(1, np.float32)
    lib().sref_sample_cosine_hemisphere(u0, u1, _p(out), _p(pdf))
    return out, float(pdf[0])


def build_onb(n):
    T, B = np.zeros(3, np.float32), np.zeros(3, np.float32)
    lib().sref_build_onb(_p(_f3(n)), _p(T), _p(B))
    return T, B


def vmf_sample(mu, kappa, u0, u1):
    d, pdf = np.zeros(3, np.float32), np.zeros(1, np.float32)
    lib().sref_vmf_sample(_p(_f3(mu)), kappa, u0, u1, _p(d), _p(pdf))
    return d, float(pdf[0])


def vmf_pdf(mu, kappa, d):
    return lib().sref_vmf_pdf(_p(_f3(mu)), kappa, _p(_f3(d)))


def guiding_cell_index(pos, bsdf, cam_pos, gp) -> int:
    return lib().sref_guiding_cell_index(_p(_f3(pos)), bsdf, _p(_f3(cam_pos)), C.byref(gp))


def guiding_splat(accum, pos, dirs, bsdf, cam_pos, gp):
    pos, dirs = np.ascontiguousarray(pos, np.float32), np.ascontiguousarray(dirs, np.float32)
    bsdf = np.ascontiguousarray(bsdf, np.uint32)
    lib().sref_guiding_splat(_p(accum), _p(pos), _p(dirs), _p(bsdf), len(bsdf), _p(_f3(cam_pos)), C.byref(gp))


def guiding_fit(accum, fitted, gp):
    lib().sref_guiding_fit(_p(accum), _p(fitted), C.byref(gp))


def pathtrace(scene: RefScene, cam, frame_seed: int, max_bounces: int, spp: int = 1, region=None, nthreads=None):
    W, H = cam.screen_width, cam.screen_height
    x0, y0, w, h = region if region is not None else (0, 0, W, H)
    out = np.zeros((spp, h, w, 4), np.float32)
    lib().sref_pathtrace(scene.handle, C.addressof(cam), frame_seed, max_bounces, spp, x0, y0, w, h, _p(out),
                         nthreads or O.threads())
    return out


def accumulate(radiance: np.ndarray, acc: np.ndarray, camera_moved: int, spp: int) -> None:
    H, W = acc.shape[0], acc.shape[1]
    lib().sref_accumulate(_p(radiance), _p(acc), W, H, camera_moved, spp)


def restir_di(stage: int, scene: RefScene, cam, p, gpos, gnrm, res_curr, res_prev, out, nthreads=None):
    lib().sref_restir_di(stage, scene.handle, C.addressof(cam), C.byref(p), _p(gpos), _p(gnrm), _p(res_curr),
                         _p(res_prev), _p(out), nthreads or O.threads())


def atrous_iteration(inp, gpos, gnrm, out, stride, sp=0.25, sn=0.20, sl=1.0, nthreads=None):
    H, W = inp.shape[0], inp.shape[1]
    lib().sref_atrous_iteration(_p(inp), _p(gpos), _p(gnrm), _p(out), W, H, stride, sp, sn, sl,
                                nthreads or O.threads())


def atrous(inp, gpos, gnrm, iterations=5, sp=0.25, sn=0.20, sl=1.0):
    """AtrousPass::execute semantics (AtrousPass.cpp:243-306): iterations
    clamped to 1..7, stride 1 << i, ping-pong."""
    it = min(max(iterations, 1), 7)
    ping = [np.empty_like(inp), np.empty_like(inp)]
    read = inp
    for i in range(it):
        atrous_iteration(read, gpos, gnrm, ping[i & 1], 1 << i, sp, sn, sl)
        read = ping[i & 1]
    return read


def restir_pt(stage: int, scene: RefScene, cam, p, images, nthreads=None):
    lib().sref_restir_pt(stage, scene.handle, C.addressof(cam), C.byref(p), C.byref(images), nthreads or O.threads())


def restir_gi(stage: int, scene: RefScene, cam, p, images, nthreads=None):
    lib().sref_restir_gi(stage, scene.handle, C.addressof(cam), C.byref(p), C.byref(images), nthreads or O.threads())
