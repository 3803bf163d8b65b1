"""CPU checks of the C ABI library: it loads, exports every declared entry
point, its host-side factories match an independent restatement of the
reference, and argument errors come back as status codes (no GPU needed)."""
import ctypes as C
import re
import subprocess
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parent.parent


def declared_functions():
    names = set()
    for h in ("rr_cuda.h", "rr_host.h"):
        text = (ROOT / "include" / h).read_text()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"\b(rr_[a-z0-9_]+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol(rr):
    L = rr.lib()
    names = declared_functions()
    assert len(names) >= 30
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    out = subprocess.run(["nm", "-D", "--defined-only", str(rr.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if ln.strip()}
    assert not [n for n in names if n not in exported]
    # the Python binding declares exactly the header's functions
    assert set(rr.EXPORTED) == set(names)


def test_abi_version_and_status_strings(rr):
    assert rr.lib().rr_abi_version() == 1
    assert rr.lib().rr_status_string(0) == b"RR_OK"
    assert rr.lib().rr_status_string(5) == b"RR_ERR_QUEUE_OVERFLOW"


def test_struct_sizes_match_headers(rr):
    assert C.sizeof(rr.GpuCameraData) == 304
    assert C.sizeof(rr.PtParams) == 16 and C.sizeof(rr.AccParams) == 16
    assert C.sizeof(rr.DIParams) == 32 and C.sizeof(rr.AtrousParams) == 32 and C.sizeof(rr.GuidingParams) == 32
    assert C.sizeof(rr.SceneStats) == 48


def test_traversal_variant_widths(rr):
    """Variants 3, 4 and 6 walk the 4-wide tree (128-byte nodes), the others
    the binary one; out-of-range variants report width 0."""
    L = rr.lib()
    assert [L.rr_pathtracer_variant_width(v) for v in range(rr.PT_VARIANT_COUNT)] == [2, 2, 2, 4, 4, 2, 4, 2]
    assert L.rr_pathtracer_variant_width(-1) == 0 and L.rr_pathtracer_variant_width(rr.PT_VARIANT_COUNT) == 0


def test_cornell_factory_matches_reference_restatement(rr):
    from cornell import MATERIALS, cornell_triangles
    hs = rr.HostScene.cornell(0)
    a = hs.arrays
    assert len(a["meshes"]) == 8 and len(a["instances"]) == 8 and hs.triangle_count() == 36
    tris = []
    for inst in a["instances"]:
        m = a["meshes"][inst["mesh_index"]]
        T = inst["transform"].reshape(4, 4).astype(np.float64)
        ib = m["index_byte_offset"] // 4
        for j in range(m["index_count"] // 3):
            idx = a["indices"][ib + 3 * j: ib + 3 * j + 3] + m["vertex_base"]
            p = a["vertices"]["pos"][idx].astype(np.float64)
            tris.append((T[:3, :3] @ p.T).T + T[:3, 3])
    ref, ref_mats = cornell_triangles()
    np.testing.assert_allclose(np.array(tris), ref, atol=2e-6)
    for k, (base, emit) in enumerate(MATERIALS):
        np.testing.assert_allclose(a["materials"]["base_color"][k][:3], base, rtol=1e-7)
        np.testing.assert_allclose(a["materials"]["emissive"][k], emit)
    assert a["materials"]["roughness"].tolist() == [1.0] * 4
    L = a["lights"][0]
    assert L["type"] == 0 and np.allclose(L["position"], [0, 0.9, 0]) and np.allclose(L["emission"], [15, 15, 12])
    v1 = rr.HostScene.cornell(1).arrays
    np.testing.assert_allclose(v1["materials"]["emissive"][3], [17, 12, 4])


def test_camera_matches_reference_restatement(rr):
    from cornell import camera_matrices
    cd = rr.camera_desc(320, 200, eye=(0.5, 1.0, 3.0), center=(0.0, 0.2, 0.0))
    cam = rr.camera_data(cd)
    V, Pm = camera_matrices(np.array(cam.position, np.float64), cd.yaw_deg, cd.pitch_deg, 45.0, 320 / 200, 0.01,
                            1000.0)
    np.testing.assert_allclose(np.array(cam.view).reshape(4, 4), V, atol=1e-5)
    np.testing.assert_allclose(np.array(cam.inv_view).reshape(4, 4), np.linalg.inv(V), atol=1e-5)
    np.testing.assert_allclose(np.array(cam.inv_proj).reshape(4, 4), np.linalg.inv(Pm), rtol=1e-5, atol=1e-6)
    assert (cam.screen_width, cam.screen_height) == (320, 200)
    # the primary ray through the image centre follows the camera direction
    import oracle as O
    o, d, _ = O.primary_ray(cam, 160, 100, 0)
    fwd = np.array(cam.direction)
    assert float(d @ fwd) > 0.999


def test_procedural_scene_shape(rr):
    hs = rr.HostScene.procedural(seed=7, target_triangles=200_000, emissive_triangles=64, box_half=20.0)
    a = hs.arrays
    assert hs.triangle_count() >= 200_000
    assert len(a["lights"]) == 64
    emissive = (a["materials"]["emissive"] > 0).any(axis=1)
    assert emissive.sum() == 64
    L = a["materials"]["emissive"][emissive].max(axis=1)
    assert L.min() >= 0.06 and L.max() <= 100.0
    r = a["materials"]["roughness"][~emissive]
    assert r.min() >= 0.05 and r.max() <= 1.0
    assert set(np.unique(a["materials"]["metallic"][~emissive])) <= {0.0, 1.0}
    # deterministic for a seed
    b = rr.HostScene.procedural(seed=7, target_triangles=200_000, emissive_triangles=64, box_half=20.0).arrays
    assert np.array_equal(a["vertices"], b["vertices"])


def test_instanced_scene_shape(rr):
    hs = rr.HostScene.instanced(seed=5, base_meshes=4, tris_per_mesh=200, instance_count=50, emissive_triangles=8)
    a = hs.arrays
    assert len(a["instances"]) == 50 + 8
    assert (a["meshes"]["index_count"][:4] // 3 == 200).all()


def test_context_requires_gpu_or_reports(rr):
    import torch
    if torch.cuda.is_available():
        pytest.skip("GPU present")
    h = C.c_void_p()
    st = rr.lib().rr_ctx_create(0, C.byref(h))
    assert st in (2, 1)  # RR_ERR_CUDA without a device
    assert rr.lib().rr_ctx_destroy(None) == 1
    assert rr.lib().rr_scene_create(None, None, None) == 1
    assert rr.lib().rr_pathtracer_execute(None, None, None, None, None, None) == 1


def test_null_arguments_rejected_without_device(rr):
    L = rr.lib()
    assert L.rr_accumulate_execute(None, None, 0, None, None, None, None) == 1
    assert L.rr_atrous_execute(None, None, None, None, None, None, None, None, None) == 1
    assert L.rr_guiding_fit(None, None, None, None, None) == 1
    assert L.rr_host_scene_cornell(7, C.byref(C.c_void_p())) == 1
    assert L.rr_camera_build(None, None, None) == 1


def test_inputs_library_builds_the_same_scenes_and_cameras(rr, O):
    """The CPU reference arm builds its scene and camera with
    oracle/librr_inputs.so (the generator source without CUDA); it must give
    the same bytes as the product library's factories."""
    I = O.inputs_lib()
    pairs = [
        (rr.HostScene.procedural(seed=0x5EED0002, target_triangles=60_000, emissive_triangles=256, box_half=20.0),
         rr.HostScene.procedural(seed=0x5EED0002, target_triangles=60_000, emissive_triangles=256, box_half=20.0,
                                 L=I)),
        (rr.HostScene.instanced(seed=7, base_meshes=4, tris_per_mesh=500, instance_count=64, emissive_triangles=64,
                                box_half=50.0),
         rr.HostScene.instanced(seed=7, base_meshes=4, tris_per_mesh=500, instance_count=64, emissive_triangles=64,
                                box_half=50.0, L=I)),
        (rr.HostScene.cornell(0), rr.HostScene.cornell(0, L=I)),
    ]
    for a, b in pairs:
        for k, v in a.arrays.items():
            assert v.tobytes() == b.arrays[k].tobytes(), k
    for eye, center in (((0.0, 4.0, 34.0), (0.0, -3.0, 0.0)), (None, None)):
        ca = rr.camera_data(rr.camera_desc(1920, 1080, eye=eye, center=center))
        cb = rr.camera_data(rr.camera_desc(1920, 1080, eye=eye, center=center, L=I), L=I)
        assert bytes(ca) == bytes(cb)


def test_scene_without_emitter_point_lights(rr):
    """RR_SCENE_NO_EMITTER_LIGHTS keeps the geometry and materials and drops
    only the emitters' point lights."""
    a = rr.HostScene.procedural(seed=3, target_triangles=30_000, emissive_triangles=50).arrays
    b = rr.HostScene.procedural(seed=3, target_triangles=30_000, emissive_triangles=50,
                                flags=rr.SCENE_NO_EMITTER_LIGHTS).arrays
    assert len(a["lights"]) == 50 and len(b["lights"]) == 0
    for k in ("vertices", "indices", "meshes", "materials", "instances"):
        assert a[k].tobytes() == b[k].tobytes(), k
