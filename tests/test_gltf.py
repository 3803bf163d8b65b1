"""glTF 2.0 loading (rr_host_scene_gltf, GltfLoader::load + Scene::upload) on
the CPU: the library's loader against the restatement in oracle/gltf_ref.py,
bit-exact, on generated files in the three storage forms (.gltf with a
base64 buffer, .gltf with an external .bin, .glb); interleaved attributes;
and the error paths (every one an RRError with a reason, nothing read out of
range)."""
import json

import numpy as np
import pytest

import gltf_files
import gltf_ref


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).view(np.uint32)


def _compare(hs, ref):
    a = hs.arrays
    v = a["vertices"]
    got_v = np.concatenate([v["pos"], v["normal"], v["uv"], v["tangent"]], axis=1)
    np.testing.assert_array_equal(_bits(got_v), _bits(ref["vertices"]))
    np.testing.assert_array_equal(a["indices"], ref["indices"])
    m = a["meshes"]
    got_m = np.stack([m["vertex_base"], m["vertex_count"], m["index_byte_offset"], m["index_count"],
                      m["material_index"]], 1)
    np.testing.assert_array_equal(got_m, ref["meshes"])
    mt = a["materials"]
    got_mt = np.concatenate([mt["base_color"], mt["metallic"][:, None], mt["roughness"][:, None], mt["emissive"],
                             mt["ior"][:, None]], axis=1)
    np.testing.assert_array_equal(_bits(got_mt), _bits(ref["materials"]))
    assert (mt["albedo_tex_idx"] == 0xFFFFFFFF).all() and (mt["sampler_idx"] == 0).all()
    ins = a["instances"]
    np.testing.assert_array_equal(_bits(ins["transform"]), _bits(ref["transforms"]))
    np.testing.assert_array_equal(ins["mesh_index"], ref["mesh_index"])
    assert len(a["lights"]) == 0


@pytest.mark.parametrize("mode,ext", [("embedded", "gltf"), ("external", "gltf"), ("glb", "glb")])
@pytest.mark.parametrize("seed", [1, 2])
def test_gltf_matches_restatement(rr, tmp_path, mode, ext, seed):
    path = str(tmp_path / f"scene.{ext}")
    gltf_files.feature_scene(seed).save(path, mode)
    hs = rr.HostScene.gltf(path)
    ref = gltf_ref.load(path)
    # the feature scene: 4 triangle meshes (the LINES primitive skipped), scene 1's trees:
    # node 0 -> (1 -> 2: mesh 0), (3: mesh 1); node 5 (mesh 2) -> 6 (mesh 3)
    assert len(ref["meshes"]) == 4 and list(ref["mesh_index"]) == [0, 1, 2, 3]
    _compare(hs, ref)
    hs.close()


def test_gltf_transform_semantics(rr, tmp_path):
    """T * R * S against a hand-built matrix, and parent * child composition."""
    g = gltf_files.Builder()
    p = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], "<f4")
    g.doc["meshes"] = [{"primitives": [{"attributes": {"POSITION": g.accessor(p, "VEC3")}}]}]
    s2 = float(np.sqrt(0.5))
    g.doc["nodes"] = [{"translation": [1.0, 2.0, 3.0], "rotation": [0.0, 0.0, s2, s2], "scale": [2.0, 2.0, 2.0],
                       "children": [1]},
                      {"mesh": 0, "translation": [1.0, 0.0, 0.0]}]
    g.doc["scenes"] = [{"nodes": [0]}]
    path = str(tmp_path / "t.gltf")
    g.save(path)
    hs = rr.HostScene.gltf(path)
    T = hs.arrays["instances"]["transform"][0].reshape(4, 4)   # row-major
    # parent: translate (1,2,3), rotate 90 deg about z, scale 2; child: translate (1,0,0)
    want = np.array([[0, -2, 0, 1], [2, 0, 0, 4], [0, 0, 2, 3], [0, 0, 0, 1]], np.float64)
    np.testing.assert_allclose(T, want, atol=1e-6)
    assert len(hs.arrays["materials"]) == 1   # no materials in the file: one default Material
    mt = hs.arrays["materials"][0]
    assert tuple(mt["base_color"]) == (1, 1, 1, 1) and mt["metallic"] == 0 and mt["roughness"] == 1
    hs.close()


def test_gltf_interleaved_attributes(rr, tmp_path):
    """byteStride is honoured (positions and normals interleaved in one view)."""
    g = gltf_files.Builder()
    rng = np.random.default_rng(5)
    P = rng.uniform(-1, 1, (6, 3)).astype("<f4")
    N = rng.uniform(-1, 1, (6, 3)).astype("<f4")
    inter = np.concatenate([P, N], 1).astype("<f4")
    v = g.view(inter.tobytes(), stride=24)
    pa = g.accessor(P, "VEC3", view=v)
    na = g.accessor(N, "VEC3", view=v, offset=12)
    g.doc["meshes"] = [{"primitives": [{"attributes": {"POSITION": pa, "NORMAL": na}}]}]
    g.doc["nodes"] = [{"mesh": 0}]
    g.doc["scenes"] = [{"nodes": [0]}]
    path = str(tmp_path / "i.glb")
    g.save(path, "glb")
    hs = rr.HostScene.gltf(path)
    np.testing.assert_array_equal(hs.arrays["vertices"]["pos"], P)
    np.testing.assert_array_equal(hs.arrays["vertices"]["normal"], N)
    hs.close()


def _broken(tmp_path, edit, name="b.gltf"):
    g = gltf_files.feature_scene(3)
    edit(g)
    path = str(tmp_path / name)
    g.save(path)
    return path


@pytest.mark.parametrize("case,edit,msg", [
    ("index", lambda g: g.doc["meshes"][0]["primitives"][0].update(indices=999), "index out of range"),
    ("accessor_range", lambda g: g.doc["accessors"][0].update(count=10_000), "outside its bufferView"),
    ("cycle", lambda g: g.doc["nodes"][2].update(children=[0]), "cycle"),
    ("position_type", lambda g: g.doc["accessors"][0].update(componentType=5123), "POSITION must be FLOAT"),
    ("vertex_index", lambda g: g.doc["accessors"][3].update(componentType=5125, count=9), "index past"),
    ("sparse", lambda g: g.doc["accessors"][1].update(sparse={"count": 1}), "sparse"),
    ("material", lambda g: g.doc["meshes"][0]["primitives"][0].update(material=42), "missing material"),
    ("mesh", lambda g: g.doc["nodes"][5].update(mesh=17), "missing mesh"),
    ("no_version", lambda g: g.doc.pop("asset"), "asset.version"),
])
def test_gltf_errors(rr, tmp_path, case, edit, msg):
    path = _broken(tmp_path, edit)
    with pytest.raises(rr.RRError, match=msg):
        rr.HostScene.gltf(path)


def test_gltf_bad_files(rr, tmp_path):
    with pytest.raises(rr.RRError, match="cannot open"):
        rr.HostScene.gltf(str(tmp_path / "missing.gltf"))
    bad = tmp_path / "bad.gltf"
    bad.write_text('{"asset": {"version": "2.0"}, "meshes": [}')
    with pytest.raises(rr.RRError, match="JSON"):
        rr.HostScene.gltf(str(bad))
    deep = tmp_path / "deep.gltf"
    deep.write_text("[" * 1000 + "]" * 1000)
    with pytest.raises(rr.RRError, match="nesting"):
        rr.HostScene.gltf(str(deep))
    trunc = tmp_path / "t.glb"
    g = gltf_files.feature_scene(4)
    g.save(str(trunc), "glb")
    data = trunc.read_bytes()
    trunc.write_bytes(data[:len(data) // 2])
    with pytest.raises(rr.RRError):
        rr.HostScene.gltf(str(trunc))
    # short buffer: byteLength larger than the data
    sb = tmp_path / "short.gltf"
    g.save(str(sb))
    doc = json.loads(sb.read_text())
    doc["buffers"][0]["byteLength"] += 64
    sb.write_text(json.dumps(doc))
    with pytest.raises(rr.RRError, match="shorter"):
        rr.HostScene.gltf(str(sb))


def test_gltf_json_escapes_and_empty_scene(rr, tmp_path):
    path = tmp_path / "e.gltf"
    path.write_text('{"asset": {"version": "2.0", "generator": "\\u00e9\\ud83d\\ude00 \\"q\\" \\\\ \\/"},'
                    ' "scenes": [{"nodes": []}], "scene": 0}')
    hs = rr.HostScene.gltf(str(path))
    assert len(hs.arrays["vertices"]) == 0 and len(hs.arrays["instances"]) == 0
    hs.close()
