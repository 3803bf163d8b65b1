"""CPU restatement of the reference's glTF scene loading — test infrastructure
only (the checker of rr_host_scene_gltf, never shipped or measured).

Restates GltfLoader::load (src/scene/GltfLoader.cpp:79-365) and the CPU side
of Scene::upload (src/scene/Scene.cpp:255-345): the GpuScene arrays the
reference would upload for a glTF 2.0 file. The reference parses files with
tinygltf 2.9.7 (vcpkg.json:30), which is not part of the reference tree; its
document defaults are the glTF 2.0 ones (primitive mode 4, baseColorFactor
(1,1,1,1), metallicFactor 1, roughnessFactor 1, emissiveFactor (0,0,0),
material / indices -1, defaultScene -1). Parity is unpinned: the reference
cannot run here and ships no glTF test files or expected arrays, so this
restatement and the CUDA library's loader are checked against each other on
generated files. Arithmetic follows glm (float32, column-major, left-to-right
sums); numbers go text -> binary64 -> binary32 as tinygltf's JSON reader and
the loader's casts take them.

Only what the reference reads well is restated: tightly packed float
attributes, u8/u16/u32 indices, no sparse accessors.
"""
import base64
import json
import os
import struct
from urllib.parse import unquote

import numpy as np

f32 = np.float32


def _identity():
    return [[f32(1.0) if r == c else f32(0.0) for r in range(4)] for c in range(4)]   # m[c][r]


def _mul(A, B):   # glm operator*(mat4, mat4)
    return [[A[0][r] * B[i][0] + A[1][r] * B[i][1] + A[2][r] * B[i][2] + A[3][r] * B[i][3] for r in range(4)]
            for i in range(4)]


def _translate(m, v):   # glm::translate
    R = [list(c) for c in m]
    R[3] = [m[0][r] * v[0] + m[1][r] * v[1] + m[2][r] * v[2] + m[3][r] for r in range(4)]
    return R


def _scale(m, v):   # glm::scale
    return [[m[0][r] * v[0] for r in range(4)], [m[1][r] * v[1] for r in range(4)],
            [m[2][r] * v[2] for r in range(4)], list(m[3])]


def _quat_to_mat4(w, x, y, z):   # glm::mat4_cast(glm::quat(w, x, y, z))
    one, two = f32(1.0), f32(2.0)
    qxx, qyy, qzz = x * x, y * y, z * z
    qxz, qxy, qyz = x * z, x * y, y * z
    qwx, qwy, qwz = w * x, w * y, w * z
    R = _identity()
    R[0][0] = one - two * (qyy + qzz); R[0][1] = two * (qxy + qwz); R[0][2] = two * (qxz - qwy)
    R[1][0] = two * (qxy - qwz); R[1][1] = one - two * (qxx + qzz); R[1][2] = two * (qyz + qwx)
    R[2][0] = two * (qxz + qwy); R[2][1] = two * (qyz - qwx); R[2][2] = one - two * (qxx + qyy)
    return R


def _node_transform(node):   # GltfLoader.cpp:33-61
    if "matrix" in node:
        mat = node["matrix"]
        m = _identity()
        for r in range(4):
            for c in range(4):
                m[c][r] = f32(float(mat[r * 4 + c]))
        return m
    t = _identity()
    if "translation" in node:
        t = _translate(t, [f32(float(a)) for a in node["translation"]])
    if "rotation" in node:
        q = [f32(float(a)) for a in node["rotation"]]
        t = _mul(t, _quat_to_mat4(q[3], q[0], q[1], q[2]))
    if "scale" in node:
        t = _scale(t, [f32(float(a)) for a in node["scale"]])
    return t


_CT = {5121: ("<u1", 1), 5123: ("<u2", 2), 5125: ("<u4", 4), 5126: ("<f4", 4)}
_NC = {"SCALAR": 1, "VEC2": 2, "VEC3": 3, "VEC4": 4}


def _read_document(path):
    raw = open(path, "rb").read()
    bin_chunk = None
    if raw[:4] == b"glTF":
        total = struct.unpack_from("<I", raw, 8)[0]
        o, doc = 12, None
        while o + 8 <= total:
            ln, ty = struct.unpack_from("<II", raw, o)
            body = raw[o + 8:o + 8 + ln]
            if ty == 0x4E4F534A and doc is None:
                doc = json.loads(body.decode("utf-8"))
            elif ty == 0x004E4942 and bin_chunk is None:
                bin_chunk = body
            o += 8 + ((ln + 3) & ~3)
    else:
        doc = json.loads(raw.decode("utf-8"))
    base = os.path.dirname(path)
    buffers = []
    for b, B in enumerate(doc.get("buffers", [])):
        uri = B.get("uri")
        if uri is None:
            data = bin_chunk
        elif uri.startswith("data:"):
            data = base64.b64decode(uri[uri.index(",") + 1:])
        else:
            data = open(os.path.join(base, unquote(uri)), "rb").read()
        buffers.append(data[:B["byteLength"]])
    return doc, buffers


def _accessor(doc, buffers, idx):   # accessor_data (GltfLoader.cpp:64-75), packed elements
    acc = doc["accessors"][idx]
    bv = doc["bufferViews"][acc["bufferView"]]
    dt, size = _CT[acc["componentType"]]
    n = _NC[acc["type"]]
    start = bv.get("byteOffset", 0) + acc.get("byteOffset", 0)
    a = np.frombuffer(buffers[bv["buffer"]], dtype=dt, count=acc["count"] * n, offset=start)
    return a.reshape(acc["count"], n) if n > 1 else a


def load(path):
    """Returns dict(vertices (N, 12) float32 [pos, normal, uv, tangent], indices uint32,
    meshes (M, 5) uint32 [vertex_base, vertex_count, index_byte_offset, index_count, material],
    materials (K, 10) float32 [base rgba, metallic, roughness, emissive rgb, ior],
    transforms (I, 16) float32 row-major, mesh_index (I,) uint32)."""
    doc, buffers = _read_document(path)
    materials = []
    for m in doc.get("materials", []):   # GltfLoader.cpp:101-155
        pbr = m.get("pbrMetallicRoughness", {})
        bc = pbr.get("baseColorFactor", [1.0, 1.0, 1.0, 1.0])
        em = m.get("emissiveFactor", [0.0, 0.0, 0.0])
        materials.append([f32(float(c)) for c in bc] + [f32(float(pbr.get("metallicFactor", 1.0))),
                                                        f32(float(pbr.get("roughnessFactor", 1.0)))]
                         + [f32(float(c)) for c in em] + [f32(1.5)])
    verts, idx, meshes = [], [], []
    prim_mesh = []
    need_default = False
    for mesh in doc.get("meshes", []):   # GltfLoader.cpp:201-326
        ids = []
        for prim in mesh["primitives"]:
            ids.append(None)
            if prim.get("mode", 4) != 4 or "POSITION" not in prim["attributes"]:
                continue
            at = prim["attributes"]
            pos = _accessor(doc, buffers, at["POSITION"])
            n = len(pos)
            v = np.zeros((n, 12), np.float32)
            v[:, 0:3] = pos
            v[:, 3:6] = _accessor(doc, buffers, at["NORMAL"])[:n] if "NORMAL" in at else (0.0, 1.0, 0.0)
            if "TEXCOORD_0" in at:
                v[:, 6:8] = _accessor(doc, buffers, at["TEXCOORD_0"])[:n]
            v[:, 8:12] = _accessor(doc, buffers, at["TANGENT"])[:n] if "TANGENT" in at else (1.0, 0.0, 0.0, 1.0)
            ind = (_accessor(doc, buffers, prim["indices"]).astype(np.uint32) if "indices" in prim
                   else np.arange(n, dtype=np.uint32))
            mat = prim.get("material", -1)
            if mat < 0 and not materials:
                need_default = True
            vb = sum(len(a) for a in verts)
            ib = sum(len(a) for a in idx)
            ids[-1] = len(meshes)
            meshes.append([vb, n, ib * 4, len(ind), max(mat, 0)])
            verts.append(v)
            idx.append(ind)
        prim_mesh.append(ids)
    if need_default:   # Material{} (Scene.h:36-48)
        materials.append([f32(1.0)] * 4 + [f32(0.0), f32(1.0), f32(0.0), f32(0.0), f32(0.0), f32(1.5)])
    transforms, mesh_index = [], []

    def walk(ni, parent):   # GltfLoader.cpp:328-355
        node = doc["nodes"][ni]
        world = _mul(parent, _node_transform(node))
        if node.get("mesh", -1) >= 0:
            for gm in prim_mesh[node["mesh"]]:
                if gm is None:
                    continue
                transforms.append([world[c][r] for r in range(4) for c in range(4)])   # Scene.cpp:333-339
                mesh_index.append(gm)
        for ch in node.get("children", []):
            walk(ch, world)

    if doc.get("scenes"):
        scene = doc["scenes"][doc.get("scene", 0) if doc.get("scene", -1) >= 0 else 0]
        for r in scene.get("nodes", []):
            walk(r, _identity())
    return dict(vertices=np.concatenate(verts) if verts else np.zeros((0, 12), np.float32),
                indices=np.concatenate(idx) if idx else np.zeros(0, np.uint32),
                meshes=np.array(meshes, np.uint32).reshape(-1, 5),
                materials=np.array(materials, np.float32).reshape(-1, 10),
                transforms=np.array(transforms, np.float32).reshape(-1, 16),
                mesh_index=np.array(mesh_index, np.uint32))
