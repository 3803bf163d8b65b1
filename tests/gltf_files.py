"""Writers of small glTF 2.0 test scenes (.gltf with embedded or external
buffers, .glb) from numpy arrays, seeded. Used by the glTF loader tests."""
import base64
import json
import math
import struct

import numpy as np


class Builder:
    def __init__(self):
        self.doc = {"asset": {"version": "2.0", "generator": "research_b200 tests"},
                    "buffers": [], "bufferViews": [], "accessors": [], "meshes": [], "materials": [],
                    "nodes": [], "scenes": []}
        self.blob = bytearray()

    def view(self, data: bytes, stride=None) -> int:
        while len(self.blob) % 4:
            self.blob.append(0)
        bv = {"buffer": 0, "byteOffset": len(self.blob), "byteLength": len(data)}
        if stride:
            bv["byteStride"] = stride
        self.blob += data
        self.doc["bufferViews"].append(bv)
        return len(self.doc["bufferViews"]) - 1

    def accessor(self, arr, type_, ctype=None, view=None, offset=0, count=None) -> int:
        arr = np.ascontiguousarray(arr)
        if ctype is None:
            ctype = {np.dtype("<f4"): 5126, np.dtype("<u4"): 5125, np.dtype("<u2"): 5123,
                     np.dtype("u1"): 5121}[arr.dtype]
        if view is None:
            view = self.view(arr.tobytes())
        acc = {"bufferView": view, "componentType": ctype, "type": type_,
               "count": int(count if count is not None else arr.shape[0])}
        if offset:
            acc["byteOffset"] = offset
        self.doc["accessors"].append(acc)
        return len(self.doc["accessors"]) - 1

    def save(self, path, mode="embedded", bin_name="scene data.bin"):
        doc = json.loads(json.dumps(self.doc))
        blob = bytes(self.blob)
        if mode == "embedded":
            doc["buffers"] = [{"byteLength": len(blob), "uri": "data:application/octet-stream;base64,"
                               + base64.b64encode(blob).decode()}]
            open(path, "w").write(json.dumps(doc, indent=1))
        elif mode == "external":
            doc["buffers"] = [{"byteLength": len(blob), "uri": bin_name.replace(" ", "%20")}]
            open(path, "w").write(json.dumps(doc))
            open(str(path).rsplit("/", 1)[0] + "/" + bin_name, "wb").write(blob)
        elif mode == "glb":
            doc["buffers"] = [{"byteLength": len(blob)}]
            j = json.dumps(doc).encode()
            j += b" " * ((4 - len(j) % 4) % 4)
            b = blob + b"\0" * ((4 - len(blob) % 4) % 4)
            out = struct.pack("<III", 0x46546C67, 2, 12 + 8 + len(j) + 8 + len(b))
            out += struct.pack("<II", len(j), 0x4E4F534A) + j + struct.pack("<II", len(b), 0x004E4942) + b
            open(path, "wb").write(out)
        else:
            raise ValueError(mode)


def _unit_quat(rng):
    q = rng.normal(size=4)
    return (q / np.linalg.norm(q)).tolist()


def feature_scene(seed=1) -> Builder:
    """Materials with full, partial and absent factors; a two-primitive mesh
    (TRIANGLES with u16 indices, normals and uv, and a skipped LINES one), a
    non-indexed mesh without normals but with tangents, a u8-indexed mesh
    without a material, a u32-indexed grid; a node tree with TRS, matrix and
    rotation-only nodes three levels deep; two scenes, the second the default."""
    rng = np.random.default_rng(seed)
    g = Builder()
    g.doc["materials"] = [
        {"pbrMetallicRoughness": {"baseColorFactor": [0.8, 0.2, 0.1, 1.0], "metallicFactor": 0.25,
                                  "roughnessFactor": 0.4}},
        {"emissiveFactor": [5.0, 4.0, 3.0], "pbrMetallicRoughness": {}},
        {},
        {"pbrMetallicRoughness": {"roughnessFactor": 0.05}, "emissiveFactor": [0.0, 0.0, 0.1]},
    ]
    # mesh 0: box-ish soup with u16 indices + a lines primitive
    p0 = rng.uniform(-1, 1, (24, 3)).astype("<f4")
    n0 = rng.normal(size=(24, 3)).astype("<f4")
    uv0 = rng.uniform(0, 1, (24, 2)).astype("<f4")
    i0 = rng.integers(0, 24, 36).astype("<u2")
    prim_a = {"attributes": {"POSITION": g.accessor(p0, "VEC3"), "NORMAL": g.accessor(n0, "VEC3"),
                             "TEXCOORD_0": g.accessor(uv0, "VEC2")},
              "indices": g.accessor(i0, "SCALAR"), "material": 0}
    prim_b = {"attributes": {"POSITION": g.accessor(p0[:4], "VEC3")}, "mode": 1, "material": 1}
    g.doc["meshes"].append({"name": "soup", "primitives": [prim_a, prim_b]})
    # mesh 1: non-indexed, tangents, no normals
    p1 = rng.uniform(-2, 2, (9, 3)).astype("<f4")
    t1 = rng.uniform(-1, 1, (9, 4)).astype("<f4")
    g.doc["meshes"].append({"primitives": [{"attributes": {"POSITION": g.accessor(p1, "VEC3"),
                                                           "TANGENT": g.accessor(t1, "VEC4")}, "material": 2}]})
    # mesh 2: u8 indices, no material; the accessor starts inside its view
    p2 = rng.uniform(-1, 1, (10, 3)).astype("<f4")
    n2 = rng.normal(size=(10, 3)).astype("<f4")
    pad = np.zeros((2, 3), "<f4")
    v2 = g.view(np.concatenate([pad, p2]).tobytes())
    i2 = rng.integers(0, 10, 12).astype("u1")
    g.doc["meshes"].append({"primitives": [{"attributes": {"POSITION": g.accessor(p2, "VEC3", view=v2, offset=24),
                                                           "NORMAL": g.accessor(n2, "VEC3")},
                                            "indices": g.accessor(i2, "SCALAR")}]})
    # mesh 3: a 5x5 grid with u32 indices, emissive material
    xs, zs = np.meshgrid(np.linspace(-1, 1, 5), np.linspace(-1, 1, 5))
    p3 = np.stack([xs.ravel(), np.zeros(25), zs.ravel()], 1).astype("<f4")
    q = [(r * 5 + c, r * 5 + c + 5, r * 5 + c + 1) for r in range(4) for c in range(4)]
    q += [(r * 5 + c + 1, r * 5 + c + 5, r * 5 + c + 6) for r in range(4) for c in range(4)]
    i3 = np.array(q, "<u4").ravel()
    g.doc["meshes"].append({"primitives": [{"attributes": {"POSITION": g.accessor(p3, "VEC3")},
                                            "indices": g.accessor(i3, "SCALAR"), "material": 3}]})
    m = rng.uniform(-1, 1, 16)
    g.doc["nodes"] = [
        {"translation": [1.0, -2.0, 0.5], "rotation": _unit_quat(rng), "scale": [2.0, 1.0, 0.5],
         "children": [1, 3]},
        {"matrix": m.tolist(), "children": [2]},
        {"mesh": 0, "translation": [0.1, 0.2, 0.3]},
        {"mesh": 1, "rotation": _unit_quat(rng)},
        {"mesh": 2},
        {"mesh": 2, "scale": [-1.0, 1.0, 1.0], "children": [6]},
        {"mesh": 3, "translation": [0.0, 3.0, 0.0], "rotation": [0.0, 0.0, 0.0, 1.0]},
    ]
    g.doc["scenes"] = [{"nodes": [4]}, {"nodes": [0, 5]}]
    g.doc["scene"] = 1
    return g


def room_scene() -> Builder:
    """A closed box room (inward-facing quads) with an emissive ceiling patch
    and two blocks, for rendering: every triangle faces into the room."""
    g = Builder()
    g.doc["materials"] = [
        {"pbrMetallicRoughness": {"baseColorFactor": [0.73, 0.73, 0.73, 1.0], "metallicFactor": 0.0,
                                  "roughnessFactor": 0.8}},
        {"pbrMetallicRoughness": {"baseColorFactor": [0.65, 0.05, 0.05, 1.0], "metallicFactor": 0.0}},
        {"pbrMetallicRoughness": {"baseColorFactor": [0.9, 0.8, 0.6, 1.0], "metallicFactor": 1.0,
                                  "roughnessFactor": 0.3}},
        {"emissiveFactor": [17.0, 12.0, 4.0], "pbrMetallicRoughness": {"baseColorFactor": [0, 0, 0, 1]}},
    ]

    def quad(a, b, c, d, n):
        p = np.array([a, b, c, d], "<f4")
        return p, np.tile(np.array(n, "<f4"), (4, 1))

    def mesh(quads, mat):
        P = np.concatenate([q[0] for q in quads])
        N = np.concatenate([q[1] for q in quads])
        idx = np.concatenate([np.array([0, 1, 2, 0, 2, 3], "<u2") + 4 * k for k in range(len(quads))])
        g.doc["meshes"].append({"primitives": [{"attributes": {"POSITION": g.accessor(P, "VEC3"),
                                                               "NORMAL": g.accessor(N, "VEC3")},
                                                "indices": g.accessor(idx.astype("<u2"), "SCALAR"),
                                                "material": mat}]})
        return len(g.doc["meshes"]) - 1

    walls = mesh([quad((-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1), (0, 0, 1)),      # back
                  quad((-1, -1, 1), (1, -1, 1), (1, -1, -1), (-1, -1, -1), (0, 1, 0)),      # floor
                  quad((-1, 1, -1), (1, 1, -1), (1, 1, 1), (-1, 1, 1), (0, -1, 0)),         # ceiling
                  quad((1, -1, 1), (1, -1, -1), (1, 1, -1), (1, 1, 1), (-1, 0, 0))], 0)     # right
    red = mesh([quad((-1, -1, -1), (-1, -1, 1), (-1, 1, 1), (-1, 1, -1), (1, 0, 0))], 1)  # left
    light = mesh([quad((-0.3, 0.99, -0.3), (0.3, 0.99, -0.3), (0.3, 0.99, 0.3), (-0.3, 0.99, 0.3), (0, -1, 0))], 3)
    b = 0.5
    A, B_, C_, D = (-b, -b, -b), (b, -b, -b), (b, -b, b), (-b, -b, b)
    E, F, G, H = (-b, b, -b), (b, b, -b), (b, b, b), (-b, b, b)
    block = mesh([quad(E, F, G, H, (0, 1, 0)), quad(D, H, G, C_, (0, 0, 1)), quad(B_, F, E, A, (0, 0, -1)),
                  quad(A, E, H, D, (-1, 0, 0)), quad(C_, G, F, B_, (1, 0, 0))], 2)
    c15 = math.cos(math.radians(15.0))
    s15 = math.sin(math.radians(15.0))
    g.doc["nodes"] = [{"mesh": walls}, {"mesh": red}, {"mesh": light},
                      {"mesh": block, "translation": [-0.35, -0.6, -0.3], "scale": [0.6, 0.8, 0.6],
                       "rotation": [0.0, s15, 0.0, c15]},
                      {"children": [5], "translation": [0.4, -0.8, 0.3]},
                      {"mesh": block, "scale": [0.4, 0.4, 0.4]}]
    g.doc["scenes"] = [{"nodes": [0, 1, 2, 3, 4]}]
    return g
