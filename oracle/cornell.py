"""Independent numpy restatement of Scene::build_cornell_box (Scene.cpp:144-251)
and Camera::rebuild_matrices (Camera.cpp:120-145), used only to check the
library's host-side factories. TEST INFRASTRUCTURE ONLY.
"""
import math

import numpy as np

# (name, corners a,b,c,d, normal, material) — Scene.cpp:176-219
WALLS = [
    ("back_wall", [(-1, -1, -1), (1, -1, -1), (1, 1, -1), (-1, 1, -1)], (0, 0, 1), 0),
    ("floor", [(-1, -1, 1), (1, -1, 1), (1, -1, -1), (-1, -1, -1)], (0, 1, 0), 0),
    ("ceiling", [(-1, 1, -1), (1, 1, -1), (1, 1, 1), (-1, 1, 1)], (0, -1, 0), 0),
    ("left_wall", [(-1, -1, -1), (-1, -1, 1), (-1, 1, 1), (-1, 1, -1)], (1, 0, 0), 1),
    ("right_wall", [(1, -1, 1), (1, -1, -1), (1, 1, -1), (1, 1, 1)], (-1, 0, 0), 2),
    ("ceiling_light", [(-0.25, 0.999, -0.25), (0.25, 0.999, -0.25), (0.25, 0.999, 0.25), (-0.25, 0.999, 0.25)],
     (0, -1, 0), 3),
]
# Scene.cpp:151-174
MATERIALS = [((0.73, 0.73, 0.73), (0, 0, 0)), ((0.65, 0.05, 0.05), (0, 0, 0)), ((0.12, 0.45, 0.15), (0, 0, 0)),
             ((1.0, 1.0, 1.0), (15.0, 15.0, 15.0))]


def box_quads(mn, mx):
    """Scene.cpp:121-141"""
    a = (mn[0], mn[1], mn[2]); b = (mx[0], mn[1], mn[2]); c = (mx[0], mn[1], mx[2]); d = (mn[0], mn[1], mx[2])
    e = (mn[0], mx[1], mn[2]); f = (mx[0], mx[1], mn[2]); g = (mx[0], mx[1], mx[2]); h = (mn[0], mx[1], mx[2])
    return [([d, c, b, a], (0, -1, 0)), ([e, f, g, h], (0, 1, 0)), ([d, h, g, c], (0, 0, 1)),
            ([b, f, e, a], (0, 0, -1)), ([a, e, h, d], (-1, 0, 0)), ([c, g, f, b], (1, 0, 0))]


def rot_y(t, deg):
    a = np.float32(deg) * np.float32(math.pi / 180.0)
    c, s = np.float32(math.cos(a)), np.float32(math.sin(a))
    m = np.eye(4, dtype=np.float32)
    m[0, 0], m[0, 2], m[2, 0], m[2, 2] = c, s, -s, c
    m[:3, 3] = t
    return m


def cornell_triangles():
    """World-space triangles (n, 3, 3) in instance order with their material."""
    tris, mats = [], []
    for _, q, _, mat in WALLS:
        q = np.array(q, np.float32)
        for t in ((0, 1, 2), (0, 2, 3)):
            tris.append(q[list(t)]); mats.append(mat)
    for mn, mx, t, deg in [((-0.25, -1.0, -0.25), (0.25, -0.5, 0.25), (0.35, 0.0, -0.35), 18.0),
                           ((-0.25, -1.0, -0.25), (0.25, 0.0, 0.25), (-0.35, 0.0, -0.2), -15.0)]:
        M = rot_y(np.array(t, np.float32), deg)
        for q, _ in box_quads(mn, mx):
            q = np.array(q, np.float32)
            qw = (M[:3, :3] @ q.T).T + M[:3, 3]
            for tt in ((0, 1, 2), (0, 2, 3)):
                tris.append(qw[list(tt)]); mats.append(0)
    return np.array(tris, np.float32), np.array(mats)


def camera_forward(yaw_deg, pitch_deg):
    y, p = math.radians(yaw_deg), math.radians(pitch_deg)
    v = np.array([math.cos(p) * math.cos(y), math.sin(p), math.cos(p) * math.sin(y)])
    return v / np.linalg.norm(v)


def camera_matrices(pos, yaw_deg, pitch_deg, fov_deg, aspect, near, far):
    """view, proj (with Vulkan Y flip), row-major float64."""
    f = camera_forward(yaw_deg, pitch_deg)
    r = np.cross(f, [0, 1, 0]); r /= np.linalg.norm(r)
    u = np.cross(r, f); u /= np.linalg.norm(u)
    s = np.cross(f, u); s /= np.linalg.norm(s)
    uu = np.cross(s, f)
    V = np.eye(4)
    V[0, :3], V[1, :3], V[2, :3] = s, uu, -f
    V[0, 3], V[1, 3], V[2, 3] = -s @ pos, -uu @ pos, f @ pos
    th = math.tan(math.radians(fov_deg) / 2)
    Pm = np.zeros((4, 4))
    Pm[0, 0] = 1 / (aspect * th); Pm[1, 1] = -1 / th
    Pm[2, 2] = -(far + near) / (far - near); Pm[2, 3] = -(2 * far * near) / (far - near); Pm[3, 2] = -1
    return V, Pm
