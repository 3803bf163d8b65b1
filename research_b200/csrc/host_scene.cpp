// host_scene.cpp — scene factories and camera math (rr_host.h).
//
// Cornell box: restates Scene::build_cornell_box (Scene.cpp:144-251) with
// its add_quad / add_box helpers (Scene.cpp:94-141): quads are two triangles
// (0,1,2), (0,2,3) with one flat normal, tangent (1,0,0,1), uv corners
// (0,0),(1,0),(1,1),(0,1); transforms are row-major (Scene.cpp:87-90).
// Camera: restates Camera::forward / rebuild_matrices (Camera.cpp:120-145),
// glm::lookAt and glm::perspective (right-handed, depth -1..1, then the
// Vulkan Y flip proj[1][1] *= -1); inverses are evaluated in closed form in
// double precision and rounded to binary32.

#include "rr_host_internal.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

namespace {

struct F3 { float x, y, z; };
inline F3 f3(float x, float y, float z) { return F3{x, y, z}; }
inline F3 add(F3 a, F3 b) { return f3(a.x + b.x, a.y + b.y, a.z + b.z); }
inline F3 sub(F3 a, F3 b) { return f3(a.x - b.x, a.y - b.y, a.z - b.z); }
inline F3 scl(F3 a, float s) { return f3(a.x * s, a.y * s, a.z * s); }
inline float dot3(F3 a, F3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline F3 cross3(F3 a, F3 b) { return f3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
inline F3 norm3(F3 a) { float l = std::sqrt(dot3(a, a)); return l > 0 ? scl(a, 1.0f / l) : a; }

void identity(float* m) { for (int i = 0; i < 16; ++i) m[i] = (i % 5 == 0) ? 1.0f : 0.0f; }

GpuMaterial make_material(F3 base, float metallic, float roughness, F3 emissive) {
    GpuMaterial m{};
    m.base_color[0] = base.x; m.base_color[1] = base.y; m.base_color[2] = base.z; m.base_color[3] = 1.0f;
    m.metallic = metallic; m.roughness = roughness;
    m.emissive[0] = emissive.x; m.emissive[1] = emissive.y; m.emissive[2] = emissive.z;
    m.ior = 1.5f;  // Scene.h:43
    m.albedo_tex_idx = m.normal_tex_idx = m.metallic_roughness_tex_idx = m.emissive_tex_idx = 0xffffffffu;
    m.sampler_idx = 0;
    return m;
}

GpuVertex make_vertex(F3 p, F3 n, float u, float v) {
    GpuVertex gv{};
    gv.pos[0] = p.x; gv.pos[1] = p.y; gv.pos[2] = p.z;
    gv.normal[0] = n.x; gv.normal[1] = n.y; gv.normal[2] = n.z;
    gv.uv[0] = u; gv.uv[1] = v;
    gv.tangent[0] = 1; gv.tangent[1] = 0; gv.tangent[2] = 0; gv.tangent[3] = 1;
    return gv;
}

// Scene::add_mesh (Scene.cpp:32-50) followed by add_instance.
uint32_t add_mesh(rr_host_scene& s, const std::vector<GpuVertex>& v, const std::vector<uint32_t>& idx,
                  uint32_t material, const float* transform /*row-major, nullable*/) {
    GpuMesh m{};
    m.vertex_base = uint32_t(s.vertices.size());
    m.vertex_count = uint32_t(v.size());
    m.index_byte_offset = uint32_t(s.indices.size() * 4);
    m.index_count = uint32_t(idx.size());
    m.material_index = material;
    s.vertices.insert(s.vertices.end(), v.begin(), v.end());
    s.indices.insert(s.indices.end(), idx.begin(), idx.end());
    const uint32_t mesh_idx = uint32_t(s.meshes.size());
    s.meshes.push_back(m);
    GpuInstance inst{};
    if (transform) std::memcpy(inst.transform, transform, 64); else identity(inst.transform);
    inst.mesh_index = mesh_idx;
    s.instances.push_back(inst);
    return mesh_idx;
}

// Scene.cpp:94-118
void add_quad(std::vector<GpuVertex>& v, std::vector<uint32_t>& idx, F3 a, F3 b, F3 c, F3 d, F3 n) {
    const uint32_t base = uint32_t(v.size());
    v.push_back(make_vertex(a, n, 0, 0));
    v.push_back(make_vertex(b, n, 1, 0));
    v.push_back(make_vertex(c, n, 1, 1));
    v.push_back(make_vertex(d, n, 0, 1));
    for (uint32_t k : {0u, 1u, 2u, 0u, 2u, 3u}) idx.push_back(base + k);
}

// Scene.cpp:121-141
void add_box(std::vector<GpuVertex>& v, std::vector<uint32_t>& idx, F3 mn, F3 mx) {
    F3 a{mn.x, mn.y, mn.z}, b{mx.x, mn.y, mn.z}, c{mx.x, mn.y, mx.z}, d{mn.x, mn.y, mx.z};
    F3 e{mn.x, mx.y, mn.z}, f{mx.x, mx.y, mn.z}, g{mx.x, mx.y, mx.z}, h{mn.x, mx.y, mx.z};
    add_quad(v, idx, d, c, b, a, f3(0, -1, 0));
    add_quad(v, idx, e, f, g, h, f3(0, 1, 0));
    add_quad(v, idx, d, h, g, c, f3(0, 0, 1));
    add_quad(v, idx, b, f, e, a, f3(0, 0, -1));
    add_quad(v, idx, a, e, h, d, f3(-1, 0, 0));
    add_quad(v, idx, c, g, f, b, f3(1, 0, 0));
}

// glm::translate(I, t) * glm::rotate(I, radians(deg), (0,1,0)), row-major.
void translate_rotate_y(float* m, F3 t, float deg) {
    const float a = deg * 0.01745329251994329576923690768489f;  // glm::radians
    const float c = std::cos(a), s = std::sin(a);
    const float one_minus_c = 1.0f - c;
    identity(m);
    m[0] = c;                  m[2] = s;  m[3] = t.x;
    m[5] = c + one_minus_c;               m[7] = t.y;
    m[8] = -s;                 m[10] = c; m[11] = t.z;
}

// ── deterministic host RNG (splitmix64) and value noise ───────────────────
struct Rng {
    uint64_t s;
    uint64_t next() {
        uint64_t z = (s += 0x9e3779b97f4a7c15ull);
        z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
        z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
        return z ^ (z >> 31);
    }
    float uni() { return float(next() >> 40) * (1.0f / 16777216.0f); }
    float uni(float a, float b) { return a + (b - a) * uni(); }
};

inline float lattice(int x, int y, int z, uint32_t seed) {
    uint32_t h = uint32_t(x) * 0x8da6b343u ^ uint32_t(y) * 0xd8163841u ^ uint32_t(z) * 0xcb1ab31fu ^ seed * 0x9e3779b9u;
    h ^= h >> 15; h *= 0x2c1b3c6du; h ^= h >> 12; h *= 0x297a2d39u; h ^= h >> 15;
    return float(h >> 8) * (2.0f / 16777216.0f) - 1.0f;
}
inline float smooth(float t) { return t * t * (3.0f - 2.0f * t); }
float value_noise(float x, float y, float z, uint32_t seed) {
    const float fx = std::floor(x), fy = std::floor(y), fz = std::floor(z);
    const int ix = int(fx), iy = int(fy), iz = int(fz);
    const float tx = smooth(x - fx), ty = smooth(y - fy), tz = smooth(z - fz);
    float c[2][2][2];
    for (int a = 0; a < 2; ++a) for (int b = 0; b < 2; ++b) for (int d = 0; d < 2; ++d)
        c[a][b][d] = lattice(ix + a, iy + b, iz + d, seed);
    auto lerpf = [](float a, float b, float t) { return a + (b - a) * t; };
    const float x00 = lerpf(c[0][0][0], c[1][0][0], tx), x10 = lerpf(c[0][1][0], c[1][1][0], tx);
    const float x01 = lerpf(c[0][0][1], c[1][0][1], tx), x11 = lerpf(c[0][1][1], c[1][1][1], tx);
    return lerpf(lerpf(x00, x10, ty), lerpf(x01, x11, ty), tz);
}
float fbm(float x, float y, float z, uint32_t seed, int octaves) {
    float sum = 0.0f, amp = 0.5f, f = 1.0f;
    for (int o = 0; o < octaves; ++o) { sum += amp * value_noise(x * f, y * f, z * f, seed + uint32_t(o)); amp *= 0.5f; f *= 2.0f; }
    return sum;
}

void smooth_normals(std::vector<GpuVertex>& v, const std::vector<uint32_t>& idx) {
    std::vector<F3> acc(v.size(), f3(0, 0, 0));
    for (size_t t = 0; t + 2 < idx.size(); t += 3) {
        const GpuVertex &a = v[idx[t]], &b = v[idx[t + 1]], &c = v[idx[t + 2]];
        const F3 pa = f3(a.pos[0], a.pos[1], a.pos[2]), pb = f3(b.pos[0], b.pos[1], b.pos[2]), pc = f3(c.pos[0], c.pos[1], c.pos[2]);
        const F3 n = cross3(sub(pb, pa), sub(pc, pa));
        for (int k = 0; k < 3; ++k) acc[idx[t + k]] = add(acc[idx[t + k]], n);
    }
    for (size_t i = 0; i < v.size(); ++i) {
        F3 n = norm3(acc[i]);
        if (!(dot3(n, n) > 0.5f)) n = f3(0, 1, 0);
        v[i].normal[0] = n.x; v[i].normal[1] = n.y; v[i].normal[2] = n.z;
    }
}

// Unit icosphere with `subdiv` midpoint subdivisions.
void icosphere(int subdiv, std::vector<F3>& pts, std::vector<uint32_t>& idx) {
    const float t = (1.0f + std::sqrt(5.0f)) * 0.5f;
    pts = {f3(-1, t, 0), f3(1, t, 0), f3(-1, -t, 0), f3(1, -t, 0), f3(0, -1, t), f3(0, 1, t),
           f3(0, -1, -t), f3(0, 1, -t), f3(t, 0, -1), f3(t, 0, 1), f3(-t, 0, -1), f3(-t, 0, 1)};
    for (auto& p : pts) p = norm3(p);
    idx = {0, 11, 5, 0, 5, 1, 0, 1, 7, 0, 7, 10, 0, 10, 11, 1, 5, 9, 5, 11, 4, 11, 10, 2, 10, 7, 6, 7, 1, 8,
           3, 9, 4, 3, 4, 2, 3, 2, 6, 3, 6, 8, 3, 8, 9, 4, 9, 5, 2, 4, 11, 6, 2, 10, 8, 6, 7, 9, 8, 1};
    for (int s = 0; s < subdiv; ++s) {
        std::vector<uint32_t> out;
        out.reserve(idx.size() * 4);
        std::vector<std::pair<uint64_t, uint32_t>> cache;
        cache.reserve(idx.size() * 3 / 2);
        // midpoint lookup via sorted edge keys
        std::vector<uint64_t> keys;
        keys.reserve(idx.size());
        for (size_t k = 0; k < idx.size(); k += 3)
            for (int e = 0; e < 3; ++e) {
                uint32_t a = idx[k + e], b = idx[k + (e + 1) % 3];
                if (a > b) std::swap(a, b);
                keys.push_back((uint64_t(a) << 32) | b);
            }
        std::sort(keys.begin(), keys.end());
        keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
        const uint32_t base = uint32_t(pts.size());
        for (uint64_t key : keys) {
            const F3 a = pts[key >> 32], b = pts[key & 0xffffffffu];
            pts.push_back(norm3(scl(add(a, b), 0.5f)));
        }
        auto mid = [&](uint32_t a, uint32_t b) {
            if (a > b) std::swap(a, b);
            const uint64_t key = (uint64_t(a) << 32) | b;
            return base + uint32_t(std::lower_bound(keys.begin(), keys.end(), key) - keys.begin());
        };
        for (size_t k = 0; k < idx.size(); k += 3) {
            const uint32_t a = idx[k], b = idx[k + 1], c = idx[k + 2];
            const uint32_t ab = mid(a, b), bc = mid(b, c), ca = mid(c, a);
            for (uint32_t q : {a, ab, ca, b, bc, ab, c, ca, bc, ab, bc, ca}) out.push_back(q);
        }
        idx.swap(out);
    }
}

// One single-triangle emitter mesh + material (+ a point light at it when
// point_light: the same geometry and random draws either way).
void add_emitter(rr_host_scene& s, Rng& rng, float box_half, float size_lo, float size_hi, bool point_light) {
    const F3 c = f3(rng.uni(-box_half, box_half), rng.uni(-box_half, box_half), rng.uni(-box_half, box_half));
    F3 n = norm3(f3(rng.uni(-1, 1), rng.uni(-1, 1), rng.uni(-1, 1)));
    if (!(dot3(n, n) > 0.5f)) n = f3(0, -1, 0);
    const F3 up = std::fabs(n.x) < 0.9f ? f3(1, 0, 0) : f3(0, 1, 0);
    const F3 t = norm3(cross3(up, n)), b = cross3(n, t);
    const float size = rng.uni(size_lo, size_hi);
    const float phase = rng.uni(0.0f, 6.2831853f);
    std::vector<GpuVertex> v;
    for (int k = 0; k < 3; ++k) {
        const float a = phase + float(k) * 2.0943951f;
        const F3 p = add(c, add(scl(t, size * std::cos(a)), scl(b, size * std::sin(a))));
        v.push_back(make_vertex(p, n, 0, 0));
    }
    // counter-clockwise around n
    std::vector<uint32_t> idx = {0, 1, 2};
    const F3 e = cross3(sub(f3(v[1].pos[0], v[1].pos[1], v[1].pos[2]), f3(v[0].pos[0], v[0].pos[1], v[0].pos[2])),
                        sub(f3(v[2].pos[0], v[2].pos[1], v[2].pos[2]), f3(v[0].pos[0], v[0].pos[1], v[0].pos[2])));
    if (dot3(e, n) < 0) std::swap(idx[1], idx[2]);
    // radiance log-uniform in [0.1, 100] with a mild tint
    const float L = 0.1f * std::pow(1000.0f, rng.uni());
    const F3 emit = f3(L * rng.uni(0.6f, 1.0f), L * rng.uni(0.6f, 1.0f), L * rng.uni(0.6f, 1.0f));
    const uint32_t mat = uint32_t(s.materials.size());
    s.materials.push_back(make_material(f3(1, 1, 1), 0.0f, 1.0f, emit));
    add_mesh(s, v, idx, mat, nullptr);
    if (!point_light) return;
    const float area = 0.5f * std::sqrt(dot3(e, e));
    GpuLight l{};
    const F3 lp = add(c, scl(n, 0.05f));
    l.position[0] = lp.x; l.position[1] = lp.y; l.position[2] = lp.z;
    l.type = 0;
    l.direction[0] = 0; l.direction[1] = -1; l.direction[2] = 0;
    l.emission[0] = emit.x; l.emission[1] = emit.y; l.emission[2] = emit.z;
    l.intensity = area;
    s.lights.push_back(l);
}

GpuMaterial random_material(Rng& rng) {
    const float rough = rng.uni(0.05f, 1.0f);
    const float metal = rng.uni() < 0.3f ? 1.0f : 0.0f;
    const F3 base = f3(rng.uni(0.05f, 0.95f), rng.uni(0.05f, 0.95f), rng.uni(0.05f, 0.95f));
    return make_material(base, metal, rough, f3(0, 0, 0));
}

// ── camera (Camera.cpp) ────────────────────────────────────────────────────
void copy_rowmajor(float* dst, const double m[4][4]) {
    for (int r = 0; r < 4; ++r) for (int c = 0; c < 4; ++c) dst[r * 4 + c] = float(m[r][c]);
}

struct CamMats { double view[4][4], inv_view[4][4], proj[4][4], inv_proj[4][4]; F3 fwd; };

CamMats camera_matrices(const rr_camera_desc& c) {
    CamMats M{};
    // Camera::forward (Camera.cpp:120-128), float like glm
    const float yaw = c.yaw_deg * 0.01745329251994329576923690768489f;
    const float pitch = c.pitch_deg * 0.01745329251994329576923690768489f;
    const F3 fwd = norm3(f3(std::cos(pitch) * std::cos(yaw), std::sin(pitch), std::cos(pitch) * std::sin(yaw)));
    M.fwd = fwd;
    F3 right = norm3(cross3(fwd, f3(0, 1, 0)));
    if (std::sqrt(dot3(right, right)) < 1e-5f) right = f3(1, 0, 0);
    const F3 up = norm3(cross3(right, fwd));
    // glm::lookAt(eye, eye + fwd, up), right-handed
    const F3 eye = f3(c.position[0], c.position[1], c.position[2]);
    const F3 center = add(eye, fwd);
    const F3 f = norm3(sub(center, eye));
    const F3 s = norm3(cross3(f, up));
    const F3 u = cross3(s, f);
    const double V[4][4] = {{s.x, s.y, s.z, -double(dot3(s, eye))},
                            {u.x, u.y, u.z, -double(dot3(u, eye))},
                            {-f.x, -f.y, -f.z, double(dot3(f, eye))},
                            {0, 0, 0, 1}};
    std::memcpy(M.view, V, sizeof(V));
    // inverse of [R t; 0 1] = [R^T, -R^T t; 0 1]
    for (int r = 0; r < 3; ++r) {
        for (int k = 0; k < 3; ++k) M.inv_view[r][k] = V[k][r];
        M.inv_view[r][3] = -(V[0][r] * V[0][3] + V[1][r] * V[1][3] + V[2][r] * V[2][3]);
    }
    M.inv_view[3][0] = M.inv_view[3][1] = M.inv_view[3][2] = 0.0; M.inv_view[3][3] = 1.0;
    // glm::perspective RH, depth -1..1, then proj[1][1] *= -1 (Camera.cpp:140-142)
    const double aspect = double(c.width) / double(c.height ? c.height : 1);
    const double th = std::tan(double(c.fov_y_deg) * 3.14159265358979323846 / 360.0);
    const double n = c.near_plane, fa = c.far_plane;
    const double a = 1.0 / (aspect * th), b = -1.0 / th;
    const double cc = -(fa + n) / (fa - n), d = -(2.0 * fa * n) / (fa - n);
    const double P[4][4] = {{a, 0, 0, 0}, {0, b, 0, 0}, {0, 0, cc, d}, {0, 0, -1, 0}};
    std::memcpy(M.proj, P, sizeof(P));
    const double IP[4][4] = {{1.0 / a, 0, 0, 0}, {0, 1.0 / b, 0, 0}, {0, 0, 0, -1}, {0, 0, 1.0 / d, cc / d}};
    std::memcpy(M.inv_proj, IP, sizeof(IP));
    return M;
}

} // namespace

extern "C" {

rr_status rr_host_scene_cornell(int variant, rr_host_scene** out) {
    if (!out || (variant != 0 && variant != 1)) return RR_ERR_INVALID_ARGUMENT;
    rr_host_scene* s = new (std::nothrow) rr_host_scene;
    if (!s) return RR_ERR_OUT_OF_MEMORY;
    const uint32_t white = 0, red = 1, green = 2, light = 3;
    s->materials.push_back(make_material(f3(0.73f, 0.73f, 0.73f), 0.0f, 1.0f, f3(0, 0, 0)));
    s->materials.push_back(make_material(f3(0.65f, 0.05f, 0.05f), 0.0f, 1.0f, f3(0, 0, 0)));
    s->materials.push_back(make_material(f3(0.12f, 0.45f, 0.15f), 0.0f, 1.0f, f3(0, 0, 0)));
    s->materials.push_back(make_material(f3(1, 1, 1), 0.0f, 1.0f,
                                         variant == 0 ? f3(15.0f, 15.0f, 15.0f) : f3(17.0f, 12.0f, 4.0f)));
    auto quad_mesh = [&](F3 a, F3 b, F3 c, F3 d, F3 n, uint32_t mat) {
        std::vector<GpuVertex> v; std::vector<uint32_t> i;
        add_quad(v, i, a, b, c, d, n);
        add_mesh(*s, v, i, mat, nullptr);
    };
    quad_mesh(f3(-1, -1, -1), f3(1, -1, -1), f3(1, 1, -1), f3(-1, 1, -1), f3(0, 0, 1), white);   // back
    quad_mesh(f3(-1, -1, 1), f3(1, -1, 1), f3(1, -1, -1), f3(-1, -1, -1), f3(0, 1, 0), white);   // floor
    quad_mesh(f3(-1, 1, -1), f3(1, 1, -1), f3(1, 1, 1), f3(-1, 1, 1), f3(0, -1, 0), white);      // ceiling
    quad_mesh(f3(-1, -1, -1), f3(-1, -1, 1), f3(-1, 1, 1), f3(-1, 1, -1), f3(1, 0, 0), red);     // left
    quad_mesh(f3(1, -1, 1), f3(1, -1, -1), f3(1, 1, -1), f3(1, 1, 1), f3(-1, 0, 0), green);      // right
    quad_mesh(f3(-0.25f, 0.999f, -0.25f), f3(0.25f, 0.999f, -0.25f), f3(0.25f, 0.999f, 0.25f),
              f3(-0.25f, 0.999f, 0.25f), f3(0, -1, 0), light);                                   // area light
    {
        std::vector<GpuVertex> v; std::vector<uint32_t> i;
        add_box(v, i, f3(-0.25f, -1.0f, -0.25f), f3(0.25f, -0.5f, 0.25f));
        float m[16];
        translate_rotate_y(m, f3(0.35f, 0.0f, -0.35f), 18.0f);
        add_mesh(*s, v, i, white, m);                                                            // short box
    }
    {
        std::vector<GpuVertex> v; std::vector<uint32_t> i;
        add_box(v, i, f3(-0.25f, -1.0f, -0.25f), f3(0.25f, 0.0f, 0.25f));
        float m[16];
        translate_rotate_y(m, f3(-0.35f, 0.0f, -0.2f), -15.0f);
        add_mesh(*s, v, i, white, m);                                                            // tall box
    }
    GpuLight l{};
    l.position[0] = 0.0f; l.position[1] = 0.9f; l.position[2] = 0.0f;
    l.type = 0;
    l.direction[0] = 0; l.direction[1] = -1; l.direction[2] = 0;  // Scene.h:62 default
    l.radius = 0.0f;
    l.emission[0] = 15.0f; l.emission[1] = 15.0f; l.emission[2] = 12.0f;
    l.intensity = 1.0f;
    s->lights.push_back(l);
    *out = s;
    return RR_OK;
}

rr_status rr_host_scene_procedural(const rr_procedural_params* p, rr_host_scene** out) {
    if (!p || !out || p->target_triangles == 0 || !(p->box_half > 0.0f)) return RR_ERR_INVALID_ARGUMENT;
    rr_host_scene* s = new (std::nothrow) rr_host_scene;
    if (!s) return RR_ERR_OUT_OF_MEMORY;
    Rng rng{p->seed};
    const float H = p->box_half;
    uint64_t tris = 0;
    // An open-fronted room: a heightfield floor (256..512 vertices a side) and
    // three heightfield walls (128..256 a side), displaced by value noise.
    // Local grid (u, v) in [-H, H]^2 with height h; `frame` maps it to world.
    auto heightfield = [&](int G, int frame) {
        const uint32_t nseed = uint32_t(rng.next());
        std::vector<GpuVertex> v; std::vector<uint32_t> idx;
        v.reserve(size_t(G) * G);
        for (int j = 0; j < G; ++j)
            for (int i = 0; i < G; ++i) {
                const float u = -H + 2.0f * H * float(i) / float(G - 1);
                const float w = -H + 2.0f * H * float(j) / float(G - 1);
                const float h = 0.08f * H * fbm(u * 0.15f, 0.0f, w * 0.15f, nseed, 4);
                F3 q;
                switch (frame) {
                case 0: q = f3(u, -0.5f * H + h, w); break;  // floor
                case 1: q = f3(u, w, -H + h); break;         // back wall
                case 2: q = f3(-H + h, w, u); break;         // left wall
                default: q = f3(H - h, w, u); break;         // right wall
                }
                v.push_back(make_vertex(q, f3(0, 1, 0), float(i) / float(G - 1), float(j) / float(G - 1)));
            }
        for (int j = 0; j + 1 < G; ++j)
            for (int i = 0; i + 1 < G; ++i) {
                const uint32_t a = uint32_t(j * G + i), b = a + 1, c = a + uint32_t(G), d = c + 1;
                for (uint32_t q : {a, c, b, b, c, d}) idx.push_back(q);
            }
        smooth_normals(v, idx);
        const uint32_t mat = uint32_t(s->materials.size());
        s->materials.push_back(random_material(rng));
        tris += idx.size() / 3;
        add_mesh(*s, v, idx, mat, nullptr);
    };
    // Below 1M triangles the drawn grid sizes are capped (floor at 30 % of
    // the target, each wall at 7 %) so that small scenes keep the mix of
    // heightfields and icospheres; from 1M on the draws are used as they are.
    const bool small = p->target_triangles < 1000000u;
    auto capped = [&](int G, double share) {
        if (!small) return G;
        const double cap = share * double(p->target_triangles);
        if (2.0 * double(G - 1) * double(G - 1) <= cap) return G;
        return std::max(8, int(std::sqrt(cap / 2.0)) + 1);
    };
    heightfield(capped(256 + int(rng.next() % 257), 0.30), 0);
    for (int wall = 1; wall <= 3; ++wall) heightfield(capped(128 + int(rng.next() % 129), 0.07), wall);
    // displaced icospheres (subdivision 3..5) inside the room until the
    // triangle target is met
    std::vector<F3> base_pts[3];
    std::vector<uint32_t> base_idx[3];
    for (int k = 0; k < 3; ++k) icosphere(3 + k, base_pts[k], base_idx[k]);
    const uint64_t target = p->target_triangles > p->emissive_triangles ? p->target_triangles - p->emissive_triangles : 0;
    while (tris < target) {
        const int level = int(rng.next() % 3);
        const float scale = rng.uni(0.05f, 2.0f) * (H / 20.0f);
        const F3 c = f3(rng.uni(-0.9f * H, 0.9f * H), rng.uni(-0.45f * H, 0.6f * H), rng.uni(-0.9f * H, 0.9f * H));
        const uint32_t nseed = uint32_t(rng.next());
        const float amp = rng.uni(0.05f, 0.35f), freq = rng.uni(1.0f, 4.0f);
        std::vector<GpuVertex> v;
        v.reserve(base_pts[level].size());
        for (const F3& q : base_pts[level]) {
            const float disp = 1.0f + amp * fbm(q.x * freq, q.y * freq, q.z * freq, nseed, 3);
            v.push_back(make_vertex(add(c, scl(q, scale * disp)), q, 0, 0));
        }
        smooth_normals(v, base_idx[level]);
        const uint32_t mat = uint32_t(s->materials.size());
        s->materials.push_back(random_material(rng));
        tris += base_idx[level].size() / 3;
        add_mesh(*s, v, base_idx[level], mat, nullptr);
    }
    for (uint32_t e = 0; e < p->emissive_triangles; ++e) add_emitter(*s, rng, 0.9f * H, 0.004f * H, 0.015f * H,
                                                                  (p->flags & RR_SCENE_NO_EMITTER_LIGHTS) == 0);
    *out = s;
    return RR_OK;
}

rr_status rr_host_scene_instanced(const rr_instanced_params* p, rr_host_scene** out) {
    if (!p || !out || p->base_meshes == 0 || p->instance_count == 0 || p->tris_per_mesh < 8 || !(p->box_half > 0.0f))
        return RR_ERR_INVALID_ARGUMENT;
    rr_host_scene* s = new (std::nothrow) rr_host_scene;
    if (!s) return RR_ERR_OUT_OF_MEMORY;
    Rng rng{p->seed};
    // base meshes: noise-displaced tori on an Nu x Nv periodic grid
    const uint32_t quads = std::max(4u, p->tris_per_mesh / 2);
    // largest divisor of the quad count not above sqrt(quads / 2), so that the
    // Nu x Nv grid has exactly tris_per_mesh / 2 quads when possible
    uint32_t nv = std::max(1u, uint32_t(std::sqrt(double(quads) / 2.0)));
    while (nv > 1 && quads % nv != 0) --nv;
    if (nv < 2) nv = 2;
    const uint32_t nu = std::max(2u, quads / nv);
    std::vector<uint32_t> mesh_ids;
    for (uint32_t m = 0; m < p->base_meshes; ++m) {
        const float R = 1.0f, r = rng.uni(0.25f, 0.5f);
        const uint32_t nseed = uint32_t(rng.next());
        std::vector<GpuVertex> v; std::vector<uint32_t> idx;
        for (uint32_t j = 0; j < nv; ++j)
            for (uint32_t i = 0; i < nu; ++i) {
                const float u = 6.2831853f * float(i) / float(nu), w = 6.2831853f * float(j) / float(nv);
                const F3 dir = f3(std::cos(u), 0.0f, std::sin(u));
                const F3 q = f3(std::cos(u) * std::cos(w), std::sin(w), std::sin(u) * std::cos(w));
                const float rr = r * (1.0f + 0.3f * fbm(q.x * 3.0f + u, q.y * 3.0f, q.z * 3.0f + w, nseed, 3));
                v.push_back(make_vertex(add(scl(dir, R), scl(q, rr)), q, float(i) / nu, float(j) / nv));
            }
        for (uint32_t j = 0; j < nv; ++j)
            for (uint32_t i = 0; i < nu; ++i) {
                const uint32_t a = j * nu + i, b = j * nu + (i + 1) % nu;
                const uint32_t c = ((j + 1) % nv) * nu + i, d = ((j + 1) % nv) * nu + (i + 1) % nu;
                for (uint32_t q : {a, c, b, b, c, d}) idx.push_back(q);
            }
        smooth_normals(v, idx);
        GpuMesh gm{};
        gm.vertex_base = uint32_t(s->vertices.size());
        gm.vertex_count = uint32_t(v.size());
        gm.index_byte_offset = uint32_t(s->indices.size() * 4);
        gm.index_count = uint32_t(idx.size());
        gm.material_index = uint32_t(s->materials.size());
        s->materials.push_back(random_material(rng));
        s->vertices.insert(s->vertices.end(), v.begin(), v.end());
        s->indices.insert(s->indices.end(), idx.begin(), idx.end());
        mesh_ids.push_back(uint32_t(s->meshes.size()));
        s->meshes.push_back(gm);
    }
    for (uint32_t k = 0; k < p->instance_count; ++k) {
        // random rotation from a unit quaternion, uniform scale, translation
        float q[4];
        float len2;
        do {
            for (float& x : q) x = rng.uni(-1.0f, 1.0f);
            len2 = q[0] * q[0] + q[1] * q[1] + q[2] * q[2] + q[3] * q[3];
        } while (len2 > 1.0f || len2 < 1e-4f);
        const float il = 1.0f / std::sqrt(len2);
        for (float& x : q) x *= il;
        const float w = q[0], x = q[1], y = q[2], z = q[3];
        const float sc = rng.uni(0.2f, 3.0f);
        const F3 t = f3(rng.uni(-p->box_half, p->box_half), rng.uni(-p->box_half, p->box_half), rng.uni(-p->box_half, p->box_half));
        GpuInstance inst{};
        const float Rm[9] = {1 - 2 * (y * y + z * z), 2 * (x * y - w * z), 2 * (x * z + w * y),
                             2 * (x * y + w * z), 1 - 2 * (x * x + z * z), 2 * (y * z - w * x),
                             2 * (x * z - w * y), 2 * (y * z + w * x), 1 - 2 * (x * x + y * y)};
        for (int r = 0; r < 3; ++r) {
            for (int c = 0; c < 3; ++c) inst.transform[r * 4 + c] = Rm[r * 3 + c] * sc;
        }
        inst.transform[3] = t.x; inst.transform[7] = t.y; inst.transform[11] = t.z;
        inst.transform[12] = inst.transform[13] = inst.transform[14] = 0.0f; inst.transform[15] = 1.0f;
        inst.mesh_index = mesh_ids[rng.next() % mesh_ids.size()];
        s->instances.push_back(inst);
    }
    for (uint32_t e = 0; e < p->emissive_triangles; ++e) add_emitter(*s, rng, p->box_half, 0.3f, 1.5f,
                                                                  (p->flags & RR_SCENE_NO_EMITTER_LIGHTS) == 0);
    *out = s;
    return RR_OK;
}

rr_status rr_host_scene_desc(const rr_host_scene* s, rr_scene_desc* d) {
    if (!s || !d) return RR_ERR_INVALID_ARGUMENT;
    d->vertices = s->vertices.data();   d->vertex_count = uint32_t(s->vertices.size());
    d->indices = s->indices.data();     d->index_count = uint32_t(s->indices.size());
    d->meshes = s->meshes.data();       d->mesh_count = uint32_t(s->meshes.size());
    d->materials = s->materials.data(); d->material_count = uint32_t(s->materials.size());
    d->instances = s->instances.data(); d->instance_count = uint32_t(s->instances.size());
    d->lights = s->lights.empty() ? nullptr : s->lights.data();
    d->light_count = uint32_t(s->lights.size());
    return RR_OK;
}

rr_status rr_host_scene_destroy(rr_host_scene* s) {
    if (!s) return RR_ERR_INVALID_ARGUMENT;
    delete s;
    return RR_OK;
}

rr_status rr_camera_default(uint32_t width, uint32_t height, rr_camera_desc* c) {
    if (!c) return RR_ERR_INVALID_ARGUMENT;
    std::memset(c, 0, sizeof(*c));
    c->position[0] = 0.0f; c->position[1] = 0.0f; c->position[2] = 3.0f;
    c->yaw_deg = -90.0f; c->pitch_deg = 0.0f;
    c->fov_y_deg = 45.0f; c->near_plane = 0.01f; c->far_plane = 1000.0f;
    c->width = width; c->height = height;
    return RR_OK;
}

rr_status rr_camera_look_at(rr_camera_desc* c, const float eye[3], const float center[3]) {
    if (!c || !eye || !center) return RR_ERR_INVALID_ARGUMENT;
    const F3 dir = norm3(f3(center[0] - eye[0], center[1] - eye[1], center[2] - eye[2]));
    c->position[0] = eye[0]; c->position[1] = eye[1]; c->position[2] = eye[2];
    c->pitch_deg = std::asin(dir.y) * 57.295779513082320876798154814105f;
    c->yaw_deg = std::atan2(dir.z, dir.x) * 57.295779513082320876798154814105f;
    return RR_OK;
}

rr_status rr_camera_build(const rr_camera_desc* c, const rr_camera_desc* prev, GpuCameraData* out) {
    if (!c || !out || c->width == 0 || c->height == 0) return RR_ERR_INVALID_ARGUMENT;
    const CamMats M = camera_matrices(*c);
    const CamMats P = prev ? camera_matrices(*prev) : M;
    std::memset(out, 0, sizeof(*out));
    copy_rowmajor(out->view, M.view);
    copy_rowmajor(out->inv_view, M.inv_view);
    copy_rowmajor(out->inv_proj, M.inv_proj);
    double vp[4][4];
    for (int r = 0; r < 4; ++r)
        for (int k = 0; k < 4; ++k) {
            double acc = 0.0;
            for (int j = 0; j < 4; ++j) acc += P.proj[r][j] * P.view[j][k];
            vp[r][k] = acc;
        }
    copy_rowmajor(out->prev_view_proj, vp);
    out->position[0] = c->position[0]; out->position[1] = c->position[1]; out->position[2] = c->position[2];
    out->near_plane = c->near_plane;
    out->direction[0] = M.fwd.x; out->direction[1] = M.fwd.y; out->direction[2] = M.fwd.z;
    out->far_plane = c->far_plane;
    out->frame_index = c->frame_index;
    out->screen_width = c->width;
    out->screen_height = c->height;
    return RR_OK;
}

} // extern "C"
