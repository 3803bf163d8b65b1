// gltf.cpp — glTF 2.0 scene loading (rr_host_scene_gltf), restating
// GltfLoader::load (GltfLoader.cpp:79-365) followed by the CPU side of
// Scene::upload (Scene.cpp:255-345), so that the arrays equal the GpuScene
// buffers the reference uploads for the same file:
//   - materials: pbrMetallicRoughness baseColorFactor / metallicFactor /
//     roughnessFactor and emissiveFactor with the glTF defaults (1,1,1,1),
//     1, 1, (0,0,0); ior 1.5; texture indices 0xFFFFFFFF and sampler 0, as
//     Scene::upload writes them (Scene.cpp:310-330);
//   - meshes: one GpuMesh per TRIANGLES primitive (other modes skipped),
//     POSITION required, NORMAL default (0,1,0), TEXCOORD_0 default (0,0),
//     TANGENT default (1,0,0,1); indices u8/u16/u32, or 0..n-1 when absent;
//     material -1 -> 0;
//   - instances: the default scene's node tree, world = parent * local,
//     local = node.matrix read as GltfLoader.cpp:36-42 reads it, else
//     T * R * S; one GpuInstance per primitive of a node's mesh, transform
//     stored row-major (Scene.cpp:333-339);
//   - no lights (the loader adds none) and no texture images (the path's
//     materials never sample them: Scene::upload binds none).
// The JSON reader, the .glb container and base64 data URIs are parsed here
// (the reference uses tinygltf). Differences, each a case the reference
// reads out of bounds or misreads: accessors honour byteStride and reject
// non-float vertex attributes and sparse accessors; every index is checked;
// a file without materials gets one default Material (Scene.h:36-48) for
// primitives without a material.

#include "rr_host_internal.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <new>
#include <string>
#include <utility>
#include <vector>

namespace {

// ── JSON ───────────────────────────────────────────────────────────────────
struct Json {
    enum Kind { Null, Bool, Num, Str, Arr, Obj } kind = Null;
    bool b = false;
    double num = 0.0;
    std::string str;
    std::vector<Json> arr;
    std::vector<std::pair<std::string, Json>> obj;

    const Json* get(const char* key) const {
        if (kind != Obj) return nullptr;
        for (const auto& kv : obj)
            if (kv.first == key) return &kv.second;
        return nullptr;
    }
    size_t size() const { return kind == Arr ? arr.size() : 0; }
};

struct LoadError {
    std::string msg;
};

class JsonReader {
public:
    JsonReader(const char* p, size_t n) : p_(p), end_(p + n) {}
    Json parse() {
        Json v = value(0);
        ws();
        if (p_ != end_) fail("trailing characters after the JSON value");
        return v;
    }

private:
    const char* p_;
    const char* end_;

    [[noreturn]] void fail(const char* what) { throw LoadError{std::string("JSON: ") + what}; }
    void ws() {
        while (p_ < end_ && (*p_ == ' ' || *p_ == '\t' || *p_ == '\n' || *p_ == '\r')) ++p_;
    }
    bool lit(const char* s) {
        const size_t n = std::strlen(s);
        if (size_t(end_ - p_) < n || std::memcmp(p_, s, n) != 0) return false;
        p_ += n;
        return true;
    }
    Json value(int depth) {
        if (depth > 128) fail("nesting deeper than 128");
        ws();
        if (p_ >= end_) fail("unexpected end of input");
        Json v;
        const char c = *p_;
        if (c == '{') {
            v.kind = Json::Obj;
            ++p_;
            ws();
            if (p_ < end_ && *p_ == '}') { ++p_; return v; }
            for (;;) {
                ws();
                if (p_ >= end_ || *p_ != '"') fail("expected a member name");
                std::string key = string();
                ws();
                if (p_ >= end_ || *p_ != ':') fail("expected ':'");
                ++p_;
                Json m = value(depth + 1);
                v.obj.emplace_back(std::move(key), std::move(m));
                ws();
                if (p_ < end_ && *p_ == ',') { ++p_; continue; }
                if (p_ < end_ && *p_ == '}') { ++p_; return v; }
                fail("expected ',' or '}'");
            }
        }
        if (c == '[') {
            v.kind = Json::Arr;
            ++p_;
            ws();
            if (p_ < end_ && *p_ == ']') { ++p_; return v; }
            for (;;) {
                v.arr.push_back(value(depth + 1));
                ws();
                if (p_ < end_ && *p_ == ',') { ++p_; continue; }
                if (p_ < end_ && *p_ == ']') { ++p_; return v; }
                fail("expected ',' or ']'");
            }
        }
        if (c == '"') { v.kind = Json::Str; v.str = string(); return v; }
        if (lit("true")) { v.kind = Json::Bool; v.b = true; return v; }
        if (lit("false")) { v.kind = Json::Bool; v.b = false; return v; }
        if (lit("null")) return v;
        v.kind = Json::Num;
        v.num = number();
        return v;
    }
    double number() {
        const char* s = p_;
        if (p_ < end_ && *p_ == '-') ++p_;
        const char* digits = p_;
        while (p_ < end_ && *p_ >= '0' && *p_ <= '9') ++p_;
        if (p_ == digits) fail("bad number");
        if (p_ < end_ && *p_ == '.') {
            ++p_;
            const char* f = p_;
            while (p_ < end_ && *p_ >= '0' && *p_ <= '9') ++p_;
            if (p_ == f) fail("bad number");
        }
        if (p_ < end_ && (*p_ == 'e' || *p_ == 'E')) {
            ++p_;
            if (p_ < end_ && (*p_ == '+' || *p_ == '-')) ++p_;
            const char* e = p_;
            while (p_ < end_ && *p_ >= '0' && *p_ <= '9') ++p_;
            if (p_ == e) fail("bad number");
        }
        const std::string text(s, p_);
        return std::strtod(text.c_str(), nullptr);  // correctly rounded to binary64
    }
    static void utf8(std::string& out, uint32_t cp) {
        if (cp < 0x80) {
            out += char(cp);
        } else if (cp < 0x800) {
            out += char(0xC0 | (cp >> 6)); out += char(0x80 | (cp & 0x3F));
        } else if (cp < 0x10000) {
            out += char(0xE0 | (cp >> 12)); out += char(0x80 | ((cp >> 6) & 0x3F)); out += char(0x80 | (cp & 0x3F));
        } else {
            out += char(0xF0 | (cp >> 18)); out += char(0x80 | ((cp >> 12) & 0x3F));
            out += char(0x80 | ((cp >> 6) & 0x3F)); out += char(0x80 | (cp & 0x3F));
        }
    }
    uint32_t hex4() {
        if (end_ - p_ < 4) fail("bad \\u escape");
        uint32_t v = 0;
        for (int k = 0; k < 4; ++k) {
            const char h = *p_++;
            v <<= 4;
            if (h >= '0' && h <= '9') v |= uint32_t(h - '0');
            else if (h >= 'a' && h <= 'f') v |= uint32_t(h - 'a' + 10);
            else if (h >= 'A' && h <= 'F') v |= uint32_t(h - 'A' + 10);
            else fail("bad \\u escape");
        }
        return v;
    }
    std::string string() {
        ++p_;  // opening quote
        std::string out;
        for (;;) {
            if (p_ >= end_) fail("unterminated string");
            const char c = *p_++;
            if (c == '"') return out;
            if (c != '\\') { out += c; continue; }
            if (p_ >= end_) fail("unterminated string");
            const char e = *p_++;
            switch (e) {
                case '"': out += '"'; break;
                case '\\': out += '\\'; break;
                case '/': out += '/'; break;
                case 'b': out += '\b'; break;
                case 'f': out += '\f'; break;
                case 'n': out += '\n'; break;
                case 'r': out += '\r'; break;
                case 't': out += '\t'; break;
                case 'u': {
                    uint32_t cp = hex4();
                    if (cp >= 0xD800 && cp < 0xDC00 && end_ - p_ >= 6 && p_[0] == '\\' && p_[1] == 'u') {
                        p_ += 2;
                        const uint32_t lo = hex4();
                        if (lo >= 0xDC00 && lo < 0xE000) cp = 0x10000 + ((cp - 0xD800) << 10) + (lo - 0xDC00);
                        else fail("bad surrogate pair");
                    }
                    utf8(out, cp);
                    break;
                }
                default: fail("bad escape");
            }
        }
    }
};

// ── helpers over the document ──────────────────────────────────────────────
[[noreturn]] void fail(const std::string& m) { throw LoadError{m}; }

int64_t int_of(const Json* v, int64_t def) {
    if (!v) return def;
    if (v->kind != Json::Num || v->num != std::floor(v->num) || std::fabs(v->num) > 9.0e15)
        fail("expected an integer");
    return int64_t(v->num);
}
double num_of(const Json* v, double def) {
    if (!v) return def;
    if (v->kind != Json::Num) fail("expected a number");
    return v->num;
}
// n numbers from an array member, or the defaults when absent
void nums_of(const Json* v, size_t n, const double* def, double* out) {
    if (!v) { for (size_t k = 0; k < n; ++k) out[k] = def[k]; return; }
    if (v->kind != Json::Arr || v->arr.size() != n) fail("expected an array of " + std::to_string(n) + " numbers");
    for (size_t k = 0; k < n; ++k) out[k] = num_of(&v->arr[k], 0.0);
}
const Json& at(const Json* arr, int64_t i, const char* what) {
    if (!arr || arr->kind != Json::Arr || i < 0 || size_t(i) >= arr->arr.size())
        fail(std::string("index out of range: ") + what + " " + std::to_string(i));
    return arr->arr[size_t(i)];
}

std::vector<uint8_t> read_file(const std::string& path) {
    FILE* f = std::fopen(path.c_str(), "rb");
    if (!f) fail("cannot open '" + path + "'");
    std::vector<uint8_t> data;
    uint8_t chunk[1 << 16];
    size_t got;
    while ((got = std::fread(chunk, 1, sizeof chunk, f)) > 0) data.insert(data.end(), chunk, chunk + got);
    const bool bad = std::ferror(f) != 0;
    std::fclose(f);
    if (bad) fail("read error on '" + path + "'");
    return data;
}

std::vector<uint8_t> base64(const std::string& s, size_t from) {
    auto val = [](char c) -> int {
        if (c >= 'A' && c <= 'Z') return c - 'A';
        if (c >= 'a' && c <= 'z') return c - 'a' + 26;
        if (c >= '0' && c <= '9') return c - '0' + 52;
        if (c == '+' || c == '-') return 62;
        if (c == '/' || c == '_') return 63;
        return -1;
    };
    std::vector<uint8_t> out;
    uint32_t acc = 0;
    int bits = 0;
    for (size_t i = from; i < s.size(); ++i) {
        const char c = s[i];
        if (c == '=') break;
        const int v = val(c);
        if (v < 0) fail("bad base64 data URI");
        acc = (acc << 6) | uint32_t(v);
        bits += 6;
        if (bits >= 8) {
            bits -= 8;
            out.push_back(uint8_t((acc >> bits) & 0xFF));
        }
    }
    return out;
}

std::string uri_decode(const std::string& u) {
    std::string out;
    for (size_t i = 0; i < u.size(); ++i) {
        if (u[i] == '%' && i + 2 < u.size()) {
            char h[3] = {u[i + 1], u[i + 2], 0};
            char* e = nullptr;
            const long v = std::strtol(h, &e, 16);
            if (e == h + 2) { out += char(v); i += 2; continue; }
        }
        out += u[i];
    }
    return out;
}

// ── glm-style 4x4 matrices (column-major: m[c*4 + r] is row r of column c) ──
struct M4 {
    float m[16];
};
M4 identity4() {
    M4 a{};
    a.m[0] = a.m[5] = a.m[10] = a.m[15] = 1.0f;
    return a;
}
// (A * B): column i = A0*B[i][0] + A1*B[i][1] + A2*B[i][2] + A3*B[i][3],
// summed left to right per component
M4 mul(const M4& A, const M4& B) {
    M4 R;
    for (int i = 0; i < 4; ++i)
        for (int r = 0; r < 4; ++r)
            R.m[i * 4 + r] = A.m[0 * 4 + r] * B.m[i * 4 + 0] + A.m[1 * 4 + r] * B.m[i * 4 + 1] +
                             A.m[2 * 4 + r] * B.m[i * 4 + 2] + A.m[3 * 4 + r] * B.m[i * 4 + 3];
    return R;
}
// translate(m, v): column 3 = m0*v0 + m1*v1 + m2*v2 + m3
M4 translate(const M4& A, float x, float y, float z) {
    M4 R = A;
    for (int r = 0; r < 4; ++r) R.m[12 + r] = A.m[0 + r] * x + A.m[4 + r] * y + A.m[8 + r] * z + A.m[12 + r];
    return R;
}
// scale(m, v): columns 0..2 scaled by v
M4 scale(const M4& A, float x, float y, float z) {
    M4 R = A;
    for (int r = 0; r < 4; ++r) { R.m[r] = A.m[r] * x; R.m[4 + r] = A.m[4 + r] * y; R.m[8 + r] = A.m[8 + r] * z; }
    return R;
}
// Rotation matrix of the unit quaternion (w, x, y, z), the standard
// expansion 1 - 2(y^2 + z^2), 2(xy + wz), ... written per column.
M4 quat_matrix(float w, float x, float y, float z) {
    const float xx = x * x, yy = y * y, zz = z * z;
    const float xz = x * z, xy = x * y, yz = y * z;
    const float wx = w * x, wy = w * y, wz = w * z;
    M4 R = identity4();
    R.m[0] = 1.0f - 2.0f * (yy + zz); R.m[1] = 2.0f * (xy + wz);        R.m[2] = 2.0f * (xz - wy);
    R.m[4] = 2.0f * (xy - wz);        R.m[5] = 1.0f - 2.0f * (xx + zz); R.m[6] = 2.0f * (yz + wx);
    R.m[8] = 2.0f * (xz + wy);        R.m[9] = 2.0f * (yz - wx);        R.m[10] = 1.0f - 2.0f * (xx + yy);
    return R;
}

// node_transform (GltfLoader.cpp:33-61)
M4 node_transform(const Json& node) {
    if (const Json* mat = node.get("matrix")) {
        double v[16];
        static const double id[16] = {1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1, 0, 0, 0, 0, 1};
        nums_of(mat, 16, id, v);
        M4 m;
        // the reference fills m[c][r] = matrix[r * 4 + c] (GltfLoader.cpp:38-41)
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) m.m[c * 4 + r] = float(v[r * 4 + c]);
        return m;
    }
    M4 t = identity4();
    if (const Json* tr = node.get("translation")) {
        double v[3];
        nums_of(tr, 3, nullptr, v);
        t = translate(t, float(v[0]), float(v[1]), float(v[2]));
    }
    if (const Json* rq = node.get("rotation")) {
        double q[4];
        nums_of(rq, 4, nullptr, q);  // glTF order x, y, z, w
        t = mul(t, quat_matrix(float(q[3]), float(q[0]), float(q[1]), float(q[2])));
    }
    if (const Json* sc = node.get("scale")) {
        double v[3];
        nums_of(sc, 3, nullptr, v);
        t = scale(t, float(v[0]), float(v[1]), float(v[2]));
    }
    return t;
}

// ── the document ───────────────────────────────────────────────────────────
struct Doc {
    Json root;
    std::vector<std::vector<uint8_t>> buffers;
};

size_t comp_size(int64_t ct) {
    switch (ct) {
        case 5120: case 5121: return 1;   // BYTE, UNSIGNED_BYTE
        case 5122: case 5123: return 2;   // SHORT, UNSIGNED_SHORT
        case 5125: case 5126: return 4;   // UNSIGNED_INT, FLOAT
        default: fail("bad accessor componentType " + std::to_string(ct));
    }
}
size_t comp_count(const std::string& t) {
    if (t == "SCALAR") return 1;
    if (t == "VEC2") return 2;
    if (t == "VEC3") return 3;
    if (t == "VEC4") return 4;
    if (t == "MAT2") return 4;
    if (t == "MAT3") return 9;
    if (t == "MAT4") return 16;
    fail("bad accessor type '" + t + "'");
}

struct View {
    const uint8_t* base = nullptr;  // first element
    size_t count = 0, stride = 0, comps = 0;
    int64_t ctype = 0;
};

// accessor_data (GltfLoader.cpp:64-75) with bounds, stride and type checks
View accessor(const Doc& d, int64_t idx, const char* what) {
    const Json& acc = at(d.root.get("accessors"), idx, "accessor");
    if (acc.get("sparse")) fail(std::string("sparse accessors are not supported (") + what + ")");
    const Json* bvi = acc.get("bufferView");
    if (!bvi) fail(std::string("accessor without bufferView (") + what + ")");
    const Json& bv = at(d.root.get("bufferViews"), int_of(bvi, -1), "bufferView");
    const int64_t bi = int_of(bv.get("buffer"), -1);
    if (bi < 0 || size_t(bi) >= d.buffers.size()) fail("bufferView names a missing buffer");
    const std::vector<uint8_t>& buf = d.buffers[size_t(bi)];
    const int64_t bv_off = int_of(bv.get("byteOffset"), 0), bv_len = int_of(bv.get("byteLength"), -1);
    if (bv_off < 0 || bv_len < 0 || uint64_t(bv_off) + uint64_t(bv_len) > buf.size())
        fail("bufferView outside its buffer");
    View v;
    v.ctype = int_of(acc.get("componentType"), -1);
    const Json* type = acc.get("type");
    if (!type || type->kind != Json::Str) fail("accessor without type");
    v.comps = comp_count(type->str);
    const size_t elem = comp_size(v.ctype) * v.comps;
    const int64_t stride = int_of(bv.get("byteStride"), 0);
    if (stride != 0 && (stride < int64_t(elem) || stride > 252)) fail("bad byteStride");
    v.stride = stride ? size_t(stride) : elem;
    const int64_t cnt = int_of(acc.get("count"), -1), off = int_of(acc.get("byteOffset"), 0);
    if (cnt < 0 || off < 0) fail("bad accessor count or offset");
    v.count = size_t(cnt);
    if (v.count > 0 && uint64_t(off) + uint64_t(v.count - 1) * v.stride + elem > uint64_t(bv_len))
        fail(std::string("accessor outside its bufferView (") + what + ")");
    v.base = buf.data() + bv_off + off;
    return v;
}

float read_float(const View& v, size_t i, size_t c) {
    float f;
    std::memcpy(&f, v.base + i * v.stride + c * 4, 4);
    return f;
}

uint32_t read_index(const View& v, size_t i) {
    const uint8_t* p = v.base + i * v.stride;
    switch (v.ctype) {
        case 5121: return p[0];
        case 5123: { uint16_t x; std::memcpy(&x, p, 2); return x; }
        case 5125: { uint32_t x; std::memcpy(&x, p, 4); return x; }
        default: fail("index accessor must be UNSIGNED_BYTE, UNSIGNED_SHORT or UNSIGNED_INT");
    }
}

Doc open_document(const std::string& path) {
    Doc d;
    const std::vector<uint8_t> file = read_file(path);
    const uint8_t* bin = nullptr;
    size_t bin_len = 0;
    auto u32 = [&](size_t o) {
        uint32_t x;
        std::memcpy(&x, file.data() + o, 4);
        return x;
    };
    if (file.size() >= 12 && u32(0) == 0x46546C67u) {  // "glTF": binary container
        if (u32(4) != 2u) fail("unsupported .glb version " + std::to_string(u32(4)));
        const size_t total = std::min<size_t>(u32(8), file.size());
        size_t o = 12;
        const uint8_t* json = nullptr;
        size_t json_len = 0;
        while (o + 8 <= total) {
            const size_t len = u32(o), type = u32(o + 4);
            if (o + 8 + len > total) fail(".glb chunk outside the file");
            if (type == 0x4E4F534Au && !json) { json = file.data() + o + 8; json_len = len; }
            else if (type == 0x004E4942u && !bin) { bin = file.data() + o + 8; bin_len = len; }
            o += 8 + ((len + 3) & ~size_t(3));
        }
        if (!json) fail(".glb without a JSON chunk");
        d.root = JsonReader(reinterpret_cast<const char*>(json), json_len).parse();
    } else {
        d.root = JsonReader(reinterpret_cast<const char*>(file.data()), file.size()).parse();
    }
    if (d.root.kind != Json::Obj) fail("the document is not a JSON object");
    const std::string dir = [&] {
        const size_t s = path.find_last_of('/');
        return s == std::string::npos ? std::string() : path.substr(0, s + 1);
    }();
    if (const Json* bufs = d.root.get("buffers")) {
        if (bufs->kind != Json::Arr) fail("buffers is not an array");
        for (size_t b = 0; b < bufs->arr.size(); ++b) {
            const Json& B = bufs->arr[b];
            const int64_t len = int_of(B.get("byteLength"), -1);
            if (len < 0) fail("buffer without byteLength");
            std::vector<uint8_t> data;
            const Json* uri = B.get("uri");
            if (!uri) {
                if (b != 0 || !bin) fail("buffer " + std::to_string(b) + " has no uri and no .glb BIN chunk");
                data.assign(bin, bin + bin_len);
            } else {
                if (uri->kind != Json::Str) fail("buffer uri is not a string");
                const std::string& u = uri->str;
                if (u.compare(0, 5, "data:") == 0) {
                    const size_t comma = u.find(',');
                    if (comma == std::string::npos || u.rfind(";base64", comma) == std::string::npos)
                        fail("only base64 data URIs are supported");
                    data = base64(u, comma + 1);
                } else {
                    data = read_file(dir + uri_decode(u));
                }
            }
            if (data.size() < size_t(len)) fail("buffer " + std::to_string(b) + " is shorter than its byteLength");
            data.resize(size_t(len));
            d.buffers.push_back(std::move(data));
        }
    }
    return d;
}

GpuMaterial default_material() {  // Material{} (Scene.h:36-48) as Scene::upload writes it
    GpuMaterial m{};
    m.base_color[0] = m.base_color[1] = m.base_color[2] = m.base_color[3] = 1.0f;
    m.metallic = 0.0f;
    m.roughness = 1.0f;
    m.ior = 1.5f;
    m.albedo_tex_idx = m.normal_tex_idx = m.metallic_roughness_tex_idx = m.emissive_tex_idx = 0xffffffffu;
    m.sampler_idx = 0;
    return m;
}

void load(const std::string& path, rr_host_scene& s) {
    const Doc d = open_document(path);
    const Json& R = d.root;
    // tinygltf's default section check (REQUIRE_VERSION): asset.version must exist
    const Json* asset = R.get("asset");
    const Json* version = asset ? asset->get("version") : nullptr;
    if (!version || version->kind != Json::Str) fail("missing asset.version");
    // materials (GltfLoader.cpp:101-155)
    size_t n_materials = 0;
    if (const Json* mats = R.get("materials")) {
        if (mats->kind != Json::Arr) fail("materials is not an array");
        n_materials = mats->arr.size();
        for (const Json& M : mats->arr) {
            GpuMaterial g = default_material();
            const Json* pbr = M.get("pbrMetallicRoughness");
            static const double one4[4] = {1, 1, 1, 1}, zero3[3] = {0, 0, 0};
            double bc[4], em[3];
            nums_of(pbr ? pbr->get("baseColorFactor") : nullptr, 4, one4, bc);
            for (int k = 0; k < 4; ++k) g.base_color[k] = float(bc[k]);
            g.metallic = float(num_of(pbr ? pbr->get("metallicFactor") : nullptr, 1.0));
            g.roughness = float(num_of(pbr ? pbr->get("roughnessFactor") : nullptr, 1.0));
            nums_of(M.get("emissiveFactor"), 3, zero3, em);
            for (int k = 0; k < 3; ++k) g.emissive[k] = float(em[k]);
            s.materials.push_back(g);
        }
    }
    bool need_default_material = false;
    // meshes (GltfLoader.cpp:201-326): one GpuMesh per triangle primitive
    std::vector<std::vector<int64_t>> prim_mesh;
    if (const Json* meshes = R.get("meshes")) {
        if (meshes->kind != Json::Arr) fail("meshes is not an array");
        prim_mesh.resize(meshes->arr.size());
        for (size_t mi = 0; mi < meshes->arr.size(); ++mi) {
            const Json* prims = meshes->arr[mi].get("primitives");
            if (!prims || prims->kind != Json::Arr) fail("mesh without primitives");
            prim_mesh[mi].assign(prims->arr.size(), -1);
            for (size_t pi = 0; pi < prims->arr.size(); ++pi) {
                const Json& P = prims->arr[pi];
                if (int_of(P.get("mode"), 4) != 4) continue;
                const Json* attrs = P.get("attributes");
                const Json* pos_a = attrs ? attrs->get("POSITION") : nullptr;
                if (!pos_a) continue;
                const View pos = accessor(d, int_of(pos_a, -1), "POSITION");
                if (pos.ctype != 5126 || pos.comps != 3) fail("POSITION must be FLOAT VEC3");
                View nor, uv, tan;
                if (const Json* a = attrs->get("NORMAL")) {
                    nor = accessor(d, int_of(a, -1), "NORMAL");
                    if (nor.ctype != 5126 || nor.comps != 3) fail("NORMAL must be FLOAT VEC3");
                    if (nor.count < pos.count) fail("NORMAL has fewer elements than POSITION");
                }
                if (const Json* a = attrs->get("TEXCOORD_0")) {
                    uv = accessor(d, int_of(a, -1), "TEXCOORD_0");
                    if (uv.ctype != 5126 || uv.comps != 2) fail("TEXCOORD_0 must be FLOAT VEC2");
                    if (uv.count < pos.count) fail("TEXCOORD_0 has fewer elements than POSITION");
                }
                if (const Json* a = attrs->get("TANGENT")) {
                    tan = accessor(d, int_of(a, -1), "TANGENT");
                    if (tan.ctype != 5126 || tan.comps != 4) fail("TANGENT must be FLOAT VEC4");
                    if (tan.count < pos.count) fail("TANGENT has fewer elements than POSITION");
                }
                std::vector<uint32_t> idx;
                if (const Json* ia = P.get("indices")) {
                    const View iv = accessor(d, int_of(ia, -1), "indices");
                    if (iv.comps != 1) fail("indices must be SCALAR");
                    idx.resize(iv.count);
                    for (size_t k = 0; k < iv.count; ++k) {
                        idx[k] = read_index(iv, k);
                        if (idx[k] >= pos.count) fail("index past the primitive's vertices");
                    }
                } else {
                    idx.resize(pos.count);
                    for (size_t k = 0; k < pos.count; ++k) idx[k] = uint32_t(k);
                }
                GpuMesh g{};
                g.vertex_base = uint32_t(s.vertices.size());
                g.vertex_count = uint32_t(pos.count);
                g.index_byte_offset = uint32_t(s.indices.size() * 4);
                g.index_count = uint32_t(idx.size());
                const int64_t mat = int_of(P.get("material"), -1);
                if (mat >= int64_t(n_materials)) fail("primitive names a missing material");
                if (mat < 0 && n_materials == 0) need_default_material = true;
                g.material_index = mat >= 0 ? uint32_t(mat) : 0u;
                for (size_t k = 0; k < pos.count; ++k) {
                    GpuVertex v{};
                    for (int c = 0; c < 3; ++c) v.pos[c] = read_float(pos, k, c);
                    if (nor.base) { for (int c = 0; c < 3; ++c) v.normal[c] = read_float(nor, k, c); }
                    else { v.normal[0] = 0.0f; v.normal[1] = 1.0f; v.normal[2] = 0.0f; }
                    if (uv.base) { v.uv[0] = read_float(uv, k, 0); v.uv[1] = read_float(uv, k, 1); }
                    if (tan.base) { for (int c = 0; c < 4; ++c) v.tangent[c] = read_float(tan, k, c); }
                    else { v.tangent[0] = 1.0f; v.tangent[1] = 0.0f; v.tangent[2] = 0.0f; v.tangent[3] = 1.0f; }
                    s.vertices.push_back(v);
                }
                s.indices.insert(s.indices.end(), idx.begin(), idx.end());
                prim_mesh[mi][pi] = int64_t(s.meshes.size());
                s.meshes.push_back(g);
            }
        }
    }
    if (need_default_material) s.materials.push_back(default_material());
    // nodes (GltfLoader.cpp:328-355): the default scene's trees
    const Json* scenes = R.get("scenes");
    if (!scenes || scenes->size() == 0) {
        if (!s.meshes.empty()) fail("the document has meshes but no scene");
        return;
    }
    const int64_t si = int_of(R.get("scene"), 0);
    const Json& scene = at(scenes, si < 0 ? 0 : si, "scene");
    const Json* nodes = R.get("nodes");
    const size_t n_nodes = nodes ? nodes->size() : 0;
    std::vector<uint8_t> on_path(n_nodes, 0);
    struct Walker {
        const Json* nodes;
        const std::vector<std::vector<int64_t>>& prim_mesh;
        std::vector<uint8_t>& on_path;
        rr_host_scene& s;
        void walk(int64_t ni, const M4& parent, int depth) {
            const Json& node = at(nodes, ni, "node");
            if (on_path[size_t(ni)] || depth > 1024) fail("the node graph has a cycle");
            on_path[size_t(ni)] = 1;
            const M4 world = mul(parent, node_transform(node));
            const int64_t mesh = int_of(node.get("mesh"), -1);
            if (mesh >= 0) {
                if (size_t(mesh) >= prim_mesh.size()) fail("node names a missing mesh");
                for (int64_t gm : prim_mesh[size_t(mesh)]) {
                    if (gm < 0) continue;
                    GpuInstance inst{};
                    for (int r = 0; r < 4; ++r)
                        for (int c = 0; c < 4; ++c) inst.transform[r * 4 + c] = world.m[c * 4 + r];
                    inst.mesh_index = uint32_t(gm);
                    s.instances.push_back(inst);
                }
            }
            if (const Json* ch = node.get("children")) {
                if (ch->kind != Json::Arr) fail("node children is not an array");
                for (const Json& c : ch->arr) walk(int_of(&c, -1), world, depth + 1);
            }
            on_path[size_t(ni)] = 0;
        }
    } w{nodes, prim_mesh, on_path, s};
    if (const Json* roots = scene.get("nodes")) {
        if (roots->kind != Json::Arr) fail("scene nodes is not an array");
        for (const Json& r : roots->arr) w.walk(int_of(&r, -1), identity4(), 0);
    }
}

void set_err(char* err, size_t n, const std::string& m) {
    if (!err || n == 0) return;
    const size_t k = std::min(n - 1, m.size());
    std::memcpy(err, m.data(), k);
    err[k] = 0;
}

} // namespace

extern "C" rr_status rr_host_scene_gltf(const char* path, rr_host_scene** out, char* err, size_t err_size) {
    set_err(err, err_size, "");
    if (!path || !out) {
        set_err(err, err_size, "glTF: null argument");
        return RR_ERR_INVALID_ARGUMENT;
    }
    *out = nullptr;
    std::unique_ptr<rr_host_scene> s(new (std::nothrow) rr_host_scene());
    if (!s) return RR_ERR_OUT_OF_MEMORY;
    try {
        load(path, *s);
    } catch (const LoadError& e) {
        set_err(err, err_size, std::string("glTF '") + path + "': " + e.msg);
        return RR_ERR_INVALID_ARGUMENT;
    } catch (const std::bad_alloc&) {
        set_err(err, err_size, "glTF: out of host memory");
        return RR_ERR_OUT_OF_MEMORY;
    }
    *out = s.release();
    return RR_OK;
}
