// slang_shim.h — the Slang/HLSL vocabulary that the reference's shader text
// needs in order to compile as C++ (TEST INFRASTRUCTURE ONLY).
//
// oracle/make_ref.py rewrites the reference's .slang files mechanically into
// C++ (parameter qualifiers, swizzles, literal suffixes, constructor syntax)
// and compiles them against this header, so that the reference's own source
// text, not a restatement of it, computes the same images as the
// hand-written oracle on the CPU. The header defines:
//   - vector types floatN / intN / uintN / boolN (N = 2, 3, 4), scalar-layout
//     (4-byte aligned, 12-byte float3: the layout of the reference's scene
//     buffers, GpuScene.slang), with component-wise arithmetic;
//   - float3x3 / float4x4 (row-major, as the reference's Slang session
//     compiles them) and mul(M, v);
//   - the intrinsics the shaders call, with the definitions both the oracle
//     and the CUDA kernels use (stated in the design notes): dot and mul sum
//     left to right, normalize(v) = v * (1 / sqrt(dot(v, v))), length =
//     sqrt(dot), lerp(x, y, s) = x + (y - x) * s, reflect(i, n) =
//     i - n * (2 dot(i, n)), rsqrt(x) = 1 / sqrt(x), frac(x) = x - floor(x),
//     round = round half to even, max(a, b) = a > b ? a : b; sin, cos, exp,
//     log are the deterministic functions of rr_detmath.h (the reference
//     leaves their precision to the Vulkan driver);
//   - the bindless resources (ByteAddressBuffer, RWByteAddressBuffer,
//     RWTexture2D<float4>, Texture2D) as views of host arrays, and the heap
//     arrays gScene / gSceneRW / gStorageImages / gTextures / gTLAS that the
//     harness fills before a dispatch;
//   - RayQuery over a closest-hit callback: the reference traces against a
//     driver-built BLAS/TLAS on ray-tracing hardware, which has no source to
//     rewrite; the harness supplies the oracle's watertight intersector
//     (opaque, two-sided: every instance disables facing culling).
#pragma once

#include <cstdint>
#include <cstring>
#include <cmath>

#include "rr_detmath.h"

namespace slang {

typedef uint32_t uint;

// ── vectors ────────────────────────────────────────────────────────────────
template <class T> struct V2;
template <class T> struct V3;
template <class T> struct V4;

template <class T>
struct V2 {
    union { struct { T x, y; }; struct { T r, g; }; };
    V2() : x(T()), y(T()) {}
    V2(T s) : x(s), y(s) {}
    template <class A, class B> V2(A a, B b) : x(T(a)), y(T(b)) {}
    template <class U> explicit V2(const V2<U>& o) : x(T(o.x)), y(T(o.y)) {}
    V2(const V2&) = default;
    V2& operator=(const V2&) = default;
    V2 xy() const { return *this; }
};

template <class T>
struct V3 {
    union { struct { T x, y, z; }; struct { T r, g, b; }; };
    V3() : x(T()), y(T()), z(T()) {}
    V3(T s) : x(s), y(s), z(s) {}
    template <class A, class B, class C> V3(A a, B b, C c) : x(T(a)), y(T(b)), z(T(c)) {}
    template <class U, class B> V3(const V2<U>& v, B b) : x(T(v.x)), y(T(v.y)), z(T(b)) {}
    template <class U> explicit V3(const V3<U>& o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
    V3(const V3&) = default;
    V3& operator=(const V3&) = default;
    V2<T> xy() const { return V2<T>(x, y); }
    V3 xyz() const { return *this; }
};

template <class T>
struct V4 {
    union { struct { T x, y, z, w; }; struct { T r, g, b, a; }; };
    V4() : x(T()), y(T()), z(T()), w(T()) {}
    V4(T s) : x(s), y(s), z(s), w(s) {}
    template <class A, class B, class C, class D>
    V4(A a, B b, C c, D d) : x(T(a)), y(T(b)), z(T(c)), w(T(d)) {}
    template <class U, class D> V4(const V3<U>& v, D d) : x(T(v.x)), y(T(v.y)), z(T(v.z)), w(T(d)) {}
    template <class U> explicit V4(const V4<U>& o) : x(T(o.x)), y(T(o.y)), z(T(o.z)), w(T(o.w)) {}
    V4(const V4&) = default;
    V4& operator=(const V4&) = default;
    V2<T> xy() const { return V2<T>(x, y); }
    V3<T> xyz() const { return V3<T>(x, y, z); }
};

typedef V2<float> float2;
typedef V3<float> float3;
typedef V4<float> float4;
typedef V2<int> int2;
typedef V3<int> int3;
typedef V4<int> int4;
typedef V2<uint> uint2;
typedef V3<uint> uint3;
typedef V4<uint> uint4;
typedef V2<bool> bool2;
typedef V3<bool> bool3;
typedef V4<bool> bool4;

static_assert(sizeof(float3) == 12 && sizeof(float4) == 16 && sizeof(uint3) == 12, "scalar layout");

// component-wise operators (vector op vector, vector op scalar, scalar op vector)
#define SLANG_VEC_BINOP(OP)                                                                            \
    template <class T> V2<T> operator OP(const V2<T>& a, const V2<T>& b) { return V2<T>(a.x OP b.x, a.y OP b.y); } \
    template <class T> V3<T> operator OP(const V3<T>& a, const V3<T>& b) {                             \
        return V3<T>(a.x OP b.x, a.y OP b.y, a.z OP b.z);                                              \
    }                                                                                                  \
    template <class T> V4<T> operator OP(const V4<T>& a, const V4<T>& b) {                             \
        return V4<T>(a.x OP b.x, a.y OP b.y, a.z OP b.z, a.w OP b.w);                                  \
    }                                                                                                  \
    template <class T> V2<T> operator OP(const V2<T>& a, T s) { return V2<T>(a.x OP s, a.y OP s); }    \
    template <class T> V3<T> operator OP(const V3<T>& a, T s) { return V3<T>(a.x OP s, a.y OP s, a.z OP s); } \
    template <class T> V4<T> operator OP(const V4<T>& a, T s) {                                        \
        return V4<T>(a.x OP s, a.y OP s, a.z OP s, a.w OP s);                                          \
    }                                                                                                  \
    template <class T> V2<T> operator OP(T s, const V2<T>& a) { return V2<T>(s OP a.x, s OP a.y); }    \
    template <class T> V3<T> operator OP(T s, const V3<T>& a) { return V3<T>(s OP a.x, s OP a.y, s OP a.z); } \
    template <class T> V4<T> operator OP(T s, const V4<T>& a) {                                        \
        return V4<T>(s OP a.x, s OP a.y, s OP a.z, s OP a.w);                                          \
    }                                                                                                  \
    template <class T, class V> V& operator OP##=(V& a, const T& b) { return a = a OP b; }
SLANG_VEC_BINOP(+)
SLANG_VEC_BINOP(-)
SLANG_VEC_BINOP(*)
SLANG_VEC_BINOP(/)
#undef SLANG_VEC_BINOP

template <class T> V2<T> operator-(const V2<T>& a) { return V2<T>(-a.x, -a.y); }
template <class T> V3<T> operator-(const V3<T>& a) { return V3<T>(-a.x, -a.y, -a.z); }
template <class T> V4<T> operator-(const V4<T>& a) { return V4<T>(-a.x, -a.y, -a.z, -a.w); }

#define SLANG_VEC_CMP(OP)                                                                                \
    template <class T> bool2 operator OP(const V2<T>& a, T s) { return bool2(a.x OP s, a.y OP s); }      \
    template <class T> bool3 operator OP(const V3<T>& a, T s) { return bool3(a.x OP s, a.y OP s, a.z OP s); } \
    template <class T> bool3 operator OP(const V3<T>& a, const V3<T>& b) {                               \
        return bool3(a.x OP b.x, a.y OP b.y, a.z OP b.z);                                                \
    }                                                                                                    \
    template <class T> bool2 operator OP(const V2<T>& a, const V2<T>& b) { return bool2(a.x OP b.x, a.y OP b.y); }
SLANG_VEC_CMP(>)
SLANG_VEC_CMP(<)
SLANG_VEC_CMP(>=)
SLANG_VEC_CMP(<=)
SLANG_VEC_CMP(==)
SLANG_VEC_CMP(!=)
#undef SLANG_VEC_CMP

inline bool any(const bool2& v) { return v.x || v.y; }
inline bool any(const bool3& v) { return v.x || v.y || v.z; }
inline bool any(const bool4& v) { return v.x || v.y || v.z || v.w; }
inline bool all(const bool2& v) { return v.x && v.y; }
inline bool all(const bool3& v) { return v.x && v.y && v.z; }
inline bool all(const bool4& v) { return v.x && v.y && v.z && v.w; }

// ── matrices (row-major: m[row][col]) ──────────────────────────────────────
struct float4x4 { float m[4][4]; };
struct float3x3 { float m[3][3]; };
static_assert(sizeof(float4x4) == 64, "scalar layout");

inline float3x3 to_float3x3(const float4x4& a) {
    float3x3 r;
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) r.m[i][j] = a.m[i][j];
    return r;
}
inline float4 mul(const float4x4& M, const float4& v) {
    return float4(M.m[0][0] * v.x + M.m[0][1] * v.y + M.m[0][2] * v.z + M.m[0][3] * v.w,
                  M.m[1][0] * v.x + M.m[1][1] * v.y + M.m[1][2] * v.z + M.m[1][3] * v.w,
                  M.m[2][0] * v.x + M.m[2][1] * v.y + M.m[2][2] * v.z + M.m[2][3] * v.w,
                  M.m[3][0] * v.x + M.m[3][1] * v.y + M.m[3][2] * v.z + M.m[3][3] * v.w);
}
inline float3 mul(const float3x3& M, const float3& v) {
    return float3(M.m[0][0] * v.x + M.m[0][1] * v.y + M.m[0][2] * v.z,
                  M.m[1][0] * v.x + M.m[1][1] * v.y + M.m[1][2] * v.z,
                  M.m[2][0] * v.x + M.m[2][1] * v.y + M.m[2][2] * v.z);
}

// ── intrinsics ─────────────────────────────────────────────────────────────
inline float max(float a, float b) { return a > b ? a : b; }
inline float min(float a, float b) { return a < b ? a : b; }
inline uint max(uint a, uint b) { return a > b ? a : b; }
inline uint min(uint a, uint b) { return a < b ? a : b; }
inline int max(int a, int b) { return a > b ? a : b; }
inline int min(int a, int b) { return a < b ? a : b; }
template <class T> V2<T> max(const V2<T>& a, const V2<T>& b) { return V2<T>(max(a.x, b.x), max(a.y, b.y)); }
template <class T> V3<T> max(const V3<T>& a, const V3<T>& b) {
    return V3<T>(max(a.x, b.x), max(a.y, b.y), max(a.z, b.z));
}
template <class T> V2<T> min(const V2<T>& a, const V2<T>& b) { return V2<T>(min(a.x, b.x), min(a.y, b.y)); }
template <class T> V3<T> min(const V3<T>& a, const V3<T>& b) {
    return V3<T>(min(a.x, b.x), min(a.y, b.y), min(a.z, b.z));
}
inline float clamp(float x, float lo, float hi) { return min(max(x, lo), hi); }
inline uint clamp(uint x, uint lo, uint hi) { return min(max(x, lo), hi); }
inline int clamp(int x, int lo, int hi) { return min(max(x, lo), hi); }
template <class T> V2<T> clamp(const V2<T>& x, const V2<T>& lo, const V2<T>& hi) {
    return V2<T>(clamp(x.x, lo.x, hi.x), clamp(x.y, lo.y, hi.y));
}
template <class T> V3<T> clamp(const V3<T>& x, const V3<T>& lo, const V3<T>& hi) {
    return V3<T>(clamp(x.x, lo.x, hi.x), clamp(x.y, lo.y, hi.y), clamp(x.z, lo.z, hi.z));
}
inline float saturate(float x) { return clamp(x, 0.0f, 1.0f); }
inline float abs(float x) { return std::fabs(x); }
inline int abs(int x) { return x < 0 ? -x : x; }
inline float2 abs(const float2& v) { return float2(abs(v.x), abs(v.y)); }
inline float3 abs(const float3& v) { return float3(abs(v.x), abs(v.y), abs(v.z)); }
inline float sqrt(float x) { return std::sqrt(x); }
inline float rsqrt(float x) { return 1.0f / std::sqrt(x); }
inline float floor(float x) { return std::floor(x); }
inline float2 floor(const float2& v) { return float2(floor(v.x), floor(v.y)); }
inline float3 floor(const float3& v) { return float3(floor(v.x), floor(v.y), floor(v.z)); }
inline float frac(float x) { return x - floor(x); }
inline float2 frac(const float2& v) { return float2(frac(v.x), frac(v.y)); }
inline float3 frac(const float3& v) { return float3(frac(v.x), frac(v.y), frac(v.z)); }
inline float round(float x) { return std::nearbyint(x); }   // round half to even (default FP environment)
inline float sin(float x) { return rr_sinf(x); }
inline float cos(float x) { return rr_cosf(x); }
inline float exp(float x) { return rr_expf(x); }
inline float log(float x) { return rr_logf(x); }

inline float dot(const float2& a, const float2& b) { return a.x * b.x + a.y * b.y; }
inline float dot(const float3& a, const float3& b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline float dot(const float4& a, const float4& b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
inline float length(const float3& v) { return sqrt(dot(v, v)); }
inline float length(const float2& v) { return sqrt(dot(v, v)); }
inline float3 normalize(const float3& v) { return v * (1.0f / sqrt(dot(v, v))); }
inline float2 normalize(const float2& v) { return v * (1.0f / sqrt(dot(v, v))); }
inline float3 cross(const float3& a, const float3& b) {
    return float3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline float lerp(float x, float y, float s) { return x + (y - x) * s; }
inline float3 lerp(const float3& x, const float3& y, float s) { return x + (y - x) * s; }
inline float3 lerp(const float3& x, const float3& y, const float3& s) { return x + (y - x) * s; }
inline float3 reflect(const float3& i, const float3& n) { return i - n * (2.0f * dot(i, n)); }

inline float asfloat(uint u) { float f; std::memcpy(&f, &u, 4); return f; }
inline float asfloat(int u) { float f; std::memcpy(&f, &u, 4); return f; }
inline uint asuint(float f) { uint u; std::memcpy(&u, &f, 4); return u; }
inline uint asuint(int i) { return uint(i); }
inline uint asuint(uint u) { return u; }
inline int asint(uint u) { return int(u); }
inline int asint(float f) { int i; std::memcpy(&i, &f, 4); return i; }

// ── bindless resources ─────────────────────────────────────────────────────
struct ByteAddressBuffer {
    const unsigned char* data = nullptr;
    size_t size = 0;
    template <class T> T Load(int64_t offset) const {
        T v;
        std::memcpy(&v, data + offset, sizeof(T));
        return v;
    }
};

struct RWByteAddressBuffer {
    unsigned char* data = nullptr;
    size_t size = 0;
    template <class T> T Load(int64_t offset) const {
        T v;
        std::memcpy(&v, data + offset, sizeof(T));
        return v;
    }
    template <class T> void Store(int64_t offset, T v) { std::memcpy(data + offset, &v, sizeof(T)); }
    // integer adds commute: threads of a dispatch may splat in any order
    void InterlockedAdd(int64_t offset, uint v, uint& original) {
        original = __atomic_fetch_add(reinterpret_cast<uint*>(data + offset), v, __ATOMIC_RELAXED);
    }
};

// A view of `width` x `height` pixels whose first pixel is the image's pixel
// (ox, oy): a dispatch over a region writes into a region-sized array.
struct RWTexture2D {
    float4* data = nullptr;
    uint width = 0, height = 0;
    uint ox = 0, oy = 0;
    float4& operator[](const uint2& p) const { return data[size_t(p.y - oy) * width + (p.x - ox)]; }
    float4& operator[](const int2& p) const { return data[size_t(uint(p.y) - oy) * width + (uint(p.x) - ox)]; }
};

struct Texture2D {
    const float4* data = nullptr;
    uint width = 0, height = 0;
    float4 Load(const int3& p) const { return data[size_t(p.y) * width + p.x]; }
};

// ── inline ray tracing ─────────────────────────────────────────────────────
struct RayDesc {
    float3 Origin;
    float TMin = 0.0f;
    float3 Direction;
    float TMax = 0.0f;
};

// Closest hit in [tmin, tmax]: returns true and fills t, the barycentrics of
// v1 and v2, the instance (its custom index) and the mesh-local primitive.
typedef bool (*ClosestHitFn)(const void* scene, const float origin[3], const float dir[3], float tmin, float tmax,
                             float* t, float* u, float* v, uint* instance, uint* primitive);

struct RaytracingAccelerationStructure {
    const void* scene = nullptr;
    ClosestHitFn closest_hit = nullptr;
};

constexpr uint RAY_FLAG_NONE = 0u;
constexpr uint RAY_FLAG_CULL_BACK_FACING_TRIANGLES = 0x10u;
constexpr uint RAY_FLAG_ACCEPT_FIRST_HIT_AND_END_SEARCH = 0x4u;
constexpr uint CANDIDATE_NON_OPAQUE_TRIANGLE = 0u;
constexpr uint CANDIDATE_PROCEDURAL_PRIMITIVE = 1u;
constexpr uint COMMITTED_NOTHING = 0u;
constexpr uint COMMITTED_TRIANGLE_HIT = 1u;

// Every instance of the reference's TLAS sets the facing-cull-disable flag and
// every geometry is opaque, so a query commits the closest hit and never
// yields a candidate: Proceed() returns false at once.
template <uint kFlags>
struct RayQuery {
    bool hit = false;
    float t = 0.0f, u = 0.0f, v = 0.0f;
    uint instance = 0, primitive = 0;
    void TraceRayInline(const RaytracingAccelerationStructure& as, uint, uint, const RayDesc& ray) {
        const float o[3] = {ray.Origin.x, ray.Origin.y, ray.Origin.z};
        const float d[3] = {ray.Direction.x, ray.Direction.y, ray.Direction.z};
        hit = as.closest_hit(as.scene, o, d, ray.TMin, ray.TMax, &t, &u, &v, &instance, &primitive);
    }
    bool Proceed() { return false; }
    uint CandidateType() const { return CANDIDATE_NON_OPAQUE_TRIANGLE; }
    void CommitNonOpaqueTriangleHit() {}
    uint CommittedStatus() const { return hit ? COMMITTED_TRIANGLE_HIT : COMMITTED_NOTHING; }
    float CommittedRayT() const { return t; }
    uint CommittedInstanceID() const { return instance; }
    uint CommittedInstanceIndex() const { return instance; }
    uint CommittedPrimitiveIndex() const { return primitive; }
    float2 CommittedTriangleBarycentrics() const { return float2(u, v); }
};

// The heaps a dispatch reads (filled by the harness before each dispatch).
extern ByteAddressBuffer gScene[16];
extern RWByteAddressBuffer gSceneRW[16];
extern RWTexture2D gStorageImages[32];
extern Texture2D gTextures[32];
extern RaytracingAccelerationStructure gTLAS[1];

} // namespace slang
