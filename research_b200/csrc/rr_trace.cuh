// rr_trace.cuh — BVH traversal and watertight ray/triangle intersection.
//
// Replaces the hardware RayQuery of pathtracer.slang:45-120 /
// restir_di.slang:86-146 (driver-built BLAS/TLAS, AccelStructure.cpp:98-330).
// Semantics kept from the reference: opaque geometry, closest hit in
// [t_min, t_max], no face culling (every TLAS instance sets
// TRIANGLE_FACING_CULL_DISABLE, AccelStructure.cpp:90), hit reports the
// instance index, the mesh-local primitive index and the barycentric weights
// of vertices 1 and 2. Ties on t go to the lowest (instance, primitive).
//
// Geometry is flattened to world space at scene creation (one BVH over every
// instance's triangles), so a ray is never transformed per instance.
#pragma once

#include "rr_dev.cuh"

namespace rr {

// One BVH2 node holds the boxes of both children (64 bytes):
//   a = (c0.lo.x, c0.hi.x, c0.lo.y, c0.hi.y)
//   b = (c1.lo.x, c1.hi.x, c1.lo.y, c1.hi.y)
//   c = (c0.lo.z, c0.hi.z, c1.lo.z, c1.hi.z)
//   d = (child0, child1, count0, count1); child >= 0 is an inner node,
//       child < 0 a leaf whose triangles start at ~child (count in d.z/d.w).
// One triangle record (48 bytes): (v0.xyz, v1.x), (v1.yz, v2.xy),
// (v2.z, instance, primitive, flattened id).
struct DevScene {
    const float4* nodes;
    const float4* tris;
    const float4* nodes4;     // the same tree 4-wide (see trace_step4)
    const float4* vertices;   // GpuVertex as 3 float4
    const uint32_t* indices;
    const uint4* meshes;      // GpuMesh as 2 uint4
    const float4* instances;  // GpuInstance as 5 float4
    const float4* materials;  // (base.rgb, metallic), (emissive.rgb, roughness)
    const float4* lights;     // GpuLight as 3 float4
    uint32_t num_lights;
    uint32_t num_instances;
    uint32_t num_tris;
    uint32_t num_materials;
    uint32_t num_nodes;
    uint32_t num_nodes4;
    // Emissive triangles (RR_PT_FLAG_EMITTERS): world-space (p0, Le.r),
    // (e1, Le.g), (e2, Le.b) per emitter, instance-major; emit_alias is an
    // alias table over their powers luminance(Le) * area (emitter_pick),
    // emit_total the total power.
    const float4* emitters;
    const float2* emit_alias;
    uint32_t num_emitters;
    float emit_total;
};

// An emitter drawn with probability proportional to its power from two
// uniforms: u picks a column of the alias table, uc keeps it or takes its
// alias (one table read instead of a search of prefix sums).
RR_D uint32_t emitter_pick(const DevScene& s, float u, float uc) {
    const uint32_t n = s.num_emitters;
    const uint32_t k = min(uint32_t(u * float(n)), n - 1u);
    const float2 t = __ldg(s.emit_alias + k);
    return uc < t.x ? k : __float_as_uint(t.y);
}

// A ray with its shear constants (triangle test) and its slab-test
// constants: a box plane x is at t = fma(x, inv, alo) for a lower plane and
// fma(x, inv, ahi) for an upper one (see make_ray).
struct Ray {
    float3 o, d, inv;
    float3 alo, ahi;
    float Sx, Sy, Sz;
    int kx, ky, kz;
};

RR_D float comp(float3 v, int k) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

// Per-ray shear constants (Woop, Benthin, Wald, JCGT 2013).
RR_D Ray make_ray(float3 o, float3 d) {
    Ray r;
    r.o = o; r.d = d;
    int kz = 0;
    if (fabsf(d.y) > fabsf(comp(d, kz))) kz = 1;
    if (fabsf(d.z) > fabsf(comp(d, kz))) kz = 2;
    int kx = kz + 1; if (kx == 3) kx = 0;
    int ky = kx + 1; if (ky == 3) ky = 0;
    const float dz = comp(d, kz);
    if (dz < 0.0f) { const int t = kx; kx = ky; ky = t; }
    r.kx = kx; r.ky = ky; r.kz = kz;
    r.Sx = comp(d, kx) / dz;
    r.Sy = comp(d, ky) / dz;
    r.Sz = 1.0f / dz;
    const float sx = fabsf(d.x) < 1e-20f ? copysignf(1e-20f, d.x) : d.x;
    const float sy = fabsf(d.y) < 1e-20f ? copysignf(1e-20f, d.y) : d.y;
    const float sz = fabsf(d.z) < 1e-20f ? copysignf(1e-20f, d.z) : d.z;
    r.inv = f3(1.0f / sx, 1.0f / sy, 1.0f / sz);
    // Slab offsets: t(x) = (x - o) inv is evaluated as fma(x, inv, a) with
    // a = -fl(o inv) -/+ m. The fma rounds once and fl(o inv) and a carry
    // at most 3 u |o inv| between them (u = 2^-24), so m = 2^-22 |o inv|
    // moves near planes nearer and far planes farther than every rounding
    // error; which of a box's lower / upper planes is near follows the sign
    // of inv. Culling therefore stays conservative, as with (x - o) * inv.
    auto offsets = [](float o, float inv, float& alo, float& ahi) {
        const float oi = o * inv;
        const float m = fabsf(oi) * 2.384185791015625e-7f;
        const float anear = -oi - m, afar = -oi + m;
        alo = inv >= 0.0f ? anear : afar;
        ahi = inv >= 0.0f ? afar : anear;
    };
    offsets(o.x, r.inv.x, r.alo.x, r.ahi.x);
    offsets(o.y, r.inv.y, r.alo.y, r.ahi.y);
    offsets(o.z, r.inv.z, r.alo.z, r.ahi.z);
    return r;
}

// Watertight test; two-sided. On hit writes t and the weights of v1, v2.
RR_D bool intersect_triangle(const Ray& r, float3 p0, float3 p1, float3 p2, float tmin,
                             float tmax, float& t, float& bu, float& bv) {
    const float3 A = p0 - r.o, B = p1 - r.o, C = p2 - r.o;
    const float Az0 = comp(A, r.kz), Bz0 = comp(B, r.kz), Cz0 = comp(C, r.kz);
    const float Ax = comp(A, r.kx) - r.Sx * Az0, Ay = comp(A, r.ky) - r.Sy * Az0;
    const float Bx = comp(B, r.kx) - r.Sx * Bz0, By = comp(B, r.ky) - r.Sy * Bz0;
    const float Cx = comp(C, r.kx) - r.Sx * Cz0, Cy = comp(C, r.ky) - r.Sy * Cz0;
    const float U = Cx * By - Cy * Bx;
    const float V = Ax * Cy - Ay * Cx;
    const float W = Bx * Ay - By * Ax;
    if ((U < 0.0f || V < 0.0f || W < 0.0f) && (U > 0.0f || V > 0.0f || W > 0.0f)) return false;
    const float det = U + V + W;
    if (det == 0.0f) return false;
    const float Az = r.Sz * Az0, Bz = r.Sz * Bz0, Cz = r.Sz * Cz0;
    const float T = U * Az + V * Bz + W * Cz;
    const float rcp = 1.0f / det;
    const float tt = T * rcp;
    if (!(tt >= tmin && tt <= tmax)) return false;
    t = tt; bu = V * rcp; bv = W * rcp;
    return true;
}

// Conservative slab test of both children of a node, one fma per plane
// (offsets from make_ray). The far distance is also widened by a few ulps
// for the product's rounding (Ize, JCGT 2013), and the closest-hit bound
// too, so that a box holding a triangle at exactly the current t is opened
// and ties go to the lowest key whatever the visiting order.
RR_D void box_pair(const Ray& r, float4 a, float4 b, float4 c, float tmin, float tmax,
                   bool& h0, bool& h1, float& n0, float& n1) {
    const float ix = r.inv.x, iy = r.inv.y, iz = r.inv.z;
    const float tlim = tmax * 1.00001f;
    {
        const float tx0 = __fmaf_rn(a.x, ix, r.alo.x), tx1 = __fmaf_rn(a.y, ix, r.ahi.x);
        const float ty0 = __fmaf_rn(a.z, iy, r.alo.y), ty1 = __fmaf_rn(a.w, iy, r.ahi.y);
        const float tz0 = __fmaf_rn(c.x, iz, r.alo.z), tz1 = __fmaf_rn(c.y, iz, r.ahi.z);
        const float nn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
        const float ff = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1)) * 1.000002f;
        h0 = nn <= fminf(ff, tlim);
        n0 = nn;
    }
    {
        const float tx0 = __fmaf_rn(b.x, ix, r.alo.x), tx1 = __fmaf_rn(b.y, ix, r.ahi.x);
        const float ty0 = __fmaf_rn(b.z, iy, r.alo.y), ty1 = __fmaf_rn(b.w, iy, r.ahi.y);
        const float tz0 = __fmaf_rn(c.z, iz, r.alo.z), tz1 = __fmaf_rn(c.w, iz, r.ahi.z);
        const float nn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
        const float ff = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1)) * 1.000002f;
        h1 = nn <= fminf(ff, tlim);
        n1 = nn;
    }
}

struct HitRec {
    float t, u, v;
    uint32_t inst, prim, key;
};

constexpr int kStackSize = 64;

// Work counters of one traversal (only maintained when Count = true).
struct TraceWork {
    uint32_t nodes = 0;
    uint32_t tris = 0;
};

// Traversal state of one ray between node steps. node < 0: no inner node
// left, only the postponed leaf (pend_count > 0) to intersect.
struct TravState {
    int node;
    int sp;
    bool found;
    uint32_t visits;
    int pend_first, pend_count;
};

RR_D void trav_begin(TravState& st, HitRec& hit, float tmax) {
    st.node = 0; st.sp = 0; st.found = false; st.visits = 0;
    st.pend_first = 0; st.pend_count = 0;
    hit.t = tmax; hit.key = kNoIndex;
}

// The triangles [first, first + count) of a leaf against the ray; closest
// hit: keeps the lowest (t, key); any hit: returns true at the first hit.
template <bool AnyHit, bool Count>
RR_D bool leaf_tris(const DevScene& s, const Ray& r, float tmin, HitRec& hit, TravState& st, int first, int count,
                    TraceWork* work) {
    for (int i = first; i < first + count; ++i) {
        if (Count) work->tris++;
        const float4 t0 = __ldg(s.tris + i * 3 + 0);
        const float4 t1 = __ldg(s.tris + i * 3 + 1);
        const float4 t2 = __ldg(s.tris + i * 3 + 2);
        float tt, uu, vv;
        if (intersect_triangle(r, f3(t0.x, t0.y, t0.z), f3(t0.w, t1.x, t1.y), f3(t1.z, t1.w, t2.x), tmin, hit.t,
                               tt, uu, vv)) {
            const uint32_t key = __float_as_uint(t2.w);
            if (AnyHit) { hit.t = tt; st.found = true; return true; }
            if (!st.found || tt < hit.t || (tt == hit.t && key < hit.key)) {
                st.found = true;
                hit.t = tt; hit.u = uu; hit.v = vv; hit.key = key;
                hit.inst = __float_as_uint(t2.y); hit.prim = __float_as_uint(t2.z);
            }
        }
    }
    return false;
}

// Traversal stacks of (node, near distance) entries. LocalStack: all in
// local memory. SplitStack: the bottom S entries in shared memory, one
// column per thread of a block of Threads (entry j of a thread at
// col[j * Threads], so a warp's accesses to one depth are consecutive
// words), the deeper ones in local memory. Shared-memory entries do not
// compete with node and triangle fetches for L1 lines.
// N entries: kStackSize for the binary tree (one push per level, at most 60
// levels), kStackSize4 for the 4-wide tree (at most three pushes per level).
constexpr int kStackSize4 = 192;
template <int N = kStackSize>
struct LocalStackN {
    int2 e[N];
    RR_D void put(int i, int2 v) { e[i] = v; }
    RR_D int2 get(int i) const { return e[i]; }
};
using LocalStack = LocalStackN<kStackSize>;
template <int S, int Threads, int N = kStackSize>
struct SplitStack {
    int2* col;
    int2 e[N - S];
    RR_D void put(int i, int2 v) {
        if (i < S) col[i * Threads] = v;
        else e[i - S] = v;
    }
    RR_D int2 get(int i) const { return i < S ? col[i * Threads] : e[i - S]; }
};

// Pops the next stacked node not beyond the current hit; false when none is left.
template <class Stack>
RR_D bool pop_node(TravState& st, const Stack& stack, const HitRec& hit) {
    while (st.sp > 0) {
        --st.sp;
        const int2 e = stack.get(st.sp);
        if (__int_as_float(e.y) <= hit.t) { st.node = e.x; return true; }
    }
    return false;
}

// One node of a closest-hit (AnyHit = false) or any-hit traversal: tests the
// node's two child boxes, intersects the triangles of hit leaf children right
// away, descends into one inner child and pushes the other: closest hit the
// nearer first; any hit the farther first (a shadow ray toward a light sample
// is blocked near its light end more often than near its surface end: 28 %
// fewer node visits on the 1M-triangle room). An any-hit ray only reports
// whether a triangle lies in [tmin, tmax], which no visiting order changes.
// Returns true once the traversal is finished (stack empty, or any hit).
// Postpone: a lane keeps its first leaf child for later and goes on with
// inner nodes; the step intersects the kept leaf once every lane of the warp
// still traversing holds one (or the lane has no inner node left), so the
// warp runs its leaves' triangle loops side by side instead of one lane's
// at a time (Aila and Laine 2009). Culling meanwhile uses the hit found so
// far, which only visits more, and the kept (t, key) minimum does not depend
// on the order, so the result is the same.
template <bool AnyHit, bool Count, bool Postpone = false, class Stack>
RR_D bool trace_step(const DevScene& s, const Ray& r, float tmin, HitRec& hit, TravState& st,
                     Stack& stack, TraceWork* work) {
    if constexpr (Postpone) {
        const bool all_hold = __all_sync(__activemask(), st.pend_count > 0);
        if (st.pend_count > 0 && (st.node < 0 || all_hold)) {
            if (leaf_tris<AnyHit, Count>(s, r, tmin, hit, st, st.pend_first, st.pend_count, work)) return true;
            st.pend_count = 0;
            if (st.node >= 0) return false;
            return !pop_node(st, stack, hit);
        }
    }
    // A tree visits each inner node at most once; the bound only guards
    // against a malformed node array turning into an endless loop.
    if (++st.visits > s.num_nodes + 1) return true;
    const int node = st.node;
    const float4 a = __ldg(s.nodes + node * 4 + 0);
    const float4 b = __ldg(s.nodes + node * 4 + 1);
    const float4 c = __ldg(s.nodes + node * 4 + 2);
    const int4 d = __ldg(reinterpret_cast<const int4*>(s.nodes) + node * 4 + 3);
    if (Count) work->nodes++;
    bool h0, h1; float n0, n1;
    box_pair(r, a, b, c, tmin, hit.t, h0, h1, n0, n1);
    #pragma unroll
    for (int k = 0; k < 2; ++k) {
        const bool hk = k == 0 ? h0 : h1;
        const int child = k == 0 ? d.x : d.y;
        if (hk && child < 0) {
            const int first = ~child;
            const int count = k == 0 ? d.z : d.w;
            if constexpr (Postpone) {
                if (st.pend_count == 0) { st.pend_first = first; st.pend_count = count; continue; }
            }
            if (leaf_tris<AnyHit, Count>(s, r, tmin, hit, st, first, count, work)) return true;
        }
    }
    const bool i0 = h0 && d.x >= 0 && n0 <= hit.t;
    const bool i1 = h1 && d.y >= 0 && n1 <= hit.t;
    if (i0 && i1) {
        const bool first0 = AnyHit ? n0 > n1 : n0 <= n1;
        stack.put(st.sp, make_int2(first0 ? d.y : d.x, __float_as_int(first0 ? n1 : n0)));
        ++st.sp;
        st.node = first0 ? d.x : d.y;
    } else if (i0) {
        st.node = d.x;
    } else if (i1) {
        st.node = d.y;
    } else {
        if (pop_node(st, stack, hit)) return false;
        if constexpr (Postpone) {
            if (st.pend_count > 0) { st.node = -1; return false; }
        }
        return true;
    }
    return false;
}

// One node of the 4-wide tree (8 float4 per node: lo.x, hi.x, lo.y, hi.y,
// lo.z, hi.z of children 0..3, their references and their triangle counts;
// unused slots hold a point box at 1e30, never reached). The four child
// boxes are tested with box_pair's arithmetic, hit leaf children are
// intersected right away, and the hit inner children are visited in
// distance order (closest hit nearest first, any hit farthest first, ties
// by slot): the first goes on, the others are pushed so that they pop in
// that order. One step reads one 128-byte line where the binary tree's
// steps read 64 bytes each, and a ray takes about half as many steps.
RR_D void box_quad(const Ray& r, float4 lx, float4 hx, float4 ly, float4 hy, float4 lz, float4 hz, float tmin,
                   float tmax, bool* h, float* nr) {
    const float ix = r.inv.x, iy = r.inv.y, iz = r.inv.z;
    const float tlim = tmax * 1.00001f;
    const float Lx[4] = {lx.x, lx.y, lx.z, lx.w}, Hx[4] = {hx.x, hx.y, hx.z, hx.w};
    const float Ly[4] = {ly.x, ly.y, ly.z, ly.w}, Hy[4] = {hy.x, hy.y, hy.z, hy.w};
    const float Lz[4] = {lz.x, lz.y, lz.z, lz.w}, Hz[4] = {hz.x, hz.y, hz.z, hz.w};
    #pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float tx0 = __fmaf_rn(Lx[k], ix, r.alo.x), tx1 = __fmaf_rn(Hx[k], ix, r.ahi.x);
        const float ty0 = __fmaf_rn(Ly[k], iy, r.alo.y), ty1 = __fmaf_rn(Hy[k], iy, r.ahi.y);
        const float tz0 = __fmaf_rn(Lz[k], iz, r.alo.z), tz1 = __fmaf_rn(Hz[k], iz, r.ahi.z);
        const float nn = fmaxf(fmaxf(fminf(tx0, tx1), fminf(ty0, ty1)), fmaxf(fminf(tz0, tz1), tmin));
        const float ff = fminf(fminf(fmaxf(tx0, tx1), fmaxf(ty0, ty1)), fmaxf(tz0, tz1)) * 1.000002f;
        h[k] = nn <= fminf(ff, tlim);
        nr[k] = nn;
    }
}

template <bool AnyHit, bool Count, class Stack>
RR_D bool trace_step4(const DevScene& s, const Ray& r, float tmin, HitRec& hit, TravState& st, Stack& stack,
                      TraceWork* work) {
    if (++st.visits > s.num_nodes4 + 1) return true;
    const float4* q = s.nodes4 + size_t(st.node) * 8;
    const float4 lx = __ldg(q + 0), hx = __ldg(q + 1), ly = __ldg(q + 2), hy = __ldg(q + 3);
    const float4 lz = __ldg(q + 4), hz = __ldg(q + 5);
    const int4 ref = __ldg(reinterpret_cast<const int4*>(q + 6));
    const int4 cnt = __ldg(reinterpret_cast<const int4*>(q + 7));
    if (Count) work->nodes++;
    bool h[4];
    float nr[4];
    box_quad(r, lx, hx, ly, hy, lz, hz, tmin, hit.t, h, nr);
    const int R[4] = {ref.x, ref.y, ref.z, ref.w}, K[4] = {cnt.x, cnt.y, cnt.z, cnt.w};
    #pragma unroll
    for (int k = 0; k < 4; ++k)
        if (h[k] && R[k] < 0 && leaf_tris<AnyHit, Count>(s, r, tmin, hit, st, ~R[k], K[k], work)) return true;
    // inner children still in reach, as (key, node) with misses at +inf; a
    // sorting network orders them (closest hit ascending distance, any hit
    // descending), ties keep slot order
    float key[4];
    int nd[4];
    int m = 0;
    #pragma unroll
    for (int k = 0; k < 4; ++k) {
        const bool in = h[k] && R[k] >= 0 && nr[k] <= hit.t;
        m += in ? 1 : 0;
        key[k] = in ? (AnyHit ? -nr[k] : nr[k]) : INFINITY;
        nd[k] = R[k];
    }
    auto cswap = [&](int i, int j) {
        const bool sw = key[j] < key[i];
        const float ki = key[i], kj = key[j];
        const int ni = nd[i], nj = nd[j];
        key[i] = sw ? kj : ki; key[j] = sw ? ki : kj;
        nd[i] = sw ? nj : ni; nd[j] = sw ? ni : nj;
    };
    cswap(0, 1); cswap(2, 3); cswap(0, 2); cswap(1, 3); cswap(1, 2);
    if (m == 0) return !pop_node(st, stack, hit);
    // push entries m-1 .. 1 (the farthest in visiting order deepest), go on with entry 0
    #pragma unroll
    for (int k = 3; k >= 1; --k) {
        if (k < m) {
            stack.put(st.sp, make_int2(nd[k], __float_as_int(AnyHit ? -key[k] : key[k])));
            ++st.sp;
        }
    }
    st.node = nd[0];
    return false;
}

// Closest hit (AnyHit = false) or any hit (AnyHit = true) in [tmin, tmax],
// one ray per thread. Returns true on hit; `hit` is filled for closest hit.
template <bool AnyHit, bool Count = false>
RR_D bool trace(const DevScene& s, const Ray& r, float tmin, float tmax, HitRec& hit, TraceWork* work = nullptr) {
    LocalStack stack;
    TravState st;
    trav_begin(st, hit, tmax);
    while (!trace_step<AnyHit, Count>(s, r, tmin, hit, st, stack, work)) {}
    return st.found;
}

// trace() over the 4-wide tree.
template <bool AnyHit, bool Count = false>
RR_D bool trace4(const DevScene& s, const Ray& r, float tmin, float tmax, HitRec& hit, TraceWork* work = nullptr) {
    LocalStackN<kStackSize4> stack;
    TravState st;
    trav_begin(st, hit, tmax);
    while (!trace_step4<AnyHit, Count>(s, r, tmin, hit, st, stack, work)) {}
    return st.found;
}

// Hit attributes (pathtracer.slang:69-118 / restir_di.slang:108-144):
// instance -> mesh -> 3 indices -> 3 vertices, barycentric interpolation in
// object space, then the row-major instance transform (normals use the upper
// 3x3, not the inverse transpose, as the reference does).
struct Surface {
    float3 pos, normal;
    uint32_t material;
};

// The hit triangle's unit geometric normal in world space, from its
// vertices transformed as the scene's world-space triangles are.
RR_D float3 hit_geometric_normal(const DevScene& s, uint32_t inst_idx, uint32_t prim) {
    const float4* ip = s.instances + inst_idx * 5;
    const float4 r0 = __ldg(ip + 0), r1 = __ldg(ip + 1), r2 = __ldg(ip + 2);
    const uint32_t mesh_index = __float_as_uint(__ldg(ip + 4).x);
    const uint4 m0 = __ldg(s.meshes + mesh_index * 2 + 0);
    const uint32_t base = m0.z / 4u + prim * 3u;
    const uint32_t i0 = __ldg(s.indices + base), i1 = __ldg(s.indices + base + 1), i2 = __ldg(s.indices + base + 2);
    const float3 p0 = mul_rows_point(r0, r1, r2, xyz(__ldg(s.vertices + (m0.x + i0) * 3)), 1.0f);
    const float3 p1 = mul_rows_point(r0, r1, r2, xyz(__ldg(s.vertices + (m0.x + i1) * 3)), 1.0f);
    const float3 p2 = mul_rows_point(r0, r1, r2, xyz(__ldg(s.vertices + (m0.x + i2) * 3)), 1.0f);
    return normalize(cross(p1 - p0, p2 - p0));
}

RR_D Surface hit_surface(const DevScene& s, uint32_t inst_idx, uint32_t prim, float bu, float bv) {
    const float4* ip = s.instances + inst_idx * 5;
    const float4 r0 = __ldg(ip + 0), r1 = __ldg(ip + 1), r2 = __ldg(ip + 2);
    const uint32_t mesh_index = __float_as_uint(__ldg(ip + 4).x);
    const uint4 m0 = __ldg(s.meshes + mesh_index * 2 + 0);  // vertex_base, vertex_count, index_byte_offset, index_count
    const uint4 m1 = __ldg(s.meshes + mesh_index * 2 + 1);  // material_index, pad
    const uint32_t base = m0.z / 4u + prim * 3u;
    const uint32_t i0 = __ldg(s.indices + base), i1 = __ldg(s.indices + base + 1), i2 = __ldg(s.indices + base + 2);
    const float4 va0 = __ldg(s.vertices + (m0.x + i0) * 3), vb0 = __ldg(s.vertices + (m0.x + i0) * 3 + 1);
    const float4 va1 = __ldg(s.vertices + (m0.x + i1) * 3), vb1 = __ldg(s.vertices + (m0.x + i1) * 3 + 1);
    const float4 va2 = __ldg(s.vertices + (m0.x + i2) * 3), vb2 = __ldg(s.vertices + (m0.x + i2) * 3 + 1);
    const float b0 = 1.0f - bu - bv;
    const float3 lp = b0 * xyz(va0) + bu * xyz(va1) + bv * xyz(va2);
    const float3 n0 = f3(va0.w, vb0.x, vb0.y), n1 = f3(va1.w, vb1.x, vb1.y), n2 = f3(va2.w, vb2.x, vb2.y);
    const float3 ln = normalize(b0 * n0 + bu * n1 + bv * n2);
    Surface sf;
    sf.pos = mul_rows_point(r0, r1, r2, lp, 1.0f);
    sf.normal = normalize(mul_rows_dir(r0, r1, r2, ln));
    sf.material = m1.x;
    return sf;
}

} // namespace rr
