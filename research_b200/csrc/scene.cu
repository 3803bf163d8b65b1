// scene.cu — context and scene entry points of rr_cuda.h.
//
// rr_scene_create replaces Scene::upload (Scene.cpp:255-515): the flat
// GpuScene arrays go to the device unchanged (vertices, indices, meshes,
// instances, lights), materials are repacked to two float4 per material,
// and instead of the driver BLAS/TLAS build (Scene.cpp:449-507) every
// instance's triangles are transformed to world space on the host
// (mul(transform, float4(p, 1)), row-major) and one BVH2 is built over them.

#include "rr_internal.h"

#include <chrono>
#include <cmath>
#include <cstring>
#include <thread>

rr_status rr_fail(rr_ctx* ctx, rr_status st, const char* fmt, ...) {
    if (ctx) {
        char buf[1024];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof(buf), fmt, ap);
        va_end(ap);
        ctx->last_error = buf;
    }
    return st;
}

extern "C" {

uint32_t rr_abi_version(void) { return RR_ABI_VERSION; }

const char* rr_status_string(rr_status s) {
    switch (s) {
    case RR_OK: return "RR_OK";
    case RR_ERR_INVALID_ARGUMENT: return "RR_ERR_INVALID_ARGUMENT";
    case RR_ERR_CUDA: return "RR_ERR_CUDA";
    case RR_ERR_OUT_OF_MEMORY: return "RR_ERR_OUT_OF_MEMORY";
    case RR_ERR_NOT_INITIALIZED: return "RR_ERR_NOT_INITIALIZED";
    case RR_ERR_QUEUE_OVERFLOW: return "RR_ERR_QUEUE_OVERFLOW";
    case RR_ERR_TIMEOUT: return "RR_ERR_TIMEOUT";
    case RR_ERR_UNSUPPORTED: return "RR_ERR_UNSUPPORTED";
    }
    return "RR_ERR_UNKNOWN";
}

rr_status rr_ctx_create(int device_ordinal, rr_ctx** out) {
    if (!out) return RR_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || n == 0) return RR_ERR_CUDA;
    if (device_ordinal < 0 || device_ordinal >= n) return RR_ERR_INVALID_ARGUMENT;
    if (cudaSetDevice(device_ordinal) != cudaSuccess) return RR_ERR_CUDA;
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, device_ordinal) != cudaSuccess) return RR_ERR_CUDA;
    if (prop.major < 10) return RR_ERR_UNSUPPORTED;  // built for sm_100a only
    rr_ctx* ctx = new rr_ctx;
    ctx->device = device_ordinal;
    ctx->sm_count = prop.multiProcessorCount;
    if (cudaMalloc(&ctx->counters, sizeof(uint32_t) * kCounterWords) != cudaSuccess) {
        delete ctx;
        return RR_ERR_OUT_OF_MEMORY;
    }
    cudaMemset(ctx->counters, 0, sizeof(uint32_t) * kCounterWords);
    if (cudaMalloc(&ctx->work64, sizeof(unsigned long long) * 4) != cudaSuccess) {
        cudaFree(ctx->counters);
        delete ctx;
        return RR_ERR_OUT_OF_MEMORY;
    }
    cudaMemset(ctx->work64, 0, sizeof(unsigned long long) * 4);
    *out = ctx;
    return RR_OK;
}

static void free_queues(rr_ctx* ctx) {
    rr_pt_queues& q = ctx->pt;
    for (int i = 0; i < 2; ++i) { cudaFree(q.ray_a[i]); cudaFree(q.ray_b[i]); cudaFree(q.ray_c[i]); }
    cudaFree(q.hits); cudaFree(q.shadow_a); cudaFree(q.shadow_b); cudaFree(q.shadow_c);
    q = rr_pt_queues();
}

rr_status rr_ctx_destroy(rr_ctx* ctx) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    cudaSetDevice(ctx->device);
    free_queues(ctx);
    cudaDeviceSynchronize();
    for (const rr_stage_event& ev : ctx->pending) { cudaEventDestroy(ev.start); cudaEventDestroy(ev.stop); }
    for (cudaEvent_t e : ctx->event_pool) cudaEventDestroy(e);
    cudaFree(ctx->counters);
    cudaFree(ctx->work64);
    cudaFree(ctx->mse_partial);
    cudaFree(ctx->atrous_nrm);
    cudaFree(ctx->atrous_wt);
    if (ctx->atrous_error) cudaFreeHost(ctx->atrous_error);
    for (int b = 0; b < kMaxBounces; ++b) {
        if (ctx->shaded[b]) cudaEventDestroy(ctx->shaded[b]);
        if (ctx->shadowed[b]) cudaEventDestroy(ctx->shadowed[b]);
    }
    if (ctx->side) cudaStreamDestroy(ctx->side);
    cudaFree(ctx->wave_state);
    cudaFree(ctx->wave_counters);
    delete ctx;
    return RR_OK;
}

rr_status rr_ctx_set_queue_limit(rr_ctx* ctx, uint64_t max_entries) {
    if (!ctx) return RR_ERR_INVALID_ARGUMENT;
    ctx->queue_limit = size_t(max_entries);
    return RR_OK;
}

rr_status rr_last_error(const rr_ctx* ctx, char* buf, size_t n) {
    if (!ctx || !buf || n == 0) return RR_ERR_INVALID_ARGUMENT;
    std::strncpy(buf, ctx->last_error.c_str(), n - 1);
    buf[n - 1] = '\0';
    return RR_OK;
}

static inline float row_point(const float* M, int r, const float* p) {
    return M[r * 4 + 0] * p[0] + M[r * 4 + 1] * p[1] + M[r * 4 + 2] * p[2] + M[r * 4 + 3] * 1.0f;
}

// Vose's alias table over weights w (FP64, w_k > 0): column k keeps a draw
// with probability prob_k and hands it to alias_k otherwise, so that column
// k is picked with probability w_k / sum(w). Entry k is (prob_k, alias_k as
// float bits). Columns are paired in stack order (the last "small" with the
// last "large"); columns left over by rounding keep every draw.
static std::vector<float2> alias_table(const std::vector<double>& w) {
    const size_t n = w.size();
    std::vector<float2> t(n);
    if (n == 0) return t;
    double total = 0.0;
    for (double x : w) total += x;
    std::vector<double> sc(n);
    std::vector<uint32_t> small, large;
    for (size_t i = 0; i < n; ++i) {
        sc[i] = w[i] * double(n) / total;
        (sc[i] < 1.0 ? small : large).push_back(uint32_t(i));
    }
    std::vector<float> prob(n, 1.0f);
    std::vector<uint32_t> alias(n);
    for (size_t i = 0; i < n; ++i) alias[i] = uint32_t(i);
    while (!small.empty() && !large.empty()) {
        const uint32_t a = small.back();
        small.pop_back();
        const uint32_t b = large.back();
        large.pop_back();
        prob[a] = float(sc[a]);
        alias[a] = b;
        sc[b] = (sc[b] + sc[a]) - 1.0;
        (sc[b] < 1.0 ? small : large).push_back(b);
    }
    for (size_t i = 0; i < n; ++i) {
        t[i].x = prob[i];
        std::memcpy(&t[i].y, &alias[i], 4);
    }
    return t;
}

rr_status rr_scene_create(rr_ctx* ctx, const rr_scene_desc* d, rr_scene** out) {
    if (!ctx || !d || !out) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "null argument");
    *out = nullptr;
    // Scene::upload throws on an empty scene (Scene.cpp:261-262).
    if (d->vertex_count == 0 || !d->vertices) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "scene has no vertices");
    if (d->index_count == 0 || !d->indices) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "scene has no indices");
    if (d->mesh_count == 0 || !d->meshes) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "scene has no meshes");
    if (d->material_count == 0 || !d->materials) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "scene has no materials");
    if (d->instance_count == 0 || !d->instances) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "scene has no instances");
    if (d->light_count > 0 && !d->lights) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "null light array");
    for (uint32_t m = 0; m < d->mesh_count; ++m) {
        const GpuMesh& g = d->meshes[m];
        if (g.index_byte_offset % 4u != 0 || g.index_count % 3u != 0)
            return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "mesh %u: misaligned index range", m);
        const uint64_t end = uint64_t(g.index_byte_offset / 4u) + g.index_count;
        if (end > d->index_count) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "mesh %u: index range out of bounds", m);
        if (g.material_index >= d->material_count)
            return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "mesh %u: material %u out of range", m, g.material_index);
        for (uint64_t k = g.index_byte_offset / 4u; k < end; ++k)
            if (uint64_t(g.vertex_base) + d->indices[k] >= d->vertex_count)
                return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "mesh %u: vertex index out of range", m);
    }
    uint64_t ntri64 = 0;
    for (uint32_t i = 0; i < d->instance_count; ++i) {
        if (d->instances[i].mesh_index >= d->mesh_count)
            return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "instance %u: mesh out of range", i);
        ntri64 += d->meshes[d->instances[i].mesh_index].index_count / 3u;
    }
    if (ntri64 == 0 || ntri64 >= (1ull << 31)) return rr_fail(ctx, RR_ERR_INVALID_ARGUMENT, "bad triangle count");
    const uint32_t ntri = uint32_t(ntri64);

    // Flatten to world space, instance-major (the tie-break key order).
    auto t0 = std::chrono::steady_clock::now();
    std::vector<float> world(size_t(ntri) * 9);
    std::vector<uint32_t> tri_inst(ntri), tri_prim(ntri);
    {
        uint32_t k = 0;
        for (uint32_t i = 0; i < d->instance_count; ++i) {
            const float* M = d->instances[i].transform;
            const GpuMesh& g = d->meshes[d->instances[i].mesh_index];
            const uint32_t nt = g.index_count / 3u, ib = g.index_byte_offset / 4u;
            for (uint32_t j = 0; j < nt; ++j, ++k) {
                for (int c = 0; c < 3; ++c) {
                    const float* p = d->vertices[g.vertex_base + d->indices[ib + 3 * j + c]].pos;
                    for (int r = 0; r < 3; ++r) world[size_t(k) * 9 + c * 3 + r] = row_point(M, r, p);
                }
                tri_inst[k] = i; tri_prim[k] = j;
            }
        }
    }
    const int threads = int(std::max(1u, std::thread::hardware_concurrency()));
    rr::BvhBuild bvh = rr::build_bvh(world, threads);
    auto t1 = std::chrono::steady_clock::now();

    std::vector<float4> trirec(size_t(ntri) * 3);
    for (uint32_t i = 0; i < ntri; ++i) {
        const uint32_t t = bvh.order[i];
        const float* w = &world[size_t(t) * 9];
        float4 a, b, c;
        a.x = w[0]; a.y = w[1]; a.z = w[2]; a.w = w[3];
        b.x = w[4]; b.y = w[5]; b.z = w[6]; b.w = w[7];
        c.x = w[8];
        std::memcpy(&c.y, &tri_inst[t], 4);
        std::memcpy(&c.z, &tri_prim[t], 4);
        std::memcpy(&c.w, &t, 4);
        trirec[size_t(i) * 3] = a; trirec[size_t(i) * 3 + 1] = b; trirec[size_t(i) * 3 + 2] = c;
    }
    // Emitter table: every triangle of an emissive material with non-zero
    // area, instance-major, and an alias table over their powers
    // luminance(Le) * area (alias_table below).
    std::vector<float4> emit;
    std::vector<double> emit_power;
    float emit_total = 0.0f;
    {
        double acc = 0.0;
        for (uint32_t k = 0; k < ntri; ++k) {
            const GpuMaterial& g = d->materials[d->meshes[d->instances[tri_inst[k]].mesh_index].material_index];
            if (!(g.emissive[0] > 0.0f || g.emissive[1] > 0.0f || g.emissive[2] > 0.0f)) continue;
            const float* w = &world[size_t(k) * 9];
            const float e1[3] = {w[3] - w[0], w[4] - w[1], w[5] - w[2]};
            const float e2[3] = {w[6] - w[0], w[7] - w[1], w[8] - w[2]};
            const float c[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2],
                                e1[0] * e2[1] - e1[1] * e2[0]};
            const float area = 0.5f * std::sqrt(c[0] * c[0] + c[1] * c[1] + c[2] * c[2]);
            if (!(area > 0.0f)) continue;
            const float lum = 0.2126f * g.emissive[0] + 0.7152f * g.emissive[1] + 0.0722f * g.emissive[2];
            acc += double(lum) * double(area);
            emit.push_back(make_float4(w[0], w[1], w[2], g.emissive[0]));
            emit.push_back(make_float4(e1[0], e1[1], e1[2], g.emissive[1]));
            emit.push_back(make_float4(e2[0], e2[1], e2[2], g.emissive[2]));
            emit_power.push_back(double(lum) * double(area));
        }
        emit_total = float(acc);
    }
    const std::vector<float2> emit_alias = alias_table(emit_power);
    std::vector<float4> mats(size_t(d->material_count) * 2);
    for (uint32_t m = 0; m < d->material_count; ++m) {
        const GpuMaterial& g = d->materials[m];
        mats[2 * m] = make_float4(g.base_color[0], g.base_color[1], g.base_color[2], g.metallic);
        mats[2 * m + 1] = make_float4(g.emissive[0], g.emissive[1], g.emissive[2], g.roughness);
    }

    rr_scene* s = new rr_scene;
    s->ctx = ctx;
    RR_TRY_CUDA(ctx, cudaSetDevice(ctx->device));
    auto upload = [&](const void* src, size_t bytes, void** dst) -> rr_status {
        if (bytes == 0) bytes = 16;
        void* p = nullptr;
        cudaError_t e = cudaMalloc(&p, bytes);
        if (e != cudaSuccess) return rr_fail(ctx, RR_ERR_OUT_OF_MEMORY, "cudaMalloc(%zu): %s", bytes, cudaGetErrorString(e));
        s->allocations.push_back(p);
        s->stats.device_bytes += bytes;
        if (src) {
            e = cudaMemcpy(p, src, bytes, cudaMemcpyHostToDevice);
            if (e != cudaSuccess) return rr_fail(ctx, RR_ERR_CUDA, "cudaMemcpy: %s", cudaGetErrorString(e));
        }
        *dst = p;
        return RR_OK;
    };
    void* p;
    rr_status st;
#define RR_UP(src, bytes, field, type)                                           \
    if ((st = upload((src), (bytes), &p)) != RR_OK) { rr_scene_destroy(s); return st; } \
    s->dev.field = reinterpret_cast<type>(p);
    RR_UP(bvh.nodes.data(), bvh.nodes.size() * sizeof(float4), nodes, const float4*);
    RR_UP(bvh.nodes4.data(), bvh.nodes4.size() * sizeof(float4), nodes4, const float4*);
    RR_UP(trirec.data(), trirec.size() * sizeof(float4), tris, const float4*);
    RR_UP(d->vertices, size_t(d->vertex_count) * sizeof(GpuVertex), vertices, const float4*);
    RR_UP(d->indices, size_t(d->index_count) * 4, indices, const uint32_t*);
    RR_UP(d->meshes, size_t(d->mesh_count) * sizeof(GpuMesh), meshes, const uint4*);
    RR_UP(d->instances, size_t(d->instance_count) * sizeof(GpuInstance), instances, const float4*);
    RR_UP(mats.data(), mats.size() * sizeof(float4), materials, const float4*);
    RR_UP(d->light_count ? d->lights : nullptr, size_t(d->light_count) * sizeof(GpuLight), lights, const float4*);
    RR_UP(emit.empty() ? nullptr : emit.data(), emit.size() * sizeof(float4), emitters, const float4*);
    RR_UP(emit_alias.empty() ? nullptr : emit_alias.data(), emit_alias.size() * sizeof(float2), emit_alias,
          const float2*);
#undef RR_UP
    s->dev.num_emitters = uint32_t(emit_power.size());
    s->dev.emit_total = emit_total;
    s->dev.num_lights = d->light_count;
    s->dev.num_instances = d->instance_count;
    s->dev.num_tris = ntri;
    s->dev.num_materials = d->material_count;
    s->dev.num_nodes = uint32_t(bvh.nodes.size() / 4);
    s->dev.num_nodes4 = uint32_t(bvh.nodes4.size() / 8);
    auto t2 = std::chrono::steady_clock::now();
    s->stats.triangle_count = ntri;
    s->stats.bvh_node_count = uint32_t(bvh.nodes.size() / 4);
    s->stats.bvh_max_depth = bvh.max_depth;
    s->stats.bvh4_node_count = uint32_t(bvh.nodes4.size() / 8);
    s->stats.light_count = d->light_count;
    s->stats.build_ms = std::chrono::duration<double, std::milli>(t1 - t0).count();
    s->stats.upload_ms = std::chrono::duration<double, std::milli>(t2 - t1).count();
    *out = s;
    return RR_OK;
}

rr_status rr_scene_destroy(rr_scene* s) {
    if (!s) return RR_ERR_INVALID_ARGUMENT;
    if (s->ctx) cudaSetDevice(s->ctx->device);
    for (void* p : s->allocations) cudaFree(p);
    delete s;
    return RR_OK;
}

rr_status rr_scene_get_stats(const rr_scene* s, rr_scene_stats* out) {
    if (!s || !out) return RR_ERR_INVALID_ARGUMENT;
    *out = s->stats;
    return RR_OK;
}

} // extern "C"
