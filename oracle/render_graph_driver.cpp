// render_graph_driver.cpp — drives the CUDA RenderPass adapters
// (research_b200/adapters/rr_passes.h) through the reference renderer's own
// rr::render::RenderGraph (src/render/RenderGraph.cpp, compiled unmodified
// from the reference checkout by oracle/Makefile, target `ref`), the way the
// reference's Application wires its accumulate-mode and ReSTIR DI passes
// (Application.cpp:218-266): path tracer → accumulate, ReSTIR DI → A-trous
// on the DI output with the DI G-buffer. TEST INFRASTRUCTURE ONLY: the tests
// call it through ctypes and compare the images with the oracle.

#include "render/FrameContext.h"
#include "render/RenderGraph.h"

#include "rr_passes.h"

#include <cuda_runtime.h>

#include <memory>
#include <vector>

namespace {

using namespace rr::cuda_passes;

struct Graph {
    rr::render::RenderGraph graph;
    PathTracerCudaPass* pt = nullptr;
    AccumulateCudaPass* acc = nullptr;
    ReSTIRDICudaPass* di = nullptr;
    AtrousCudaPass* atrous = nullptr;
    std::vector<CudaPassBase*> passes;
    uint32_t frame_index = 0;
};

template <class T> T* add(Graph* g, std::unique_ptr<T> p) {
    T* raw = p.get();
    g->passes.push_back(raw);
    g->graph.add_pass(std::move(p));
    return raw;
}

} // namespace

extern "C" {

// di = {num_initial_candidates, spatial_num_neighbors, spatial_radius}
void* rrg_create(rr_ctx* ctx, const rr_scene* scene, uint32_t width, uint32_t height, uint32_t max_bounces,
                 const uint32_t di[3], uint32_t atrous_iterations) {
    auto* g = new Graph;
    const rr::rhi::Extent2D ext{width, height};
    g->pt = add(g, std::make_unique<PathTracerCudaPass>(ctx, ext));
    g->acc = add(g, std::make_unique<AccumulateCudaPass>(ctx, ext));
    g->di = add(g, std::make_unique<ReSTIRDICudaPass>(ctx, ext));
    g->atrous = add(g, std::make_unique<AtrousCudaPass>(ctx, ext));
    g->pt->set_scene(scene);
    g->pt->max_bounces = max_bounces;
    g->acc->set_input(g->pt->radiance());
    g->acc->camera_moved = true;
    g->di->set_scene(scene);
    g->di->num_initial_candidates = di[0];
    g->di->spatial_num_neighbors = di[1];
    g->di->spatial_radius = di[2];
    g->atrous->set_input(g->di->output());
    g->atrous->set_gbuffer(g->di->gbuffer_position(), g->di->gbuffer_normal());
    g->atrous->iterations = atrous_iterations;
    return g;
}

void rrg_destroy(void* gv) { delete static_cast<Graph*>(gv); }

int rrg_pass_count(void* gv) { return int(static_cast<Graph*>(gv)->passes.size()); }

const char* rrg_pass_name(void* gv, int i) { return static_cast<Graph*>(gv)->passes[size_t(i)]->name(); }

// The first output's name, format and extent from reflect().
const char* rrg_pass_output(void* gv, int i, int* format, uint32_t* width, uint32_t* height) {
    static thread_local std::string name;
    const auto r = static_cast<Graph*>(gv)->passes[size_t(i)]->reflect();
    name = r.outputs.empty() ? std::string() : r.outputs[0].name;
    *format = r.outputs.empty() ? 0 : int(r.outputs[0].format);
    *width = r.outputs.empty() ? 0u : r.outputs[0].extent.width;
    *height = r.outputs.empty() ? 0u : r.outputs[0].extent.height;
    return name.c_str();
}

void rrg_set_enabled(void* gv, int i, int enabled) {
    static_cast<Graph*>(gv)->passes[size_t(i)]->set_enabled(enabled != 0);
}

void rrg_set_camera(void* gv, const GpuCameraData* cam) {
    auto* g = static_cast<Graph*>(gv);
    g->pt->set_camera(*cam);
    g->di->set_camera(*cam);
}

void rrg_set_stream(void* gv, void* stream) {
    for (CudaPassBase* p : static_cast<Graph*>(gv)->passes) p->set_stream(stream);
}

// One frame: RenderGraph::execute over the enabled passes in insertion order.
void rrg_execute(void* gv) {
    auto* g = static_cast<Graph*>(gv);
    rr::render::FrameContext fc{};
    fc.frame_index = g->frame_index++;
    g->graph.execute(fc);
}

int rrg_status(void* gv, int i) { return int(static_cast<Graph*>(gv)->passes[size_t(i)]->last_status()); }

// 0 radiance, 1 accumulated, 2 G-buffer position, 3 G-buffer normal, 4 DI output, 5 A-trous output
const float* rrg_image(void* gv, int which) {
    auto* g = static_cast<Graph*>(gv);
    switch (which) {
    case 0: return g->pt->radiance();
    case 1: return g->acc->accumulated();
    case 2: return g->di->gbuffer_position();
    case 3: return g->di->gbuffer_normal();
    case 4: return g->di->output();
    default: return g->atrous->output();
    }
}

// Copies image `which` (W x H RGBA32F) to host memory; 0 on success.
int rrg_read_image(void* gv, int which, float* host, size_t bytes) {
    return cudaMemcpy(host, rrg_image(gv, which), bytes, cudaMemcpyDeviceToHost) == cudaSuccess ? 0 : 1;
}

} // extern "C"
