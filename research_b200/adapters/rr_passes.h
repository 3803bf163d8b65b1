// rr_passes.h — the CUDA passes as rr::render::RenderPass subclasses, for a
// host that keeps the reference renderer's pass interface
// (src/render/RenderPass.h:11-48, src/render/FrameContext.h:26-41; build
// with the reference's src/ on the include path). Each class stands in for
// one reference pass, with its name()-visible role, its public tuning fields
// and its wiring setters, and calls the C ABI (include/rr_cuda.h):
//
//   PathTracerCudaPass  ← rr::passes::pathtracer::PathTracerPass
//                         (PathTracerPass.h:21-60, execute PathTracerPass.cpp:170-224)
//   AccumulateCudaPass  ← rr::passes::accumulate::AccumulatePass
//                         (AccumulatePass.h:15-47, execute AccumulatePass.cpp:167-218)
//   ReSTIRDICudaPass    ← rr::passes::restir_di::ReSTIRDIPass
//                         (ReSTIRDIPass.h:24-93, execute ReSTIRDIPass.cpp:306-446)
//   AtrousCudaPass      ← rr::passes::denoise::AtrousPass
//                         (AtrousPass.h:15-58, execute AtrousPass.cpp:243-306)
//
// What changes at the boundary, and why:
//   - initialize(Device&, SlangSession&, BindlessRegistry&, Extent2D)
//     becomes the constructor (rr_ctx*, Extent2D): there is no Vulkan device,
//     shader session or bindless heap; each pass allocates its output images
//     in device memory as the reference's create_images does, and
//     on_resize() re-creates them.
//   - Bindless indices become device pointers: the wiring setters take the
//     producing pass's images (set_input, set_gbuffer), and output images are
//     returned by accessors.
//   - The scene and the camera block: FrameContext carries the reference's
//     rr::scene::Scene, which a CUDA host does not have, so set_scene() takes
//     the uploaded rr_scene and set_camera() the frame's GpuCameraData (the
//     block Scene::update_camera writes, Scene.cpp:554-585).
//   - Work is enqueued on the CUDA stream given to set_stream() (default:
//     the legacy default stream) instead of FrameContext::command_recorder.
//   - execute() returns silently when the pass is not ready, as the
//     reference's passes do (PathTracerPass.cpp:172-174,
//     AtrousPass.cpp:245-247); last_status() reports why (the C ABI status of
//     the last call, RR_ERR_NOT_INITIALIZED when inputs were missing).
#pragma once

#include "render/FrameContext.h"
#include "render/RenderPass.h"
#include "rhi/Types.h"

#include "rr_cuda.h"

#include <cstdint>

namespace rr::cuda_passes {

// A W x H RGBA32F image in device memory, owned by a pass.
class DeviceImage {
public:
    DeviceImage() = default;
    ~DeviceImage();
    DeviceImage(const DeviceImage&) = delete;
    DeviceImage& operator=(const DeviceImage&) = delete;
    rr_status allocate(rr::rhi::Extent2D extent);   // zero-filled
    void release();
    [[nodiscard]] float* data() const noexcept { return data_; }
private:
    float* data_ = nullptr;
};

// Common plumbing: the context, the stream, the extent and the status.
class CudaPassBase : public rr::render::RenderPass {
public:
    void set_stream(void* stream) noexcept { stream_ = stream; }
    [[nodiscard]] rr_status last_status() const noexcept { return status_; }
    [[nodiscard]] rr::rhi::Extent2D extent() const noexcept { return extent_; }
protected:
    CudaPassBase(rr_ctx* ctx, rr::rhi::Extent2D extent) : ctx_(ctx), extent_(extent) {}
    Reflection one_output(const char* name) const;
    rr_ctx* ctx_;
    rr::rhi::Extent2D extent_;
    void* stream_ = nullptr;
    rr_status status_ = RR_OK;
};

class PathTracerCudaPass final : public CudaPassBase {
public:
    PathTracerCudaPass(rr_ctx* ctx, rr::rhi::Extent2D extent);
    [[nodiscard]] const char* name() const override { return "PathTracerPass"; }
    [[nodiscard]] Reflection reflect() const override;
    void on_resize(rr::rhi::Extent2D new_extent) override;
    void execute(rr::render::FrameContext& fc) override;

    void set_scene(const rr_scene* scene) noexcept { scene_ = scene; }
    void set_camera(const GpuCameraData& camera) noexcept { camera_ = camera; has_camera_ = true; }
    [[nodiscard]] const float* radiance() const noexcept { return radiance_.data(); }

    uint32_t max_bounces = 5;   // PathTracerPass.h:46
    bool emitter_sampling = false;   // RR_PT_FLAG_EMITTERS (not in the reference)
private:
    const rr_scene* scene_ = nullptr;
    GpuCameraData camera_{};
    bool has_camera_ = false;
    uint32_t frame_count_ = 0;   // frame_seed = frame_count_++ (PathTracerPass.cpp:215)
    DeviceImage radiance_;
};

class AccumulateCudaPass final : public CudaPassBase {
public:
    AccumulateCudaPass(rr_ctx* ctx, rr::rhi::Extent2D extent);
    [[nodiscard]] const char* name() const override { return "AccumulatePass"; }
    [[nodiscard]] Reflection reflect() const override;
    void on_resize(rr::rhi::Extent2D new_extent) override;
    void execute(rr::render::FrameContext& fc) override;

    // The radiance image to accumulate (PathTracerCudaPass::radiance()).
    void set_input(const float* radiance) noexcept { input_ = radiance; }
    [[nodiscard]] const float* accumulated() const noexcept { return accumulated_.data(); }

    bool camera_moved = false;     // AccumulatePass.h:46-47
    uint32_t accumulated_spp = 0;
private:
    const float* input_ = nullptr;
    DeviceImage accumulated_;
};

class ReSTIRDICudaPass final : public CudaPassBase {
public:
    ReSTIRDICudaPass(rr_ctx* ctx, rr::rhi::Extent2D extent);
    [[nodiscard]] const char* name() const override { return "ReSTIRDIPass"; }
    [[nodiscard]] Reflection reflect() const override;
    void on_resize(rr::rhi::Extent2D new_extent) override;
    void execute(rr::render::FrameContext& fc) override;

    void set_scene(const rr_scene* scene) noexcept { scene_ = scene; }
    void set_camera(const GpuCameraData& camera) noexcept { camera_ = camera; has_camera_ = true; }
    // ReSTIRDIPass.h:80-85
    void reset_history() noexcept { reservoir_flip_ = 0; frame_count_ = 0; }
    [[nodiscard]] const float* output() const noexcept { return output_.data(); }
    [[nodiscard]] const float* gbuffer_position() const noexcept { return gbuf_pos_.data(); }
    [[nodiscard]] const float* gbuffer_normal() const noexcept { return gbuf_norm_.data(); }
    [[nodiscard]] const float* reservoir(int slot) const noexcept { return reservoir_[slot & 1].data(); }

    // ReSTIRDIPass.h:89-93
    bool temporal_enable = true;
    bool spatial_enable = true;
    uint32_t num_initial_candidates = 16;
    uint32_t spatial_num_neighbors = 4;
    uint32_t spatial_radius = 15;
    bool emitter_candidates = false;   // RR_DI_FLAG_EMITTERS (not in the reference)
private:
    const rr_scene* scene_ = nullptr;
    GpuCameraData camera_{};
    bool has_camera_ = false;
    uint32_t frame_count_ = 0;
    uint32_t reservoir_flip_ = 0;
    DeviceImage gbuf_pos_, gbuf_norm_, output_;
    DeviceImage reservoir_[2];
};

class AtrousCudaPass final : public CudaPassBase {
public:
    AtrousCudaPass(rr_ctx* ctx, rr::rhi::Extent2D extent);
    [[nodiscard]] const char* name() const override { return "AtrousPass"; }
    [[nodiscard]] Reflection reflect() const override;
    void on_resize(rr::rhi::Extent2D new_extent) override;
    void execute(rr::render::FrameContext& fc) override;

    void set_input(const float* radiance) noexcept { input_ = radiance; }
    void set_gbuffer(const float* position, const float* normal) noexcept { gbuf_pos_ = position; gbuf_norm_ = normal; }
    // the image the last execute() wrote (ping-pong slot (iterations-1)&1, AtrousPass.cpp:199,205)
    [[nodiscard]] const float* output() const noexcept { return ping_[out_slot_].data(); }

    // AtrousPass.h:55-58
    uint32_t iterations = 5;
    float sigma_position = 0.25f;
    float sigma_normal = 0.20f;
    float sigma_luminance = 1.00f;
private:
    const float* input_ = nullptr;
    const float* gbuf_pos_ = nullptr;
    const float* gbuf_norm_ = nullptr;
    uint32_t out_slot_ = 0;
    DeviceImage ping_[2];
};

} // namespace rr::cuda_passes
