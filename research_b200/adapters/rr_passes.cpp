// rr_passes.cpp — the RenderPass adapters of rr_passes.h over the C ABI.

#include "rr_passes.h"

#include <cuda_runtime.h>

namespace rr::cuda_passes {

namespace {
constexpr size_t kPixelBytes = 16;   // RGBA32F

rr::render::RenderPass::ResourceDesc rgba32f(const char* name, rr::rhi::Extent2D extent) {
    return {name, rr::render::RenderPass::ResourceDesc::Kind::Texture, rr::rhi::Format::R32G32B32A32_Sfloat, extent};
}
} // namespace

DeviceImage::~DeviceImage() { release(); }

rr_status DeviceImage::allocate(rr::rhi::Extent2D extent) {
    release();
    const size_t bytes = size_t(extent.width) * extent.height * kPixelBytes;
    if (bytes == 0) return RR_ERR_INVALID_ARGUMENT;
    if (cudaMalloc(reinterpret_cast<void**>(&data_), bytes) != cudaSuccess) {
        data_ = nullptr;
        return RR_ERR_OUT_OF_MEMORY;
    }
    return cudaMemset(data_, 0, bytes) == cudaSuccess ? RR_OK : RR_ERR_CUDA;
}

void DeviceImage::release() {
    if (data_) cudaFree(data_);
    data_ = nullptr;
}

rr::render::RenderPass::Reflection CudaPassBase::one_output(const char* name) const {
    Reflection r;
    r.outputs.push_back(rgba32f(name, extent_));
    return r;
}

// ── PathTracerPass ──────────────────────────────────────────────────────────
PathTracerCudaPass::PathTracerCudaPass(rr_ctx* ctx, rr::rhi::Extent2D extent) : CudaPassBase(ctx, extent) {
    if (ctx_) status_ = radiance_.allocate(extent_);
}

rr::render::RenderPass::Reflection PathTracerCudaPass::reflect() const { return one_output("radiance_image"); }

void PathTracerCudaPass::on_resize(rr::rhi::Extent2D new_extent) {
    extent_ = new_extent;
    if (ctx_) status_ = radiance_.allocate(extent_);
}

void PathTracerCudaPass::execute(rr::render::FrameContext&) {
    if (!ctx_ || !scene_ || !has_camera_ || !radiance_.data()) {
        status_ = RR_ERR_NOT_INITIALIZED;
        return;
    }
    if (camera_.screen_width != extent_.width || camera_.screen_height != extent_.height) {
        status_ = RR_ERR_INVALID_ARGUMENT;
        return;
    }
    const rr_pt_params p{frame_count_++, max_bounces, 1u, emitter_sampling ? RR_PT_FLAG_EMITTERS : 0u};
    status_ = rr_pathtracer_execute(ctx_, scene_, &camera_, &p, radiance_.data(), stream_);
}

// ── AccumulatePass ──────────────────────────────────────────────────────────
AccumulateCudaPass::AccumulateCudaPass(rr_ctx* ctx, rr::rhi::Extent2D extent) : CudaPassBase(ctx, extent) {
    if (ctx_) status_ = accumulated_.allocate(extent_);
}

rr::render::RenderPass::Reflection AccumulateCudaPass::reflect() const { return one_output("accumulated_image"); }

void AccumulateCudaPass::on_resize(rr::rhi::Extent2D new_extent) {
    extent_ = new_extent;
    if (ctx_) status_ = accumulated_.allocate(extent_);
    camera_moved = true;
}

void AccumulateCudaPass::execute(rr::render::FrameContext&) {
    if (!ctx_ || !input_ || !accumulated_.data()) {
        status_ = RR_ERR_NOT_INITIALIZED;
        return;
    }
    const rr_acc_params p{extent_.width, extent_.height, camera_moved ? 1u : 0u, accumulated_spp};
    status_ = rr_accumulate_execute(ctx_, input_, 1, accumulated_.data(), nullptr, &p, stream_);
    if (status_ != RR_OK) return;
    // AccumulatePass.cpp:211-217
    accumulated_spp = camera_moved ? 1u : accumulated_spp + 1u;
    camera_moved = false;
}

// ── ReSTIRDIPass ────────────────────────────────────────────────────────────
ReSTIRDICudaPass::ReSTIRDICudaPass(rr_ctx* ctx, rr::rhi::Extent2D extent) : CudaPassBase(ctx, extent) {
    on_resize(extent);
}

rr::render::RenderPass::Reflection ReSTIRDICudaPass::reflect() const { return one_output("restir_di_output"); }

void ReSTIRDICudaPass::on_resize(rr::rhi::Extent2D new_extent) {
    extent_ = new_extent;
    if (!ctx_) return;
    for (DeviceImage* img : {&gbuf_pos_, &gbuf_norm_, &output_, &reservoir_[0], &reservoir_[1]}) {
        status_ = img->allocate(extent_);
        if (status_ != RR_OK) return;
    }
    reservoir_flip_ = 0;   // ReSTIRDIPass.cpp:285
}

void ReSTIRDICudaPass::execute(rr::render::FrameContext&) {
    if (!ctx_ || !scene_ || !has_camera_ || !output_.data() || !reservoir_[1].data()) {
        status_ = RR_ERR_NOT_INITIALIZED;
        return;
    }
    if (camera_.screen_width != extent_.width || camera_.screen_height != extent_.height) {
        status_ = RR_ERR_INVALID_ARGUMENT;
        return;
    }
    rr_di_params p{};
    p.frame_seed = frame_count_++;
    p.num_initial_candidates = num_initial_candidates;
    p.temporal_enable = temporal_enable ? 1u : 0u;
    p.spatial_enable = spatial_enable ? 1u : 0u;
    p.spatial_num_neighbors = spatial_num_neighbors;
    p.spatial_radius = spatial_radius;
    p.m_cap_factor = 20u;   // restir_di.slang:300
    p.flags = emitter_candidates ? RR_DI_FLAG_EMITTERS : 0u;
    status_ = rr_restir_di_execute(ctx_, scene_, &camera_, &p, gbuf_pos_.data(), gbuf_norm_.data(),
                                   reservoir_[reservoir_flip_].data(), reservoir_[1u - reservoir_flip_].data(),
                                   output_.data(), stream_);
    if (status_ == RR_OK) reservoir_flip_ ^= 1u;   // ReSTIRDIPass.cpp:444
}

// ── AtrousPass ──────────────────────────────────────────────────────────────
AtrousCudaPass::AtrousCudaPass(rr_ctx* ctx, rr::rhi::Extent2D extent) : CudaPassBase(ctx, extent) {
    on_resize(extent);
}

rr::render::RenderPass::Reflection AtrousCudaPass::reflect() const { return one_output("atrous_output"); }

void AtrousCudaPass::on_resize(rr::rhi::Extent2D new_extent) {
    extent_ = new_extent;
    if (!ctx_) return;
    for (DeviceImage* img : {&ping_[0], &ping_[1]}) {
        status_ = img->allocate(extent_);
        if (status_ != RR_OK) return;
    }
}

void AtrousCudaPass::execute(rr::render::FrameContext&) {
    if (!ctx_ || !input_ || !gbuf_pos_ || !gbuf_norm_ || !ping_[1].data()) {
        status_ = RR_ERR_NOT_INITIALIZED;
        return;
    }
    rr_atrous_params p{};
    p.width = extent_.width;
    p.height = extent_.height;
    p.iterations = iterations;   // clamped to 1..7 by the library (AtrousPass.cpp:265)
    p.sigma_position = sigma_position;
    p.sigma_normal = sigma_normal;
    p.sigma_luminance = sigma_luminance;
    uint32_t slot = 0;
    status_ = rr_atrous_execute(ctx_, input_, gbuf_pos_, gbuf_norm_, ping_[0].data(), ping_[1].data(), &p, &slot,
                                stream_);
    if (status_ == RR_OK) out_slot_ = slot;
}

} // namespace rr::cuda_passes
