// rr_bvh.h — host BVH builder interface (host-only header).
#pragma once

#include <cstdint>
#include <vector>
#include <vector_types.h>

namespace rr {
struct BvhBuild {
    std::vector<float4> nodes;     // 4 float4 per node (layout in rr_trace.cuh)
    std::vector<float4> nodes4;    // the same tree collapsed 4-wide: 8 float4 per node (layout in rr_trace.cuh)
    std::vector<uint32_t> order;   // leaf order -> flattened triangle id
    uint32_t max_depth = 0;
};
// tri_world: 9 floats per triangle (v0, v1, v2 in world space).
BvhBuild build_bvh(const std::vector<float>& tri_world, int threads);
} // namespace rr
