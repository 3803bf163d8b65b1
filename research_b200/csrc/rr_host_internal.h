// rr_host_internal.h — the host scene object behind rr_host.h: the flat
// GpuScene arrays a factory or loader fills (Scene::all_vertices_,
// all_indices_, meshes_, materials_, instances_, lights_ after
// Scene::upload's conversion, Scene.cpp:255-345).
#pragma once

#include "rr_host.h"

#include <vector>

struct rr_host_scene {
    std::vector<GpuVertex> vertices;
    std::vector<uint32_t> indices;
    std::vector<GpuMesh> meshes;
    std::vector<GpuMaterial> materials;
    std::vector<GpuInstance> instances;
    std::vector<GpuLight> lights;
};
