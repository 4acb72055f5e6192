// internal.h — scene preparation shared by the pass objects of pathtracer.cu
// and batch.cu (not part of the C ABI).
#pragma once
#include <cuda_runtime.h>

#include "../../include/strelka_b200.h"
#include "traverse.cuh"

namespace sb {

// sRGB-to-linear table of the 256 texel values (texturemanager.cpp:79's
// R8G8B8A8_SRGB decode).
void srgb_lut_host(float* lut);
// Argument checks of a scene descriptor shared by every entry point.
int validate_scene_desc(const PathTracerDesc* d);
// Device tables derived from a scene's BVH, all in one allocation of
// scene_tables_bytes(numNodes) bytes: the leaf-triangle records (3 float4 per
// leaf, at most numNodes/2 + 1 leaves), each node's compact leaf index (4 B
// per node), the 4-wide BVH (8 float4 per node, at most numNodes/2 + 1
// nodes) and the scratch of its build (16 B per node).
struct SceneTables {
    float4* rec = nullptr;
    uint32_t recCap = 0;
    float4* shade = nullptr;  // 6 float4 per leaf: its triangle's shading vertex data (k_prep_shade)
    uint32_t* leafOf = nullptr;
    float4* wide = nullptr;
    uint32_t wideCap = 0;
    uint32_t* parent = nullptr;
    uint32_t* flag = nullptr;
    uint32_t* map = nullptr;
    uint32_t* extra = nullptr;  // pointer-jumping parities
    uint32_t* deep = nullptr;   // set when the tree is too deep for the walk-up
    void* scan = nullptr;
    size_t scanBytes = 0;
};
size_t scene_tables_bytes(uint32_t numNodes);
// The tables of a scene of numNodes nodes carved out of `base`.
SceneTables scene_tables(void* base, uint32_t numNodes);
// Builds the tables of a scene on `st` (no host synchronisation).
int launch_prep_tables(const BVHNode* nodes, uint32_t numNodes, const InstanceConstants* inst, uint32_t numInstances,
                       const uint32_t* ib, uint32_t numIndices, const Vertex* vb, uint32_t numVertices,
                       const SceneTables& t, uint32_t* status, int numSMs, cudaStream_t st);
// The device view of a descriptor's scene with its derived tables.
DevScene scene_from_desc(const PathTracerDesc* d, const SceneTables& t, const float* srgbLut, uint32_t* status);

}  // namespace sb
