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
// Builds the node-pair record table (4 float4 per node) of a scene on `st`.
int launch_prep_records(const BVHNode* nodes, uint32_t numNodes, const InstanceConstants* inst, uint32_t numInstances,
                        const uint32_t* ib, uint32_t numIndices, const Vertex* vb, uint32_t numVertices, float4* rec,
                        uint32_t* status, int numSMs, cudaStream_t st);
// The device view of a descriptor's scene with its record table.
DevScene scene_from_desc(const PathTracerDesc* d, const float4* rec, const float* srgbLut, uint32_t* status);

}  // namespace sb
