// wave.cuh — wavefront path state shared by the single-job and the batched
// renderers: structure-of-arrays slots, flag packing and warp-aggregated
// queue pushes.
#pragma once
#include "shading.cuh"

namespace sb {

// Wavefront state (structure of arrays, one slot per path of the chunk).
struct Wave {
    float4* ray_o;   // origin, tmax
    float4* ray_d;   // direction, last BSDF pdf
    float4* thr;     // throughput, flags (depth | specular << 16 | inside << 17)
    float4* col;     // color
    uint32_t* rng;
    float4* hit;     // u, v, t, instId (SB_INVALID = miss)
    uint32_t* hitPrim;
    uint32_t* queue[2];
    float4* sh_o;    // origin, tmax
    float4* sh_d;    // direction, slot
    float4* sh_cd;   // diffuse contribution, kind
    float4* sh_cg;   // glossy contribution
    uint32_t* counters;  // [0],[1] queue sizes, [2] shadow queue size
};

__device__ __forceinline__ uint32_t pack_flags(const PathState& ps)
{
    return (uint32_t)ps.depth | ((uint32_t)ps.specular << 16) | ((uint32_t)ps.inside << 17) |
           ((uint32_t)ps.nrcReady << 18);
}

__device__ __forceinline__ uint32_t warp_push(uint32_t* counter, bool pred)
{
    const unsigned mask = __ballot_sync(0xffffffffu, pred);
    const int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (mask != 0) {
        const int leader = __ffs(mask) - 1;
        if (lane == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
        base = __shfl_sync(0xffffffffu, base, leader);
    }
    return base + __popc(mask & ((1u << lane) - 1u));
}

}  // namespace sb
