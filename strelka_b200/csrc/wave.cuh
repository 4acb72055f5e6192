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
    uint32_t* hitRef;  // the hit primitive id (batch) or its compact leaf index (single-job passes)
    uint32_t* queue[2];
    float4* sh_o;    // origin, tmax
    float4* sh_d;    // direction, slot
    float4* sh_cd;   // diffuse contribution, kind
    float4* sh_cg;   // glossy contribution
    uint32_t* counters;  // [0],[1] queue sizes, [2] shadow queue size, [3..5] work-queue
                         // heads of extend, shade and shadow (kWaveCounters entries)
};

constexpr int kWaveCounters = 8;

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

// A warp's share of an atomic work queue: the warp takes `chunk` items at a
// time from *counter and hands them to the lanes that ask, so lanes whose
// work ends early pick up new items while the rest of the warp continues.
// Returns the item of a lane that asked and got one, else SB_INVALID (the
// queue is then empty).  Warp-uniform state; called by the whole warp.
struct WarpPool {
    uint32_t next, end;
    int dry;
};

__device__ __forceinline__ uint32_t pool_take(WarpPool& p, uint32_t* counter, uint32_t total, uint32_t chunk, bool need)
{
    const int lane = threadIdx.x & 31;
    unsigned mask = __ballot_sync(0xffffffffu, need);
    uint32_t got = SB_INVALID;
    while (mask) {
        if (p.next >= p.end) {
            if (p.dry) break;
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(counter, chunk);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base >= total) {
                p.dry = 1;
                break;
            }
            p.next = base;
            p.end = (uint32_t)min((uint64_t)base + chunk, (uint64_t)total);
        }
        const uint32_t avail = p.end - p.next;
        const uint32_t rank = (uint32_t)__popc(mask & ((1u << lane) - 1u));
        const bool served = ((mask >> lane) & 1u) && rank < avail;
        if (served) got = p.next + rank;
        p.next += min((uint32_t)__popc(mask), avail);
        mask &= ~__ballot_sync(0xffffffffu, served);
    }
    return got;
}

}  // namespace sb
