// traverse.cuh — stackless BVH traversal over the reference's flattened
// depth-first node array (shaders/raytracing.h:198-286), sm_100a.
//
// Nodes are fetched as two 16-byte read-only loads (ld.global.nc.v4).  The
// leaf triangle of node i is read from a derived table (3 float4 per node:
// v0|instId, e0|primId, e1|0) computed once per scene version with exactly
// the arithmetic of getTriangle (raytracing.h:134-153), so the intersection
// results are bit-identical to evaluating getTriangle at every visit while
// each leaf visit reads 32 + 48 bytes instead of an instance record, three
// indices and three vertices.
//
// Closest hit visits nodes in the reference's depth-first order and
// additionally skips an inner node whose entry distance exceeds the best hit
// so far by a relative 2^-12 (the reference never prunes); the winner under
// the strict t < minHit rule is unchanged.  Any hit is the reference
// traversal verbatim (its result depends on the visit order).
#pragma once
#include "device_math.cuh"

namespace sb {

// Scene view passed to every kernel by value.
struct DevScene {
    const float4* nodes;  // 2 float4 per BVHNode
    const float4* tris;   // 3 float4 per node (leaf slots only)
    uint32_t numNodes;
    uint32_t numVertices;
    const Vertex* vb;
    const uint32_t* ib;
    uint32_t numIndices;
    uint32_t numInstances;
    const InstanceConstants* inst;
    const UniformLight* lights;
    uint32_t lightCapacity;
    uint32_t numMaterials;
    const uint8_t* argBlock;
    uint64_t argBlockBytes;
    const MdlMaterial* materials;
    const Mdl_resource_info* resInfos;
    uint32_t numResInfos;
    uint32_t numTextures;
    const StrelkaTexture* textures;
    const float* srgbLut;  // 256 entries
    StrelkaEnvMap env;
    int hasEnv;
    uint32_t* status;      // device status word (STRELKA_DEV_* bits)
};

#define SB_PRUNE_SCALE (1.0f + 0x1p-12f)

__device__ __forceinline__ void raise_status(const DevScene& s, uint32_t bits)
{
    if (s.status) atomicOr(s.status, bits);
}

// raytracing.h:36-88
__device__ __forceinline__ bool ray_triangle(v3 orig, v3 dir, v3 v0, v3 e0, v3 e1, float& t, float& bu, float& bv)
{
    t = 1e9f;
    v3 pvec = vcross(dir, e1);
    float det = vdot(e0, pvec);
    if (fabsf(det) < 1e-6f) return false;
    float invDet = 1.0f / det;
    v3 tvec = vsub(orig, v0);
    float u = vdot(tvec, pvec) * invDet;
    if (u < 0.0f || u > 1.0f) return false;
    v3 qvec = vcross(tvec, e0);
    float v = vdot(dir, qvec) * invDet;
    if (v < 0.0f || (u + v) > 1.0f) return false;
    t = vdot(e1, qvec) * invDet;
    if (t < 1e-6f) return false;
    bu = u;
    bv = v;
    return true;
}

// ray.h:35-48 with HLSL min/max as fminf/fmaxf
__device__ __forceinline__ bool ray_box(v3 o, v3 inv, float4 lo, float4 hi, float& t)
{
    float fx = (hi.x - o.x) * inv.x, fy = (hi.y - o.y) * inv.y, fz = (hi.z - o.z) * inv.z;
    float nx = (lo.x - o.x) * inv.x, ny = (lo.y - o.y) * inv.y, nz = (lo.z - o.z) * inv.z;
    float t1 = fminf(fmaxf(fx, nx), fminf(fmaxf(fy, ny), fmaxf(fz, nz)));
    float t0 = fmaxf(fmaxf(fminf(fx, nx), fmaxf(fminf(fy, ny), fminf(fz, nz))), 0.0f);
    t = t0;
    return t1 >= t0;
}

struct HitRec {
    float u, v, t;
    uint32_t instId, primId;
};

// raytracing.h:198-247 (+ pruning, see file comment)
template <bool COUNT>
__device__ __forceinline__ bool trace_closest(const DevScene& s, v3 o, float tmax, v3 d, HitRec& hit,
                                              uint32_t& nInner, uint32_t& nLeaf)
{
    const v3 inv = V(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    float minHit = 1e9f;
    bool found = false;
    uint32_t node = 0;
    const uint32_t cap = 2u * s.numNodes + 2u;
    uint32_t visits = 0;
    while (node != SB_INVALID) {
        if (node >= s.numNodes) { raise_status(s, STRELKA_DEV_NODE_OOB); break; }
        if (++visits > cap) { raise_status(s, STRELKA_DEV_TRAVERSAL_CAP); break; }
        const float4 lo = __ldg(&s.nodes[2 * (size_t)node]);
        const float4 hi = __ldg(&s.nodes[2 * (size_t)node + 1]);
        const uint32_t instId = __float_as_uint(lo.w);
        if (instId != SB_INVALID) {
            if (COUNT) ++nLeaf;
            const float4* tp = &s.tris[3 * (size_t)node];
            const float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
            float t, bu, bv;
            if (ray_triangle(o, d, xyz(a), xyz(b), xyz(c), t, bu, bv) && (t < tmax) && (t < minHit)) {
                minHit = t;
                hit.t = t;
                hit.u = bu;
                hit.v = bv;
                hit.instId = instId;
                hit.primId = __float_as_uint(lo.x);
                found = true;
            }
            node = __float_as_uint(hi.w);
            continue;
        }
        if (COUNT) ++nInner;
        float boxT;
        if (ray_box(o, inv, lo, hi, boxT)) {
            if (boxT > tmax || boxT > minHit * SB_PRUNE_SCALE) {
                node = __float_as_uint(hi.w);
                continue;
            }
            ++node;
            continue;
        }
        node = __float_as_uint(hi.w);
    }
    return found;
}

// raytracing.h:249-286
template <bool COUNT>
__device__ __forceinline__ bool trace_any(const DevScene& s, v3 o, float tmax, v3 d, HitRec& hit, uint32_t& nInner,
                                          uint32_t& nLeaf)
{
    const v3 inv = V(1.0f / d.x, 1.0f / d.y, 1.0f / d.z);
    uint32_t node = 0;
    const uint32_t cap = 2u * s.numNodes + 2u;
    uint32_t visits = 0;
    while (node != SB_INVALID) {
        if (node >= s.numNodes) { raise_status(s, STRELKA_DEV_NODE_OOB); break; }
        if (++visits > cap) { raise_status(s, STRELKA_DEV_TRAVERSAL_CAP); break; }
        const float4 lo = __ldg(&s.nodes[2 * (size_t)node]);
        const float4 hi = __ldg(&s.nodes[2 * (size_t)node + 1]);
        const uint32_t instId = __float_as_uint(lo.w);
        if (instId != SB_INVALID) {
            if (COUNT) ++nLeaf;
            const float4* tp = &s.tris[3 * (size_t)node];
            const float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
            float t, bu, bv;
            bool isect = ray_triangle(o, d, xyz(a), xyz(b), xyz(c), t, bu, bv);
            hit.t = t;
            if (isect && (t < tmax)) {
                hit.instId = instId;
                hit.primId = __float_as_uint(lo.x);
                return true;
            }
        } else {
            if (COUNT) ++nInner;
            float boxT;
            if (ray_box(o, inv, lo, hi, boxT)) {
                if (boxT > tmax) {
                    node = __float_as_uint(hi.w);
                    continue;
                }
                ++node;
                continue;
            }
        }
        node = __float_as_uint(hi.w);
    }
    return false;
}

}  // namespace sb
