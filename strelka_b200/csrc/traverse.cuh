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
// trace_closest / trace_any below are the reference's stackless loops over
// the node array (used by the allocation-free ray query); closest hit adds
// the 2^-12 relative pruning of subtrees whose entry lies beyond the best
// hit.  The kernels of the passes use the 4-wide traversal further down.
#pragma once
#include "device_math.cuh"

namespace sb {

// Scene view passed to every kernel by value.
struct DevScene {
    const float4* nodes;  // 2 float4 per BVHNode
    const float4* tris;   // 3 float4 per node (leaf slots only)
    const float4* rec;    // 3 float4 per leaf, at the leaf's compact index
    const uint32_t* leafOf;  // per node: its compact leaf index (leaves only)
    uint32_t numRec;      // capacity of `rec` in leaves
    const float4* shadeRec;  // 6 float4 per leaf at its compact index: shading vertex data (k_prep_shade)
    const float4* wide;   // 8 float4 per 4-wide node (see below)
    uint32_t numWide;     // capacity of `wide` in nodes
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
    const uint8_t* roData;  // MDL read-only data segment
    uint64_t roDataBytes;
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

// ===========================================================================
// 4-wide traversal.
//
// Derived tables, built once per scene version on the GPU (pathtracer.cu):
//   compact leaf index of every node: a leaf's rank among the leaves in the
//     depth-first node order (leafOf, an exclusive scan of the leaf flags);
//   record table, 3 float4 per leaf at its compact index: the triangle
//     [0] = v0 | instId  [1] = e0 | primId  [2] = e1 | 0;
//   shading table, 6 float4 per leaf at its compact index: the triangle's
//     world-space vertex positions and normals and its UVs (k_prep_shade;
//     read by shade(), which receives the hit's compact leaf index);
//   4-wide BVH, 8 float4 per node: the binary inner nodes at even depth of
//     the reference's tree (children L = n+1 and R = escape(n+1), the
//     implicit tree of the depth-first layout, bvh.cpp:182-220).  Node w:
//     [0..2] = min x / y / z of its 4 entries, [3..5] = max x / y / z,
//     [6] = the 4 entry refs.  The entries, in the reference's order, are for
//     each binary child c: c itself when it is a leaf (ref | SB_LEAF_BIT |
//     SB_NOBOX_BIT: tested without a box, as the reference does, except at
//     the root, where the root's box gates it), otherwise c's two children:
//     an inner one with its own box (ref = its 4-wide index), a leaf one
//     gated by c's box (ref = its compact index | SB_LEAF_BIT).
// A child's box test passing implies its parent's (the slab arithmetic
// rounds monotonically and a parent box contains its children's), so testing
// only the even-depth boxes leaves the set of triangles a query tests
// exactly the reference's.  One step reads one 4-wide node (112 bytes, with
// four 256-bit loads of its 128-byte line) and tests four boxes: half the
// dependent fetches of a binary traversal.  The slab subtractions and
// products of the four boxes run as packed pairs (sub/mul.rn.f32x2, each
// half rounded exactly as the scalar instruction), and the ray's reciprocal
// direction is __frcp_rn, the correctly rounded 1/x, so every value equals
// the reference's expression evaluated in single precision.
//
// Closest hit tests all entry boxes, then the leaves that passed, continues
// with the nearest passing inner entry and keeps the others on a per-thread
// stack with their entry distances (sorted, farthest first), dropping any
// subtree whose entry exceeds the best hit by more than a relative 2^-12.  A
// tie in t goes to the leaf with the smaller compact index, the first in
// depth-first order: the reference's winner under its strict t < minHit rule.
// Any hit keeps the reference's depth-first order exactly: a node's passing
// entries go onto the stack in reverse order, and leaves are tested when
// reached.  A full stack falls back to the reference's stackless loop from
// the root (closest: with the best hit so far).  tests/test_traversal_rule.py
// checks the rule, replayed by the oracle, against the reference loop bit for
// bit; tests/test_gpu_trace.py checks the kernels against both.  The
// ray-query kernels and the large-scene wavefront passes run closest hit with
// its leaf tests deferred across the warp (closest_defer_*, below) and keep
// the top of each stack in shared memory (SplitStack); the results are the
// same.
// ===========================================================================

namespace sb {

#ifndef SB_STACK
#define SB_STACK 64
#endif
#define SB_LEAF_BIT 0x80000000u   // a ref to a leaf triangle (its compact index in the record table)
#define SB_NOBOX_BIT 0x40000000u  // a leaf tested without a box (a leaf child of the node itself)

struct RayQ {
    v3 o, d, inv;
    float tmax;
};

__device__ __forceinline__ RayQ make_ray(v3 o, float tmax, v3 d)
{
    RayQ r;
    r.o = o;
    r.d = d;
    r.tmax = tmax;
    // __frcp_rn is the reciprocal correctly rounded to nearest: the value of
    // the IEEE division 1.0f / x for every x (zeros, infinities, subnormals)
    r.inv = V(__frcp_rn(d.x), __frcp_rn(d.y), __frcp_rn(d.z));
    return r;
}

// triangle of leaf `leaf` (its compact index: the leaf's rank in the
// depth-first node order) in the record table
__device__ __forceinline__ bool rec_triangle(const DevScene& s, const RayQ& r, uint32_t leaf, float& t, float& bu, float& bv,
                                             uint32_t& instId, uint32_t& primId)
{
    const float4* tp = &s.rec[3 * (size_t)leaf];
    const float4 a = __ldg(tp), b = __ldg(tp + 1), c = __ldg(tp + 2);
    instId = __float_as_uint(a.w);
    primId = __float_as_uint(b.w);
    return ray_triangle(r.o, r.d, xyz(a), xyz(b), xyz(c), t, bu, bv);
}

// Result of a stackless fallback (returned by value so that the caller's
// traversal state can stay in registers).
struct Fallback {
    HitRec hit;
    float minHit;
    uint32_t leaf;  // compact index of the best hit's leaf
    uint32_t nInner, nLeaf;
    bool found;
};

// The reference's stackless closest-hit loop over the node array, reading
// leaf triangles from the record table; runs from the root with the best hit
// so far (used when the stack overflows).
template <bool COUNT>
__device__ __noinline__ Fallback closest_stackless_rec(const DevScene s, const RayQ r, float minHit, uint32_t best, HitRec hit,
                                                       bool found)
{
    Fallback f;
    f.nInner = 0;
    f.nLeaf = 0;
    uint32_t node = 0;
    const uint32_t cap = 2u * s.numNodes + 2u;
    uint32_t visits = 0;
    while (node != SB_INVALID) {
        if (node >= s.numNodes) { raise_status(s, STRELKA_DEV_NODE_OOB); break; }
        if (++visits > cap) { raise_status(s, STRELKA_DEV_TRAVERSAL_CAP); break; }
        const float4 lo = __ldg(&s.nodes[2 * (size_t)node]);
        const float4 hi = __ldg(&s.nodes[2 * (size_t)node + 1]);
        if (__float_as_uint(lo.w) != SB_INVALID) {
            if (COUNT) ++f.nLeaf;
            float t, bu, bv;
            uint32_t iid, pid;
            const uint32_t li = __ldg(&s.leafOf[node]);
            if (li >= s.numRec) {
                raise_status(s, STRELKA_DEV_NODE_OOB);
                break;
            }
            if (rec_triangle(s, r, li, t, bu, bv, iid, pid) && (t < r.tmax) &&
                (t < minHit || (t == minHit && li < best))) {
                minHit = t;
                best = li;
                hit.t = t;
                hit.u = bu;
                hit.v = bv;
                hit.instId = iid;
                hit.primId = pid;
                found = true;
            }
            node = __float_as_uint(hi.w);
            continue;
        }
        if (COUNT) ++f.nInner;
        float boxT;
        if (ray_box(r.o, r.inv, lo, hi, boxT) && !(boxT > r.tmax) && !(boxT > minHit * SB_PRUNE_SCALE)) {
            ++node;
            continue;
        }
        node = __float_as_uint(hi.w);
    }
    f.hit = hit;
    f.minHit = minHit;
    f.leaf = best;
    f.found = found;
    return f;
}

// The reference's stackless any-hit loop from `node` (raytracing.h:249-286),
// inlined into the any-hit kernels (any_stackless_loop) and called out of
// line elsewhere (any_stackless_rec).
template <bool COUNT>
__device__ __forceinline__ Fallback any_stackless_loop(const DevScene& s, const RayQ& r, uint32_t node, HitRec hit)
{
    Fallback f;
    f.nInner = 0;
    f.nLeaf = 0;
    f.found = false;
    f.minHit = 0.0f;
    const uint32_t cap = 2u * s.numNodes + 2u;
    uint32_t visits = 0;
    while (node != SB_INVALID) {
        if (node >= s.numNodes) { raise_status(s, STRELKA_DEV_NODE_OOB); break; }
        if (++visits > cap) { raise_status(s, STRELKA_DEV_TRAVERSAL_CAP); break; }
        const float4 lo = __ldg(&s.nodes[2 * (size_t)node]);
        const float4 hi = __ldg(&s.nodes[2 * (size_t)node + 1]);
        if (__float_as_uint(lo.w) != SB_INVALID) {
            if (COUNT) ++f.nLeaf;
            float t, bu, bv;
            uint32_t iid, pid;
            const uint32_t li = __ldg(&s.leafOf[node]);
            if (li >= s.numRec) {
                raise_status(s, STRELKA_DEV_NODE_OOB);
                break;
            }
            bool isect = rec_triangle(s, r, li, t, bu, bv, iid, pid);
            hit.t = t;
            if (isect && (t < r.tmax)) {
                hit.instId = iid;
                hit.primId = pid;
                f.found = true;
                break;
            }
        } else {
            if (COUNT) ++f.nInner;
            float boxT;
            if (ray_box(r.o, r.inv, lo, hi, boxT)) {
                if (boxT > r.tmax) {
                    node = __float_as_uint(hi.w);
                    continue;
                }
                ++node;
                continue;
            }
        }
        node = __float_as_uint(hi.w);
    }
    f.hit = hit;
    return f;
}
template <bool COUNT>
__device__ __noinline__ Fallback any_stackless_rec(const DevScene s, const RayQ r, uint32_t node, HitRec hit)
{
    return any_stackless_loop<COUNT>(s, r, node, hit);
}

// Per-query traversal state for the step functions.
struct Trav {
    RayQ r;
    float minHit;
    uint32_t leaf;  // closest hit: compact index of the best hit's leaf
    uint32_t cur;  // 4-wide node to process next, a leaf ref (SB_LEAF_BIT), or SB_INVALID = pop
    int sp;
    uint32_t steps;
    bool found;
    HitRec hit;
};

// The traversal's first entry: the 4-wide root, the root leaf, or nothing.
__device__ __forceinline__ uint32_t trav_root(const DevScene& s)
{
    if (!s.numNodes) return SB_INVALID;
    return __float_as_uint(__ldg(&s.nodes[0]).w) != SB_INVALID ? (SB_LEAF_BIT | SB_NOBOX_BIT) : 0u;
}
__device__ __forceinline__ void trav_init_root(Trav& T, v3 o, float tmax, v3 d, bool any, uint32_t root)
{
    T.r = make_ray(o, tmax, d);
    T.minHit = 1e9f;
    T.leaf = SB_INVALID;
    T.sp = 0;
    T.steps = 0;
    T.found = false;
    T.hit.u = 0.0f;
    T.hit.v = 0.0f;
    T.hit.t = any ? 0.0f : 1e9f;
    T.hit.instId = SB_INVALID;
    T.hit.primId = SB_INVALID;
    T.cur = root;
}
__device__ __forceinline__ void trav_init(const DevScene& s, Trav& T, v3 o, float tmax, v3 d, bool any)
{
    T.r = make_ray(o, tmax, d);
    T.minHit = 1e9f;
    T.leaf = SB_INVALID;
    T.sp = 0;
    T.steps = 0;
    T.found = false;
    T.hit.u = 0.0f;
    T.hit.v = 0.0f;
    T.hit.t = any ? 0.0f : 1e9f;
    T.hit.instId = SB_INVALID;
    T.hit.primId = SB_INVALID;
    if (!s.numNodes) T.cur = SB_INVALID;
    else if (__float_as_uint(__ldg(&s.nodes[0]).w) != SB_INVALID) T.cur = SB_LEAF_BIT | SB_NOBOX_BIT;  // the root is a leaf
    else T.cur = 0u;  // the 4-wide root
}

// The four entries of 4-wide node w.
struct WideNode {
    float4 lx, ly, lz, hx, hy, hz;
    uint32_t ref[4];
};
// Two float4 from one 32-byte-aligned address with one 256-bit read-only load.
__device__ __forceinline__ void ldg_pair(const float4* p, float4& a, float4& b)
{
    const size_t g = __cvta_generic_to_global(p);
    asm("ld.global.nc.v8.f32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=f"(a.x), "=f"(a.y), "=f"(a.z), "=f"(a.w), "=f"(b.x), "=f"(b.y), "=f"(b.z), "=f"(b.w)
        : "l"(g));
}
// A 4-wide node (128 bytes, 128-byte aligned) in four 256-bit loads.
__device__ __forceinline__ WideNode load_wide(const DevScene& s, uint32_t w)
{
    const float4* p = &s.wide[8 * (size_t)w];
    WideNode n;
    float4 rf, pad;
    ldg_pair(p, n.lx, n.ly);
    ldg_pair(p + 2, n.lz, n.hx);
    ldg_pair(p + 4, n.hy, n.hz);
    ldg_pair(p + 6, rf, pad);
    (void)pad;
    n.ref[0] = __float_as_uint(rf.x);
    n.ref[1] = __float_as_uint(rf.y);
    n.ref[2] = __float_as_uint(rf.z);
    n.ref[3] = __float_as_uint(rf.w);
    return n;
}
// Packed pairs of floats (sm_100 f32x2 arithmetic: each half rounded as the
// scalar instruction would round it).
__device__ __forceinline__ unsigned long long f2pack(float a, float b)
{
    unsigned long long r;
    asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(a), "f"(b));
    return r;
}
__device__ __forceinline__ void f2unpack(unsigned long long v, float& a, float& b)
{
    asm("mov.b64 {%0, %1}, %2;" : "=f"(a), "=f"(b) : "l"(v));
}
__device__ __forceinline__ unsigned long long f2sub(unsigned long long a, unsigned long long b)
{
    unsigned long long r;
    asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
__device__ __forceinline__ unsigned long long f2mul(unsigned long long a, unsigned long long b)
{
    unsigned long long r;
    asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(r) : "l"(a), "l"(b));
    return r;
}
// (b[k] - o) * inv for the four entries k of one bound row
__device__ __forceinline__ void slab4(float4 b, unsigned long long oo, unsigned long long ii, float t[4])
{
    f2unpack(f2mul(f2sub(f2pack(b.x, b.y), oo), ii), t[0], t[1]);
    f2unpack(f2mul(f2sub(f2pack(b.z, b.w), oo), ii), t[2], t[3]);
}
// The four entry boxes of a 4-wide node with the reference's slab arithmetic
// (ray.h:35-48): t0[k] the entry distance, bit k of the result whether box k is hit.
__device__ __forceinline__ unsigned wide_boxes(const RayQ& r, const WideNode& n, float t0[4])
{
    float fx[4], fy[4], fz[4], nx[4], ny[4], nz[4];
    {
        const unsigned long long ox = f2pack(r.o.x, r.o.x), ix = f2pack(r.inv.x, r.inv.x);
        slab4(n.hx, ox, ix, fx);
        slab4(n.lx, ox, ix, nx);
    }
    {
        const unsigned long long oy = f2pack(r.o.y, r.o.y), iy = f2pack(r.inv.y, r.inv.y);
        slab4(n.hy, oy, iy, fy);
        slab4(n.ly, oy, iy, ny);
    }
    {
        const unsigned long long oz = f2pack(r.o.z, r.o.z), iz = f2pack(r.inv.z, r.inv.z);
        slab4(n.hz, oz, iz, fz);
        slab4(n.lz, oz, iz, nz);
    }
    unsigned m = 0;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const float t1 = fminf(fmaxf(fx[k], nx[k]), fminf(fmaxf(fy[k], ny[k]), fmaxf(fz[k], nz[k])));
        t0[k] = fmaxf(fmaxf(fminf(fx[k], nx[k]), fmaxf(fminf(fy[k], ny[k]), fminf(fz[k], nz[k]))), 0.0f);
        if (t1 >= t0[k]) m |= 1u << k;
    }
    return m;
}

__device__ __forceinline__ void cswap(float& ta, uint32_t& ra, float& tb, uint32_t& rb)
{
    if (tb < ta) {
        const float t = ta;
        ta = tb;
        tb = t;
        const uint32_t x = ra;
        ra = rb;
        rb = x;
    }
}

// Closest-hit test of one leaf triangle.  On a tie in t the leaf with the
// smaller compact index wins: compact indices follow the depth-first node
// order, so that is the leaf the reference visits first and keeps (its test
// is the strict t < minHit), whatever order this traversal reaches them in.
__device__ __forceinline__ void closest_leaf(const DevScene& s, Trav& T, uint32_t leaf)
{
    float t, bu, bv;
    uint32_t iid, pid;
    if (rec_triangle(s, T.r, leaf, t, bu, bv, iid, pid) && (t < T.r.tmax) &&
        (t < T.minHit || (t == T.minHit && leaf < T.leaf))) {
        T.minHit = t;
        T.leaf = leaf;
        T.hit.t = t;
        T.hit.u = bu;
        T.hit.v = bv;
        T.hit.instId = iid;
        T.hit.primId = pid;
        T.found = true;
    }
}

// Traversal stacks: closest hit keeps (entry ref, entry distance) pairs,
// any hit entry refs.  LocalStack / LocalStackN are per-thread arrays (local
// memory).  SplitStack / SplitStackN keep the entries below depth S in shared
// memory, entry i of a thread at sm[i * STRIDE] (consecutive threads in
// consecutive words, so a warp's accesses are free of bank conflicts whatever
// depths its lanes are at), and deeper ones in local memory: a pop then costs
// a shared-memory read instead of a local load that mostly misses L1 behind
// the node stream.
struct LocalStack {
    uint32_t n[SB_STACK];
    float t[SB_STACK];
    __device__ __forceinline__ void set(int i, uint32_t r, float d)
    {
        n[i] = r;
        t[i] = d;
    }
    __device__ __forceinline__ uint32_t ref(int i) const { return n[i]; }
    __device__ __forceinline__ float dist(int i) const { return t[i]; }
};
struct LocalStackN {
    uint32_t n[SB_STACK];
    __device__ __forceinline__ void set(int i, uint32_t ref) { n[i] = ref; }
    __device__ __forceinline__ uint32_t get(int i) const { return n[i]; }
};
template <int STRIDE, int S>
struct SplitStack {
    uint2* sm;
    uint2 deep[SB_STACK - S];
    __device__ __forceinline__ void set(int i, uint32_t ref, float d)
    {
        const uint2 v = make_uint2(ref, __float_as_uint(d));
        if (i < S) sm[i * STRIDE] = v;
        else deep[i - S] = v;
    }
    __device__ __forceinline__ uint2 get(int i) const { return i < S ? sm[i * STRIDE] : deep[i - S]; }
    __device__ __forceinline__ uint32_t ref(int i) const { return get(i).x; }
    __device__ __forceinline__ float dist(int i) const { return __uint_as_float(get(i).y); }
};
template <int STRIDE, int S>
struct SplitStackN {
    uint32_t* sm;
    uint32_t deep[SB_STACK - S];
    __device__ __forceinline__ void set(int i, uint32_t ref)
    {
        if (i < S) sm[i * STRIDE] = ref;
        else deep[i - S] = ref;
    }
    __device__ __forceinline__ uint32_t get(int i) const { return i < S ? sm[i * STRIDE] : deep[i - S]; }
};

// Pops until an entry within the best hit is found (T.cur stays SB_INVALID
// when the stack runs out).  PAIR reads an entry's ref and distance with one
// access (split stacks only) instead of the distance first; both forms
// compute the same, and each kernel uses the one that compiles to fewer
// spilled registers.
template <bool PAIR = false, class STK>
__device__ __forceinline__ void closest_pop(Trav& T, const STK& st)
{
    const float lim = T.minHit * SB_PRUNE_SCALE;
    while (T.sp > 0) {
        --T.sp;
        if constexpr (PAIR) {
            const uint2 e = st.get(T.sp);
            if (!(__uint_as_float(e.y) > lim)) {
                T.cur = e.x;
                return;
            }
        } else {
            if (!(st.dist(T.sp) > lim)) {
                T.cur = st.ref(T.sp);
                return;
            }
        }
    }
}

// One closest-hit step: processes the 4-wide node T.cur (or the root leaf),
// then pops until a node to process is found.  Returns true when finished.
template <bool COUNT, class STK>
__device__ __forceinline__ bool closest_step(const DevScene& s, Trav& T, STK& st, uint32_t& nInner, uint32_t& nLeaf)
{
    const uint32_t cur = T.cur;
    if (cur != SB_INVALID) {
        if (++T.steps > s.numNodes + 1u) {
            raise_status(s, STRELKA_DEV_TRAVERSAL_CAP);
            return true;
        }
        if (cur & SB_LEAF_BIT) {
            if (COUNT) ++nLeaf;
            closest_leaf(s, T, cur & ~(SB_LEAF_BIT | SB_NOBOX_BIT));
            T.cur = SB_INVALID;
        } else {
            if (cur >= s.numWide) {
                raise_status(s, STRELKA_DEV_NODE_OOB);
                return true;
            }
            if (COUNT) ++nInner;
            // boxes first (so that the node's bounds are dead before the
            // triangle tests), then the leaves hit in the reference's order;
            // inner children hit within tmax become candidates
            uint32_t ref[4];
            float bt[4];
            bool pass[4];
            {
                const WideNode n = load_wide(s, cur);
                const float lim0 = T.minHit * SB_PRUNE_SCALE;
                const unsigned hitm = wide_boxes(T.r, n, bt);
#pragma unroll
                for (int k = 0; k < 4; ++k) {
                    ref[k] = n.ref[k];
                    pass[k] = ref[k] != SB_INVALID &&
                              ((ref[k] & SB_NOBOX_BIT) || (((hitm >> k) & 1u) && !(bt[k] > T.r.tmax) && !(bt[k] > lim0)));
                    if (ref[k] & SB_NOBOX_BIT) bt[k] = 0.0f;
                }
            }
            float ct[4];
            uint32_t cr[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                ct[k] = __int_as_float(0x7f800000);  // +inf: no candidate
                cr[k] = SB_INVALID;
                if (!pass[k]) continue;
                if (ref[k] & SB_LEAF_BIT) {
                    if (COUNT) ++nLeaf;
                    closest_leaf(s, T, ref[k] & ~(SB_LEAF_BIT | SB_NOBOX_BIT));
                } else {
                    ct[k] = bt[k];
                    cr[k] = ref[k];
                }
            }
            // nearest first: sort the (up to four) candidates by entry distance
            cswap(ct[0], cr[0], ct[1], cr[1]);
            cswap(ct[2], cr[2], ct[3], cr[3]);
            cswap(ct[0], cr[0], ct[2], cr[2]);
            cswap(ct[1], cr[1], ct[3], cr[3]);
            cswap(ct[1], cr[1], ct[2], cr[2]);
            const float lim = T.minHit * SB_PRUNE_SCALE;
            T.cur = (cr[0] != SB_INVALID && !(ct[0] > lim)) ? cr[0] : SB_INVALID;
            // the others onto the stack, farthest first
#pragma unroll
            for (int k = 3; k >= 1; --k) {
                if (cr[k] == SB_INVALID || ct[k] > lim) continue;
                if (T.sp < SB_STACK) {
                    st.set(T.sp, cr[k], ct[k]);
                    ++T.sp;
                } else {
                    // stack full: finish with the stackless loop from the root
                    const Fallback f = closest_stackless_rec<COUNT>(s, T.r, T.minHit, T.leaf, T.hit, T.found);
                    T.hit = f.hit;
                    T.minHit = f.minHit;
                    T.leaf = f.leaf;
                    T.found = f.found;
                    if (COUNT) {
                        nInner += f.nInner;
                        nLeaf += f.nLeaf;
                    }
                    T.cur = SB_INVALID;
                    T.sp = 0;
                    return true;
                }
            }
        }
    }
    if (T.cur == SB_INVALID) {
        closest_pop(T, st);
        if (T.cur == SB_INVALID) return true;
    }
    return false;
}

// ---------------------------------------------------------------------------
// Closest hit with leaf tests deferred and run together across the warp.
//
// A triangle test is about 70 instructions and a node step finds a passing
// leaf only about once in three, so testing leaves at the node that reaches
// them runs the test code with a few lanes of the warp active.  Here the
// passing leaves of a node join the thread's pending list (SB_DEFER_CAP
// entries in shared memory; entry j of a thread at pend[j * STRIDE]), the
// traversal goes on with the nearest inner entry, and every lane that waits
// tests its latest pending leaf when at least SB_DEFER_LANES lanes of the
// warp wait, or when a waiting lane cannot go on (nothing left to traverse,
// or no room for another node's leaves).  Pruning uses the best hit known at
// the time, which is never closer than the one the immediate order would
// know, so no subtree holding the closest hit is dropped; the tie rule on
// compact leaf indices makes the result independent of the test order.  The
// results are the reference's bit for bit; the nodes and tests counted depend
// on the warp's mix of rays.
#ifndef SB_DEFER_CAP
#define SB_DEFER_CAP 12
#endif
#ifndef SB_DEFER_LANES
#define SB_DEFER_LANES 16
#endif


// One node of the deferred traversal (T.cur is a 4-wide node or the root
// leaf; the caller guarantees room for four more pending leaves): passing
// leaves join the pending list, the nearest passing inner entry is next and
// the others go onto the stack, farthest first.  Returns true when the
// traversal ended early (a fault, the step cap, or the stackless fallback,
// which tests every leaf itself, pending ones included).
template <bool COUNT, int STRIDE, class STK>
__device__ __forceinline__ bool closest_defer_node(const DevScene& s, Trav& T, STK& st, uint32_t* pend, uint32_t& np,
                                                   uint32_t& nInner, uint32_t& nLeaf)
{
    const uint32_t cur = T.cur;
    if (++T.steps > s.numNodes + 1u) {
        raise_status(s, STRELKA_DEV_TRAVERSAL_CAP);
        return true;
    }
    if (cur & SB_LEAF_BIT) {
        pend[(np++) * STRIDE] = cur & ~(SB_LEAF_BIT | SB_NOBOX_BIT);
        T.cur = SB_INVALID;
        return false;
    }
    if (cur >= s.numWide) {
        raise_status(s, STRELKA_DEV_NODE_OOB);
        return true;
    }
    if (COUNT) ++nInner;
    float ct[4];
    uint32_t cr[4];
    {
        const WideNode n = load_wide(s, cur);
        const float lim0 = T.minHit * SB_PRUNE_SCALE;
        float bt[4];
        const unsigned hitm = wide_boxes(T.r, n, bt);
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const uint32_t ref = n.ref[k];
            const bool pass = ref != SB_INVALID &&
                              ((ref & SB_NOBOX_BIT) || (((hitm >> k) & 1u) && !(bt[k] > T.r.tmax) && !(bt[k] > lim0)));
            ct[k] = __int_as_float(0x7f800000);  // +inf: no candidate
            cr[k] = SB_INVALID;
            if (pass && (ref & SB_LEAF_BIT)) {
                pend[(np++) * STRIDE] = ref & ~(SB_LEAF_BIT | SB_NOBOX_BIT);
            } else if (pass) {
                ct[k] = bt[k];
                cr[k] = ref;
            }
        }
    }
    // nearest first; every candidate is within the best hit (tested above)
    cswap(ct[0], cr[0], ct[1], cr[1]);
    cswap(ct[2], cr[2], ct[3], cr[3]);
    cswap(ct[0], cr[0], ct[2], cr[2]);
    cswap(ct[1], cr[1], ct[3], cr[3]);
    cswap(ct[1], cr[1], ct[2], cr[2]);
    T.cur = cr[0];
#pragma unroll
    for (int k = 3; k >= 1; --k) {
        if (cr[k] == SB_INVALID) continue;
        if (T.sp < SB_STACK) {
            st.set(T.sp, cr[k], ct[k]);
            ++T.sp;
        } else {
            // stack full: finish with the stackless loop from the root
            const Fallback f = closest_stackless_rec<COUNT>(s, T.r, T.minHit, T.leaf, T.hit, T.found);
            T.hit = f.hit;
            T.minHit = f.minHit;
            T.leaf = f.leaf;
            T.found = f.found;
            if (COUNT) {
                nInner += f.nInner;
                nLeaf += f.nLeaf;
            }
            T.cur = SB_INVALID;
            T.sp = 0;
            return true;
        }
    }
    return false;
}

// The warp's deferred leaf tests.  All 32 lanes call it; `have` says whether
// the lane holds a query.
template <bool COUNT, int STRIDE>
__device__ __forceinline__ void closest_defer_leaves(const DevScene& s, Trav& T, bool have, const uint32_t* pend, uint32_t& np,
                                                     uint32_t& nLeaf)
{
    const bool wait = have && np != 0;
    const unsigned waiting = __ballot_sync(0xffffffffu, wait);
    const bool stuck = wait && (T.cur == SB_INVALID || np > SB_DEFER_CAP - 4);
    if (waiting && (__popc(waiting) >= SB_DEFER_LANES || __any_sync(0xffffffffu, stuck))) {
        if (wait) {
            --np;
            if (COUNT) ++nLeaf;
            closest_leaf(s, T, pend[np * STRIDE]);
        }
    }
}

// One any-hit step (the reference's depth-first order).  Returns true when
// finished; T.found tells whether a hit with t < tmax was found.
template <bool COUNT, bool INLINE_FALLBACK = false, class STK>
__device__ __forceinline__ bool any_step(const DevScene& s, Trav& T, STK& st, uint32_t& nInner, uint32_t& nLeaf)
{
    const uint32_t cur = T.cur;
    if (cur != SB_INVALID && !(cur & SB_LEAF_BIT)) {
        if (++T.steps > s.numNodes + 1u || cur >= s.numWide) {
            raise_status(s, cur >= s.numWide ? STRELKA_DEV_NODE_OOB : STRELKA_DEV_TRAVERSAL_CAP);
            return true;
        }
        if (COUNT) ++nInner;
        // the entries visited, in order: an ungated leaf always, a gated leaf
        // or an inner child when its box is hit within tmax (the reference
        // reaches the same leaves and nodes, raytracing.h:249-286); the first
        // is next, the others wait on the stack in order
        uint32_t ref[4];
        bool pass[4];
        {
            const WideNode n = load_wide(s, cur);
            float bt[4];
            const unsigned hitm = wide_boxes(T.r, n, bt);
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                ref[k] = n.ref[k];
                pass[k] = ref[k] != SB_INVALID &&
                          ((ref[k] & SB_NOBOX_BIT) || (((hitm >> k) & 1u) && !(bt[k] > T.r.tmax)));
            }
        }
        uint32_t first = SB_INVALID;
#pragma unroll
        for (int k = 3; k >= 0; --k) {
            if (!pass[k]) continue;
            if (first != SB_INVALID) {
                if (T.sp < SB_STACK) {
                    st.set(T.sp++, first);
                } else {
                    // stack full: the reference's stackless loop from the root
                    // gives the same first hit
                    const Fallback f = INLINE_FALLBACK ? any_stackless_loop<COUNT>(s, T.r, 0u, T.hit)
                                                       : any_stackless_rec<COUNT>(s, T.r, 0u, T.hit);
                    T.hit = f.hit;
                    T.found = f.found;
                    if (COUNT) {
                        nInner += f.nInner;
                        nLeaf += f.nLeaf;
                    }
                    T.cur = SB_INVALID;
                    T.sp = 0;
                    return true;
                }
            }
            first = ref[k];
        }
        T.cur = first;
    }
    // leaves reached as the next entry (the first of a node, or popped)
    for (;;) {
        if (T.cur == SB_INVALID) {
            if (T.sp == 0) return true;
            T.cur = st.get(--T.sp);
        }
        if (!(T.cur & SB_LEAF_BIT)) return false;
        if (COUNT) ++nLeaf;
        float t, bu, bv;
        uint32_t iid, pid;
        const bool isect = rec_triangle(s, T.r, T.cur & ~(SB_LEAF_BIT | SB_NOBOX_BIT), t, bu, bv, iid, pid);
        T.hit.t = t;
        if (isect && (t < T.r.tmax)) {
            T.hit.instId = iid;
            T.hit.primId = pid;
            T.found = true;
            return true;
        }
        T.cur = SB_INVALID;
    }
}

// LEAF_REF: the record's primId holds the hit's compact leaf index instead
// (for shade(), which reads the leaf's shading record).
template <bool COUNT, bool LEAF_REF = false>
__device__ __forceinline__ bool trace_closest_rec(const DevScene& s, v3 o, float tmax, v3 d, HitRec& hit, uint32_t& nInner,
                                                  uint32_t& nLeaf)
{
    LocalStack st;
    Trav T;
    trav_init(s, T, o, tmax, d, false);
    if (T.cur != SB_INVALID)
        while (!closest_step<COUNT>(s, T, st, nInner, nLeaf)) {
        }
    hit = T.hit;
    if (LEAF_REF) hit.primId = T.leaf;
    return T.found;
}

template <bool COUNT>
__device__ __forceinline__ bool trace_any_rec(const DevScene& s, v3 o, float tmax, v3 d, HitRec& hit, uint32_t& nInner,
                                              uint32_t& nLeaf)
{
    LocalStackN st;
    Trav T;
    trav_init(s, T, o, tmax, d, true);
    if (T.cur != SB_INVALID)
        while (!any_step<COUNT>(s, T, st, nInner, nLeaf)) {
        }
    hit = T.hit;
    return T.found;
}

}  // namespace sb
