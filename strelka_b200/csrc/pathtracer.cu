// pathtracer.cu — the path tracer pass (megakernel and wavefront forms) and
// the ray-query microbenchmark entry points, sm_100a.
//
// PathTracer::execute (src/render/pathtracer.cpp:50-59) dispatches
// computeMain (shaders/pathtracerMdl.hlsl:406-423) over W*H*spp threads.
// Here the same work runs either as
//   * a megakernel: one thread per (pixel, sample), the reference's shape, or
//   * a wavefront: per chunk of paths, generate -> [extend -> shade -> shadow]
//     x maxDepth -> finalize, each a separate kernel over structure-of-arrays
//     path state, with the surviving paths compacted by warp ballot into a
//     queue between bounces.
// Both forms call the same shade()/apply_shadow() device code.
#include <type_traits>
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include <cub/device/device_scan.cuh>

#include "common.h"
#include "nrc.h"
#include "refine.cuh"
#include "internal.h"
#include "shading.cuh"
#include "wave.cuh"

using namespace sb;

namespace {

constexpr int kExtendBlock = 128;
// Traversal stack entries kept in shared memory per thread (deeper ones in
// local memory), measured fastest per kernel: the wavefront closest-hit pass
// 8, its any-hit pass and the ray-query kernels 16.
constexpr int kExtendStackShared = 8;
constexpr int kShadowStackShared = 16;
#ifndef SB_TRACE_STACK_SHARED_CLOSEST
#define SB_TRACE_STACK_SHARED_CLOSEST 16
#endif
#ifndef SB_TRACE_STACK_SHARED_ANY
#define SB_TRACE_STACK_SHARED_ANY 16
#endif
constexpr int kShadeBlock = 128;
constexpr int kSmallBlock = 256;
constexpr uint32_t kMaxSortKeys = 4096;
constexpr uint32_t kDefaultQueueChunk = 32;
constexpr uint32_t kDefaultTailDepth = 5;  // first bounce finished by k_tail

// Minimum resident blocks per SM requested for the any-hit (shadow) kernel:
// 9 blocks of 128 threads fit its registers without spills (10 spill) and
// measured fastest (52.6 ms per large frame against 53.3 at 8 and 7).
#ifndef SB_SHADOW_MINBLOCKS
#define SB_SHADOW_MINBLOCKS 9
#endif
// The closest-hit kernel is latency-bound: 8 resident blocks (64 registers,
// 8 bytes spilled) beat 9 (56 registers, 110 bytes spilled) and 7.
// Shadow queries of bounce k overlap the closest-hit queries of bounce k+1.
#ifndef SB_OVERLAP_SHADOW
#define SB_OVERLAP_SHADOW 1
#endif
#ifndef SB_EXTEND_MINBLOCKS
#define SB_EXTEND_MINBLOCKS 8
#endif

enum KernelClass {
    KC_GENERATE = 0,
    KC_EXTEND,
    KC_SHADE,
    KC_SHADOW,
    KC_FINALIZE,
    KC_MEGAKERNEL,
    KC_PREP,
    KC_NRC_PATHS,
    KC_NRC_TRAIN,
    KC_NRC_INFER,
    KC_SORT,
    KC_TAIL,
    KC_COUNT
};
const char* kKernelNames[KC_COUNT] = {"generate",  "extend",    "shade",     "shadow",    "finalize", "megakernel",
                                      "prep",      "nrc_paths", "nrc_train", "nrc_infer", "sort", "tail"};

// ---------------------------------------------------------------------------
// Scene preparation: the record table of traverse.cuh, one record per leaf
// at the leaf's compact index leafOf[i] (its rank among the leaves in the
// depth-first node order): the triangle exactly as getTriangle computes it
// (raytracing.h:134-153).
__global__ void k_leaf_flag(const float4* __restrict__ nodes, uint32_t numNodes, uint32_t* __restrict__ flag)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < numNodes; i += gridDim.x * blockDim.x)
        flag[i] = __float_as_uint(nodes[2 * (size_t)i].w) != SB_INVALID ? 1u : 0u;
}

// Per-leaf shading record, 6 float4 at the leaf's compact index: the
// world-space positions and normals of its triangle's vertices and their
// UVs, with exactly the arithmetic the shade kernel applies at a hit
// (pathtracerMdl.hlsl:237-267), so reading them gives the same bits while a
// shaded hit reads 96 contiguous bytes instead of three indices and three
// vertices behind its instance record:
// [0] p0|u0  [1] p1|v0  [2] p2|u1  [3] n0|v1  [4] n1|u2  [5] n2|v2.
// Leaves that k_prep_rec rejects are never hit and are skipped here.
__global__ void k_prep_shade(const float4* __restrict__ nodes, uint32_t numNodes, const InstanceConstants* __restrict__ inst,
                             uint32_t numInstances, const uint32_t* __restrict__ ib, uint32_t numIndices,
                             const Vertex* __restrict__ vb, uint32_t numVertices, const uint32_t* __restrict__ leafOf,
                             uint32_t recCap, float4* __restrict__ out)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < numNodes; i += gridDim.x * blockDim.x) {
        const float4 lo = nodes[2 * (size_t)i];
        const uint32_t instId = __float_as_uint(lo.w);
        if (instId == SB_INVALID || instId >= numInstances) continue;
        const uint32_t li = leafOf[i];
        if (li >= recCap) continue;
        const InstanceConstants* ic = &inst[instId];
        const uint32_t base = (uint32_t)ic->indexOffset + __float_as_uint(lo.x) * 3u;
        if ((uint64_t)base + 2 >= numIndices) continue;
        const uint32_t i0 = ib[base], i1 = ib[base + 1], i2 = ib[base + 2];
        if (i0 >= numVertices || i1 >= numVertices || i2 >= numVertices) continue;
        const float* o2w = ic->objectToWorld.m;
        const float* nrm = ic->normalMatrix.m;
        const Vertex& V0 = vb[i0];
        const Vertex& V1 = vb[i1];
        const Vertex& V2 = vb[i2];
        const v3 p0 = mat_mul_point(o2w, V(V0.position[0], V0.position[1], V0.position[2]), 1.0f);
        const v3 p1 = mat_mul_point(o2w, V(V1.position[0], V1.position[1], V1.position[2]), 1.0f);
        const v3 p2 = mat_mul_point(o2w, V(V2.position[0], V2.position[1], V2.position[2]), 1.0f);
        const v3 n0 = mat_mul_dir3(nrm, unpack_normal(V0.normal));
        const v3 n1 = mat_mul_dir3(nrm, unpack_normal(V1.normal));
        const v3 n2 = mat_mul_dir3(nrm, unpack_normal(V2.normal));
        float uv0[2], uv1[2], uv2[2];
        unpack_uv(V0.uv, uv0[0], uv0[1]);
        unpack_uv(V1.uv, uv1[0], uv1[1]);
        unpack_uv(V2.uv, uv2[0], uv2[1]);
        float4* r = &out[6 * (size_t)li];
        r[0] = f4(p0, uv0[0]);
        r[1] = f4(p1, uv0[1]);
        r[2] = f4(p2, uv1[0]);
        r[3] = f4(n0, uv1[1]);
        r[4] = f4(n1, uv2[0]);
        r[5] = f4(n2, uv2[1]);
    }
}

__global__ void k_prep_rec(const float4* __restrict__ nodes, uint32_t numNodes, const InstanceConstants* __restrict__ inst,
                           uint32_t numInstances, const uint32_t* __restrict__ ib, uint32_t numIndices,
                           const Vertex* __restrict__ vb, uint32_t numVertices, const uint32_t* __restrict__ leafOf,
                           uint32_t recCap, float4* __restrict__ rec, uint32_t* status)
{
    const float qnan = __int_as_float(0x7fc00000);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < numNodes; i += gridDim.x * blockDim.x) {
        const float4 lo = nodes[2 * (size_t)i];
        const float4 hi = nodes[2 * (size_t)i + 1];
        const uint32_t instId = __float_as_uint(lo.w);
        const uint32_t esc = __float_as_uint(hi.w);
        if (esc != SB_INVALID && esc >= numNodes) atomicOr(status, STRELKA_DEV_NODE_OOB);
        if (instId == SB_INVALID) continue;  // inner nodes live in the 4-wide BVH
        const uint32_t li = leafOf[i];
        if (li >= recCap) {  // more leaves than a binary tree of numNodes nodes has
            atomicOr(status, STRELKA_DEV_NODE_OOB);
            continue;
        }
        float4* out = &rec[3 * (size_t)li];
        const float4 bad = make_float4(qnan, qnan, qnan, 0.0f);
        if (instId >= numInstances) {
            atomicOr(status, STRELKA_DEV_INSTANCE_OOB);
            out[0] = bad; out[1] = bad; out[2] = bad;
            continue;
        }
        const InstanceConstants* ic = &inst[instId];
        const uint32_t prim = __float_as_uint(lo.x);
        const uint32_t base = (uint32_t)ic->indexOffset + prim * 3u;
        if ((uint64_t)base + 2 >= numIndices) {
            atomicOr(status, STRELKA_DEV_INDEX_OOB);
            out[0] = bad; out[1] = bad; out[2] = bad;
            continue;
        }
        const uint32_t i0 = ib[base], i1 = ib[base + 1], i2 = ib[base + 2];
        if (i0 >= numVertices || i1 >= numVertices || i2 >= numVertices) {
            atomicOr(status, STRELKA_DEV_INDEX_OOB);
            out[0] = bad; out[1] = bad; out[2] = bad;
            continue;
        }
        const float* m = ic->objectToWorld.m;
        v3 v0 = mat_mul_point(m, V(vb[i0].position[0], vb[i0].position[1], vb[i0].position[2]), 1.0f);
        v3 e0 = vsub(mat_mul_point(m, V(vb[i1].position[0], vb[i1].position[1], vb[i1].position[2]), 1.0f), v0);
        v3 e1 = vsub(mat_mul_point(m, V(vb[i2].position[0], vb[i2].position[1], vb[i2].position[2]), 1.0f), v0);
        out[0] = f4(v0, __uint_as_float(instId));
        out[1] = f4(e0, __uint_as_float(prim));
        out[2] = f4(e1, 0.0f);
    }
}

// ---------------------------------------------------------------------------
// Megakernel: computeMain, one thread per (pixel, sample).
// ---------------------------------------------------------------------------
// The 4-wide BVH of traverse.cuh, derived from the reference's binary tree
// (implicit children: L = n+1, R = escape(n+1), bvh.cpp:182-220).  Its nodes
// are the binary inner nodes at even depth; each holds the children of its
// two binary children, in order:
//   a leaf child       -> an ungated leaf entry (tested whenever the node is;
//                         at the root, gated by the root's box, which the
//                         reference tests first);
//   an inner child c   -> c's two children: an inner one with its own box, a
//                         leaf one gated by c's box.
// A node's box test implies its parent's (the slab arithmetic rounds
// monotonically and a parent box contains its children's), so skipping the
// odd-depth boxes leaves the set of triangles a query tests unchanged.

// parent of every node (the root keeps SB_INVALID)
__global__ void k_wide_parent(const float4* __restrict__ nodes, uint32_t numNodes, uint32_t* __restrict__ parent)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < numNodes; i += gridDim.x * blockDim.x) {
        if (__float_as_uint(nodes[2 * (size_t)i].w) != SB_INVALID) continue;  // leaf
        const uint32_t L = i + 1;
        if (L >= numNodes) continue;
        parent[L] = i;
        const uint32_t R = __float_as_uint(nodes[2 * (size_t)L + 1].w);
        if (R != SB_INVALID && R < numNodes) parent[R] = i;
    }
}

// Steps a thread walks up towards the root in k_wide_flag before leaving
// the node to the pointer-jumping pass (deep trees, chains).
constexpr uint32_t kWideWalkCap = 1024;

// 1 for the inner nodes at even depth, by walking up to the root.  A walk
// longer than kWideWalkCap sets *deep instead, and the pointer-jumping pass
// below recomputes every node's parity, so a chain-shaped tree costs
// O(n log n), not O(n^2).
__global__ void k_wide_flag(const float4* __restrict__ nodes, uint32_t numNodes, const uint32_t* __restrict__ parent,
                            uint32_t* __restrict__ flag, uint32_t* deep, uint32_t* status)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < numNodes; i += gridDim.x * blockDim.x) {
        uint32_t f = 0;
        if (__float_as_uint(nodes[2 * (size_t)i].w) == SB_INVALID) {
            uint32_t p = i, depth = 0;
            bool ok = true;
            while (p != 0) {
                p = parent[p];
                if (p == SB_INVALID) {
                    ok = false;
                    break;
                }
                if (++depth > kWideWalkCap) {
                    atomicOr(deep, 1u);
                    break;
                }
            }
            if (!ok) atomicOr(status, STRELKA_DEV_NODE_OOB);
            f = ok && (depth & 1u) == 0 ? 1u : 0u;
        }
        flag[i] = f;
    }
}

// Pointer jumping (only when *deep): anc[i] is the ancestor 2^r levels up and
// par[i] the parity of that distance; after ceil(log2 n) + 1 rounds every
// ancestor is past the root and par[i] is the parity of the depth.
__global__ void k_wide_jump_init(uint32_t numNodes, const uint32_t* __restrict__ parent, uint32_t* __restrict__ par,
                                 const uint32_t* deep)
{
    if (!*deep) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < numNodes; i += gridDim.x * blockDim.x)
        par[i] = parent[i] != SB_INVALID ? 1u : 0u;
}
__global__ void k_wide_jump(uint32_t numNodes, const uint32_t* __restrict__ ancIn, const uint32_t* __restrict__ parIn,
                            uint32_t* __restrict__ ancOut, uint32_t* __restrict__ parOut, const uint32_t* deep)
{
    if (!*deep) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < numNodes; i += gridDim.x * blockDim.x) {
        const uint32_t a = ancIn[i];
        if (a == SB_INVALID || a >= numNodes) {
            ancOut[i] = a;
            parOut[i] = parIn[i];
        } else {
            ancOut[i] = ancIn[a];
            parOut[i] = parIn[i] ^ parIn[a];
        }
    }
}
__global__ void k_wide_jump_finish(const float4* __restrict__ nodes, uint32_t numNodes, const uint32_t* __restrict__ anc,
                                   const uint32_t* __restrict__ par, uint32_t* __restrict__ flag, const uint32_t* deep,
                                   uint32_t* status)
{
    if (!*deep) return;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < numNodes; i += gridDim.x * blockDim.x) {
        uint32_t f = 0;
        if (__float_as_uint(nodes[2 * (size_t)i].w) == SB_INVALID) {
            // an ancestor left means the parents form a cycle
            if (anc[i] != SB_INVALID) atomicOr(status, STRELKA_DEV_NODE_OOB);
            else f = par[i] == 0 ? 1u : 0u;
        }
        flag[i] = f;
    }
}

__global__ void k_wide_build(const float4* __restrict__ nodes, uint32_t numNodes, const uint32_t* __restrict__ flag,
                             const uint32_t* __restrict__ map, const uint32_t* __restrict__ leafOf, uint32_t recCap,
                             float4* __restrict__ wide, uint32_t wideCap, uint32_t* status)
{
    for (uint32_t P = blockIdx.x * blockDim.x + threadIdx.x; P < numNodes; P += gridDim.x * blockDim.x) {
        if (!flag[P]) continue;
        const uint32_t w = map[P];
        if (w >= wideCap) {
            atomicOr(status, STRELKA_DEV_NODE_OOB);
            continue;
        }
        float lo[3][4], hi[3][4];
        uint32_t ref[4] = {SB_INVALID, SB_INVALID, SB_INVALID, SB_INVALID};
        for (int a = 0; a < 3; ++a)
            for (int k = 0; k < 4; ++k) lo[a][k] = hi[a][k] = 0.0f;
        int e = 0;
        auto right_of = [&](uint32_t left) -> uint32_t {
            const uint32_t r = __float_as_uint(nodes[2 * (size_t)left + 1].w);
            return r < numNodes ? r : SB_INVALID;
        };
        auto put = [&](uint32_t r, uint32_t boxNode) {
            ref[e] = r;
            if (boxNode != SB_INVALID) {
                const float4 b0 = nodes[2 * (size_t)boxNode], b1 = nodes[2 * (size_t)boxNode + 1];
                lo[0][e] = b0.x; lo[1][e] = b0.y; lo[2][e] = b0.z;
                hi[0][e] = b1.x; hi[1][e] = b1.y; hi[2][e] = b1.z;
            }
            ++e;
        };
        const uint32_t L = P + 1 < numNodes ? P + 1 : SB_INVALID;
        const uint32_t child[2] = {L, L != SB_INVALID ? right_of(L) : SB_INVALID};
        bool bad = child[0] == SB_INVALID || child[1] == SB_INVALID;
        // a leaf's ref is its compact record index
        auto leaf_ref = [&](uint32_t node) -> uint32_t {
            const uint32_t li = leafOf[node];
            if (li >= recCap) {
                bad = true;
                return SB_INVALID;
            }
            return li;
        };
        for (int k = 0; k < 2; ++k) {
            const uint32_t c = child[k];
            if (c == SB_INVALID) continue;
            if (__float_as_uint(nodes[2 * (size_t)c].w) != SB_INVALID) {
                // below the root a node is entered only after its box passed;
                // the root's own box is tested here, before its leaf children
                const uint32_t li = leaf_ref(c);
                if (li == SB_INVALID) put(SB_INVALID, SB_INVALID);
                else if (P == 0) put(li | SB_LEAF_BIT, P);
                else put(li | SB_LEAF_BIT | SB_NOBOX_BIT, SB_INVALID);
                continue;
            }
            const uint32_t g0 = c + 1 < numNodes ? c + 1 : SB_INVALID;
            const uint32_t grand[2] = {g0, g0 != SB_INVALID ? right_of(g0) : SB_INVALID};
            bad = bad || grand[0] == SB_INVALID || grand[1] == SB_INVALID;
            for (int j = 0; j < 2; ++j) {
                const uint32_t g = grand[j];
                if (g == SB_INVALID) continue;
                if (__float_as_uint(nodes[2 * (size_t)g].w) != SB_INVALID) {
                    const uint32_t li = leaf_ref(g);
                    put(li == SB_INVALID ? SB_INVALID : (li | SB_LEAF_BIT), c);
                }
                else if (flag[g] && map[g] < wideCap) put(map[g], g);
                else bad = true;
            }
        }
        if (bad) atomicOr(status, STRELKA_DEV_NODE_OOB);
        float4* out = &wide[8 * (size_t)w];
        out[0] = make_float4(lo[0][0], lo[0][1], lo[0][2], lo[0][3]);
        out[1] = make_float4(lo[1][0], lo[1][1], lo[1][2], lo[1][3]);
        out[2] = make_float4(lo[2][0], lo[2][1], lo[2][2], lo[2][3]);
        out[3] = make_float4(hi[0][0], hi[0][1], hi[0][2], hi[0][3]);
        out[4] = make_float4(hi[1][0], hi[1][1], hi[1][2], hi[1][3]);
        out[5] = make_float4(hi[2][0], hi[2][1], hi[2][2], hi[2][3]);
        out[6] = make_float4(__uint_as_float(ref[0]), __uint_as_float(ref[1]), __uint_as_float(ref[2]),
                             __uint_as_float(ref[3]));
        out[7] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
}

__global__ void __launch_bounds__(kExtendBlock) k_megakernel(DevScene s, PathTracerParam ubo, float* __restrict__ sampleBuffer,
                                                             uint64_t first, uint64_t count)
{
    const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    const uint64_t idx = first + t;
    PathState ps;
    init_path(ubo, idx, ps);
    const int maxDepth = (int)ubo.maxDepth;
    while (ps.depth < maxDepth) {
        HitRec h;
        uint32_t a = 0, b = 0;
        bool found = s.numNodes != 0 && trace_closest_rec<false, true>(s, ps.ro, ps.tmax, ps.rd, h, a, b);
        ShadowReq sr;
        bool cont = shade(s, ubo, ps, found, h, sr);
        if (sr.kind != 0 && shadow_visible(s, sr.kind, sr.o, sr.tmax, sr.d)) apply_shadow(ps.color, sr.cd, sr.cg);
        if (!cont) break;
        ++ps.depth;
    }
    sampleBuffer[idx * 3 + 0] = ps.color.x;
    sampleBuffer[idx * 3 + 1] = ps.color.y;
    sampleBuffer[idx * 3 + 2] = ps.color.z;
}

constexpr int kNrcMaxVerts = 16;  // training vertices recorded per path

struct WaveBuf {
    Wave w{};
    uint32_t* sorted = nullptr;  // the shade queue in material order
    uint16_t* keys = nullptr;    // sort key of each queue entry
    size_t cap = 0;
    std::vector<void*> allocs;
};

// Radiance-cache queries of the wavefront (paths that end at a cache lookup).
struct NrcWave {
    StrelkaNrcRecord* queries;
    uint32_t* count;
    uint32_t capacity;
    int enabled;
    float diffuseRoughness;
};

// Shadow-request count of a bounce: counters[2] on even bounces, [6] on odd
// ones, so that shadow(k) can read its count while extend(k+1) resets the
// count shade(k+1) will fill.
__host__ __device__ __forceinline__ int shadow_count(int qin) { return qin ? 6 : 2; }

__global__ void __launch_bounds__(kSmallBlock) k_generate(PathTracerParam ubo, Wave w, uint64_t first, uint32_t n)
{
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        w.counters[0] = n;
        w.counters[1] = 0;
        w.counters[2] = 0;
        w.counters[3] = 0;  // extend's work-queue head
        w.counters[6] = 0;
        w.counters[7] = 0;  // the tail kernel's work-queue head
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        PathState ps;
        init_path(ubo, first + i, ps);
        w.ray_o[i] = f4(ps.ro, ps.tmax);
        w.ray_d[i] = f4(ps.rd, ps.lastPdf);
        w.thr[i] = f4(ps.throughput, __uint_as_float(pack_flags(ps)));
        w.col[i] = f4(ps.color, 0.0f);
        w.rng[i] = ps.rng;
        w.queue[0][i] = i;
    }
}

// extend: closest-hit query for every queued path.  Warps take `chunk`
// queue entries at a time from an atomic head, and a lane takes its next
// path as soon as its current query ends (the warp keeps stepping while any
// lane has work), so neither a warp nor a CTA waits for its longest ray.
// DEFER: leaf tests deferred across the warp with the split stack (for
// incoherent rays); otherwise tested where reached, on a local-memory stack
// (coherent rays, whose lanes already test the same leaves together).
template <bool COUNT, bool DEFER>
__global__ void __launch_bounds__(kExtendBlock, SB_EXTEND_MINBLOCKS) k_extend(DevScene s, Wave w, int qin, uint32_t chunk,
                                                         unsigned long long* visitCounters)
{
    const uint32_t count = w.counters[qin];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        w.counters[qin ^ 1] = 0;           // consumed by shade(k-1); refilled by shade(k)
        w.counters[shadow_count(qin)] = 0; // consumed by shadow(k-2); refilled by shade(k)
        w.counters[4] = 0;                 // shade's work-queue head
    }
    const uint32_t* __restrict__ q = qin ? w.queue[1] : w.queue[0];
    using Stack = std::conditional_t<DEFER, SplitStack<kExtendBlock, kExtendStackShared>, LocalStack>;
    __shared__ uint2 sStack[DEFER ? kExtendStackShared * kExtendBlock : 1];
    __shared__ uint32_t sPend[DEFER ? SB_DEFER_CAP * kExtendBlock : 1];  // deferred leaf tests
    Stack st;
    if constexpr (DEFER) st.sm = &sStack[threadIdx.x];
    uint32_t* pend = &sPend[DEFER ? threadIdx.x : 0];
    uint32_t nI = 0, nL = 0, nR = 0;
    WarpPool pool{0, 0, 0};
    uint32_t slot = 0;
    Trav T;
    const uint32_t root = trav_root(s);
    uint32_t np = 0;
    bool have = false;
    while (true) {
        const uint32_t i = pool_take(pool, &w.counters[3], count, chunk, !have);
        if (!have && i != SB_INVALID) {
            slot = q[i];
            const float4 o = w.ray_o[slot], d = w.ray_d[slot];
            trav_init_root(T, xyz(o), o.w, xyz(d), false, root);
            np = 0;
            have = true;
        }
        if (!__any_sync(0xffffffffu, have)) break;
        if constexpr (DEFER) closest_defer_leaves<COUNT, kExtendBlock>(s, T, have, pend, np, nL);
        if (!have) continue;
        if constexpr (DEFER) {
            bool fin = false;
            if (T.cur != SB_INVALID && np <= SB_DEFER_CAP - 4) {
                fin = closest_defer_node<COUNT, kExtendBlock>(s, T, st, pend, np, nI, nL);
                if (fin) np = 0;
            }
            if (!fin && T.cur == SB_INVALID) closest_pop<true>(T, st);
            if (!fin && !(T.cur == SB_INVALID && np == 0)) continue;
        } else {
            if (!(T.cur == SB_INVALID || closest_step<COUNT>(s, T, st, nI, nL))) continue;
        }
        w.hit[slot] = T.found ? make_float4(T.hit.u, T.hit.v, T.hit.t, __uint_as_float(T.hit.instId))
                              : make_float4(0.0f, 0.0f, 1e9f, __uint_as_float(SB_INVALID));
        w.hitRef[slot] = T.found ? T.leaf : SB_INVALID;  // k_shade reads the leaf's shading record
        if (COUNT) ++nR;
        have = false;
    }
    if (COUNT) {
        atomicAdd(&visitCounters[0], (unsigned long long)nI);
        atomicAdd(&visitCounters[1], (unsigned long long)nL);
        atomicAdd(&visitCounters[4], (unsigned long long)nR);
    }
}

// Shade-queue sort (a counting sort by the hit's material, so the warps of
// k_shade see few BSDF kinds): key 0 = miss, 1 + material id, numMaterials
// + 1 for light instances and out-of-range ids.
__device__ __forceinline__ uint32_t shade_key(const DevScene& s, const Wave& w, uint32_t slot)
{
    const uint32_t inst = __float_as_uint(w.hit[slot].w);
    if (inst == SB_INVALID) return 0;
    const uint32_t nm = s.numMaterials;
    if (inst >= s.numInstances) return 1 + nm;
    const uint32_t m = (uint32_t)__ldg(&s.inst[inst].materialId);
    return 1 + (m < nm ? m : nm);
}

// Keys of the queue in queue order (keys[i] for entry i) and their histogram.
__global__ void __launch_bounds__(kSmallBlock) k_sort_count(DevScene s, Wave w, int qin, uint32_t numKeys, uint32_t* hist,
                                                            uint16_t* keys)
{
    __shared__ uint32_t sh[kMaxSortKeys];
    for (uint32_t k = threadIdx.x; k < numKeys; k += blockDim.x) sh[k] = 0;
    __syncthreads();
    const uint32_t count = w.counters[qin];
    const uint32_t* __restrict__ q = qin ? w.queue[1] : w.queue[0];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint32_t key = shade_key(s, w, q[i]);
        keys[i] = (uint16_t)key;
        atomicAdd(&sh[key], 1u);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < numKeys; k += blockDim.x)
        if (sh[k]) atomicAdd(&hist[k], sh[k]);
}

// Exclusive scan of the histogram into offsets (one block), clearing the
// histogram for the next bounce.
__global__ void __launch_bounds__(1024) k_sort_scan(uint32_t* hist, uint32_t numKeys, uint32_t* offsets)
{
    __shared__ uint32_t part[1024];
    const uint32_t per = (numKeys + 1023) / 1024;
    const uint32_t k0 = threadIdx.x * per;
    uint32_t sum = 0;
    for (uint32_t k = k0; k < min(k0 + per, numKeys); ++k) sum += hist[k];
    part[threadIdx.x] = sum;
    __syncthreads();
    for (int off = 1; off < 1024; off <<= 1) {
        const uint32_t v = threadIdx.x >= (unsigned)off ? part[threadIdx.x - off] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = part[threadIdx.x] - sum;
    for (uint32_t k = k0; k < min(k0 + per, numKeys); ++k) {
        const uint32_t h = hist[k];
        offsets[k] = run;
        run += h;
        hist[k] = 0;
    }
}

// Scatter in tiles of kSortTile entries: ranks within the tile come from
// shared-memory counters (one atomic per key per warp), and each tile
// reserves its range of every key with one global atomic per key.
constexpr int kSortPerThread = 8;
constexpr int kSortTile = kSmallBlock * kSortPerThread;

__global__ void __launch_bounds__(kSmallBlock) k_sort_scatter(Wave w, int qin, uint32_t numKeys, const uint16_t* __restrict__ keys,
                                                              uint32_t* offsets, uint32_t* sorted)
{
    __shared__ uint32_t cnt[kMaxSortKeys];
    const uint32_t count = w.counters[qin];
    const uint32_t* __restrict__ q = qin ? w.queue[1] : w.queue[0];
    const int lane = threadIdx.x & 31;
    for (uint32_t tile = blockIdx.x * (uint32_t)kSortTile; tile < count; tile += gridDim.x * (uint32_t)kSortTile) {
        for (uint32_t k = threadIdx.x; k < numKeys; k += blockDim.x) cnt[k] = 0;
        __syncthreads();
        uint32_t key[kSortPerThread], rank[kSortPerThread];
#pragma unroll
        for (int j = 0; j < kSortPerThread; ++j) {
            const uint32_t i = tile + (uint32_t)j * kSmallBlock + threadIdx.x;
            const bool valid = i < count;
            key[j] = valid ? keys[i] : 0xFFFFu;
            const unsigned peers = __match_any_sync(0xffffffffu, key[j]);
            const int leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (valid && lane == leader) base = atomicAdd(&cnt[key[j]], (uint32_t)__popc(peers));
            base = __shfl_sync(0xffffffffu, base, leader);
            rank[j] = base + __popc(peers & ((1u << lane) - 1u));
        }
        __syncthreads();
        for (uint32_t k = threadIdx.x; k < numKeys; k += blockDim.x)
            if (cnt[k]) cnt[k] = atomicAdd(&offsets[k], cnt[k]);
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kSortPerThread; ++j) {
            const uint32_t i = tile + (uint32_t)j * kSmallBlock + threadIdx.x;
            if (i < count) sorted[cnt[key[j]] + rank[j]] = q[i];
        }
        __syncthreads();
    }
}

// shade: one bounce of shading for every queued path; pushes surviving
// paths to the other queue and next-event requests to the shadow queue.
// Shading is latency-bound at the 128 registers it would take; 5 resident
// blocks (a few spills) hide more of its gathers than 4.
// First bounce whose shade queue is sorted by material: camera rays (bounce
// 0) arrive in pixel order and hit coherent materials already, so sorting
// them costs more than it saves (52.6 -> 52.2 ms per large frame without).
#ifndef SB_SORT_FROM_DEPTH
#define SB_SORT_FROM_DEPTH 1
#endif
#ifndef SB_SHADE_MINBLOCKS
#define SB_SHADE_MINBLOCKS 5
#endif

template <bool NRC>
__global__ void __launch_bounds__(kShadeBlock, SB_SHADE_MINBLOCKS) k_shade(DevScene s, PathTracerParam ubo, Wave w, int qin,
                                                       const uint32_t* order, uint32_t chunk, NrcWave nw)
{
    const uint32_t count = w.counters[qin];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        w.counters[3] = 0;  // the next extend's work-queue head
        w.counters[5] = 0;  // this bounce's shadow work-queue head
    }
    const uint32_t* __restrict__ q = order ? order : (qin ? w.queue[1] : w.queue[0]);
    uint32_t* qout = qin ? w.queue[0] : w.queue[1];
    const int maxDepth = (int)ubo.maxDepth;
    const int lane = threadIdx.x & 31;
    uint32_t next = 0, end = 0;
    while (true) {
        if (next >= end) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(&w.counters[4], chunk);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base >= count) break;
            next = base;
            end = (uint32_t)min((uint64_t)base + chunk, (uint64_t)count);
        }
        const uint32_t i = next + lane;
        next = min(next + 32u, end);
        const bool valid = i < end;
        bool cont = false;
        ShadowReq sr;
        sr.kind = 0;
        uint32_t slot = 0;
        bool query = false;
        NrcShade nq;
        nq.has = false;
        nq.terminate = false;
        v3 qdir = V(0.0f, 0.0f, 0.0f), qthr = V(0.0f, 0.0f, 0.0f);
        if (valid) {
            slot = q[i];
            const float4 o = w.ray_o[slot];
            const float4 d = w.ray_d[slot];
            const float4 t4 = w.thr[slot];
            const float4 c4 = w.col[slot];
            PathState ps;
            ps.ro = xyz(o);
            ps.tmax = o.w;
            ps.rd = xyz(d);
            ps.lastPdf = d.w;
            ps.throughput = xyz(t4);
            const uint32_t fl = __float_as_uint(t4.w);
            ps.depth = (int)(fl & 0xffffu);
            ps.specular = (fl >> 16) & 1u;
            ps.inside = (fl >> 17) & 1u;
            ps.nrcReady = (fl >> 18) & 1u;
            ps.color = xyz(c4);
            ps.rng = w.rng[slot];
            const float4 h4 = w.hit[slot];
            HitRec h;
            h.u = h4.x;
            h.v = h4.y;
            h.t = h4.z;
            h.instId = __float_as_uint(h4.w);
            h.primId = w.hitRef[slot];  // the compact leaf index (shade reads its shading record)
            const bool found = h.instId != SB_INVALID;
            if (NRC) {
                nq.mode = 2;
                nq.diffuseRoughness = nw.diffuseRoughness;
                nq.has = false;
                nq.terminate = false;
                cont = shade(s, ubo, ps, found, h, sr, &nq);
                if (nq.terminate) {
                    query = true;
                    qdir = vneg(ps.rd);
                    qthr = ps.throughput;
                }
            } else {
                cont = shade(s, ubo, ps, found, h, sr);
            }
            if (cont) {
                ++ps.depth;
                cont = ps.depth < maxDepth;
            }
            w.ray_o[slot] = f4(ps.ro, ps.tmax);
            w.ray_d[slot] = f4(ps.rd, ps.lastPdf);
            w.thr[slot] = f4(ps.throughput, __uint_as_float(pack_flags(ps)));
            w.col[slot] = f4(ps.color, 0.0f);
            w.rng[slot] = ps.rng;
        }
        const uint32_t qpos = warp_push(&w.counters[qin ^ 1], cont);
        if (cont) qout[qpos] = slot;
        if (NRC) {
            const uint32_t qpos2 = warp_push(nw.count, query);
            if (query && qpos2 < nw.capacity) {
                StrelkaNrcRecord r;
                r.pos[0] = nq.pos.x; r.pos[1] = nq.pos.y; r.pos[2] = nq.pos.z;
                r.dir[0] = qdir.x; r.dir[1] = qdir.y; r.dir[2] = qdir.z;
                r.normal[0] = nq.normal.x; r.normal[1] = nq.normal.y; r.normal[2] = nq.normal.z;
                r.roughness = nq.rough;
                r.target[0] = qthr.x; r.target[1] = qthr.y; r.target[2] = qthr.z;
                r.slot = slot;
                r.pad[0] = 0;
                r.pad[1] = 0;
                nw.queries[qpos2] = r;
            }
        }
        const bool hasShadow = sr.kind != 0;
        const uint32_t spos = warp_push(&w.counters[shadow_count(qin)], hasShadow);
        if (hasShadow) {
            w.sh_o[spos] = f4(sr.o, sr.tmax);
            w.sh_d[spos] = f4(sr.d, __uint_as_float(slot));
            w.sh_cd[spos] = f4(sr.cd, __uint_as_float((uint32_t)sr.kind));
            w.sh_cg[spos] = f4(sr.cg, 0.0f);
        }
    }
}

// shadow: any-hit query for every next-event request (reference depth-first
// order); adds the visible ones.  Work is taken from an atomic queue in
// `chunk` units as in k_extend.
// SPLIT: the split stack and the inlined stackless fallback (large scenes).
template <bool COUNT, bool SPLIT>
__global__ void __launch_bounds__(kExtendBlock, SB_SHADOW_MINBLOCKS) k_shadow(DevScene s, Wave w, int qin, uint32_t chunk,
                                                                              unsigned long long* visitCounters)
{
    const uint32_t count = w.counters[shadow_count(qin)];
    using Stack = std::conditional_t<SPLIT, SplitStackN<kExtendBlock, kShadowStackShared>, LocalStackN>;
    __shared__ uint32_t sStack[SPLIT ? kShadowStackShared * kExtendBlock : 1];
    Stack st;
    if constexpr (SPLIT) st.sm = &sStack[threadIdx.x];
    uint32_t nI = 0, nL = 0, nR = 0;
    WarpPool pool{0, 0, 0};
    uint32_t item = 0;
    Trav T;
    const uint32_t root = trav_root(s);
    bool have = false;
    while (true) {
        const uint32_t i = pool_take(pool, &w.counters[5], count, chunk, !have);
        if (!have && i != SB_INVALID) {
            item = i;
            const float4 o = w.sh_o[i], d = w.sh_d[i];
            trav_init_root(T, xyz(o), o.w, xyz(d), true, root);
            have = true;
        }
        if (!__any_sync(0xffffffffu, have)) break;
        if (!have) continue;
        const bool done = T.cur == SB_INVALID || any_step<COUNT, SPLIT>(s, T, st, nI, nL);
        if (!done) continue;
        const float4 cd = w.sh_cd[item];
        const int kind = (int)__float_as_uint(cd.w);
        const bool visible = !T.found || (kind == 1 && T.hit.instId < s.numInstances &&
                                          __ldg(&s.inst[T.hit.instId].lightId) != -1);
        if (visible) {
            const uint32_t slot = __float_as_uint(w.sh_d[item].w);
            const float4 cg = w.sh_cg[item];
            v3 c = xyz(w.col[slot]);
            apply_shadow(c, xyz(cd), xyz(cg));
            w.col[slot] = f4(c, 0.0f);
        }
        if (COUNT) ++nR;
        have = false;
    }
    if (COUNT) {
        atomicAdd(&visitCounters[2], (unsigned long long)nI);
        atomicAdd(&visitCounters[3], (unsigned long long)nL);
        atomicAdd(&visitCounters[5], (unsigned long long)nR);
    }
}

// Finishes every path still queued for bounce `depth` (queue qin) with the
// megakernel loop (closest hit, shade, shadow inline) to its end.  Used for
// the last bounces, where few paths remain and a launch sequence per bounce
// costs more than their work; each lane takes queued paths from an atomic
// head.  Same device code and order of additions as the wavefront.
__global__ void __launch_bounds__(kExtendBlock) k_tail(DevScene s, PathTracerParam ubo, Wave w, int qin, uint32_t chunk)
{
    const uint32_t count = w.counters[qin];
    const uint32_t* __restrict__ q = qin ? w.queue[1] : w.queue[0];
    const int maxDepth = (int)ubo.maxDepth;
    WarpPool pool{0, 0, 0};
    PathState ps;
    uint32_t slot = 0;
    bool have = false;
    while (true) {
        // one bounce per iteration; a lane whose path ended takes the next
        const uint32_t got = pool_take(pool, &w.counters[7], count, chunk, !have);
        if (!have && got != SB_INVALID) {
            slot = q[got];
            const float4 o = w.ray_o[slot];
            const float4 d = w.ray_d[slot];
            const float4 t4 = w.thr[slot];
            ps.ro = xyz(o);
            ps.tmax = o.w;
            ps.rd = xyz(d);
            ps.lastPdf = d.w;
            ps.throughput = xyz(t4);
            const uint32_t fl = __float_as_uint(t4.w);
            ps.depth = (int)(fl & 0xffffu);
            ps.specular = (fl >> 16) & 1u;
            ps.inside = (fl >> 17) & 1u;
            ps.nrcReady = (fl >> 18) & 1u;
            ps.color = xyz(w.col[slot]);
            ps.rng = w.rng[slot];
            have = true;
        }
        if (!__any_sync(0xffffffffu, have)) break;
        if (!have) continue;
        HitRec h;
        uint32_t a = 0, b = 0;
        const bool found = s.numNodes != 0 && trace_closest_rec<false, true>(s, ps.ro, ps.tmax, ps.rd, h, a, b);
        ShadowReq sr;
        const bool cont = shade(s, ubo, ps, found, h, sr);
        if (sr.kind != 0 && shadow_visible(s, sr.kind, sr.o, sr.tmax, sr.d)) apply_shadow(ps.color, sr.cd, sr.cg);
        if (cont && ++ps.depth < maxDepth) continue;
        w.col[slot] = f4(ps.color, 0.0f);
        have = false;
    }
}

__global__ void __launch_bounds__(kSmallBlock) k_finalize(Wave w, float* __restrict__ sampleBuffer, uint64_t first, uint32_t n)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 c = w.col[i];
        float* o = sampleBuffer + (first + i) * 3;
        o[0] = c.x;
        o[1] = c.y;
        o[2] = c.z;
    }
}

// ---------------------------------------------------------------------------
// Radiance-cache training paths: plain paths from random samples of the frame
// (a decorrelated RNG stream per batch), one thread per path; every shading
// vertex k becomes a training record with target (C_end - C_k) / T_k, where
// C_k and T_k are the path's colour and throughput on arrival at k and C_end
// its final colour.  Path i belongs to batch i / pathsPerBatch, whose records
// are appended at out + batch * capPerBatch through count[batch].  The paths
// are few and long, so they run in small blocks spread over many SMs.
constexpr int kNrcPathBlock = 32;

// Writes the training records of a finished path: every recorded vertex k
// with target (C_end - C_k) / T_k.
__device__ __forceinline__ void nrc_emit_records(const float4 (&vrec)[kNrcMaxVerts][3], const v3 (&cIn)[kNrcMaxVerts],
                                                 const v3 (&tIn)[kNrcMaxVerts], int nv, v3 cEnd, StrelkaNrcRecord* dst,
                                                 uint32_t* count, uint32_t cap)
{
    for (int k = 0; k < nv; ++k) {
        const v3 t = tIn[k];
        if (!(t.x > 0.0f && t.y > 0.0f && t.z > 0.0f)) continue;
        const v3 L = V((cEnd.x - cIn[k].x) / t.x, (cEnd.y - cIn[k].y) / t.y, (cEnd.z - cIn[k].z) / t.z);
        if (!all_finite(L)) continue;
        const uint32_t pos = atomicAdd(count, 1u);
        if (pos >= cap) continue;
        StrelkaNrcRecord r;
        r.pos[0] = vrec[k][0].x; r.pos[1] = vrec[k][0].y; r.pos[2] = vrec[k][0].z;
        r.dir[0] = vrec[k][1].x; r.dir[1] = vrec[k][1].y; r.dir[2] = vrec[k][1].z;
        r.normal[0] = vrec[k][1].w; r.normal[1] = vrec[k][2].x; r.normal[2] = vrec[k][2].y;
        r.roughness = vrec[k][0].w;
        r.target[0] = fmaxf(L.x, 0.0f);
        r.target[1] = fmaxf(L.y, 0.0f);
        r.target[2] = fmaxf(L.z, 0.0f);
        r.slot = 0;
        r.pad[0] = 0;
        r.pad[1] = 0;
        dst[pos] = r;
    }
}

// Training paths of the radiance cache: path i of batch i / pathsPerBatch
// starts at a hashed sample of the frame and is traced to its end; every
// vertex becomes a record (nrc_emit_records).  Persistent lanes: a lane takes
// path indices from an atomic head (*head, zero at launch) and, when its path
// ends, takes the next one, bounce by bounce, so no warp waits for its
// longest path.
__global__ void __launch_bounds__(kNrcPathBlock) k_nrc_train_paths(DevScene s, PathTracerParam ubo, uint32_t pathsPerBatch,
                                                                   uint32_t batches, float diffuseRoughness,
                                                                   StrelkaNrcRecord* __restrict__ out, uint32_t* count,
                                                                   uint32_t capPerBatch, uint32_t* head)
{
    const uint32_t n = pathsPerBatch * batches;
    const uint64_t total = (uint64_t)ubo.dimension[0] * (uint64_t)ubo.dimension[1] * (uint64_t)ubo.spp;
    const int maxDepth = (int)ubo.maxDepth;
    WarpPool pool{0, 0, 0};
    bool have = false;
    uint32_t batch = 0;
    PathTracerParam u = ubo;
    PathState ps;
    float4 vrec[kNrcMaxVerts][3];
    v3 cIn[kNrcMaxVerts], tIn[kNrcMaxVerts];
    int nv = 0;
    while (true) {
        const uint32_t i = pool_take(pool, head, n, 32, !have);
        if (!have && i != SB_INVALID) {
            batch = i / pathsPerBatch;
            const uint32_t fseed = jenkins_hash((ubo.frameNumber + batch * 0x2545F491u) ^ 0x5bd1e995u);
            const uint32_t h = jenkins_hash(i * 0x9E3779B9u ^ fseed);
            u.frameNumber = (ubo.frameNumber + batch * 0x2545F491u) ^ 0x3c6ef372u;
            init_path(u, (uint64_t)h % total, ps);
            nv = 0;
            have = ps.depth < maxDepth;  // else nothing to trace and no vertex to record
        }
        // (every lane reaches the vote: pool_take and __any_sync are warp-collective)
        if (!__any_sync(0xffffffffu, have)) break;
        if (!have) continue;
        HitRec hit;
        uint32_t a = 0, b = 0;
        const bool found = s.numNodes != 0 && trace_closest_rec<false, true>(s, ps.ro, ps.tmax, ps.rd, hit, a, b);
        const v3 c0 = ps.color, t0 = ps.throughput, dOut = vneg(ps.rd);
        NrcShade nq;
        nq.mode = 1;
        nq.diffuseRoughness = diffuseRoughness;
        nq.has = false;
        nq.terminate = false;
        ShadowReq sr;
        const bool cont = shade(s, u, ps, found, hit, sr, &nq);
        if (sr.kind != 0 && shadow_visible(s, sr.kind, sr.o, sr.tmax, sr.d)) apply_shadow(ps.color, sr.cd, sr.cg);
        if (nq.has && nv < kNrcMaxVerts) {
            vrec[nv][0] = f4(nq.pos, nq.rough);
            vrec[nv][1] = f4(dOut, nq.normal.x);
            vrec[nv][2] = make_float4(nq.normal.y, nq.normal.z, 0.0f, 0.0f);
            cIn[nv] = c0;
            tIn[nv] = t0;
            ++nv;
        }
        if (cont && ++ps.depth < maxDepth) continue;
        nrc_emit_records(vrec, cIn, tIn, nv, ps.color, out + (size_t)batch * capPerBatch, &count[batch], capPerBatch);
        have = false;
    }
}

// ---------------------------------------------------------------------------
// Ray-query microbenchmark kernels.
// Resident blocks asked of the ray-query kernel: 8 for closest hit and 9 for
// any hit measured fastest on the 1M-triangle soup (few spills either way).
#ifndef SB_TRACE_MINBLOCKS_CLOSEST
#define SB_TRACE_MINBLOCKS_CLOSEST 8
#endif
#ifndef SB_TRACE_MINBLOCKS_ANY
#define SB_TRACE_MINBLOCKS_ANY 9
#endif
template <bool ANY, bool COUNT, bool REFINE>
__global__ void __launch_bounds__(kExtendBlock, ANY ? SB_TRACE_MINBLOCKS_ANY : SB_TRACE_MINBLOCKS_CLOSEST)
    k_trace(DevScene s, const float4* __restrict__ rays, Hit* __restrict__ hits, uint32_t n, uint32_t* head,
            uint32_t chunk, unsigned long long* counters)
{
    // traversal stack entries kept in shared memory per thread
    constexpr int kTraceStackShared = ANY ? SB_TRACE_STACK_SHARED_ANY : SB_TRACE_STACK_SHARED_CLOSEST;
    using Stack = std::conditional_t<ANY, SplitStackN<kExtendBlock, kTraceStackShared>,
                                     SplitStack<kExtendBlock, kTraceStackShared>>;
    __shared__ std::conditional_t<ANY, uint32_t, uint2> sStack[kTraceStackShared * kExtendBlock];
    Stack st;
    st.sm = &sStack[threadIdx.x];
    uint32_t nI = 0, nL = 0;
    WarpPool pool{0, 0, 0};
    uint32_t i = 0;
    Trav T;
    const uint32_t root = trav_root(s);
    __shared__ uint32_t sPend[ANY ? 1 : SB_DEFER_CAP * kExtendBlock];  // deferred leaf tests (closest hit)
    uint32_t* pend = &sPend[ANY ? 0 : threadIdx.x];
    uint32_t np = 0;
    bool have = false;
    while (true) {
        const uint32_t got = pool_take(pool, head, n, chunk, !have);
        if (!have && got != SB_INVALID) {
            i = got;
            const float4 o = __ldg(&rays[2 * (size_t)i]), d = __ldg(&rays[2 * (size_t)i + 1]);
            trav_init_root(T, xyz(o), o.w, xyz(d), ANY, root);
            np = 0;
            have = true;
        }
        if (!__any_sync(0xffffffffu, have)) break;
        if constexpr (!ANY) closest_defer_leaves<COUNT, kExtendBlock>(s, T, have, pend, np, nL);
        if (!have) continue;
        bool done;
        if constexpr (ANY) {
            done = T.cur == SB_INVALID || any_step<COUNT, true>(s, T, st, nI, nL);
        } else {
            bool fin = false;
            if (T.cur != SB_INVALID && np <= SB_DEFER_CAP - 4) {
                fin = closest_defer_node<COUNT, kExtendBlock>(s, T, st, pend, np, nI, nL);
                if (fin) np = 0;
            }
            if (!fin && T.cur == SB_INVALID) closest_pop(T, st);
            done = fin || (T.cur == SB_INVALID && np == 0);
        }
        if (!done) continue;
        HitRec h = T.hit;
        if (REFINE && T.found) {
            const float4 o = __ldg(&rays[2 * (size_t)i]), d = __ldg(&rays[2 * (size_t)i + 1]);
            refine_hit(s, xyz(o), xyz(d), h.instId, h.primId, h.t, h.u, h.v);
        }
        if (!T.found) {
            h.instId = SB_INVALID;
            h.primId = SB_INVALID;
            if (!ANY) {
                h.t = 1e9f;
                h.u = 0.0f;
                h.v = 0.0f;
            }
        }
        uint32_t* out = reinterpret_cast<uint32_t*>(&hits[i]);
        out[0] = __float_as_uint(h.u);
        out[1] = __float_as_uint(h.v);
        out[2] = __float_as_uint(h.t);
        out[3] = h.instId;
        out[4] = h.primId;
        have = false;
    }
    if (COUNT) {
        atomicAdd(&counters[0], (unsigned long long)nI);
        atomicAdd(&counters[1], (unsigned long long)nL);
    }
}

}  // namespace

// ---------------------------------------------------------------------------
// Pass object.
struct StrelkaPathTracer {
    StrelkaPathTracerConfig cfg{};
    int device = 0;
    int numSMs = 148;
    // scene cache
    uint64_t sceneVersion = ~0ull;
    const void* keyNodes = nullptr;
    const void* keyVb = nullptr;
    const void* keyIb = nullptr;
    const void* keyInst = nullptr;
    uint32_t keyNumNodes = 0;
    void* tablesMem = nullptr;  // derived scene tables (internal.h SceneTables)
    size_t tablesCap = 0;       // nodes they were sized for
    SceneTables tables;
    float* srgbLut = nullptr;
    uint32_t* status = nullptr;
    // wavefront
    Wave wave{};
    WaveBuf main;  // the frame's paths
    // environment descriptor copy
    StrelkaEnvMap env{};
    // profiling
    struct Rec { int kc; cudaEvent_t a, b; uint32_t kernels; };
    std::vector<Rec> recs;
    std::vector<cudaEvent_t> eventPool;
    size_t eventsUsed = 0;
    int nrcPathGrid = 0;
    int extendGridCoherent = 0;
    int extendGrid = 0, shadowGrid = 0, tailGrid = 0, traceGrid = 0, traceGridAny = 0, shadeGrid = 0, shadeGridNrc = 0, smallGrid = 0;
    unsigned long long* visitCounters = nullptr;  // 6 entries (STRELKA_PT_COUNT)
    // radiance cache
    StrelkaNrc* nrc = nullptr;
    StrelkaNrcRenderConfig nrcCfg{};
    StrelkaNrcRecord* nrcTrain = nullptr;
    size_t nrcTrainCap = 0;
    StrelkaNrcRecord* nrcQueries = nullptr;
    size_t nrcQueryCap = 0;
    uint32_t* nrcCounts = nullptr;  // [0] queries, [1 + b] training records of batch b
    uint32_t nrcCountCap = 0;       // training batches the counters hold
    cudaStream_t side = nullptr;    // training runs here, beside the frame
    cudaEvent_t forkEvent = nullptr, joinEvent = nullptr;
    uint32_t* traceHead = nullptr;    // work-queue head of the ray-query kernel
    cudaStream_t aux = nullptr;       // shadow(k) beside extend(k+1)
    cudaEvent_t shadeDone = nullptr, shadowDone = nullptr;
    uint32_t* sortHist = nullptr;     // shade-queue sort histogram (cleared by each scan)
    uint32_t* sortOffsets = nullptr;
};

namespace {

void free_wave(WaveBuf& b)
{
    for (void* p : b.allocs) cudaFree(p);
    b.allocs.clear();
    b.w = Wave{};
    b.sorted = nullptr;
    b.keys = nullptr;
    b.cap = 0;
}

template <typename T>
int walloc(WaveBuf& b, T** p, size_t n)
{
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(wavefront state)");
    b.allocs.push_back(q);
    *p = static_cast<T*>(q);
    return STRELKA_OK;
}

int ensure_wave(WaveBuf& b, size_t cap)
{
    if (b.cap >= cap) return STRELKA_OK;
    free_wave(b);
    Wave& w = b.w;
    int rc;
    if ((rc = walloc(b, &w.ray_o, cap)) || (rc = walloc(b, &w.ray_d, cap)) || (rc = walloc(b, &w.thr, cap)) ||
        (rc = walloc(b, &w.col, cap)) || (rc = walloc(b, &w.rng, cap)) || (rc = walloc(b, &w.hit, cap)) ||
        (rc = walloc(b, &w.hitRef, cap)) || (rc = walloc(b, &w.queue[0], cap)) || (rc = walloc(b, &w.queue[1], cap)) ||
        (rc = walloc(b, &w.sh_o, cap)) || (rc = walloc(b, &w.sh_d, cap)) || (rc = walloc(b, &w.sh_cd, cap)) ||
        (rc = walloc(b, &w.sh_cg, cap)) || (rc = walloc(b, &w.counters, kWaveCounters)) ||
        (rc = walloc(b, &b.sorted, cap)) || (rc = walloc(b, &b.keys, cap))) {
        free_wave(b);
        return rc;
    }
    b.cap = cap;
    return STRELKA_OK;
}

cudaEvent_t next_event(StrelkaPathTracer* pt)
{
    if (pt->eventsUsed == pt->eventPool.size()) {
        cudaEvent_t e;
        if (cudaEventCreate(&e) != cudaSuccess) return nullptr;
        pt->eventPool.push_back(e);
    }
    return pt->eventPool[pt->eventsUsed++];
}

// CUDA-event interval around the `kernels` launches of one kernel class.
struct Timer {
    StrelkaPathTracer* pt;
    int kc;
    cudaStream_t st;
    uint32_t kernels;
    cudaEvent_t a = nullptr;
    Timer(StrelkaPathTracer* p, int k, cudaStream_t s, uint32_t nk = 1) : pt(p), kc(k), st(s), kernels(nk)
    {
        if (pt->cfg.flags & STRELKA_PT_PROFILE) {
            a = next_event(pt);
            if (a) cudaEventRecord(a, st);
        }
    }
    ~Timer()
    {
        if (a) {
            cudaEvent_t b = next_event(pt);
            if (b) {
                cudaEventRecord(b, st);
                pt->recs.push_back({kc, a, b, kernels});
            }
        }
    }
};

int check_scene_desc(const PathTracerDesc* d)
{
    if (!d) return fail(STRELKA_ERR_INVALID_ARGUMENT, "desc is NULL");
    if (d->numNodes > (1u << 30)) return fail(STRELKA_ERR_INVALID_ARGUMENT, "numNodes %u exceeds 2^30", d->numNodes);
    if (d->numNodes && (!d->bvhNodes || !d->vb || !d->ib || !d->instanceConst))
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "scene buffers must be non-NULL when numNodes > 0");
    if (reinterpret_cast<uintptr_t>(d->bvhNodes) & 15) return fail(STRELKA_ERR_INVALID_ARGUMENT, "bvhNodes must be 16-byte aligned");
    return STRELKA_OK;
}

// Refreshes the derived leaf-triangle table when the scene changed.
int ensure_scene(StrelkaPathTracer* pt, const BVHNode* nodes, uint32_t numNodes, const Vertex* vb, uint32_t numVertices,
                 const uint32_t* ib, uint32_t numIndices, const InstanceConstants* inst, uint32_t numInstances,
                 uint64_t version, cudaStream_t st)
{
    if (pt->sceneVersion == version && pt->keyNodes == nodes && pt->keyVb == vb && pt->keyIb == ib && pt->keyInst == inst &&
        pt->keyNumNodes == numNodes && pt->tablesMem)
        return STRELKA_OK;
    if (numNodes > pt->tablesCap || !pt->tablesMem) {
        if (pt->tablesMem) cudaFree(pt->tablesMem);
        pt->tablesMem = nullptr;
        const uint32_t cap = std::max<uint32_t>(numNodes, 1);
        SB_CUDA_TRY(cudaMalloc(&pt->tablesMem, scene_tables_bytes(cap)));
        pt->tablesCap = cap;
    }
    pt->tables = scene_tables(pt->tablesMem, numNodes);
    if (numNodes) {
        Timer t(pt, KC_PREP, st, 7);
        int rc = launch_prep_tables(nodes, numNodes, inst, numInstances, ib, numIndices, vb, numVertices, pt->tables,
                                    pt->status, pt->numSMs, st);
        if (rc) return rc;
    }
    pt->sceneVersion = version;
    pt->keyNodes = nodes;
    pt->keyVb = vb;
    pt->keyIb = ib;
    pt->keyInst = inst;
    pt->keyNumNodes = numNodes;
    return STRELKA_OK;
}

DevScene make_scene(StrelkaPathTracer* pt, const PathTracerDesc* d)
{
    return scene_from_desc(d, pt->tables, pt->srgbLut, pt->status);
}

int occupancy_grid(const void* fn, int block, int numSMs)
{
    int perSM = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fn, block, 0) != cudaSuccess || perSM < 1) perSM = 1;
    return perSM * numSMs;
}

}  // namespace

namespace sb {

void srgb_lut_host(float* lut)
{
    for (int i = 0; i < 256; ++i) {
        float x = (float)i / 255.0f;
        lut[i] = x <= 0.04045f ? x / 12.92f : powf((x + 0.055f) / 1.055f, 2.4f);
    }
}

int validate_scene_desc(const PathTracerDesc* d) { return check_scene_desc(d); }

static size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
static size_t scan_bytes(uint32_t n)
{
    size_t bytes = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, bytes, (const uint32_t*)nullptr, (uint32_t*)nullptr, (int)std::max<uint32_t>(n, 1));
    return bytes;
}

size_t scene_tables_bytes(uint32_t numNodes)
{
    const size_t n = std::max<uint32_t>(numNodes, 1);
    const size_t wideCap = n / 2 + 1, recCap = n / 2 + 1;
    return align256(recCap * 3 * sizeof(float4)) + align256(recCap * 6 * sizeof(float4)) +
           align256(wideCap * 8 * sizeof(float4)) + 5 * align256(n * 4) + 256 + align256(scan_bytes(numNodes));
}

SceneTables scene_tables(void* base, uint32_t numNodes)
{
    const size_t n = std::max<uint32_t>(numNodes, 1);
    SceneTables t;
    t.wideCap = (uint32_t)(n / 2 + 1);
    t.recCap = (uint32_t)(n / 2 + 1);  // a binary tree of n nodes has (n + 1) / 2 leaves
    char* p = static_cast<char*>(base);
    t.rec = reinterpret_cast<float4*>(p);
    p += align256((size_t)t.recCap * 3 * sizeof(float4));
    t.shade = reinterpret_cast<float4*>(p);
    p += align256((size_t)t.recCap * 6 * sizeof(float4));
    t.leafOf = reinterpret_cast<uint32_t*>(p);
    p += align256(n * 4);
    t.wide = reinterpret_cast<float4*>(p);
    p += align256((size_t)t.wideCap * 8 * sizeof(float4));
    t.parent = reinterpret_cast<uint32_t*>(p);
    p += align256(n * 4);
    t.flag = reinterpret_cast<uint32_t*>(p);
    p += align256(n * 4);
    t.map = reinterpret_cast<uint32_t*>(p);
    p += align256(n * 4);
    t.extra = reinterpret_cast<uint32_t*>(p);
    p += align256(n * 4);
    t.deep = reinterpret_cast<uint32_t*>(p);
    p += 256;
    t.scan = p;
    t.scanBytes = scan_bytes(numNodes);
    return t;
}

int launch_prep_tables(const BVHNode* nodes, uint32_t numNodes, const InstanceConstants* inst, uint32_t numInstances,
                       const uint32_t* ib, uint32_t numIndices, const Vertex* vb, uint32_t numVertices,
                       const SceneTables& t, uint32_t* status, int numSMs, cudaStream_t st)
{
    if (!numNodes) return STRELKA_OK;
    const float4* nd = reinterpret_cast<const float4*>(nodes);
    const int grid = std::min<int>((numNodes + 255) / 256, numSMs * 16);
    size_t bytes = t.scanBytes;
    // compact leaf indices: an exclusive scan of the leaf flags (held in
    // `parent` until its own use below)
    k_leaf_flag<<<grid, 256, 0, st>>>(nd, numNodes, t.parent);
    SB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(t.scan, bytes, t.parent, t.leafOf, (int)numNodes, st));
    k_prep_rec<<<grid, 256, 0, st>>>(nd, numNodes, inst, numInstances, ib, numIndices, vb, numVertices, t.leafOf,
                                     t.recCap, t.rec, status);
    k_prep_shade<<<grid, 256, 0, st>>>(nd, numNodes, inst, numInstances, ib, numIndices, vb, numVertices, t.leafOf,
                                       t.recCap, t.shade);
    SB_CUDA_TRY(cudaMemsetAsync(t.parent, 0xFF, (size_t)numNodes * 4, st));
    k_wide_parent<<<grid, 256, 0, st>>>(nd, numNodes, t.parent);
    SB_CUDA_TRY(cudaMemsetAsync(t.deep, 0, sizeof(uint32_t), st));
    k_wide_flag<<<grid, 256, 0, st>>>(nd, numNodes, t.parent, t.flag, t.deep, status);
    {
        // deep trees only (the kernels return at once unless *deep): ancestors
        // ping-pong between parent and map (map is free until the scan),
        // parities between extra and flag
        int rounds = 1;
        while (rounds < 32 && (1ull << (rounds - 1)) < (uint64_t)numNodes) ++rounds;
        k_wide_jump_init<<<grid, 256, 0, st>>>(numNodes, t.parent, t.extra, t.deep);
        uint32_t *ancIn = t.parent, *ancOut = t.map, *parIn = t.extra, *parOut = t.flag;
        for (int r = 0; r < rounds; ++r) {
            k_wide_jump<<<grid, 256, 0, st>>>(numNodes, ancIn, parIn, ancOut, parOut, t.deep);
            std::swap(ancIn, ancOut);
            std::swap(parIn, parOut);
        }
        k_wide_jump_finish<<<grid, 256, 0, st>>>(nd, numNodes, ancIn, parIn, t.flag, t.deep, status);
    }
    bytes = t.scanBytes;
    SB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(t.scan, bytes, t.flag, t.map, (int)numNodes, st));
    k_wide_build<<<grid, 256, 0, st>>>(nd, numNodes, t.flag, t.map, t.leafOf, t.recCap, t.wide, t.wideCap, status);
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}

DevScene scene_from_desc(const PathTracerDesc* d, const SceneTables& t, const float* srgbLut, uint32_t* status)
{
    DevScene s{};
    s.nodes = reinterpret_cast<const float4*>(d->bvhNodes);
    s.tris = nullptr;
    s.rec = t.rec;
    s.shadeRec = t.shade;
    s.leafOf = t.leafOf;
    s.numRec = t.recCap;
    s.wide = t.wide;
    s.numWide = t.wideCap;
    s.numNodes = d->numNodes;
    s.numVertices = d->numVertices;
    s.vb = d->vb;
    s.ib = d->ib;
    s.numIndices = d->numIndices;
    s.numInstances = d->numInstances;
    s.inst = d->instanceConst;
    s.lights = d->lights;
    s.lightCapacity = d->lights ? d->lightCapacity : 0;
    s.numMaterials = d->mdl_mdlMaterial ? d->numMaterials : 0;
    s.argBlock = d->mdl_argument_block;
    s.argBlockBytes = d->mdl_argument_block ? d->argBlockBytes : 0;
    s.roData = d->mdl_ro_data_segment;
    s.roDataBytes = d->mdl_ro_data_segment ? d->roDataBytes : 0;
    s.materials = d->mdl_mdlMaterial;
    s.resInfos = d->mdl_resource_infos;
    s.numResInfos = d->mdl_resource_infos ? d->numResourceInfos : 0;
    s.numTextures = d->matTextures ? d->numTextures : 0;
    s.textures = d->matTextures;
    s.srgbLut = srgbLut;
    s.hasEnv = d->envMap != nullptr;
    if (d->envMap) s.env = *d->envMap;
    s.status = status;
    return s;
}

}  // namespace sb

extern "C" int strelka_pathtracer_create(const StrelkaPathTracerConfig* config, StrelkaPathTracer** out)
{
    if (!out) return fail(STRELKA_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(STRELKA_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    auto* pt = new StrelkaPathTracer();
    if (config) pt->cfg = *config;
    if (pt->cfg.mode > STRELKA_MODE_MEGAKERNEL) {
        delete pt;
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "unknown mode %u", config->mode);
    }
    if ((pt->cfg.flags & STRELKA_PT_NO_SHADE_SORT) && (pt->cfg.flags & STRELKA_PT_FORCE_SHADE_SORT)) {
        delete pt;
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "STRELKA_PT_NO_SHADE_SORT and STRELKA_PT_FORCE_SHADE_SORT both set");
    }
    if (pt->cfg.queueChunk && (pt->cfg.queueChunk > 4096 || (pt->cfg.queueChunk & 31))) {
        delete pt;
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "queueChunk must be 0 or a multiple of 32 up to 4096");
    }
    if ((pt->cfg.flags & STRELKA_PT_LARGE_SCENE_KERNELS) && (pt->cfg.flags & STRELKA_PT_SMALL_SCENE_KERNELS)) {
        delete pt;
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "STRELKA_PT_LARGE_SCENE_KERNELS and STRELKA_PT_SMALL_SCENE_KERNELS together");
    }
    pt->device = dev;
    cudaDeviceGetAttribute(&pt->numSMs, cudaDevAttrMultiProcessorCount, dev);
    float lut[256];
    srgb_lut_host(lut);
    if (cudaMalloc(&pt->srgbLut, sizeof(lut)) != cudaSuccess || cudaMalloc(&pt->status, sizeof(uint32_t)) != cudaSuccess) {
        strelka_pathtracer_destroy(pt);
        return fail(STRELKA_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
    }
    cudaMemcpy(pt->srgbLut, lut, sizeof(lut), cudaMemcpyHostToDevice);
    cudaMemset(pt->status, 0, sizeof(uint32_t));
    if (cudaMalloc(&pt->visitCounters, 8 * sizeof(unsigned long long)) != cudaSuccess) {
        strelka_pathtracer_destroy(pt);
        return fail(STRELKA_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
    }
    cudaMemset(pt->visitCounters, 0, 8 * sizeof(unsigned long long));
    if (cudaMalloc(&pt->traceHead, sizeof(uint32_t)) != cudaSuccess) {
        strelka_pathtracer_destroy(pt);
        return fail(STRELKA_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
    }
    pt->extendGrid = occupancy_grid((const void*)k_extend<false, true>, kExtendBlock, pt->numSMs);
    pt->extendGridCoherent = occupancy_grid((const void*)k_extend<false, false>, kExtendBlock, pt->numSMs);
    pt->shadowGrid = occupancy_grid((const void*)k_shadow<false, true>, kExtendBlock, pt->numSMs);
    pt->tailGrid = occupancy_grid((const void*)k_tail, kExtendBlock, pt->numSMs);
    pt->nrcPathGrid = occupancy_grid((const void*)k_nrc_train_paths, kNrcPathBlock, pt->numSMs);
    pt->traceGrid = occupancy_grid((const void*)k_trace<false, false, false>, kExtendBlock, pt->numSMs);
    pt->traceGridAny = occupancy_grid((const void*)k_trace<true, false, false>, kExtendBlock, pt->numSMs);
    pt->shadeGrid = occupancy_grid((const void*)k_shade<false>, kShadeBlock, pt->numSMs);
    pt->shadeGridNrc = occupancy_grid((const void*)k_shade<true>, kShadeBlock, pt->numSMs);
    pt->smallGrid = pt->numSMs * 8;
    *out = pt;
    return STRELKA_OK;
}

extern "C" int strelka_pathtracer_destroy(StrelkaPathTracer* pt)
{
    if (!pt) return STRELKA_OK;
    free_wave(pt->main);
    if (pt->tablesMem) cudaFree(pt->tablesMem);
    if (pt->srgbLut) cudaFree(pt->srgbLut);
    if (pt->status) cudaFree(pt->status);
    if (pt->visitCounters) cudaFree(pt->visitCounters);
    if (pt->nrcTrain) cudaFree(pt->nrcTrain);
    if (pt->nrcQueries) cudaFree(pt->nrcQueries);
    if (pt->nrcCounts) cudaFree(pt->nrcCounts);
    if (pt->traceHead) cudaFree(pt->traceHead);
    if (pt->sortHist) cudaFree(pt->sortHist);
    if (pt->sortOffsets) cudaFree(pt->sortOffsets);
    if (pt->shadeDone) cudaEventDestroy(pt->shadeDone);
    if (pt->shadowDone) cudaEventDestroy(pt->shadowDone);
    if (pt->aux) cudaStreamDestroy(pt->aux);
    if (pt->forkEvent) cudaEventDestroy(pt->forkEvent);
    if (pt->joinEvent) cudaEventDestroy(pt->joinEvent);
    if (pt->side) cudaStreamDestroy(pt->side);
    for (cudaEvent_t e : pt->eventPool) cudaEventDestroy(e);
    delete pt;
    return STRELKA_OK;
}

// Radiance-cache training: `batches` batches of trainPaths training paths,
// traced in one launch, then per batch trainSteps gradient + Adam steps on
// its vertices (batch sizes read on the device).
// The wavefront passes' traversal variants.  Shared-memory stacks and
// deferred leaf tests pay on trees far beyond L1 (10M triangles: +4%); on
// small trees the shared memory they take from L1 costs more than they save
// (the 10k-triangle Cornell box: -9%); the measured crossover lies between
// 1.3M and 5M nodes.  Camera rays (bounce 0) are coherent: their lanes test
// the same leaves together, so their leaf tests are never deferred.
static bool large_scene(const StrelkaPathTracer* pt, const DevScene& s)
{
    if (pt->cfg.flags & STRELKA_PT_LARGE_SCENE_KERNELS) return true;
    if (pt->cfg.flags & STRELKA_PT_SMALL_SCENE_KERNELS) return false;
    return s.numNodes >= STRELKA_LARGE_SCENE_NODES;
}
static bool extend_defer(const StrelkaPathTracer* pt, const DevScene& s, int depth)
{
    return depth >= 1 && large_scene(pt, s);
}

static int nrc_train_frame(StrelkaPathTracer* pt, const DevScene& s, const PathTracerParam& ubo, uint32_t batches,
                           cudaStream_t st)
{
    const uint32_t nTrain = pt->nrcCfg.trainPaths;
    if (nTrain == 0 || batches == 0) return STRELKA_OK;
    if ((uint64_t)nTrain * batches > (1ull << 26))
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "trainPaths x batches exceeds 2^26");
    // counters: [0] queries, [1 + b] records of batch b, [1 + batches] the
    // training kernel's work head
    if (batches + 2 > pt->nrcCountCap) {
        if (pt->nrcCounts) cudaFree(pt->nrcCounts);
        pt->nrcCounts = nullptr;
        pt->nrcCountCap = 0;
        SB_CUDA_TRY(cudaMalloc(&pt->nrcCounts, (size_t)(batches + 2) * sizeof(uint32_t)));
        pt->nrcCountCap = batches + 2;
    }
    const size_t capPerBatch =
        (size_t)nTrain * std::min<uint32_t>(std::max<uint32_t>(ubo.maxDepth, 1u), (uint32_t)kNrcMaxVerts);
    if (capPerBatch * batches > pt->nrcTrainCap) {
        if (pt->nrcTrain) cudaFree(pt->nrcTrain);
        pt->nrcTrain = nullptr;
        pt->nrcTrainCap = 0;
        SB_CUDA_TRY(cudaMalloc(&pt->nrcTrain, capPerBatch * batches * sizeof(StrelkaNrcRecord)));
        pt->nrcTrainCap = capPerBatch * batches;
    }
    {
        Timer t(pt, KC_NRC_PATHS, st);
        SB_CUDA_TRY(cudaMemsetAsync(pt->nrcCounts + 1, 0, (batches + 1) * sizeof(uint32_t), st));
        const uint32_t n = nTrain * batches;
        const int grid = std::min<int>((int)((n + kNrcPathBlock - 1) / kNrcPathBlock), pt->nrcPathGrid);
        k_nrc_train_paths<<<grid, kNrcPathBlock, 0, st>>>(s, ubo, nTrain, batches, pt->nrcCfg.diffuseRoughness,
                                                          pt->nrcTrain, pt->nrcCounts + 1, (uint32_t)capPerBatch,
                                                          pt->nrcCounts + 1 + batches);
        SB_CUDA_TRY(cudaGetLastError());
    }
    Timer t(pt, KC_NRC_TRAIN, st);
    for (uint32_t b = 0; b < batches; ++b) {
        const StrelkaNrcRecord* recs = pt->nrcTrain + (size_t)b * capPerBatch;
        const uint32_t* cnt = pt->nrcCounts + 1 + b;
        for (uint32_t k = 0; k < std::max<uint32_t>(pt->nrcCfg.trainSteps, 1u); ++k) {
            int rc = nrc_gradients_device(pt->nrc, recs, cnt, (uint32_t)capPerBatch, st);
            if (rc) return rc;
            rc = nrc_adam_device_count(pt->nrc, 1.0f, cnt, st);
            if (rc) return rc;
        }
    }
    return STRELKA_OK;
}

extern "C" int strelka_pathtracer_execute(StrelkaPathTracer* pt, const PathTracerDesc* desc, uint32_t w, uint32_t h,
                                          uint64_t frameIndex, void* stream)
{
    (void)frameIndex;
    if (!pt) return fail(STRELKA_ERR_INVALID_ARGUMENT, "path tracer is NULL");
    int rc = check_scene_desc(desc);
    if (rc) return rc;
    const PathTracerParam& ubo = desc->constants;
    if (ubo.dimension[0] <= 0 || ubo.dimension[1] <= 0 || ubo.spp <= 0)
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "dimension and spp must be positive");
    const uint64_t total = (uint64_t)ubo.dimension[0] * (uint64_t)ubo.dimension[1] * (uint64_t)ubo.spp;
    if (total > 0xFFFFFFFFull) return fail(STRELKA_ERR_INVALID_ARGUMENT, "W*H*spp exceeds 2^32");
    if ((uint64_t)w * (h ? h : 1) != total)
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "w*h (%u*%u) must equal W*H*spp (%llu)", w, h, (unsigned long long)total);
    if (!desc->sampleBuffer) return fail(STRELKA_ERR_INVALID_ARGUMENT, "sampleBuffer is NULL");
    if (desc->envMap) {
        const StrelkaEnvMap* e = desc->envMap;
        if (!e->rgba32f || !e->marginal_cdf || !e->conditional_cdf || e->width == 0 || e->height == 0)
            return fail(STRELKA_ERR_INVALID_ARGUMENT, "incomplete environment map");
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    rc = ensure_scene(pt, desc->bvhNodes, desc->numNodes, desc->vb, desc->numVertices, desc->ib, desc->numIndices,
                      desc->instanceConst, desc->numInstances, desc->sceneVersion, st);
    if (rc) return rc;
    DevScene s = make_scene(pt, desc);

    const bool useNrc = pt->nrc && pt->nrcCfg.enable;
    if (useNrc && pt->cfg.mode == STRELKA_MODE_MEGAKERNEL)
        return fail(STRELKA_ERR_UNSUPPORTED, "the radiance cache runs with the wavefront mode");
    if (pt->cfg.mode == STRELKA_MODE_MEGAKERNEL) {
        Timer t(pt, KC_MEGAKERNEL, st);
        const uint64_t blocks = (total + kExtendBlock - 1) / kExtendBlock;
        k_megakernel<<<(unsigned)blocks, kExtendBlock, 0, st>>>(s, ubo, desc->sampleBuffer, 0, total);
        SB_CUDA_TRY(cudaGetLastError());
        return STRELKA_OK;
    }

    // wavefront
    // default: the whole frame in flight (160 bytes of state per path; a
    // 1080p x 16 spp frame is 33.2M paths, 5.3 GB)
    size_t chunk = pt->cfg.chunkPaths ? pt->cfg.chunkPaths : (size_t)1 << 25;
    chunk = std::min<size_t>(chunk, total);
    rc = ensure_wave(pt->main, chunk);
    if (rc) return rc;
    const int maxDepth = (int)ubo.maxDepth;
    const uint32_t qchunk = pt->cfg.queueChunk ? pt->cfg.queueChunk : kDefaultQueueChunk;
    // shadow(k) beside extend(k+1) on the auxiliary stream, unless the
    // caller asked for the serial order
    const bool overlap = SB_OVERLAP_SHADOW && !(pt->cfg.flags & STRELKA_PT_SERIAL_SHADOW);
    if (overlap && !pt->aux) {
        SB_CUDA_TRY(cudaStreamCreateWithFlags(&pt->aux, cudaStreamNonBlocking));
        SB_CUDA_TRY(cudaEventCreateWithFlags(&pt->shadeDone, cudaEventDisableTiming));
        SB_CUDA_TRY(cudaEventCreateWithFlags(&pt->shadowDone, cudaEventDisableTiming));
    }
    // shade-queue sort by material: one key per material + miss + light/invalid.
    // Not with the radiance cache: its paths end at the first diffuse-ish
    // vertex, so the queues of bounces >= 1 are short and sorting them costs
    // more than it saves (time to the plain relMSE 0.411 -> 0.407 x plain).
    // Not on small chunks either, where its three short launches per bounce
    // are mostly latency (Cornell 512^2 x 1 spp: 332 -> 349 Mpaths/s without;
    // the 1080p x 16 spp frame gains 0.4% with it).
    uint32_t sortKeys = 0;
    const bool sortBySize = chunk >= STRELKA_SHADE_SORT_MIN_PATHS || (pt->cfg.flags & STRELKA_PT_FORCE_SHADE_SORT);
    if (!(pt->cfg.flags & STRELKA_PT_NO_SHADE_SORT) && sortBySize && !useNrc && s.numMaterials + 2 <= kMaxSortKeys) {
        sortKeys = s.numMaterials + 2;
        if (!pt->sortHist) {
            SB_CUDA_TRY(cudaMalloc(&pt->sortHist, kMaxSortKeys * sizeof(uint32_t)));
            SB_CUDA_TRY(cudaMalloc(&pt->sortOffsets, kMaxSortKeys * sizeof(uint32_t)));
            SB_CUDA_TRY(cudaMemsetAsync(pt->sortHist, 0, kMaxSortKeys * sizeof(uint32_t), st));
        }
    }
    NrcWave nw{};
    if (useNrc) {
        if (chunk > pt->nrcQueryCap) {
            if (pt->nrcQueries) cudaFree(pt->nrcQueries);
            pt->nrcQueries = nullptr;
            SB_CUDA_TRY(cudaMalloc(&pt->nrcQueries, chunk * sizeof(StrelkaNrcRecord)));
            pt->nrcQueryCap = chunk;
        }
        if (!pt->nrcCounts) {
            SB_CUDA_TRY(cudaMalloc(&pt->nrcCounts, 2 * sizeof(uint32_t)));
            pt->nrcCountCap = 2;
        }
        if (!pt->side) {
            SB_CUDA_TRY(cudaStreamCreateWithFlags(&pt->side, cudaStreamNonBlocking));
            SB_CUDA_TRY(cudaEventCreateWithFlags(&pt->forkEvent, cudaEventDisableTiming));
            SB_CUDA_TRY(cudaEventCreateWithFlags(&pt->joinEvent, cudaEventDisableTiming));
        }
        // this frame's training runs on the side stream while the frame's
        // paths are traced; the frame waits for it before the cache inference
        SB_CUDA_TRY(cudaEventRecord(pt->forkEvent, st));
        SB_CUDA_TRY(cudaStreamWaitEvent(pt->side, pt->forkEvent, 0));
        rc = nrc_train_frame(pt, s, ubo, 1, pt->side);
        if (rc) return rc;
        SB_CUDA_TRY(cudaEventRecord(pt->joinEvent, pt->side));
        nw.queries = pt->nrcQueries;
        nw.count = pt->nrcCounts;
        nw.capacity = (uint32_t)chunk;
        nw.enabled = 1;
        nw.diffuseRoughness = pt->nrcCfg.diffuseRoughness;
    }
    for (uint64_t first = 0; first < total; first += chunk) {
        const uint32_t n = (uint32_t)std::min<uint64_t>(chunk, total - first);
        if (useNrc) SB_CUDA_TRY(cudaMemsetAsync(pt->nrcCounts, 0, sizeof(uint32_t), st));
        {
            Timer t(pt, KC_GENERATE, st);
            int grid = std::min<int>((n + kSmallBlock - 1) / kSmallBlock, pt->smallGrid);
            k_generate<<<grid, kSmallBlock, 0, st>>>(ubo, pt->main.w, first, n);
        }
        bool pendingShadow = false;
        // bounces from tailDepth on run in one k_tail launch (not with the cache)
        const int tailDepth = useNrc ? maxDepth : std::min<int>(maxDepth, (int)std::min<uint32_t>(pt->cfg.tailDepth ? pt->cfg.tailDepth : kDefaultTailDepth, 0x7FFFFFFFu));
        for (int depth = 0; depth < tailDepth; ++depth) {
            const int qin = depth & 1;
            const int gridE = std::min<int>((n + kExtendBlock - 1) / kExtendBlock, pt->extendGrid);
            const int gridW = std::min<int>((n + kExtendBlock - 1) / kExtendBlock, pt->shadowGrid);
            const int gridS =
                std::min<int>((n + kShadeBlock - 1) / kShadeBlock, useNrc ? pt->shadeGridNrc : pt->shadeGrid);
            const bool count = (pt->cfg.flags & STRELKA_PT_COUNT) != 0;
            {
                Timer t(pt, KC_EXTEND, st);
                if (extend_defer(pt, s, depth)) {
                    if (count) k_extend<true, true><<<gridE, kExtendBlock, 0, st>>>(s, pt->main.w, qin, qchunk, pt->visitCounters);
                    else k_extend<false, true><<<gridE, kExtendBlock, 0, st>>>(s, pt->main.w, qin, qchunk, nullptr);
                } else {
                    const int gridC = std::min<int>((n + kExtendBlock - 1) / kExtendBlock, pt->extendGridCoherent);
                    if (count) k_extend<true, false><<<gridC, kExtendBlock, 0, st>>>(s, pt->main.w, qin, qchunk, pt->visitCounters);
                    else k_extend<false, false><<<gridC, kExtendBlock, 0, st>>>(s, pt->main.w, qin, qchunk, nullptr);
                }
            }
            const uint32_t* order = nullptr;
            if (sortKeys && depth >= SB_SORT_FROM_DEPTH) {
                Timer t(pt, KC_SORT, st, 3);
                const int gridK = std::min<int>((n + kSmallBlock - 1) / kSmallBlock, pt->numSMs * 4);
                k_sort_count<<<gridK, kSmallBlock, 0, st>>>(s, pt->main.w, qin, sortKeys, pt->sortHist, pt->main.keys);
                k_sort_scan<<<1, 1024, 0, st>>>(pt->sortHist, sortKeys, pt->sortOffsets);
                const int gridT = std::min<int>((n + kSortTile - 1) / kSortTile, pt->numSMs * 4);
                k_sort_scatter<<<gridT, kSmallBlock, 0, st>>>(pt->main.w, qin, sortKeys, pt->main.keys, pt->sortOffsets,
                                                             pt->main.sorted);
                order = pt->main.sorted;
            }
            if (pendingShadow) SB_CUDA_TRY(cudaStreamWaitEvent(st, pt->shadowDone, 0));
            {
                Timer t(pt, KC_SHADE, st);
                if (useNrc)
                    k_shade<true><<<gridS, kShadeBlock, 0, st>>>(s, ubo, pt->main.w, qin, order, qchunk, nw);
                else
                    k_shade<false><<<gridS, kShadeBlock, 0, st>>>(s, ubo, pt->main.w, qin, order, qchunk, nw);
            }
            // shadow(k) runs on the auxiliary stream beside extend(k+1): both
            // read only shade(k)'s outputs; shade(k+1) waits for both
            cudaStream_t sst = st;
            if (overlap) {
                SB_CUDA_TRY(cudaEventRecord(pt->shadeDone, st));
                SB_CUDA_TRY(cudaStreamWaitEvent(pt->aux, pt->shadeDone, 0));
                sst = pt->aux;
            }
            {
                Timer t(pt, KC_SHADOW, sst);
                if (large_scene(pt, s)) {
                    if (count) k_shadow<true, true><<<gridW, kExtendBlock, 0, sst>>>(s, pt->main.w, qin, qchunk, pt->visitCounters);
                    else k_shadow<false, true><<<gridW, kExtendBlock, 0, sst>>>(s, pt->main.w, qin, qchunk, nullptr);
                } else {
                    if (count) k_shadow<true, false><<<gridW, kExtendBlock, 0, sst>>>(s, pt->main.w, qin, qchunk, pt->visitCounters);
                    else k_shadow<false, false><<<gridW, kExtendBlock, 0, sst>>>(s, pt->main.w, qin, qchunk, nullptr);
                }
            }
            if (overlap) {
                SB_CUDA_TRY(cudaEventRecord(pt->shadowDone, pt->aux));
                pendingShadow = true;
            }
        }
        if (pendingShadow) SB_CUDA_TRY(cudaStreamWaitEvent(st, pt->shadowDone, 0));
        if (tailDepth < maxDepth) {
            Timer t(pt, KC_TAIL, st);
            const int gridE = std::min<int>((n + kExtendBlock - 1) / kExtendBlock, pt->tailGrid);
            k_tail<<<gridE, kExtendBlock, 0, st>>>(s, ubo, pt->main.w, tailDepth & 1, qchunk);
        }
        if (useNrc) {
            if (first == 0) SB_CUDA_TRY(cudaStreamWaitEvent(st, pt->joinEvent, 0));
            Timer t(pt, KC_NRC_INFER, st);
            rc = nrc_infer_device(pt->nrc, pt->nrcQueries, pt->nrcCounts, n, nullptr, pt->main.w.col, pt->status, st);
            if (rc) return rc;
        }
        {
            Timer t(pt, KC_FINALIZE, st);
            int grid = std::min<int>((n + kSmallBlock - 1) / kSmallBlock, pt->smallGrid);
            k_finalize<<<grid, kSmallBlock, 0, st>>>(pt->main.w, desc->sampleBuffer, first, n);
        }
        SB_CUDA_TRY(cudaGetLastError());
    }
    return STRELKA_OK;
}

extern "C" int strelka_pathtracer_train_nrc(StrelkaPathTracer* pt, const PathTracerDesc* desc, uint64_t frameIndex,
                                            uint32_t batches, void* stream)
{
    (void)frameIndex;
    if (!pt) return fail(STRELKA_ERR_INVALID_ARGUMENT, "path tracer is NULL");
    if (!pt->nrc || !pt->nrcCfg.enable) return fail(STRELKA_ERR_INVALID_ARGUMENT, "no radiance cache attached");
    int rc = check_scene_desc(desc);
    if (rc) return rc;
    const PathTracerParam& ubo = desc->constants;
    if (ubo.dimension[0] <= 0 || ubo.dimension[1] <= 0 || ubo.spp <= 0)
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "dimension and spp must be positive");
    if (desc->envMap) {
        const StrelkaEnvMap* e = desc->envMap;
        if (!e->rgba32f || !e->marginal_cdf || !e->conditional_cdf || e->width == 0 || e->height == 0)
            return fail(STRELKA_ERR_INVALID_ARGUMENT, "incomplete environment map");
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    rc = ensure_scene(pt, desc->bvhNodes, desc->numNodes, desc->vb, desc->numVertices, desc->ib, desc->numIndices,
                      desc->instanceConst, desc->numInstances, desc->sceneVersion, st);
    if (rc) return rc;
    DevScene s = make_scene(pt, desc);
    return nrc_train_frame(pt, s, ubo, batches, st);
}

extern "C" int strelka_pathtracer_set_nrc(StrelkaPathTracer* pt, StrelkaNrc* nrc, const StrelkaNrcRenderConfig* cfg)
{
    if (!pt) return fail(STRELKA_ERR_INVALID_ARGUMENT, "path tracer is NULL");
    pt->nrc = nrc;
    if (cfg) pt->nrcCfg = *cfg;
    else pt->nrcCfg = StrelkaNrcRenderConfig{};
    if (nrc && !cfg) pt->nrcCfg.enable = 0;
    return STRELKA_OK;
}

extern "C" int strelka_pathtracer_get_device_status(StrelkaPathTracer* pt, void* stream, uint32_t* status)
{
    if (!pt || !status) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    SB_CUDA_TRY(cudaStreamSynchronize(st));
    SB_CUDA_TRY(cudaMemcpy(status, pt->status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    SB_CUDA_TRY(cudaMemset(pt->status, 0, sizeof(uint32_t)));
    return STRELKA_OK;
}

extern "C" int strelka_pathtracer_get_kernel_times(StrelkaPathTracer* pt, void* stream, float* ms_out, uint32_t* launches_out,
                                                   uint32_t capacity)
{
    if (!pt) return -STRELKA_ERR_INVALID_ARGUMENT;
    cudaStreamSynchronize(static_cast<cudaStream_t>(stream));
    std::vector<float> ms(KC_COUNT, 0.0f);
    std::vector<uint32_t> cnt(KC_COUNT, 0);
    for (auto& r : pt->recs) {
        float t = 0.0f;
        if (cudaEventElapsedTime(&t, r.a, r.b) == cudaSuccess) {
            ms[r.kc] += t;
            cnt[r.kc] += r.kernels;
        }
    }
    for (uint32_t i = 0; i < capacity && i < (uint32_t)KC_COUNT; ++i) {
        if (ms_out) ms_out[i] = ms[i];
        if (launches_out) launches_out[i] = cnt[i];
    }
    pt->recs.clear();
    pt->eventsUsed = 0;
    return KC_COUNT;
}

extern "C" int strelka_pathtracer_get_counters(StrelkaPathTracer* pt, void* stream, unsigned long long* out,
                                               uint32_t capacity)
{
    if (!pt || (!out && capacity)) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    unsigned long long tmp[6];
    SB_CUDA_TRY(cudaMemcpyAsync(tmp, pt->visitCounters, sizeof(tmp), cudaMemcpyDeviceToHost, st));
    SB_CUDA_TRY(cudaStreamSynchronize(st));
    SB_CUDA_TRY(cudaMemsetAsync(pt->visitCounters, 0, sizeof(tmp), st));
    for (uint32_t i = 0; i < capacity && i < 6; ++i) out[i] = tmp[i];
    return 6;
}

extern "C" const char* strelka_kernel_class_name(int i) { return (i >= 0 && i < KC_COUNT) ? kKernelNames[i] : ""; }

// ---------------------------------------------------------------------------
extern "C" int strelka_trace_execute(StrelkaPathTracer* pt, const TraceDesc* d, void* stream)
{
    if (!pt || !d) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    if (d->numNodes > (1u << 30)) return fail(STRELKA_ERR_INVALID_ARGUMENT, "numNodes exceeds 2^30");
    if (d->numNodes && (!d->bvhNodes || !d->vb || !d->ib || !d->instanceConst))
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "scene buffers must be non-NULL when numNodes > 0");
    if (d->numRays && (!d->rays || !d->hits)) return fail(STRELKA_ERR_INVALID_ARGUMENT, "rays/hits NULL");
    if ((d->flags & STRELKA_TRACE_COUNT) && !d->counters) return fail(STRELKA_ERR_INVALID_ARGUMENT, "counters NULL");
    if ((d->flags & STRELKA_TRACE_REFINE) && (d->flags & STRELKA_TRACE_ANY))
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "refine applies to closest-hit queries only");
    if (reinterpret_cast<uintptr_t>(d->rays) & 15) return fail(STRELKA_ERR_INVALID_ARGUMENT, "rays must be 16-byte aligned");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = ensure_scene(pt, d->bvhNodes, d->numNodes, d->vb, d->numVertices, d->ib, d->numIndices, d->instanceConst,
                          d->numInstances, d->sceneVersion, st);
    if (rc) return rc;
    if (d->numRays == 0) return STRELKA_OK;
    PathTracerDesc pd{};
    pd.bvhNodes = d->bvhNodes;
    pd.numNodes = d->numNodes;
    pd.vb = d->vb;
    pd.numVertices = d->numVertices;
    pd.ib = d->ib;
    pd.numIndices = d->numIndices;
    pd.instanceConst = d->instanceConst;
    pd.numInstances = d->numInstances;
    DevScene s = make_scene(pt, &pd);
    const bool any = (d->flags & 1u) != 0;
    const bool cnt = (d->flags & STRELKA_TRACE_COUNT) != 0;
    const bool refine = (d->flags & STRELKA_TRACE_REFINE) != 0;
    const int grid = std::min<int>((d->numRays + kExtendBlock - 1) / kExtendBlock, any ? pt->traceGridAny : pt->traceGrid);
    const float4* rays = reinterpret_cast<const float4*>(d->rays);
    Timer t(pt, KC_EXTEND, st);
    SB_CUDA_TRY(cudaMemsetAsync(pt->traceHead, 0, sizeof(uint32_t), st));
    const uint32_t qc = pt->cfg.queueChunk ? pt->cfg.queueChunk : kDefaultQueueChunk;
    uint32_t* hd = pt->traceHead;
    const uint32_t nr = d->numRays;
    if (any && cnt) k_trace<true, true, false><<<grid, kExtendBlock, 0, st>>>(s, rays, d->hits, nr, hd, qc, d->counters);
    else if (any) k_trace<true, false, false><<<grid, kExtendBlock, 0, st>>>(s, rays, d->hits, nr, hd, qc, nullptr);
    else if (refine && cnt)
        k_trace<false, true, true><<<grid, kExtendBlock, 0, st>>>(s, rays, d->hits, nr, hd, qc, d->counters);
    else if (refine) k_trace<false, false, true><<<grid, kExtendBlock, 0, st>>>(s, rays, d->hits, nr, hd, qc, nullptr);
    else if (cnt) k_trace<false, true, false><<<grid, kExtendBlock, 0, st>>>(s, rays, d->hits, nr, hd, qc, d->counters);
    else k_trace<false, false, false><<<grid, kExtendBlock, 0, st>>>(s, rays, d->hits, nr, hd, qc, nullptr);
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}

extern "C" int strelka_trace_host(StrelkaPathTracer* pt, const TraceDesc* desc, const Ray* hostRays, Hit* hostHits, void* stream)
{
    if (!pt || !desc || (desc->numRays && (!hostRays || !hostHits)))
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!desc->rays || !desc->hits) return fail(STRELKA_ERR_INVALID_ARGUMENT, "device staging rays/hits are NULL");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    SB_CUDA_TRY(cudaMemcpyAsync((void*)desc->rays, hostRays, (size_t)desc->numRays * sizeof(Ray), cudaMemcpyHostToDevice, st));
    int rc = strelka_trace_execute(pt, desc, stream);
    if (rc) return rc;
    SB_CUDA_TRY(cudaMemcpyAsync(hostHits, desc->hits, (size_t)desc->numRays * sizeof(Hit), cudaMemcpyDeviceToHost, st));
    SB_CUDA_TRY(cudaStreamSynchronize(st));
    return STRELKA_OK;
}
