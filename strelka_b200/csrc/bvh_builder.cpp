// bvh_builder.cpp — host SAH BVH builder emitting the reference's flattened
// depth-first node layout (replaces BvhBuilder, src/render/bvh.cpp:107-254).
//
// The reference builds a binary BVH with one triangle per leaf through
// Embree (RTC_BUILD_QUALITY_HIGH) and repacks it depth-first: a node's left
// child is the next node, nodeOffset is the escape index (the right sibling
// for a left child, the parent's escape for a right child, -1 at the end),
// a leaf stores instId and the bits of its per-instance triangle index in
// minBounds.x (bvh.cpp:169-235).  Triangle boxes are padded by +1e-6 on the
// max corner (bvh.h:138-151).  Embree is not available; this builder is a
// binned SAH builder (32 bins, all three axes) with the same output format.
//
// Because every leaf holds one triangle, a subtree over n triangles has
// exactly 2n-1 nodes, so each subtree's position in the flattened array is
// known before it is built and subtrees are built in parallel (OpenMP tasks)
// directly into the output.  The result is deterministic.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <vector>

#include "common.h"

namespace {

struct Box {
    float lo[3], hi[3];
    void reset()
    {
        for (int a = 0; a < 3; ++a) {
            lo[a] = INFINITY;
            hi[a] = -INFINITY;
        }
    }
    void grow(const Box& b)
    {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], b.lo[a]);
            hi[a] = std::max(hi[a], b.hi[a]);
        }
    }
    void grow(const float* p)
    {
        for (int a = 0; a < 3; ++a) {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a]);
        }
    }
    // include/render/bvh.h:64-72
    float half_area() const
    {
        float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
        if (!(dx >= 0)) return 0.0f;
        return dx * (dy + dz) + dy * dz;
    }
};

struct Prim {
    Box box;
    float c[3];
    uint32_t instId, primId;
};

constexpr int kBins = 32;
constexpr uint32_t kParallelThreshold = 1u << 14;

struct Builder {
    std::vector<Prim> prims;
    std::vector<uint32_t> idx;
    BVHNode* out = nullptr;

    void emit_leaf(uint32_t pos, uint32_t escape, const Prim& p)
    {
        BVHNode& n = out[pos];
        memset(&n, 0, sizeof(n));
        memcpy(&n.minBounds[0], &p.primId, 4);
        n.instId = (int32_t)p.instId;
        n.nodeOffset = (int32_t)escape;
    }

    // Chooses the split of idx[begin,end) and partitions it; returns the
    // number of primitives in the left half.
    uint32_t split(uint32_t begin, uint32_t end, const Box& cb)
    {
        const uint32_t n = end - begin;
        float bestCost = INFINITY;
        int bestAxis = -1, bestBin = -1;
        for (int axis = 0; axis < 3; ++axis) {
            const float ext = cb.hi[axis] - cb.lo[axis];
            if (!(ext > 0.0f)) continue;
            const float scale = (float)kBins / ext;
            Box bb[kBins];
            uint32_t bc[kBins];
            for (int b = 0; b < kBins; ++b) {
                bb[b].reset();
                bc[b] = 0;
            }
            for (uint32_t i = begin; i < end; ++i) {
                const Prim& p = prims[idx[i]];
                int b = (int)((p.c[axis] - cb.lo[axis]) * scale);
                b = b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
                bb[b].grow(p.box);
                bc[b]++;
            }
            float rightArea[kBins];
            uint32_t rightCount[kBins];
            Box acc;
            acc.reset();
            uint32_t cnt = 0;
            for (int b = kBins - 1; b > 0; --b) {
                if (bc[b]) acc.grow(bb[b]);
                cnt += bc[b];
                rightArea[b] = acc.half_area();
                rightCount[b] = cnt;
            }
            acc.reset();
            cnt = 0;
            for (int b = 0; b < kBins - 1; ++b) {
                if (bc[b]) acc.grow(bb[b]);
                cnt += bc[b];
                if (cnt == 0 || rightCount[b + 1] == 0) continue;
                float cost = acc.half_area() * (float)cnt + rightArea[b + 1] * (float)rightCount[b + 1];
                if (cost < bestCost) {
                    bestCost = cost;
                    bestAxis = axis;
                    bestBin = b;
                }
            }
        }
        if (bestAxis >= 0) {
            const float ext = cb.hi[bestAxis] - cb.lo[bestAxis];
            const float scale = (float)kBins / ext;
            uint32_t* first = idx.data() + begin;
            uint32_t* last = idx.data() + end;
            uint32_t* mid = std::partition(first, last, [&](uint32_t k) {
                int b = (int)((prims[k].c[bestAxis] - cb.lo[bestAxis]) * scale);
                b = b < 0 ? 0 : (b >= kBins ? kBins - 1 : b);
                return b <= bestBin;
            });
            uint32_t nl = (uint32_t)(mid - first);
            if (nl > 0 && nl < n) return nl;
        }
        // degenerate centroids: median split along the widest centroid axis,
        // ties broken by input order
        int axis = 0;
        float w = -1.0f;
        for (int a = 0; a < 3; ++a) {
            float e = cb.hi[a] - cb.lo[a];
            if (e > w) {
                w = e;
                axis = a;
            }
        }
        uint32_t half = n / 2;
        std::nth_element(idx.begin() + begin, idx.begin() + begin + half, idx.begin() + end, [&](uint32_t a, uint32_t b) {
            if (prims[a].c[axis] != prims[b].c[axis]) return prims[a].c[axis] < prims[b].c[axis];
            return a < b;
        });
        return half;
    }

    void build(uint32_t begin, uint32_t end, uint32_t pos, uint32_t escape)
    {
        const uint32_t n = end - begin;
        if (n == 1) {
            emit_leaf(pos, escape, prims[idx[begin]]);
            return;
        }
        Box bounds, cb;
        bounds.reset();
        cb.reset();
        for (uint32_t i = begin; i < end; ++i) {
            const Prim& p = prims[idx[i]];
            bounds.grow(p.box);
            cb.grow(p.c);
        }
        const uint32_t nl = split(begin, end, cb);
        const uint32_t leftPos = pos + 1;
        const uint32_t rightPos = pos + 2 * nl;  // left subtree holds 2*nl-1 nodes
        BVHNode& node = out[pos];
        memset(&node, 0, sizeof(node));
        for (int a = 0; a < 3; ++a) {
            node.minBounds[a] = bounds.lo[a];
            node.maxBounds[a] = bounds.hi[a];
        }
        node.instId = -1;
        node.nodeOffset = (int32_t)escape;
        if (n >= kParallelThreshold) {
#pragma omp task default(shared) firstprivate(begin, nl, leftPos, rightPos)
            build(begin, begin + nl, leftPos, rightPos);
#pragma omp task default(shared) firstprivate(begin, end, nl, rightPos, escape)
            build(begin + nl, end, rightPos, escape);
#pragma omp taskwait
        } else {
            build(begin, begin + nl, leftPos, rightPos);
            build(begin + nl, end, rightPos, escape);
        }
    }
};

}  // namespace

extern "C" int strelka_bvh_build(const BVHInputPosition* positions, uint32_t numPositions, BVHNode** outNodes,
                                 uint32_t* outNumNodes)
{
    if (!outNodes || !outNumNodes) return sb::fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL output");
    *outNodes = nullptr;
    *outNumNodes = 0;
    if (numPositions % 3 != 0) return sb::fail(STRELKA_ERR_INVALID_ARGUMENT, "numPositions must be a multiple of 3");
    const uint32_t numTris = numPositions / 3;
    if (numTris == 0) return STRELKA_OK;  // bvh.cpp:240-243: empty BVH
    if (!positions) return sb::fail(STRELKA_ERR_INVALID_ARGUMENT, "positions is NULL");
    if (numTris > (1u << 29)) return sb::fail(STRELKA_ERR_INVALID_ARGUMENT, "too many triangles");
    Builder b;
    b.prims.resize(numTris);
    b.idx.resize(numTris);
    const float eps = 1e-6f;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)numTris; ++i) {
        Prim& p = b.prims[i];
        const float* v0 = positions[3 * i + 0].pos;
        const float* v1 = positions[3 * i + 1].pos;
        const float* v2 = positions[3 * i + 2].pos;
        for (int a = 0; a < 3; ++a) {
            p.box.lo[a] = std::min(v0[a], std::min(v1[a], v2[a]));
            p.box.hi[a] = std::max(v0[a], std::max(v1[a], v2[a])) + eps;
            p.c[a] = (p.box.lo[a] + p.box.hi[a]) * 0.5f;
        }
        p.instId = positions[3 * i].instId;
        p.primId = positions[3 * i].primId;
        b.idx[i] = (uint32_t)i;
    }
    const uint32_t numNodes = 2 * numTris - 1;
    BVHNode* nodes = static_cast<BVHNode*>(malloc((size_t)numNodes * sizeof(BVHNode)));
    if (!nodes) return sb::fail(STRELKA_ERR_OUT_OF_MEMORY, "malloc of %u nodes failed", numNodes);
    b.out = nodes;
#pragma omp parallel
#pragma omp single nowait
    b.build(0, numTris, 0, 0xFFFFFFFFu);
    *outNodes = nodes;
    *outNumNodes = numNodes;
    return STRELKA_OK;
}
