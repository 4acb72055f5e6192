// bvh_gpu.cu — BVH construction on the GPU, emitting the same flattened
// depth-first layout as the host builder (an extension: the reference builds
// on the host with Embree, BvhBuilder::build, src/render/bvh.cpp:107-254).
//
// A linear BVH (Karras 2012, "Maximizing Parallelism in the Construction of
// BVHs, Octrees, and k-d Trees"):
//   1. one padded box per triangle (max corner + 1e-6, bvh.h:138-151) and the
//      bounds of the centroids;
//   2. 63-bit Morton codes of the centroids, sorted with their triangle index
//      (CUB radix sort);
//   3. the binary radix tree over the sorted codes (ties broken by position),
//      one internal node per thread;
//   4. boxes and subtree sizes bottom-up, the second child to arrive at a
//      node finishing it;
//   5. each node's depth-first position, summed on its path to the root (a
//      right child lands after its left sibling's subtree), and its escape
//      index = position + subtree size (-1 past the end);
//   6. the nodes written in place: inner = box, instId -1; leaf = instId and
//      the bits of the per-instance triangle index in minBounds[0].
// One triangle per leaf, 2n-1 nodes, as bvh.cpp:169-235 lays them out, so the
// traversal kernels and the oracle read the result unchanged.
//
// The default tree comes from PLOC instead of step 3-4 (Meister and Bittner
// 2018, "Parallel Locally-Ordered Clustering for Bounding Volume Hierarchy
// Construction"): over the Morton-sorted clusters, each cluster picks the
// neighbour within +-radius whose merged box has the least surface area;
// mutual pairs merge (the lower position becomes the left child), the
// survivors are compacted in order, and rounds repeat until one cluster is
// left.  It traces like a SAH tree and still builds in milliseconds.
#include <algorithm>
#include <cstring>
#include <vector>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "common.h"
#include "device_math.cuh"

using namespace sb;

namespace {

constexpr int kBlock = 256;
constexpr uint32_t kNone = 0xFFFFFFFFu;

// float <-> order-preserving uint32 for atomic min/max of bounds
__device__ __forceinline__ uint32_t ordered(float f)
{
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unordered(uint32_t u)
{
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

struct Scratch {
    float4* lo;          // n: triangle box min | instId bits
    float4* hi;          // n: triangle box max | primId bits
    uint64_t* codes[2];  // n
    uint32_t* order[2];  // n
    uint32_t* child;     // 2(n-1): left, right (>= n-1: leaf n-1+k)
    uint32_t* parent;    // 2n-1
    float4* nlo;         // n-1: internal box min
    float4* nhi;         // n-1: internal box max
    uint32_t* size;      // 2n-1: subtree node count
    uint32_t* arrive;    // n-1
    uint32_t* cbounds;   // 6: centroid bounds (ordered)
    void* cub;
    size_t cubBytes;
    // PLOC clusters (double-buffered): node id and box per cluster
    uint32_t* cid[2];
    float4* clo[2];
    float4* chi[2];
    uint32_t* nn;
    uint32_t* keep;
    uint32_t* pos;
    uint32_t* counters;  // [0] next internal node
    void* scan;
    size_t scanBytes;
};

__global__ void k_init_bounds(uint32_t* cb)
{
    if (threadIdx.x < 3) cb[threadIdx.x] = 0xFFFFFFFFu;     // min
    else if (threadIdx.x < 6) cb[threadIdx.x] = 0u;          // max
}

__global__ void __launch_bounds__(kBlock) k_prim_boxes(const BVHInputPosition* __restrict__ pos, uint32_t n, float4* lo,
                                                       float4* hi, uint32_t* cb)
{
    __shared__ uint32_t smin[3], smax[3];
    if (threadIdx.x < 3) {
        smin[threadIdx.x] = 0xFFFFFFFFu;
        smax[threadIdx.x] = 0u;
    }
    __syncthreads();
    const float eps = 1e-6f;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const BVHInputPosition a = pos[3 * (size_t)i], b = pos[3 * (size_t)i + 1], c = pos[3 * (size_t)i + 2];
        float l[3], h[3];
        for (int k = 0; k < 3; ++k) {
            l[k] = fminf(a.pos[k], fminf(b.pos[k], c.pos[k]));
            h[k] = fmaxf(a.pos[k], fmaxf(b.pos[k], c.pos[k])) + eps;
        }
        lo[i] = make_float4(l[0], l[1], l[2], __uint_as_float(a.instId));
        hi[i] = make_float4(h[0], h[1], h[2], __uint_as_float(a.primId));
        for (int k = 0; k < 3; ++k) {
            const float cen = (l[k] + h[k]) * 0.5f;
            atomicMin(&smin[k], ordered(cen));
            atomicMax(&smax[k], ordered(cen));
        }
    }
    __syncthreads();
    if (threadIdx.x < 3) {
        atomicMin(&cb[threadIdx.x], smin[threadIdx.x]);
        atomicMax(&cb[3 + threadIdx.x], smax[threadIdx.x]);
    }
}

__device__ __forceinline__ uint64_t spread21(uint32_t x)
{
    uint64_t v = x & 0x1FFFFFu;
    v = (v | (v << 32)) & 0x1F00000000FFFFull;
    v = (v | (v << 16)) & 0x1F0000FF0000FFull;
    v = (v | (v << 8)) & 0x100F00F00F00F00Full;
    v = (v | (v << 4)) & 0x10C30C30C30C30C3ull;
    v = (v | (v << 2)) & 0x1249249249249249ull;
    return v;
}

__global__ void __launch_bounds__(kBlock) k_morton(const float4* __restrict__ lo, const float4* __restrict__ hi, uint32_t n,
                                                   const uint32_t* __restrict__ cb, uint64_t* codes, uint32_t* order)
{
    float mn[3], sc[3];
    for (int k = 0; k < 3; ++k) {
        mn[k] = unordered(cb[k]);
        const float ext = unordered(cb[3 + k]) - mn[k];
        sc[k] = ext > 0.0f ? 2097151.0f / ext : 0.0f;
    }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 l = lo[i], h = hi[i];
        const float c[3] = {(l.x + h.x) * 0.5f, (l.y + h.y) * 0.5f, (l.z + h.z) * 0.5f};
        uint32_t q[3];
        for (int k = 0; k < 3; ++k) q[k] = (uint32_t)fminf(fmaxf((c[k] - mn[k]) * sc[k], 0.0f), 2097151.0f);
        codes[i] = (spread21(q[0]) << 2) | (spread21(q[1]) << 1) | spread21(q[2]);
        order[i] = i;
    }
}

// Length of the common prefix of sorted keys i and j, with the index as a
// tie-break for equal codes; -1 outside [0, n).
__device__ __forceinline__ int delta(const uint64_t* __restrict__ codes, int n, int i, int j)
{
    if (j < 0 || j >= n) return -1;
    const uint64_t a = codes[i], b = codes[j];
    if (a != b) return __clzll((long long)(a ^ b));
    return 64 + __clz((int)((uint32_t)i ^ (uint32_t)j));
}

__global__ void __launch_bounds__(kBlock) k_radix_tree(const uint64_t* __restrict__ codes, int n, uint32_t* child,
                                                       uint32_t* parent)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n - 1; i += gridDim.x * blockDim.x) {
        const int d = delta(codes, n, i, i + 1) - delta(codes, n, i, i - 1) >= 0 ? 1 : -1;
        const int dmin = delta(codes, n, i, i - d);
        int lmax = 2;
        while (delta(codes, n, i, i + lmax * d) > dmin) lmax <<= 1;
        int l = 0;
        for (int t = lmax >> 1; t >= 1; t >>= 1)
            if (delta(codes, n, i, i + (l + t) * d) > dmin) l += t;
        const int j = i + l * d;
        const int dnode = delta(codes, n, i, j);
        int s = 0;
        for (int t = (l + 1) >> 1;; t = (t + 1) >> 1) {
            if (delta(codes, n, i, i + (s + t) * d) > dnode) s += t;
            if (t == 1) break;
        }
        const int gamma = i + s * d + min(d, 0);
        const uint32_t left = (min(i, j) == gamma) ? (uint32_t)(n - 1 + gamma) : (uint32_t)gamma;
        const uint32_t right = (max(i, j) == gamma + 1) ? (uint32_t)(n - 1 + gamma + 1) : (uint32_t)(gamma + 1);
        child[2 * i] = left;
        child[2 * i + 1] = right;
        parent[left] = (uint32_t)i;
        parent[right] = (uint32_t)i;
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) parent[0] = kNone;
}

// Leaf k (node n-1+k, sorted triangle order[k]) walks up; the second of a
// node's two children to arrive computes its box and size and continues.
__global__ void __launch_bounds__(kBlock) k_bottom_up(const float4* __restrict__ lo, const float4* __restrict__ hi,
                                                      const uint32_t* __restrict__ order, uint32_t n,
                                                      const uint32_t* __restrict__ child,
                                                      const uint32_t* __restrict__ parent, float4* nlo, float4* nhi,
                                                      uint32_t* size, uint32_t* arrive)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        uint32_t node = n - 1 + k;
        size[node] = 1;
        uint32_t p = parent[node];
        uint32_t guard = 0;
        while (p != kNone && guard++ < 2 * n) {
            __threadfence();
            if (atomicAdd(&arrive[p], 1u) == 0) break;  // the sibling finishes p
            __threadfence();
            const uint32_t c0 = child[2 * p], c1 = child[2 * p + 1];
            float4 l0, h0, l1, h1;
            if (c0 >= n - 1) { l0 = lo[order[c0 - (n - 1)]]; h0 = hi[order[c0 - (n - 1)]]; }
            else { l0 = __ldcg(&nlo[c0]); h0 = __ldcg(&nhi[c0]); }
            if (c1 >= n - 1) { l1 = lo[order[c1 - (n - 1)]]; h1 = hi[order[c1 - (n - 1)]]; }
            else { l1 = __ldcg(&nlo[c1]); h1 = __ldcg(&nhi[c1]); }
            nlo[p] = make_float4(fminf(l0.x, l1.x), fminf(l0.y, l1.y), fminf(l0.z, l1.z), 0.0f);
            nhi[p] = make_float4(fmaxf(h0.x, h1.x), fmaxf(h0.y, h1.y), fmaxf(h0.z, h1.z), 0.0f);
            size[p] = 1 + __ldcg(&size[c0]) + __ldcg(&size[c1]);
            p = parent[p];
        }
    }
}

// Depth-first position of every node and the flattened node.
__global__ void __launch_bounds__(kBlock) k_flatten(const float4* __restrict__ lo, const float4* __restrict__ hi,
                                                    const uint32_t* __restrict__ order, uint32_t n,
                                                    const uint32_t* __restrict__ child, const uint32_t* __restrict__ parent,
                                                    const float4* __restrict__ nlo, const float4* __restrict__ nhi,
                                                    const uint32_t* __restrict__ size, BVHNode* out)
{
    const uint32_t total = 2 * n - 1;
    for (uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; x < total; x += gridDim.x * blockDim.x) {
        uint32_t pos = 0, c = x, p = parent[x], guard = 0;
        while (p != kNone && guard++ < total) {
            const uint32_t left = child[2 * p];
            pos += (c == left) ? 1u : 1u + size[left];
            c = p;
            p = parent[p];
        }
        const uint32_t end = pos + size[x];
        BVHNode node;
        memset(&node, 0, sizeof(node));
        node.nodeOffset = end < total ? (int32_t)end : -1;
        if (x >= n - 1) {
            const uint32_t t = order[x - (n - 1)];
            const float4 l = lo[t], h = hi[t];
            node.instId = (int32_t)__float_as_uint(l.w);
            const uint32_t prim = __float_as_uint(h.w);
            memcpy(&node.minBounds[0], &prim, 4);
        } else {
            const float4 l = nlo[x], h = nhi[x];
            node.minBounds[0] = l.x;
            node.minBounds[1] = l.y;
            node.minBounds[2] = l.z;
            node.maxBounds[0] = h.x;
            node.maxBounds[1] = h.y;
            node.maxBounds[2] = h.z;
            node.instId = -1;
        }
        out[pos] = node;
    }
}

// World-space corners of every instance's triangles (createBvhBuffer,
// ptrender.cpp:460-511), with the traversal's own transform arithmetic.
__global__ void __launch_bounds__(kBlock) k_scene_positions(const Vertex* __restrict__ vb, uint32_t numVertices,
                                                            const uint32_t* __restrict__ ib, uint32_t numIndices,
                                                            const InstanceConstants* __restrict__ inst,
                                                            const uint32_t* __restrict__ firstTri, uint32_t numInstances,
                                                            uint32_t numTris, BVHInputPosition* out, uint32_t* bad)
{
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < numTris; t += gridDim.x * blockDim.x) {
        int lo = 0, hi = (int)numInstances - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if (firstTri[mid] <= t) lo = mid;
            else hi = mid - 1;
        }
        const uint32_t j = (uint32_t)lo, prim = t - firstTri[j];
        const InstanceConstants* ic = &inst[j];
        const uint64_t base = (uint64_t)(uint32_t)ic->indexOffset + 3ull * prim;
        for (int k = 0; k < 3; ++k) {
            BVHInputPosition p;
            p.instId = j;
            p.primId = prim;
            v3 w = V(0.0f, 0.0f, 0.0f);
            if (base + k < numIndices && ib[base + k] < numVertices) {
                const Vertex& v = vb[ib[base + k]];
                w = mat_mul_point(ic->objectToWorld.m, V(v.position[0], v.position[1], v.position[2]), 1.0f);
            } else {
                atomicOr(bad, 1u);
            }
            p.pos[0] = w.x;
            p.pos[1] = w.y;
            p.pos[2] = w.z;
            out[3 * (size_t)t + k] = p;
        }
    }
}

// ---------------------------------------------------------------------------
// PLOC
__device__ __forceinline__ float half_area(float4 l, float4 h)
{
    const float dx = h.x - l.x, dy = h.y - l.y, dz = h.z - l.z;
    return dx * (dy + dz) + dy * dz;
}

__global__ void __launch_bounds__(kBlock) k_ploc_init(const float4* __restrict__ lo, const float4* __restrict__ hi,
                                                      const uint32_t* __restrict__ order, uint32_t n, uint32_t* cid,
                                                      float4* clo, float4* chi, uint32_t* size, uint32_t* parent)
{
    for (uint32_t k = blockIdx.x * blockDim.x + threadIdx.x; k < n; k += gridDim.x * blockDim.x) {
        const uint32_t t = order[k];
        cid[k] = n - 1 + k;
        clo[k] = lo[t];
        chi[k] = hi[t];
        size[n - 1 + k] = 1;
        parent[n - 1 + k] = kNone;
        if (k + 1 < n) parent[k] = kNone;
    }
}

// nearest neighbour of every cluster within +-radius (least merged area,
// ties to the lower position); boxes of a block's window staged in shared memory
constexpr int kMaxRadius = 32;

__global__ void __launch_bounds__(kBlock) k_ploc_nn(const float4* __restrict__ clo, const float4* __restrict__ chi, uint32_t C,
                                                    int radius, uint32_t* nn)
{
    __shared__ float4 slo[kBlock + 2 * kMaxRadius], shi[kBlock + 2 * kMaxRadius];
    for (uint32_t base = blockIdx.x * kBlock; base < C; base += gridDim.x * kBlock) {
        const int first = (int)base - radius;
        const int span = kBlock + 2 * radius;
        for (int t = threadIdx.x; t < span; t += kBlock) {
            const int g = first + t;
            if (g >= 0 && g < (int)C) {
                slo[t] = clo[g];
                shi[t] = chi[g];
            }
        }
        __syncthreads();
        const uint32_t i = base + threadIdx.x;
        if (i < C) {
            const int li = (int)threadIdx.x + radius;
            const float4 l = slo[li], h = shi[li];
            float best = INFINITY;
            uint32_t bj = i;
            const int j0 = max(0, (int)i - radius), j1 = min((int)C - 1, (int)i + radius);
            for (int j = j0; j <= j1; ++j) {
                if (j == (int)i) continue;
                const float4 ol = slo[j - first], oh = shi[j - first];
                const float4 ml = make_float4(fminf(l.x, ol.x), fminf(l.y, ol.y), fminf(l.z, ol.z), 0.0f);
                const float4 mh = make_float4(fmaxf(h.x, oh.x), fmaxf(h.y, oh.y), fmaxf(h.z, oh.z), 0.0f);
                const float a = half_area(ml, mh);
                if (a < best) {
                    best = a;
                    bj = (uint32_t)j;
                }
            }
            nn[i] = bj;
        }
        __syncthreads();
    }
}

// mutual nearest neighbours merge in place at the lower position
__global__ void __launch_bounds__(kBlock) k_ploc_merge(uint32_t C, const uint32_t* __restrict__ nn, uint32_t* cid, float4* clo,
                                                       float4* chi, uint32_t* keep, uint32_t* counters, uint32_t* child,
                                                       uint32_t* parent, float4* nlo, float4* nhi, uint32_t* size)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < C; i += gridDim.x * blockDim.x) {
        const uint32_t j = nn[i];
        const bool mutual = j != i && nn[j] == i;
        if (!mutual) {
            keep[i] = 1;
            continue;
        }
        if (i > j) {
            keep[i] = 0;
            continue;
        }
        const uint32_t a = cid[i], b = cid[j];
        const uint32_t node = atomicAdd(&counters[0], 1u);
        const float4 l0 = clo[i], h0 = chi[i], l1 = clo[j], h1 = chi[j];
        const float4 ml = make_float4(fminf(l0.x, l1.x), fminf(l0.y, l1.y), fminf(l0.z, l1.z), 0.0f);
        const float4 mh = make_float4(fmaxf(h0.x, h1.x), fmaxf(h0.y, h1.y), fmaxf(h0.z, h1.z), 0.0f);
        child[2 * node] = a;
        child[2 * node + 1] = b;
        parent[a] = node;
        parent[b] = node;
        nlo[node] = ml;
        nhi[node] = mh;
        size[node] = 1 + size[a] + size[b];
        cid[i] = node;
        clo[i] = ml;
        chi[i] = mh;
        keep[i] = 1;
    }
}

__global__ void __launch_bounds__(kBlock) k_ploc_compact(uint32_t C, const uint32_t* __restrict__ keep,
                                                         const uint32_t* __restrict__ pos, const uint32_t* __restrict__ cid,
                                                         const float4* __restrict__ clo, const float4* __restrict__ chi,
                                                         uint32_t* cid2, float4* clo2, float4* chi2, uint32_t* count)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < C; i += gridDim.x * blockDim.x) {
        if (keep[i]) {
            const uint32_t d = pos[i];
            cid2[d] = cid[i];
            clo2[d] = clo[i];
            chi2[d] = chi[i];
        }
        if (i == C - 1) *count = pos[i] + keep[i];
    }
}

int grid_for(uint32_t n, int sms)
{
    const uint32_t b = (n + kBlock - 1) / kBlock;
    return (int)std::max<uint32_t>(1, std::min<uint32_t>(b, (uint32_t)sms * 16));
}

}  // namespace

struct StrelkaBvhBuilder {
    int numSMs = 148;
    uint32_t mode = STRELKA_BVH_PLOC;
    uint32_t radius = 16;
    uint32_t cap = 0;  // triangles the scratch holds
    Scratch s{};
    std::vector<void*> allocs;
    BVHInputPosition* positions = nullptr;  // 3 per triangle, when built from scene buffers
    size_t posCap = 0;
    uint32_t* firstTri = nullptr;
    size_t firstTriCap = 0;
    uint32_t* bad = nullptr;
};

namespace {

void release(StrelkaBvhBuilder* b)
{
    for (void* p : b->allocs) cudaFree(p);
    b->allocs.clear();
    b->s = Scratch{};
    b->cap = 0;
}

template <typename T>
int salloc(StrelkaBvhBuilder* b, T** p, size_t n)
{
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, std::max<size_t>(n, 1) * sizeof(T));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(BVH build scratch)");
    b->allocs.push_back(q);
    *p = static_cast<T*>(q);
    return STRELKA_OK;
}

int ensure(StrelkaBvhBuilder* b, uint32_t n)
{
    if (b->cap >= n) return STRELKA_OK;
    release(b);
    Scratch& s = b->s;
    int rc;
    if ((rc = salloc(b, &s.lo, n)) || (rc = salloc(b, &s.hi, n)) || (rc = salloc(b, &s.codes[0], n)) ||
        (rc = salloc(b, &s.codes[1], n)) || (rc = salloc(b, &s.order[0], n)) || (rc = salloc(b, &s.order[1], n)) ||
        (rc = salloc(b, &s.child, 2 * (size_t)n)) || (rc = salloc(b, &s.parent, 2 * (size_t)n)) ||
        (rc = salloc(b, &s.nlo, n)) || (rc = salloc(b, &s.nhi, n)) || (rc = salloc(b, &s.size, 2 * (size_t)n)) ||
        (rc = salloc(b, &s.arrive, n)) || (rc = salloc(b, &s.cbounds, 8)) || (rc = salloc(b, &s.cid[0], n)) ||
        (rc = salloc(b, &s.cid[1], n)) || (rc = salloc(b, &s.clo[0], n)) || (rc = salloc(b, &s.clo[1], n)) ||
        (rc = salloc(b, &s.chi[0], n)) || (rc = salloc(b, &s.chi[1], n)) || (rc = salloc(b, &s.nn, n)) ||
        (rc = salloc(b, &s.keep, n)) || (rc = salloc(b, &s.pos, n)) || (rc = salloc(b, &s.counters, 4))) {
        release(b);
        return rc;
    }
    size_t scanBytes = 0;
    SB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(nullptr, scanBytes, s.keep, s.pos, (int)n));
    uint8_t* scanBuf = nullptr;
    if ((rc = salloc(b, &scanBuf, scanBytes))) {
        release(b);
        return rc;
    }
    s.scan = scanBuf;
    s.scanBytes = scanBytes;
    size_t bytes = 0;
    SB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(nullptr, bytes, s.codes[0], s.codes[1], s.order[0], s.order[1], (int)n, 0,
                                                63));
    uint8_t* cubBuf = nullptr;
    if ((rc = salloc(b, &cubBuf, bytes))) {
        release(b);
        return rc;
    }
    s.cub = cubBuf;
    s.cubBytes = bytes;
    b->cap = n;
    return STRELKA_OK;
}

// PLOC rounds over the Morton-sorted leaves; the host reads the cluster count
// after each round (one synchronisation per round) and stops when one is left
// or fails when a round makes no progress.
int ploc(StrelkaBvhBuilder* b, uint32_t n, cudaStream_t st)
{
    Scratch& s = b->s;
    k_ploc_init<<<grid_for(n, b->numSMs), kBlock, 0, st>>>(s.lo, s.hi, s.order[1], n, s.cid[0], s.clo[0], s.chi[0],
                                                           s.size, s.parent);
    SB_CUDA_TRY(cudaMemsetAsync(s.counters, 0, 4 * sizeof(uint32_t), st));
    uint32_t C = n;
    int cur = 0;
    const int radius = (int)std::min<uint32_t>(b->radius, (uint32_t)kMaxRadius);
    for (uint32_t round = 0; C > 1; ++round) {
        if (round > 4 * n) return fail(STRELKA_ERR_UNSUPPORTED, "PLOC did not converge");
        const int g = grid_for(C, b->numSMs);
        k_ploc_nn<<<g, kBlock, 0, st>>>(s.clo[cur], s.chi[cur], C, radius, s.nn);
        k_ploc_merge<<<g, kBlock, 0, st>>>(C, s.nn, s.cid[cur], s.clo[cur], s.chi[cur], s.keep, s.counters, s.child,
                                            s.parent, s.nlo, s.nhi, s.size);
        size_t bytes = s.scanBytes;
        SB_CUDA_TRY(cub::DeviceScan::ExclusiveSum(s.scan, bytes, s.keep, s.pos, (int)C, st));
        k_ploc_compact<<<g, kBlock, 0, st>>>(C, s.keep, s.pos, s.cid[cur], s.clo[cur], s.chi[cur], s.cid[cur ^ 1],
                                              s.clo[cur ^ 1], s.chi[cur ^ 1], s.counters + 1);
        SB_CUDA_TRY(cudaGetLastError());
        uint32_t next = 0;
        SB_CUDA_TRY(cudaMemcpyAsync(&next, s.counters + 1, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
        SB_CUDA_TRY(cudaStreamSynchronize(st));
        if (next >= C || next == 0) return fail(STRELKA_ERR_INVALID_ARGUMENT, "BVH build made no progress (non-finite positions?)");
        C = next;
        cur ^= 1;
    }
    return STRELKA_OK;
}

int build(StrelkaBvhBuilder* b, const BVHInputPosition* positions, uint32_t numTris, BVHNode* nodes, cudaStream_t st)
{
    int rc = ensure(b, numTris);
    if (rc) return rc;
    Scratch& s = b->s;
    const uint32_t n = numTris;
    const int g = grid_for(n, b->numSMs);
    k_init_bounds<<<1, 32, 0, st>>>(s.cbounds);
    k_prim_boxes<<<g, kBlock, 0, st>>>(positions, n, s.lo, s.hi, s.cbounds);
    k_morton<<<g, kBlock, 0, st>>>(s.lo, s.hi, n, s.cbounds, s.codes[0], s.order[0]);
    SB_CUDA_TRY(cudaGetLastError());
    size_t bytes = s.cubBytes;
    SB_CUDA_TRY(cub::DeviceRadixSort::SortPairs(s.cub, bytes, s.codes[0], s.codes[1], s.order[0], s.order[1], (int)n, 0,
                                                63, st));
    if (b->mode == STRELKA_BVH_PLOC && n > 1) {
        rc = ploc(b, n, st);
        if (rc) return rc;
    } else {
        if (n > 1) {
            k_radix_tree<<<grid_for(n - 1, b->numSMs), kBlock, 0, st>>>(s.codes[1], (int)n, s.child, s.parent);
            SB_CUDA_TRY(cudaMemsetAsync(s.arrive, 0, (size_t)(n - 1) * sizeof(uint32_t), st));
        } else {
            SB_CUDA_TRY(cudaMemsetAsync(s.parent, 0xFF, sizeof(uint32_t), st));
        }
        k_bottom_up<<<g, kBlock, 0, st>>>(s.lo, s.hi, s.order[1], n, s.child, s.parent, s.nlo, s.nhi, s.size, s.arrive);
    }
    k_flatten<<<grid_for(2 * n - 1, b->numSMs), kBlock, 0, st>>>(s.lo, s.hi, s.order[1], n, s.child, s.parent, s.nlo,
                                                                 s.nhi, s.size, nodes);
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}

}  // namespace

extern "C" int strelka_bvh_builder_create(StrelkaBvhBuilder** out)
{
    if (!out) return fail(STRELKA_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(STRELKA_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    auto* b = new StrelkaBvhBuilder();
    cudaDeviceGetAttribute(&b->numSMs, cudaDevAttrMultiProcessorCount, dev);
    if (cudaMalloc(&b->bad, sizeof(uint32_t)) != cudaSuccess) {
        delete b;
        return fail(STRELKA_ERR_OUT_OF_MEMORY, "cudaMalloc failed");
    }
    *out = b;
    return STRELKA_OK;
}

extern "C" int strelka_bvh_builder_set_mode(StrelkaBvhBuilder* b, uint32_t mode, uint32_t radius)
{
    if (!b) return fail(STRELKA_ERR_INVALID_ARGUMENT, "builder is NULL");
    if (mode != STRELKA_BVH_LBVH && mode != STRELKA_BVH_PLOC) return fail(STRELKA_ERR_INVALID_ARGUMENT, "unknown mode %u", mode);
    if (mode == STRELKA_BVH_PLOC && (radius < 1 || radius > (uint32_t)kMaxRadius))
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "radius must be in [1, %d]", kMaxRadius);
    b->mode = mode;
    if (mode == STRELKA_BVH_PLOC) b->radius = radius;
    return STRELKA_OK;
}

extern "C" int strelka_bvh_builder_destroy(StrelkaBvhBuilder* b)
{
    if (!b) return STRELKA_OK;
    release(b);
    if (b->positions) cudaFree(b->positions);
    if (b->firstTri) cudaFree(b->firstTri);
    if (b->bad) cudaFree(b->bad);
    delete b;
    return STRELKA_OK;
}

extern "C" int strelka_bvh_build_device(StrelkaBvhBuilder* b, const BVHInputPosition* positions, uint32_t numPositions,
                                        BVHNode* nodes, uint32_t nodeCapacity, uint32_t* numNodes, void* stream)
{
    if (!b || !numNodes) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    *numNodes = 0;
    if (numPositions % 3 != 0) return fail(STRELKA_ERR_INVALID_ARGUMENT, "numPositions must be a multiple of 3");
    const uint32_t numTris = numPositions / 3;
    if (numTris == 0) return STRELKA_OK;
    if (!positions || !nodes) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL buffer");
    if (numTris > (1u << 29)) return fail(STRELKA_ERR_INVALID_ARGUMENT, "too many triangles");
    if (nodeCapacity < 2 * numTris - 1)
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "nodes holds %u, the BVH needs %u", nodeCapacity, 2 * numTris - 1);
    int rc = build(b, positions, numTris, nodes, static_cast<cudaStream_t>(stream));
    if (rc) return rc;
    *numNodes = 2 * numTris - 1;
    return STRELKA_OK;
}

extern "C" int strelka_bvh_build_scene_device(StrelkaBvhBuilder* b, const Vertex* vb, uint32_t numVertices,
                                              const uint32_t* ib, uint32_t numIndices,
                                              const InstanceConstants* instances, uint32_t numInstances, BVHNode* nodes,
                                              uint32_t nodeCapacity, uint32_t* numNodes, void* stream)
{
    if (!b || !numNodes) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    *numNodes = 0;
    if (numInstances == 0) return STRELKA_OK;
    if (!vb || !ib || !instances || !nodes) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL buffer");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // per-instance triangle counts (the instance table is small; read on the host)
    std::vector<InstanceConstants> host(numInstances);
    SB_CUDA_TRY(cudaStreamSynchronize(st));
    SB_CUDA_TRY(cudaMemcpy(host.data(), instances, numInstances * sizeof(InstanceConstants), cudaMemcpyDeviceToHost));
    std::vector<uint32_t> first(numInstances);
    uint64_t total = 0;
    for (uint32_t j = 0; j < numInstances; ++j) {
        if (host[j].indexCount < 0 || host[j].indexCount % 3 != 0 || host[j].indexOffset < 0)
            return fail(STRELKA_ERR_INVALID_ARGUMENT, "instance %u: bad index range", j);
        first[j] = (uint32_t)total;
        total += (uint64_t)host[j].indexCount / 3;
    }
    if (total == 0) return STRELKA_OK;
    if (total > (1u << 29)) return fail(STRELKA_ERR_INVALID_ARGUMENT, "too many triangles");
    const uint32_t numTris = (uint32_t)total;
    if (nodeCapacity < 2 * numTris - 1)
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "nodes holds %u, the BVH needs %u", nodeCapacity, 2 * numTris - 1);
    if (3 * (size_t)numTris > b->posCap) {
        if (b->positions) cudaFree(b->positions);
        b->positions = nullptr;
        b->posCap = 0;
        SB_CUDA_TRY(cudaMalloc(&b->positions, 3 * (size_t)numTris * sizeof(BVHInputPosition)));
        b->posCap = 3 * (size_t)numTris;
    }
    if (numInstances > b->firstTriCap) {
        if (b->firstTri) cudaFree(b->firstTri);
        b->firstTri = nullptr;
        b->firstTriCap = 0;
        SB_CUDA_TRY(cudaMalloc(&b->firstTri, numInstances * sizeof(uint32_t)));
        b->firstTriCap = numInstances;
    }
    SB_CUDA_TRY(cudaMemcpyAsync(b->firstTri, first.data(), numInstances * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    SB_CUDA_TRY(cudaMemsetAsync(b->bad, 0, sizeof(uint32_t), st));
    k_scene_positions<<<grid_for(numTris, b->numSMs), kBlock, 0, st>>>(vb, numVertices, ib, numIndices, instances,
                                                                       b->firstTri, numInstances, numTris,
                                                                       b->positions, b->bad);
    SB_CUDA_TRY(cudaGetLastError());
    uint32_t bad = 0;
    SB_CUDA_TRY(cudaMemcpyAsync(&bad, b->bad, sizeof(uint32_t), cudaMemcpyDeviceToHost, st));
    SB_CUDA_TRY(cudaStreamSynchronize(st));
    if (bad) return fail(STRELKA_ERR_DEVICE_BOUNDS, "an index or vertex id is out of range");
    int rc = build(b, b->positions, numTris, nodes, st);
    if (rc) return rc;
    *numNodes = 2 * numTris - 1;
    return STRELKA_OK;
}
