// noalloc.cu — a ray-query entry point that allocates no device memory.
//
// strelka_trace_execute keeps its leaf-triangle table in memory the pass
// object allocates with cudaMalloc.  Some callers cannot let a library do
// that: an engine that hands the whole device heap to its own allocator up
// front (for example a renderer that owns device memory through Vulkan and
// imports it), or a real-time loop where an allocation's implicit device
// synchronisation would stall a frame.  strelka_trace_execute_noalloc gives
// them the same closest/any-hit queries with the scratch table in a
// file-scope __device__ array of fixed size instead.
//
// The array costs 12 MiB (+256 B) of device memory.  With CUDA's lazy module
// loading (the default since CUDA 12.2) the runtime reserves it when this
// file's module first loads on a device, which is the first call of this
// entry point there (its set-up asks for the array's address), and holds it
// until the process exits.  A caller whose allocator takes the whole heap
// should therefore make one call per device before reserving its heap; a
// call with numNodes = 0 and numRays = 0 does only that set-up.  Scenes with
// more than kNoAllocMaxNodes BVH nodes are rejected.  Every call shares the
// array, so two calls whose work overlaps on the GPU (for example on two
// streams of the same device) race on it; serialise such calls.  Each call
// rebuilds the table and clears the status word before using them, so
// nothing depends on what the previous call left behind.
#include <algorithm>
#include <mutex>

#include "common.h"
#include "traverse.cuh"

using namespace sb;

namespace {

// 262,144 nodes = scenes of up to 131,072 triangles (a one-triangle-per-leaf
// BVH over n triangles has 2n-1 nodes).
constexpr uint32_t kNoAllocMaxNodes = 1u << 18;
constexpr int kNoAllocMaxDevices = 64;

// Scratch: 3 float4 per node slot (v0|instId, e0|primId, e1), then the
// device status word.  Host code never uses these names as addresses; it
// asks the runtime for each device's address once (noalloc_setup).
static __device__ __align__(256) float4 g_noalloc_tris[3 * kNoAllocMaxNodes];
static __device__ __align__(256) uint32_t g_noalloc_status[64];

struct DeviceScratch {
    std::once_flag once;
    float4* tris = nullptr;
    uint32_t* status = nullptr;
    cudaError_t err = cudaSuccess;
};
DeviceScratch g_scratch[kNoAllocMaxDevices];

// Once per device, with that device current: the device addresses of the
// scratch arrays.  The first call on a device does this, so that call should
// come before any stream capture the caller starts.
int noalloc_setup(DeviceScratch** out)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(STRELKA_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(STRELKA_ERR_UNSUPPORTED, "device index %d beyond %d", dev,
                                                          kNoAllocMaxDevices);
    DeviceScratch& s = g_scratch[dev];
    std::call_once(s.once, [&s]() {
        s.err = cudaGetSymbolAddress(reinterpret_cast<void**>(&s.tris), g_noalloc_tris);
        if (s.err == cudaSuccess) s.err = cudaGetSymbolAddress(reinterpret_cast<void**>(&s.status), g_noalloc_status);
    });
    if (s.err != cudaSuccess) return cuda_fail(s.err, "cudaGetSymbolAddress(allocation-free scratch)");
    *out = &s;
    return STRELKA_OK;
}

// raytracing.h:134-153 per leaf node, written into the scratch table
__global__ void k_noalloc_prep(const float4* __restrict__ nodes, uint32_t numNodes, const InstanceConstants* __restrict__ inst,
                               uint32_t numInstances, const uint32_t* __restrict__ ib, uint32_t numIndices,
                               const Vertex* __restrict__ vb, uint32_t numVertices, float4* __restrict__ tris,
                               uint32_t* status)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < numNodes; i += gridDim.x * blockDim.x) {
        const float4 lo = nodes[2 * (size_t)i];
        const float4 hi = nodes[2 * (size_t)i + 1];
        const uint32_t instId = __float_as_uint(lo.w);
        const uint32_t esc = __float_as_uint(hi.w);
        if (esc != SB_INVALID && esc >= numNodes) atomicOr(status, STRELKA_DEV_NODE_OOB);
        if (instId == SB_INVALID) continue;
        float4* out = &tris[3 * (size_t)i];
        const float qnan = __int_as_float(0x7fc00000);
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

// The ray query of strelka_trace_execute, reading the scratch table.
template <bool ANY>
__global__ void __launch_bounds__(128) k_noalloc_trace(DevScene s, const float4* __restrict__ rays, Hit* __restrict__ hits,
                                                       uint32_t n)
{
    uint32_t nI = 0, nL = 0;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const float4 o = __ldg(&rays[2 * (size_t)i]);
        const float4 d = __ldg(&rays[2 * (size_t)i + 1]);
        HitRec h;
        h.u = 0.0f;
        h.v = 0.0f;
        h.t = ANY ? 0.0f : 1e9f;
        h.instId = SB_INVALID;
        h.primId = SB_INVALID;
        bool found = false;
        if (s.numNodes != 0)
            found = ANY ? trace_any<false>(s, xyz(o), o.w, xyz(d), h, nI, nL)
                        : trace_closest<false>(s, xyz(o), o.w, xyz(d), h, nI, nL);
        if (!found) {
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
    }
}

}  // namespace

extern "C" int strelka_trace_execute_noalloc(const TraceDesc* d, uint32_t* deviceStatus, void* stream)
{
    if (!d) return fail(STRELKA_ERR_INVALID_ARGUMENT, "desc is NULL");
    if (d->numNodes > kNoAllocMaxNodes)
        return fail(STRELKA_ERR_INVALID_ARGUMENT,
                    "scene has %u BVH nodes; the allocation-free ray query holds at most %u (its fixed scratch is %zu bytes)",
                    d->numNodes, kNoAllocMaxNodes, sizeof(g_noalloc_tris));
    if (d->flags & ~(uint32_t)STRELKA_TRACE_ANY)
        return fail(STRELKA_ERR_UNSUPPORTED, "the allocation-free ray query supports STRELKA_TRACE_CLOSEST/ANY only");
    if (d->numNodes && (!d->bvhNodes || !d->vb || !d->ib || !d->instanceConst))
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "scene buffers must be non-NULL when numNodes > 0");
    if (d->numRays && (!d->rays || !d->hits)) return fail(STRELKA_ERR_INVALID_ARGUMENT, "rays/hits NULL");
    if ((reinterpret_cast<uintptr_t>(d->rays) & 15) || (reinterpret_cast<uintptr_t>(d->bvhNodes) & 15))
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "rays and bvhNodes must be 16-byte aligned");
    DeviceScratch* sc = nullptr;
    int rc = noalloc_setup(&sc);
    if (rc) return rc;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the status word must start at zero for this call
    SB_CUDA_TRY(cudaMemsetAsync(sc->status, 0, sizeof(uint32_t), st));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (d->numNodes) {
        int grid = (int)std::min<uint32_t>((d->numNodes + 255) / 256, (uint32_t)sms * 16);
        k_noalloc_prep<<<grid, 256, 0, st>>>(reinterpret_cast<const float4*>(d->bvhNodes), d->numNodes, d->instanceConst,
                                             d->numInstances, d->ib, d->numIndices, d->vb, d->numVertices, sc->tris,
                                             sc->status);
        SB_CUDA_TRY(cudaGetLastError());
    }
    if (d->numRays) {
        DevScene s{};
        s.nodes = reinterpret_cast<const float4*>(d->bvhNodes);
        s.tris = sc->tris;
        s.numNodes = d->numNodes;
        s.numVertices = d->numVertices;
        s.vb = d->vb;
        s.ib = d->ib;
        s.numIndices = d->numIndices;
        s.numInstances = d->numInstances;
        s.inst = d->instanceConst;
        s.status = sc->status;
        const int grid = (int)std::min<uint32_t>((d->numRays + 127) / 128, (uint32_t)sms * 8);
        const float4* rays = reinterpret_cast<const float4*>(d->rays);
        if (d->flags & STRELKA_TRACE_ANY) k_noalloc_trace<true><<<grid, 128, 0, st>>>(s, rays, d->hits, d->numRays);
        else k_noalloc_trace<false><<<grid, 128, 0, st>>>(s, rays, d->hits, d->numRays);
        SB_CUDA_TRY(cudaGetLastError());
    }
    if (deviceStatus)
        SB_CUDA_TRY(cudaMemcpyAsync(deviceStatus, sc->status, sizeof(uint32_t), cudaMemcpyDeviceToDevice, st));
    return STRELKA_OK;
}
