// batch.cu — many scene/camera jobs of uneven size rendered as one batch,
// sm_100a.  An extension of the path tracer pass; the reference renders one
// view per PathTracer::execute (src/render/pathtracer.cpp:50-59).
//
// The jobs' paths form one index space: job j owns the global path indices
// [prefix[j], prefix[j+1]), and every kernel finds a path's job by a binary
// search of the prefix table held in shared memory.  Two execution modes:
//   * persistent: one persistent kernel; each warp takes `queueChunk` path
//     indices at a time from an atomic queue and its lanes trace whole paths
//     (one bounce per loop step), refilling from the warp's chunk as their
//     paths end, so jobs of any size and depth share the SMs;
//   * wavefront: the wavefront kernels of the single-job pass, job-aware,
//     with their persistent CTAs fed from atomic queues in `queueChunk`
//     units, and an optional counting sort of the shade queue by
//     (job, material) before shading.
// Each configuration's launch sequence is captured once into a CUDA graph
// and replayed with one cudaGraphLaunch.  Every path runs the same device
// code as the single-job pass (init_path, the node-pair traversal, shade,
// apply_shadow), so a job's samples are bit-identical to rendering it alone.
#include <algorithm>
#include <cstring>
#include <map>
#include <vector>

#include "common.h"
#include "internal.h"
#include "shading.cuh"
#include "wave.cuh"

using namespace sb;

namespace {

constexpr int kMaxJobs = STRELKA_BATCH_MAX_JOBS;
constexpr uint32_t kMaxSortKeys = 4096;
constexpr int kSmallBlock = 256;
constexpr unsigned kFull = 0xffffffffu;

struct BatchJobDev {
    DevScene s;
    PathTracerParam ubo;
    float* sampleBuffer;
    uint32_t numPaths;
    uint32_t keyBase;  // shade-sort keys [keyBase, keyBase + numMaterials] of this job (+1 for misses at 0)
};

struct BatchCtl {
    unsigned long long tStart;
    unsigned long long tDone[kMaxJobs];
    uint32_t done[kMaxJobs];
};

struct JobTable {
    const BatchJobDev* jobs;
    const uint32_t* prefix;  // numJobs + 1 entries
    int numJobs;
};

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void load_prefix(const JobTable& jt, uint32_t* sp)
{
    for (int i = threadIdx.x; i <= jt.numJobs; i += blockDim.x) sp[i] = jt.prefix[i];
    __syncthreads();
}

// The job owning global path g: the largest j < numJobs with prefix[j] <= g
// (a job without paths shares its prefix with the next job and is skipped).
__device__ __forceinline__ int find_job(const uint32_t* sp, int numJobs, uint32_t g)
{
    int lo = 0, hi = numJobs - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (sp[mid] <= g) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// Counts finished paths per job (one atomic per job per warp); the path that
// completes a job stamps the device time.  Called by the whole warp.
__device__ __forceinline__ void job_done(BatchCtl* ctl, const BatchJobDev* jobs, bool fin, int job)
{
    const int lane = threadIdx.x & 31;
    if (!__ballot_sync(kFull, fin)) return;
    const unsigned peers = __match_any_sync(kFull, fin ? job : -1 - lane);
    if (fin && lane == __ffs(peers) - 1) {
        const uint32_t n = (uint32_t)__popc(peers);
        const uint32_t old = atomicAdd(&ctl->done[job], n);
        if (old + n == jobs[job].numPaths) ctl->tDone[job] = global_ns();
    }
}

__global__ void k_batch_begin(BatchCtl* ctl, int numJobs)
{
    for (int j = threadIdx.x; j < numJobs; j += blockDim.x) {
        ctl->done[j] = 0;
        ctl->tDone[j] = 0;
    }
    if (threadIdx.x == 0) ctl->tStart = global_ns();
}

__device__ __forceinline__ void write_sample(float* sb, uint32_t idx, v3 c)
{
    float* o = sb + (size_t)idx * 3;
    o[0] = c.x;
    o[1] = c.y;
    o[2] = c.z;
}

// ---------------------------------------------------------------------------
// Persistent mode: whole paths, one bounce per loop step.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_batch_persistent(JobTable jt, uint32_t total, uint32_t chunk, uint32_t* fetch,
                                                            BatchCtl* ctl)
{
    __shared__ uint32_t sp[kMaxJobs + 1];
    load_prefix(jt, sp);
    WarpPool pool{0, 0, 0};
    bool have = false;
    int job = 0;
    uint32_t idx = 0;
    PathState ps;
    while (true) {
        const uint32_t g = pool_take(pool, fetch, total, chunk, !have);
        bool fin = false;
        if (!have && g != SB_INVALID) {
            job = find_job(sp, jt.numJobs, g);
            idx = g - sp[job];
            const BatchJobDev& J = jt.jobs[job];
            init_path(J.ubo, idx, ps);
            if ((int)J.ubo.maxDepth > 0) {
                have = true;
            } else {
                write_sample(J.sampleBuffer, idx, ps.color);
                fin = true;
            }
        }
        if (!__any_sync(kFull, have || fin)) break;
        if (have) {
            const BatchJobDev& J = jt.jobs[job];
            HitRec h;
            uint32_t a = 0, b = 0;
            const bool found = J.s.numNodes != 0 && trace_closest_rec<false, true>(J.s, ps.ro, ps.tmax, ps.rd, h, a, b);
            ShadowReq sr;
            bool cont = shade(J.s, J.ubo, ps, found, h, sr);
            if (sr.kind != 0 && shadow_visible(J.s, sr.kind, sr.o, sr.tmax, sr.d)) apply_shadow(ps.color, sr.cd, sr.cg);
            if (cont) {
                ++ps.depth;
                cont = ps.depth < (int)J.ubo.maxDepth;
            }
            if (!cont) {
                write_sample(J.sampleBuffer, idx, ps.color);
                fin = true;
                have = false;
            }
        }
        job_done(ctl, jt.jobs, fin, job);
    }
}

// ---------------------------------------------------------------------------
// Wavefront mode.  Slot i of a chunk holds global path first + i.
__global__ void __launch_bounds__(kSmallBlock) k_batch_generate(JobTable jt, Wave w, uint32_t first, uint32_t n)
{
    __shared__ uint32_t sp[kMaxJobs + 1];
    load_prefix(jt, sp);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        const uint32_t i = base + (threadIdx.x & 31u);
        bool live = false;
        if (i < n) {
            const uint32_t g = first + i;
            const int job = find_job(sp, jt.numJobs, g);
            const BatchJobDev& J = jt.jobs[job];
            PathState ps;
            init_path(J.ubo, g - sp[job], ps);
            w.ray_o[i] = f4(ps.ro, ps.tmax);
            w.ray_d[i] = f4(ps.rd, ps.lastPdf);
            w.thr[i] = f4(ps.throughput, __uint_as_float(pack_flags(ps)));
            w.col[i] = f4(ps.color, 0.0f);
            w.rng[i] = ps.rng;
            live = (int)J.ubo.maxDepth > 0;
        }
        const uint32_t pos = warp_push(&w.counters[0], live);
        if (live) w.queue[0][pos] = i;
    }
}

// Shadow-request count of a bounce: counters[2] on even bounces, [6] on odd
// ones, so that shadow(k) can read its count while extend(k+1) resets the
// one shade(k+1) fills.
__host__ __device__ __forceinline__ int batch_shadow_count(int qin) { return qin ? 6 : 2; }

// Bounces from this one on are finished by k_batch_tail.
constexpr int kBatchTailDepth = 5;

// Resident threads per SM asked of the traversal kernels: 8 x 128 for
// closest hit and 9 x 128 for any hit, as in the single-job pass.
constexpr int kExtendThreadsPerSM = 8 * 128;
constexpr int kShadowThreadsPerSM = 9 * 128;

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, kExtendThreadsPerSM / BLOCK) k_batch_extend(JobTable jt, Wave w, int qin, uint32_t first, uint32_t chunk,
                                                        uint32_t* fetch)
{
    __shared__ uint32_t sp[kMaxJobs + 1];
    load_prefix(jt, sp);
    const uint32_t count = w.counters[qin];
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        w.counters[qin ^ 1] = 0;                // refilled by this bounce's shade
        w.counters[batch_shadow_count(qin)] = 0;  // refilled by this bounce's shade
    }
    const uint32_t* __restrict__ q = qin ? w.queue[1] : w.queue[0];
    LocalStack st;
    uint32_t nI = 0, nL = 0;
    WarpPool pool{0, 0, 0};
    bool have = false;
    uint32_t slot = 0;
    const DevScene* sc = nullptr;
    Trav T;
    while (true) {
        const uint32_t i = pool_take(pool, fetch, count, chunk, !have);
        if (!have && i != SB_INVALID) {
            slot = q[i];
            sc = &jt.jobs[find_job(sp, jt.numJobs, first + slot)].s;
            const float4 o = w.ray_o[slot], d = w.ray_d[slot];
            trav_init(*sc, T, xyz(o), o.w, xyz(d), false);
            have = true;
        }
        if (!__any_sync(kFull, have)) break;
        if (!have) continue;
        const bool done = T.cur == SB_INVALID || closest_step<false>(*sc, T, st, nI, nL);
        if (!done) continue;
        w.hit[slot] = T.found ? make_float4(T.hit.u, T.hit.v, T.hit.t, __uint_as_float(T.hit.instId))
                              : make_float4(0.0f, 0.0f, 1e9f, __uint_as_float(SB_INVALID));
        w.hitRef[slot] = T.found ? T.leaf : SB_INVALID;  // k_batch_shade reads the leaf's shading record
        have = false;
    }
}

// Shade-sort key of a queued path: 0 for a miss, else 1 + the job's key base
// + the hit instance's material id (numMaterials for light instances and
// out-of-range ids).
__device__ __forceinline__ uint32_t shade_key(const JobTable& jt, const uint32_t* sp, const Wave& w, uint32_t first,
                                              uint32_t slot)
{
    const uint32_t inst = __float_as_uint(w.hit[slot].w);
    if (inst == SB_INVALID) return 0;
    const BatchJobDev& J = jt.jobs[find_job(sp, jt.numJobs, first + slot)];
    const uint32_t nm = J.s.numMaterials;
    if (inst >= J.s.numInstances) return 1 + J.keyBase + nm;
    const uint32_t m = (uint32_t)__ldg(&J.s.inst[inst].materialId);
    return 1 + J.keyBase + (m < nm ? m : nm);
}

// Keys of the shade queue in queue order (keys[i] for entry i) and their
// histogram.
__global__ void __launch_bounds__(kSmallBlock) k_batch_sort_count(JobTable jt, Wave w, int qin, uint32_t first,
                                                                  uint32_t numKeys, uint32_t* hist, uint16_t* keys)
{
    __shared__ uint32_t sp[kMaxJobs + 1];
    __shared__ uint32_t sh[kMaxSortKeys];
    for (uint32_t k = threadIdx.x; k < numKeys; k += blockDim.x) sh[k] = 0;
    load_prefix(jt, sp);
    const uint32_t count = w.counters[qin];
    const uint32_t* __restrict__ q = qin ? w.queue[1] : w.queue[0];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const uint32_t key = shade_key(jt, sp, w, first, q[i]);
        keys[i] = (uint16_t)key;
        atomicAdd(&sh[key], 1u);
    }
    __syncthreads();
    for (uint32_t k = threadIdx.x; k < numKeys; k += blockDim.x)
        if (sh[k]) atomicAdd(&hist[k], sh[k]);
}

// Exclusive scan of the histogram into offsets (one block), clearing the
// histogram for the next bounce.
__global__ void __launch_bounds__(1024) k_batch_sort_scan(uint32_t* hist, uint32_t numKeys, uint32_t* offsets)
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

// Scatter in tiles of kSortTile entries: ranks within a tile come from
// shared-memory counters (one atomic per key per warp), and each tile
// reserves its range of every key with one global atomic per key.
constexpr int kSortPerThread = 8;
constexpr int kSortTile = kSmallBlock * kSortPerThread;

__global__ void __launch_bounds__(kSmallBlock) k_batch_sort_scatter(Wave w, int qin, uint32_t numKeys,
                                                                    const uint16_t* __restrict__ keys, uint32_t* offsets,
                                                                    uint32_t* sorted)
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
            const unsigned peers = __match_any_sync(kFull, key[j]);
            const int leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (valid && lane == leader) base = atomicAdd(&cnt[key[j]], (uint32_t)__popc(peers));
            base = __shfl_sync(kFull, base, leader);
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

// One bounce of shading for every queued path (in `order`, the sorted queue,
// when not NULL); the job's scene and constants come from the job table.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_batch_shade(JobTable jt, Wave w, int qin, const uint32_t* order, uint32_t first,
                                                       uint32_t chunk, uint32_t* fetch)
{
    __shared__ uint32_t sp[kMaxJobs + 1];
    load_prefix(jt, sp);
    const uint32_t count = w.counters[qin];
    const uint32_t* __restrict__ q = order ? order : (qin ? w.queue[1] : w.queue[0]);
    uint32_t* qout = qin ? w.queue[0] : w.queue[1];
    const int lane = threadIdx.x & 31;
    uint32_t next = 0, end = 0;
    while (true) {
        if (next >= end) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(fetch, chunk);
            base = __shfl_sync(kFull, base, 0);
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
        if (valid) {
            slot = q[i];
            const BatchJobDev& J = jt.jobs[find_job(sp, jt.numJobs, first + slot)];
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
            h.primId = w.hitRef[slot];
            cont = shade(J.s, J.ubo, ps, h.instId != SB_INVALID, h, sr);
            if (cont) {
                ++ps.depth;
                cont = ps.depth < (int)J.ubo.maxDepth;
            }
            w.ray_o[slot] = f4(ps.ro, ps.tmax);
            w.ray_d[slot] = f4(ps.rd, ps.lastPdf);
            w.thr[slot] = f4(ps.throughput, __uint_as_float(pack_flags(ps)));
            w.col[slot] = f4(ps.color, 0.0f);
            w.rng[slot] = ps.rng;
        }
        const uint32_t qpos = warp_push(&w.counters[qin ^ 1], cont);
        if (cont) qout[qpos] = slot;
        const bool hasShadow = sr.kind != 0;
        const uint32_t spos = warp_push(&w.counters[batch_shadow_count(qin)], hasShadow);
        if (hasShadow) {
            w.sh_o[spos] = f4(sr.o, sr.tmax);
            w.sh_d[spos] = f4(sr.d, __uint_as_float(slot));
            w.sh_cd[spos] = f4(sr.cd, __uint_as_float((uint32_t)sr.kind));
            w.sh_cg[spos] = f4(sr.cg, 0.0f);
        }
    }
}

template <int BLOCK>
__global__ void __launch_bounds__(BLOCK, kShadowThreadsPerSM / BLOCK) k_batch_shadow(JobTable jt, Wave w, int qin, uint32_t first,
                                                        uint32_t chunk, uint32_t* fetch)
{
    __shared__ uint32_t sp[kMaxJobs + 1];
    load_prefix(jt, sp);
    const uint32_t count = w.counters[batch_shadow_count(qin)];
    LocalStackN st;
    uint32_t nI = 0, nL = 0;
    WarpPool pool{0, 0, 0};
    bool have = false;
    uint32_t item = 0;
    const DevScene* sc = nullptr;
    Trav T;
    while (true) {
        const uint32_t i = pool_take(pool, fetch, count, chunk, !have);
        if (!have && i != SB_INVALID) {
            item = i;
            const float4 o = w.sh_o[i], d = w.sh_d[i];
            sc = &jt.jobs[find_job(sp, jt.numJobs, first + __float_as_uint(d.w))].s;
            trav_init(*sc, T, xyz(o), o.w, xyz(d), true);
            have = true;
        }
        if (!__any_sync(kFull, have)) break;
        if (!have) continue;
        const bool done = T.cur == SB_INVALID || any_step<false>(*sc, T, st, nI, nL);
        if (!done) continue;
        const float4 cd = w.sh_cd[item];
        const int kind = (int)__float_as_uint(cd.w);
        const bool visible = !T.found || (kind == 1 && T.hit.instId < sc->numInstances &&
                                          __ldg(&sc->inst[T.hit.instId].lightId) != -1);
        if (visible) {
            const uint32_t slot = __float_as_uint(w.sh_d[item].w);
            const float4 cg = w.sh_cg[item];
            v3 c = xyz(w.col[slot]);
            apply_shadow(c, xyz(cd), xyz(cg));
            w.col[slot] = f4(c, 0.0f);
        }
        have = false;
    }
}

// Finishes every path queued for bounce `depth` (queue qin) with the
// persistent loop (closest hit, shade, shadow inline), each with its job's
// scene; one launch replaces the last bounces' launch sequences, where few
// paths remain.  Same device code and order of additions as the wavefront.
template <int BLOCK>
__global__ void __launch_bounds__(BLOCK) k_batch_tail(JobTable jt, Wave w, int qin, uint32_t first, uint32_t chunk,
                                                      uint32_t* fetch)
{
    __shared__ uint32_t sp[kMaxJobs + 1];
    load_prefix(jt, sp);
    const uint32_t count = w.counters[qin];
    const uint32_t* __restrict__ q = qin ? w.queue[1] : w.queue[0];
    WarpPool pool{0, 0, 0};
    PathState ps;
    uint32_t slot = 0;
    int job = 0;
    bool have = false;
    while (true) {
        const uint32_t got = pool_take(pool, fetch, count, chunk, !have);
        if (!have && got != SB_INVALID) {
            slot = q[got];
            job = find_job(sp, jt.numJobs, first + slot);
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
        if (!__any_sync(kFull, have)) break;
        if (!have) continue;
        const BatchJobDev& J = jt.jobs[job];
        HitRec h;
        uint32_t a = 0, b = 0;
        const bool found = J.s.numNodes != 0 && trace_closest_rec<false, true>(J.s, ps.ro, ps.tmax, ps.rd, h, a, b);
        ShadowReq sr;
        const bool cont = shade(J.s, J.ubo, ps, found, h, sr);
        if (sr.kind != 0 && shadow_visible(J.s, sr.kind, sr.o, sr.tmax, sr.d)) apply_shadow(ps.color, sr.cd, sr.cg);
        if (cont && ++ps.depth < (int)J.ubo.maxDepth) continue;
        w.col[slot] = f4(ps.color, 0.0f);
        have = false;
    }
}

__global__ void __launch_bounds__(kSmallBlock) k_batch_finalize(JobTable jt, Wave w, uint32_t first, uint32_t n,
                                                                BatchCtl* ctl)
{
    __shared__ uint32_t sp[kMaxJobs + 1];
    load_prefix(jt, sp);
    const uint32_t stride = gridDim.x * blockDim.x;
    for (uint32_t base = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); base < n; base += stride) {
        const uint32_t i = base + (threadIdx.x & 31u);
        const bool valid = i < n;
        int job = 0;
        if (valid) {
            const uint32_t g = first + i;
            job = find_job(sp, jt.numJobs, g);
            write_sample(jt.jobs[job].sampleBuffer, g - sp[job], xyz(w.col[i]));
        }
        job_done(ctl, jt.jobs, valid, job);
    }
}

int occupancy_grid(const void* fn, int block, int numSMs)
{
    int perSM = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&perSM, fn, block, 0) != cudaSuccess || perSM < 1) perSM = 1;
    return perSM * numSMs;
}

uint64_t config_key(const StrelkaBatchConfig& c)
{
    return (uint64_t)c.mode | ((uint64_t)c.blockSize << 4) | ((uint64_t)c.queueChunk << 16) |
           ((uint64_t)(c.materialSort ? 1 : 0) << 40) | ((uint64_t)(c.useGraph ? 1 : 0) << 41);
}

struct SceneRec {
    const BVHNode* nodes;
    uint32_t numNodes;
    const Vertex* vb;
    const uint32_t* ib;
    const InstanceConstants* inst;
    uint64_t version;
    void* mem;  // derived tables (internal.h SceneTables)
    SceneTables tables;
};

}  // namespace

struct StrelkaBatch {
    int numSMs = 148;
    std::vector<PathTracerDesc> descs;
    std::vector<BatchJobDev> jobsHost;  // by slot
    std::vector<uint32_t> order;        // slot -> the caller's job index
    std::vector<uint32_t> prefix;
    uint32_t total = 0;
    uint32_t numKeys = 0;
    int maxDepth = 0;
    BatchJobDev* jobsDev = nullptr;
    uint32_t* prefixDev = nullptr;
    BatchCtl* ctl = nullptr;
    uint32_t* status = nullptr;
    float* srgbLut = nullptr;
    std::vector<SceneRec> scenes;
    // wavefront state
    Wave w{};
    uint32_t* sorted = nullptr;
    uint16_t* keys = nullptr;
    uint32_t* hist = nullptr;
    uint32_t* offsets = nullptr;
    size_t waveCap = 0;
    std::vector<void*> waveAllocs;
    uint32_t* fetch = nullptr;
    size_t fetchCap = 0;
    // captured launch sequences
    std::map<uint64_t, cudaGraphExec_t> graphs;
    cudaStream_t capture = nullptr;
    cudaStream_t aux = nullptr;  // shadow queries beside the next bounce
    cudaEvent_t shadeDone = nullptr, shadowDone = nullptr;
    StrelkaBatchConfig tuned{};
    bool haveTuned = false;
};

namespace {

void drop_graphs(StrelkaBatch* b)
{
    for (auto& kv : b->graphs) cudaGraphExecDestroy(kv.second);
    b->graphs.clear();
}

void free_wave(StrelkaBatch* b)
{
    for (void* p : b->waveAllocs) cudaFree(p);
    b->waveAllocs.clear();
    b->w = Wave{};
    b->sorted = nullptr;
    b->keys = nullptr;
    b->waveCap = 0;
}

template <typename T>
int balloc(StrelkaBatch* b, T** p, size_t n)
{
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T));
    if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(batch wavefront state)");
    b->waveAllocs.push_back(q);
    *p = static_cast<T*>(q);
    return STRELKA_OK;
}

int ensure_wave(StrelkaBatch* b, size_t cap)
{
    if (b->waveCap >= cap) return STRELKA_OK;
    drop_graphs(b);  // graphs hold the old pointers
    free_wave(b);
    Wave& w = b->w;
    int rc;
    if ((rc = balloc(b, &w.ray_o, cap)) || (rc = balloc(b, &w.ray_d, cap)) || (rc = balloc(b, &w.thr, cap)) ||
        (rc = balloc(b, &w.col, cap)) || (rc = balloc(b, &w.rng, cap)) || (rc = balloc(b, &w.hit, cap)) ||
        (rc = balloc(b, &w.hitRef, cap)) || (rc = balloc(b, &w.queue[0], cap)) || (rc = balloc(b, &w.queue[1], cap)) ||
        (rc = balloc(b, &w.sh_o, cap)) || (rc = balloc(b, &w.sh_d, cap)) || (rc = balloc(b, &w.sh_cd, cap)) ||
        (rc = balloc(b, &w.sh_cg, cap)) || (rc = balloc(b, &w.counters, kWaveCounters)) || (rc = balloc(b, &b->sorted, cap)) ||
        (rc = balloc(b, &b->keys, cap))) {
        free_wave(b);
        return rc;
    }
    b->waveCap = cap;
    return STRELKA_OK;
}

int ensure_fetch(StrelkaBatch* b, size_t n)
{
    if (b->fetchCap >= n) return STRELKA_OK;
    drop_graphs(b);
    if (b->fetch) cudaFree(b->fetch);
    b->fetch = nullptr;
    b->fetchCap = 0;
    SB_CUDA_TRY(cudaMalloc(&b->fetch, n * sizeof(uint32_t)));
    b->fetchCap = n;
    return STRELKA_OK;
}

int check_config(const StrelkaBatch* b, const StrelkaBatchConfig& c)
{
    if (c.mode != STRELKA_BATCH_PERSISTENT && c.mode != STRELKA_BATCH_WAVEFRONT)
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "unknown batch mode %u", c.mode);
    if (c.blockSize != 64 && c.blockSize != 128 && c.blockSize != 256)
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "blockSize must be 64, 128 or 256");
    if (c.queueChunk < 32 || c.queueChunk > 4096 || (c.queueChunk & 31))
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "queueChunk must be a multiple of 32 in [32, 4096]");
    if (c.materialSort && c.mode != STRELKA_BATCH_WAVEFRONT)
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "materialSort applies to the wavefront mode");
    if (c.materialSort && b->numKeys > kMaxSortKeys)
        return fail(STRELKA_ERR_UNSUPPORTED, "%u sort keys exceed %u", b->numKeys, kMaxSortKeys);
    return STRELKA_OK;
}

template <int BLOCK>
int launch_persistent(StrelkaBatch* b, const JobTable& jt, uint32_t chunk, cudaStream_t st)
{
    const int grid = occupancy_grid((const void*)k_batch_persistent<BLOCK>, BLOCK, b->numSMs);
    k_batch_persistent<BLOCK><<<grid, BLOCK, 0, st>>>(jt, b->total, chunk, b->fetch, b->ctl);
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}

template <int BLOCK>
int launch_wavefront(StrelkaBatch* b, const JobTable& jt, const StrelkaBatchConfig& c, cudaStream_t st)
{
    const size_t chunkPaths = b->waveCap;
    const int gridE = occupancy_grid((const void*)k_batch_extend<BLOCK>, BLOCK, b->numSMs);
    const int gridS = occupancy_grid((const void*)k_batch_shade<BLOCK>, BLOCK, b->numSMs);
    const int gridW = occupancy_grid((const void*)k_batch_shadow<BLOCK>, BLOCK, b->numSMs);
    const int gridL = occupancy_grid((const void*)k_batch_tail<BLOCK>, BLOCK, b->numSMs);
    uint32_t f = 0;
    for (uint64_t first = 0; first < b->total; first += chunkPaths) {
        const uint32_t n = (uint32_t)std::min<uint64_t>(chunkPaths, b->total - first);
        SB_CUDA_TRY(cudaMemsetAsync(b->w.counters, 0, kWaveCounters * sizeof(uint32_t), st));
        const int gridG = std::min<int>((n + kSmallBlock - 1) / kSmallBlock, b->numSMs * 8);
        k_batch_generate<<<gridG, kSmallBlock, 0, st>>>(jt, b->w, (uint32_t)first, n);
        // shadow(k) runs on the auxiliary stream beside extend(k+1) and the
        // sort of bounce k+1 (it reads only shade(k)'s outputs); shade(k+1)
        // waits for it, so contributions reach each path in the same order
        const int tailDepth = std::min(b->maxDepth, kBatchTailDepth);
        bool pendingShadow = false;
        for (int depth = 0; depth < tailDepth; ++depth) {
            const int qin = depth & 1;
            k_batch_extend<BLOCK><<<gridE, BLOCK, 0, st>>>(jt, b->w, qin, (uint32_t)first, c.queueChunk, b->fetch + f++);
            const uint32_t* order = nullptr;
            if (c.materialSort) {
                const int gridK = std::min<int>((n + kSmallBlock - 1) / kSmallBlock, b->numSMs * 4);
                const int gridT = std::min<int>((n + kSortTile - 1) / kSortTile, b->numSMs * 4);
                k_batch_sort_count<<<gridK, kSmallBlock, 0, st>>>(jt, b->w, qin, (uint32_t)first, b->numKeys, b->hist,
                                                                  b->keys);
                k_batch_sort_scan<<<1, 1024, 0, st>>>(b->hist, b->numKeys, b->offsets);
                k_batch_sort_scatter<<<gridT, kSmallBlock, 0, st>>>(b->w, qin, b->numKeys, b->keys, b->offsets,
                                                                    b->sorted);
                order = b->sorted;
            }
            if (pendingShadow) SB_CUDA_TRY(cudaStreamWaitEvent(st, b->shadowDone, 0));
            k_batch_shade<BLOCK><<<gridS, BLOCK, 0, st>>>(jt, b->w, qin, order, (uint32_t)first, c.queueChunk,
                                                         b->fetch + f++);
            SB_CUDA_TRY(cudaEventRecord(b->shadeDone, st));
            SB_CUDA_TRY(cudaStreamWaitEvent(b->aux, b->shadeDone, 0));
            k_batch_shadow<BLOCK><<<gridW, BLOCK, 0, b->aux>>>(jt, b->w, qin, (uint32_t)first, c.queueChunk,
                                                              b->fetch + f++);
            SB_CUDA_TRY(cudaEventRecord(b->shadowDone, b->aux));
            pendingShadow = true;
        }
        if (pendingShadow) SB_CUDA_TRY(cudaStreamWaitEvent(st, b->shadowDone, 0));
        if (tailDepth < b->maxDepth)
            k_batch_tail<BLOCK><<<gridL, BLOCK, 0, st>>>(jt, b->w, tailDepth & 1, (uint32_t)first, c.queueChunk,
                                                        b->fetch + f++);
        k_batch_finalize<<<gridG, kSmallBlock, 0, st>>>(jt, b->w, (uint32_t)first, n, b->ctl);
    }
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}

// The launch sequence of one batch execution under configuration c.
int record(StrelkaBatch* b, const StrelkaBatchConfig& c, cudaStream_t st)
{
    JobTable jt{b->jobsDev, b->prefixDev, (int)b->jobsHost.size()};
    k_batch_begin<<<1, 64, 0, st>>>(b->ctl, jt.numJobs);
    const size_t nFetch = c.mode == STRELKA_BATCH_PERSISTENT ? 1 : b->fetchCap;
    SB_CUDA_TRY(cudaMemsetAsync(b->fetch, 0, nFetch * sizeof(uint32_t), st));
    if (c.mode == STRELKA_BATCH_PERSISTENT) {
        switch (c.blockSize) {
            case 64: return launch_persistent<64>(b, jt, c.queueChunk, st);
            case 128: return launch_persistent<128>(b, jt, c.queueChunk, st);
            default: return launch_persistent<256>(b, jt, c.queueChunk, st);
        }
    }
    switch (c.blockSize) {
        case 64: return launch_wavefront<64>(b, jt, c, st);
        case 128: return launch_wavefront<128>(b, jt, c, st);
        default: return launch_wavefront<256>(b, jt, c, st);
    }
}

int prepare(StrelkaBatch* b, const StrelkaBatchConfig& c)
{
    if (c.mode == STRELKA_BATCH_WAVEFRONT) {
        const size_t cap = std::min<size_t>(b->total, (size_t)1 << 25);
        int rc = ensure_wave(b, std::max<size_t>(cap, 1));
        if (rc) return rc;
        const size_t chunks = (b->total + b->waveCap - 1) / b->waveCap;
        rc = ensure_fetch(b, std::max<size_t>(1, chunks * (size_t)b->maxDepth * 3));
        if (rc) return rc;
        if (c.materialSort && !b->hist) {
            SB_CUDA_TRY(cudaMalloc(&b->hist, kMaxSortKeys * sizeof(uint32_t)));
            SB_CUDA_TRY(cudaMalloc(&b->offsets, kMaxSortKeys * sizeof(uint32_t)));
            SB_CUDA_TRY(cudaMemset(b->hist, 0, kMaxSortKeys * sizeof(uint32_t)));
        }
        return STRELKA_OK;
    }
    return ensure_fetch(b, 1);
}

int run(StrelkaBatch* b, const StrelkaBatchConfig& c, cudaStream_t st)
{
    int rc = check_config(b, c);
    if (rc) return rc;
    if (b->jobsHost.empty() || b->total == 0) return STRELKA_OK;
    rc = prepare(b, c);
    if (rc) return rc;
    if (!c.useGraph) return record(b, c, st);
    const uint64_t key = config_key(c);
    auto it = b->graphs.find(key);
    if (it == b->graphs.end()) {
        SB_CUDA_TRY(cudaStreamBeginCapture(b->capture, cudaStreamCaptureModeThreadLocal));
        rc = record(b, c, b->capture);
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->capture, &g);
        if (rc) {
            if (g) cudaGraphDestroy(g);
            return rc;
        }
        if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
        cudaGraphExec_t exec = nullptr;
        e = cudaGraphInstantiate(&exec, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGraphInstantiate");
        it = b->graphs.emplace(key, exec).first;
    }
    SB_CUDA_TRY(cudaGraphLaunch(it->second, st));
    return STRELKA_OK;
}

StrelkaBatchConfig default_config(const StrelkaBatch* b)
{
    StrelkaBatchConfig c{};
    c.mode = STRELKA_BATCH_WAVEFRONT;
    c.blockSize = 128;
    c.queueChunk = 256;
    c.materialSort = 0;
    c.useGraph = 1;
    (void)b;
    return c;
}

}  // namespace

extern "C" int strelka_batch_create(StrelkaBatch** out)
{
    if (!out) return fail(STRELKA_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(STRELKA_ERR_NO_DEVICE, "no CUDA device: %s", cudaGetErrorString(e));
    auto* b = new StrelkaBatch();
    cudaDeviceGetAttribute(&b->numSMs, cudaDevAttrMultiProcessorCount, dev);
    float lut[256];
    srgb_lut_host(lut);
    bool ok = cudaMalloc(&b->srgbLut, sizeof(lut)) == cudaSuccess && cudaMalloc(&b->status, sizeof(uint32_t)) == cudaSuccess &&
              cudaMalloc(&b->ctl, sizeof(BatchCtl)) == cudaSuccess &&
              cudaStreamCreateWithFlags(&b->capture, cudaStreamNonBlocking) == cudaSuccess &&
              cudaStreamCreateWithFlags(&b->aux, cudaStreamNonBlocking) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->shadeDone, cudaEventDisableTiming) == cudaSuccess &&
              cudaEventCreateWithFlags(&b->shadowDone, cudaEventDisableTiming) == cudaSuccess;
    if (!ok) {
        strelka_batch_destroy(b);
        return fail(STRELKA_ERR_OUT_OF_MEMORY, "batch allocation failed");
    }
    cudaMemcpy(b->srgbLut, lut, sizeof(lut), cudaMemcpyHostToDevice);
    cudaMemset(b->status, 0, sizeof(uint32_t));
    cudaMemset(b->ctl, 0, sizeof(BatchCtl));
    *out = b;
    return STRELKA_OK;
}

extern "C" int strelka_batch_destroy(StrelkaBatch* b)
{
    if (!b) return STRELKA_OK;
    cudaDeviceSynchronize();
    drop_graphs(b);
    free_wave(b);
    for (SceneRec& r : b->scenes) cudaFree(r.mem);
    void* ptrs[] = {b->jobsDev, b->prefixDev, b->ctl, b->status, b->srgbLut, b->fetch, b->hist, b->offsets};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (b->capture) cudaStreamDestroy(b->capture);
    if (b->aux) cudaStreamDestroy(b->aux);
    if (b->shadeDone) cudaEventDestroy(b->shadeDone);
    if (b->shadowDone) cudaEventDestroy(b->shadowDone);
    delete b;
    return STRELKA_OK;
}

extern "C" int strelka_batch_set_jobs(StrelkaBatch* b, const PathTracerDesc* jobs, uint32_t numJobs, void* stream)
{
    if (!b) return fail(STRELKA_ERR_INVALID_ARGUMENT, "batch is NULL");
    if (numJobs > (uint32_t)kMaxJobs) return fail(STRELKA_ERR_INVALID_ARGUMENT, "at most %d jobs", kMaxJobs);
    if (numJobs && !jobs) return fail(STRELKA_ERR_INVALID_ARGUMENT, "jobs is NULL");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // Shortest job first: slot k of the batch's path space holds the caller's
    // job ord[k], in ascending order of path count (ties in the caller's
    // order), so small jobs finish in the first chunks instead of waiting
    // behind large ones.  A path's arithmetic depends only on its own job
    // and its index within that job, so the order changes no result.
    std::vector<uint32_t> ord(numJobs);
    for (uint32_t j = 0; j < numJobs; ++j) ord[j] = j;
    auto paths_of = [&](uint32_t j) {
        const PathTracerParam& u = jobs[j].constants;
        return u.dimension[0] <= 0 || u.dimension[1] <= 0 || u.spp <= 0
                   ? 0ull
                   : (uint64_t)u.dimension[0] * (uint64_t)u.dimension[1] * (uint64_t)u.spp;
    };
    std::stable_sort(ord.begin(), ord.end(), [&](uint32_t a, uint32_t b2) { return paths_of(a) < paths_of(b2); });
    std::vector<uint32_t> prefix(numJobs + 1, 0);
    uint64_t total = 0;
    uint32_t numKeys = 1;
    int maxDepth = 0;
    for (uint32_t k = 0; k < numJobs; ++k) {
        const uint32_t j = ord[k];
        const PathTracerDesc& d = jobs[j];
        int rc = validate_scene_desc(&d);
        if (rc) return fail(rc, "job %u: %s", j, last_error().c_str());
        const PathTracerParam& u = d.constants;
        if (u.dimension[0] <= 0 || u.dimension[1] <= 0 || u.spp <= 0)
            return fail(STRELKA_ERR_INVALID_ARGUMENT, "job %u: dimension and spp must be positive", j);
        if (!d.sampleBuffer) return fail(STRELKA_ERR_INVALID_ARGUMENT, "job %u: sampleBuffer is NULL", j);
        if (d.envMap) {
            const StrelkaEnvMap* e = d.envMap;
            if (!e->rgba32f || !e->marginal_cdf || !e->conditional_cdf || e->width == 0 || e->height == 0)
                return fail(STRELKA_ERR_INVALID_ARGUMENT, "job %u: incomplete environment map", j);
        }
        prefix[k] = (uint32_t)total;
        total += (uint64_t)u.dimension[0] * (uint64_t)u.dimension[1] * (uint64_t)u.spp;
        if (total > 0x7FFFFFFFull) return fail(STRELKA_ERR_INVALID_ARGUMENT, "the batch exceeds 2^31 paths");
        maxDepth = std::max(maxDepth, (int)u.maxDepth);
        numKeys += (d.mdl_mdlMaterial ? d.numMaterials : 0) + 1;
    }
    prefix[numJobs] = (uint32_t)total;
    if (stream) SB_CUDA_TRY(cudaStreamSynchronize(st));
    else SB_CUDA_TRY(cudaDeviceSynchronize());
    drop_graphs(b);
    b->haveTuned = false;
    // record tables of the distinct scenes (kept across calls)
    std::vector<BatchJobDev> host(numJobs);
    uint32_t keyBase = 0;
    for (uint32_t k = 0; k < numJobs; ++k) {
        const PathTracerDesc& d = jobs[ord[k]];
        const SceneTables* tables = nullptr;
        for (SceneRec& r : b->scenes)
            if (r.nodes == d.bvhNodes && r.numNodes == d.numNodes && r.vb == d.vb && r.ib == d.ib &&
                r.inst == d.instanceConst && r.version == d.sceneVersion)
                tables = &r.tables;
        if (!tables) {
            void* mem = nullptr;
            SB_CUDA_TRY(cudaMalloc(&mem, scene_tables_bytes(d.numNodes)));
            b->scenes.push_back(SceneRec{d.bvhNodes, d.numNodes, d.vb, d.ib, d.instanceConst, d.sceneVersion, mem,
                                         scene_tables(mem, d.numNodes)});
            tables = &b->scenes.back().tables;
            int rc = launch_prep_tables(d.bvhNodes, d.numNodes, d.instanceConst, d.numInstances, d.ib, d.numIndices,
                                        d.vb, d.numVertices, *tables, b->status, b->numSMs, st);
            if (rc) return rc;
        }
        BatchJobDev& J = host[k];
        memset(&J, 0, sizeof(J));
        J.s = scene_from_desc(&d, *tables, b->srgbLut, b->status);
        J.ubo = d.constants;
        J.sampleBuffer = d.sampleBuffer;
        J.numPaths = prefix[k + 1] - prefix[k];
        J.keyBase = keyBase;
        keyBase += (d.mdl_mdlMaterial ? d.numMaterials : 0) + 1;
    }
    if (b->jobsDev) cudaFree(b->jobsDev);
    if (b->prefixDev) cudaFree(b->prefixDev);
    b->jobsDev = nullptr;
    b->prefixDev = nullptr;
    SB_CUDA_TRY(cudaMalloc(&b->jobsDev, std::max<size_t>(numJobs, 1) * sizeof(BatchJobDev)));
    SB_CUDA_TRY(cudaMalloc(&b->prefixDev, (numJobs + 1) * sizeof(uint32_t)));
    if (numJobs) SB_CUDA_TRY(cudaMemcpy(b->jobsDev, host.data(), numJobs * sizeof(BatchJobDev), cudaMemcpyHostToDevice));
    SB_CUDA_TRY(cudaMemcpy(b->prefixDev, prefix.data(), (numJobs + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice));
    b->descs.assign(jobs, jobs + numJobs);
    b->order = ord;
    b->jobsHost = host;
    b->prefix = prefix;
    b->total = (uint32_t)total;
    b->numKeys = numKeys;
    b->maxDepth = maxDepth;
    return STRELKA_OK;
}

extern "C" int strelka_batch_set_frame(StrelkaBatch* b, uint32_t frameOffset, void* stream)
{
    if (!b) return fail(STRELKA_ERR_INVALID_ARGUMENT, "batch is NULL");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // the job table is rewritten in place (the captured graphs keep its address)
    std::vector<BatchJobDev> host = b->jobsHost;
    for (size_t k = 0; k < host.size(); ++k)
        host[k].ubo.frameNumber = b->descs[b->order[k]].constants.frameNumber + frameOffset;
    if (host.empty()) return STRELKA_OK;
    SB_CUDA_TRY(cudaStreamSynchronize(st));
    SB_CUDA_TRY(cudaMemcpy(b->jobsDev, host.data(), host.size() * sizeof(BatchJobDev), cudaMemcpyHostToDevice));
    return STRELKA_OK;
}

extern "C" int strelka_batch_execute(StrelkaBatch* b, const StrelkaBatchConfig* config, void* stream)
{
    if (!b) return fail(STRELKA_ERR_INVALID_ARGUMENT, "batch is NULL");
    const StrelkaBatchConfig c = config ? *config : (b->haveTuned ? b->tuned : default_config(b));
    return run(b, c, static_cast<cudaStream_t>(stream));
}

extern "C" int strelka_batch_autotune(StrelkaBatch* b, uint32_t repeats, StrelkaBatchTuneEntry* entries, uint32_t capacity,
                                      uint32_t* numEntries, StrelkaBatchConfig* best, void* stream)
{
    if (!b) return fail(STRELKA_ERR_INVALID_ARGUMENT, "batch is NULL");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    repeats = std::max<uint32_t>(repeats, 1);
    cudaEvent_t e0, e1;
    SB_CUDA_TRY(cudaEventCreate(&e0));
    SB_CUDA_TRY(cudaEventCreate(&e1));
    std::map<uint64_t, float> measured;
    uint32_t n = 0;
    auto time_config = [&](const StrelkaBatchConfig& c, float& ms) -> int {
        const uint64_t key = config_key(c);
        auto it = measured.find(key);
        if (it != measured.end()) {
            ms = it->second;
            return STRELKA_OK;
        }
        int rc = run(b, c, st);  // warm-up (and graph capture)
        if (rc) return rc;
        std::vector<float> t(repeats);
        for (uint32_t r = 0; r < repeats; ++r) {
            SB_CUDA_TRY(cudaEventRecord(e0, st));
            rc = run(b, c, st);
            if (rc) return rc;
            SB_CUDA_TRY(cudaEventRecord(e1, st));
            SB_CUDA_TRY(cudaEventSynchronize(e1));
            SB_CUDA_TRY(cudaEventElapsedTime(&t[r], e0, e1));
        }
        std::sort(t.begin(), t.end());
        ms = t[repeats / 2];
        measured[key] = ms;
        if (entries && n < capacity) {
            entries[n].config = c;
            entries[n].ms = ms;
        }
        ++n;
        return STRELKA_OK;
    };
    // coordinate descent: mode, block size, queue chunk, material sort
    StrelkaBatchConfig cur = default_config(b);
    float curMs = 0.0f;
    int rc = time_config(cur, curMs);
    const uint32_t modes[] = {STRELKA_BATCH_PERSISTENT, STRELKA_BATCH_WAVEFRONT};
    const uint32_t blocks[] = {64, 128, 256};
    const uint32_t chunks[] = {32, 64, 128, 256, 512, 1024};
    auto consider = [&](StrelkaBatchConfig c) -> int {
        if (check_config(b, c) != STRELKA_OK) return STRELKA_OK;
        float ms = 0.0f;
        int r = time_config(c, ms);
        if (r) return r;
        if (ms < curMs) {
            cur = c;
            curMs = ms;
        }
        return STRELKA_OK;
    };
    for (uint32_t m : modes) {
        if (rc) break;
        StrelkaBatchConfig c = cur;
        c.mode = m;
        if (m != STRELKA_BATCH_WAVEFRONT) c.materialSort = 0;
        rc = consider(c);
    }
    for (uint32_t v : blocks) {
        if (rc) break;
        StrelkaBatchConfig c = cur;
        c.blockSize = v;
        rc = consider(c);
    }
    for (uint32_t v : chunks) {
        if (rc) break;
        StrelkaBatchConfig c = cur;
        c.queueChunk = v;
        rc = consider(c);
    }
    if (!rc && cur.mode == STRELKA_BATCH_WAVEFRONT) {
        for (uint32_t v : {0u, 1u}) {
            if (rc) break;
            StrelkaBatchConfig c = cur;
            c.materialSort = v;
            rc = consider(c);
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return rc;
    b->tuned = cur;
    b->haveTuned = true;
    if (best) *best = cur;
    if (numEntries) *numEntries = n;
    return STRELKA_OK;
}

extern "C" int strelka_batch_job_latency(StrelkaBatch* b, void* stream, float* ms, uint32_t capacity)
{
    if (!b) return fail(STRELKA_ERR_INVALID_ARGUMENT, "batch is NULL");
    SB_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    BatchCtl c;
    SB_CUDA_TRY(cudaMemcpy(&c, b->ctl, sizeof(c), cudaMemcpyDeviceToHost));
    const uint32_t n = (uint32_t)b->jobsHost.size();
    for (uint32_t k = 0; k < n; ++k) {
        const uint32_t j = b->order[k];  // the caller's index of slot k
        if (j >= capacity) continue;
        if (b->jobsHost[k].numPaths == 0) ms[j] = 0.0f;
        else if (c.tDone[k] == 0 || c.tDone[k] < c.tStart) ms[j] = -1.0f;
        else ms[j] = (float)((double)(c.tDone[k] - c.tStart) * 1e-6);
    }
    return (int)n;
}

extern "C" int strelka_batch_get_device_status(StrelkaBatch* b, void* stream, uint32_t* status)
{
    if (!b || !status) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    SB_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    SB_CUDA_TRY(cudaMemcpy(status, b->status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    SB_CUDA_TRY(cudaMemset(b->status, 0, sizeof(uint32_t)));
    return STRELKA_OK;
}

extern "C" int strelka_batch_info(StrelkaBatch* b, uint64_t* totalPaths, uint32_t* numJobs, uint32_t* numSortKeys)
{
    if (!b) return fail(STRELKA_ERR_INVALID_ARGUMENT, "batch is NULL");
    if (totalPaths) *totalPaths = b->total;
    if (numJobs) *numJobs = (uint32_t)b->jobsHost.size();
    if (numSortKeys) *numSortKeys = b->numKeys;
    return STRELKA_OK;
}
