// nrc.cu — online-trained neural radiance cache: multiresolution hash-grid
// encoding + a fully fused 64-wide MLP on FP16 tensor cores (FP32
// accumulation), forward and backward, with Adam.
//
// The cache predicts the outgoing radiance at a path vertex from its
// position (16-level hash grid, 2 features per level, 2^19 entries per
// level, growth 1.5; Müller et al. 2022), direction (real spherical
// harmonics of degree 4, 16 coefficients), shading normal and roughness.
// The network is 64 inputs -> 4 hidden layers of 64 (ReLU) -> 3 outputs
// (linear), no biases (a constant-1 input stands in), trained with the
// relative L2 loss (y - t)^2 / (sg(y)^2 + 0.01) (Müller et al. 2021).
//
// Both directions run on the tcgen05 tensor cores with 128-record tiles:
// inference (k_nrc_infer) keeps activations in tensor memory between
// layers; training (k_nrc_train) keeps them in shared memory, where the
// tensor core reads them for the forward pass and, transposed, for the
// weight gradients.  Details at each kernel.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <random>
#include <vector>

#include "common.h"
#include "nrc.h"
#include "tc.cuh"

namespace {

using sb::fail;
namespace tc = sb::tc;

constexpr int kLevels = 16;
constexpr int kIn = 64;
constexpr int kWidth = 64;
constexpr int kOutPad = 16;
constexpr int kMatRows = 4 * kWidth + kOutPad; // 272 rows: W0..W3 (64 each), W4 (16)
constexpr int kParams = 4 * kWidth * kIn + kOutPad * kWidth;  // 17408
constexpr float kGradScale = 1.0f / 128.0f;    // loss-gradient scale (FP16 range)
constexpr float kGradClamp = 1024.0f;          // |dL/dy| clamp before scaling

struct NrcGeom {
    float bmin[3];
    float binv[3];
    uint32_t T;      // entries per level (power of two)
    int res[kLevels];
    int dense[kLevels];
};

// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t pack2(float x, float y)
{
    __half2 h = __floats2half2_rn(x, y);
    return *reinterpret_cast<uint32_t*>(&h);
}
// ---------------------------------------------------------------------------
// Encoding.  Position -> [0,1]^3 by the scene box; level l has resolution
// res_l = floor(16 * 1.5^l); dense indexing when (res_l+1)^3 fits the table,
// otherwise the spatial hash (x * 1) ^ (y * 2654435761) ^ (z * 805459861).
struct Corner {
    uint32_t idx[8];
    float w[8];
};

__device__ __forceinline__ void level_corners(const NrcGeom& g, int l, float px, float py, float pz, Corner& c)
{
    const int res = g.res[l];
    const float x = px * (float)res, y = py * (float)res, z = pz * (float)res;
    int ix = (int)floorf(x), iy = (int)floorf(y), iz = (int)floorf(z);
    ix = ix < 0 ? 0 : (ix > res - 1 ? res - 1 : ix);
    iy = iy < 0 ? 0 : (iy > res - 1 ? res - 1 : iy);
    iz = iz < 0 ? 0 : (iz > res - 1 ? res - 1 : iz);
    const float fx = fminf(fmaxf(x - (float)ix, 0.0f), 1.0f);
    const float fy = fminf(fmaxf(y - (float)iy, 0.0f), 1.0f);
    const float fz = fminf(fmaxf(z - (float)iz, 0.0f), 1.0f);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const uint32_t cx = (uint32_t)(ix + (k & 1)), cy = (uint32_t)(iy + ((k >> 1) & 1)), cz = (uint32_t)(iz + (k >> 2));
        uint32_t idx;
        if (g.dense[l]) {
            const uint32_t s = (uint32_t)res + 1u;
            idx = cx + s * (cy + s * cz);
        } else {
            idx = (cx * 1u) ^ (cy * 2654435761u) ^ (cz * 805459861u);
        }
        c.idx[k] = (idx & (g.T - 1u)) + (uint32_t)l * g.T;
        c.w[k] = ((k & 1) ? fx : 1.0f - fx) * (((k >> 1) & 1) ? fy : 1.0f - fy) * ((k >> 2) ? fz : 1.0f - fz);
    }
}

__device__ __forceinline__ void normalized_position(const NrcGeom& g, const StrelkaNrcRecord& r, float& px, float& py,
                                                    float& pz)
{
    px = fminf(fmaxf((r.pos[0] - g.bmin[0]) * g.binv[0], 0.0f), 1.0f);
    py = fminf(fmaxf((r.pos[1] - g.bmin[1]) * g.binv[1], 0.0f), 1.0f);
    pz = fminf(fmaxf((r.pos[2] - g.bmin[2]) * g.binv[2], 0.0f), 1.0f);
}

// Real spherical harmonics, bands 0..3 (normalisation sqrt((2l+1)/4pi (l-m)!/(l+m)!) with sqrt(2) for m != 0).
__device__ __forceinline__ void sh16(float x, float y, float z, float* o)
{
    const float c00 = 0.28209479177387814f, c1 = 0.4886025119029199f, c2m2 = 1.0925484305920792f,
                c20 = 0.31539156525252005f, c22 = 0.5462742152960396f, c3m3 = 0.5900435899266435f,
                c3m2 = 2.890611442640554f, c3m1 = 0.4570457994644658f, c30 = 0.3731763325901154f,
                c32 = 1.445305721320277f;
    const float xx = x * x, yy = y * y, zz = z * z;
    o[0] = c00;
    o[1] = -c1 * y;
    o[2] = c1 * z;
    o[3] = -c1 * x;
    o[4] = c2m2 * x * y;
    o[5] = -c2m2 * y * z;
    o[6] = c20 * (3.0f * zz - 1.0f);
    o[7] = -c2m2 * x * z;
    o[8] = c22 * (xx - yy);
    o[9] = -c3m3 * y * (3.0f * xx - yy);
    o[10] = c3m2 * x * y * z;
    o[11] = -c3m1 * y * (5.0f * zz - 1.0f);
    o[12] = c30 * z * (5.0f * zz - 3.0f);
    o[13] = -c3m1 * x * (5.0f * zz - 1.0f);
    o[14] = c32 * z * (xx - yy);
    o[15] = -c3m3 * x * (xx - 3.0f * yy);
}

// ---------------------------------------------------------------------------
// Inference on the tcgen05 tensor cores.  A CTA owns tiles of 128 records;
// record i of a tile lives in TMEM lane i.  Its two warpgroups both reach
// every lane (a warp addresses lanes 32*(warp % 4) .. +31) and split the
// work by columns: warpgroup 0 encodes grid levels 0..7 plus the direction /
// normal / roughness inputs, warpgroup 1 levels 8..15.  One thread issues
// each layer as four 128xNx16 MMAs (A = activations in TMEM, B = the layer's
// weights in shared memory, D = FP32 in TMEM).  Between layers each
// warpgroup reads its 32 columns of D, applies ReLU, rounds to FP16 and
// writes them back as its half of the next layer's A, so activations never
// leave tensor memory.
constexpr int kTcTile = 128;
constexpr int kTcThreads = 256;
constexpr int kTcBlocksPerSM = 3;  // resident CTAs per SM: the register bound of the launch bounds
constexpr uint32_t kTcLayerBytes = kWidth * kIn * 2;                      // 8192
constexpr uint32_t kTcWeightBytes = 4 * kTcLayerBytes + kOutPad * kIn * 2;  // 34816
constexpr uint32_t kTcColD = 0;     // accumulator, 64 columns
constexpr uint32_t kTcColA = 64;    // activations, 32 columns (64 halves)
constexpr uint32_t kTcCols = 128;   // TMEM columns per CTA
constexpr uint64_t kTcWaitNs = 1000000000ull;  // MMA completion wait limit (1 s)
// Shared memory per CTA: the weights, the mbarrier and the TMEM address.
constexpr uint32_t kTcSmem = kTcWeightBytes + 64;
// Shared-memory carveout (percent of the maximum), chosen so that at most
// three CTAs fit by shared memory (3 x 128 TMEM columns <= 512) and the L1
// keeps about half the SM's memory for the hash-grid gathers.
constexpr int kTcCarveoutPercent = 50;

// Byte offset of weight (row r, input k) in the K-major core-matrix layout:
// 8x8 blocks of 128 contiguous bytes, 128 B apart along K, 1024 B apart
// along the rows.
__device__ __forceinline__ uint32_t core_offset(int r, int k)
{
    return (uint32_t)((r >> 3) * 1024 + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Corner weights of level l and the 8 grid entries they blend (loads issued).
__device__ __forceinline__ void level_fetch(const NrcGeom& g, const __half2* __restrict__ grid, int l, float px, float py,
                                            float pz, float (&w)[8], uint32_t (&v)[8])
{
    Corner c;
    level_corners(g, l, px, py, pz, c);
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        w[k] = c.w[k];
        // grid entries are kept in L1 ahead of other lines: corners along x
        // often share a sector, and the coarse levels are reused across records
        uint32_t r;
        asm volatile("ld.global.nc.L1::evict_last.b32 %0, [%1];"
                     : "=r"(r)
                     : "l"(reinterpret_cast<const unsigned int*>(grid) + c.idx[k]));
        v[k] = r;
    }
}
// trilinear blend of one level's two features, as an FP16 pair
__device__ __forceinline__ uint32_t level_mix(const float (&w)[8], const uint32_t (&v)[8])
{
    float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const float2 x = __half22float2(*reinterpret_cast<const __half2*>(&v[k]));
        f0 += w[k] * x.x;
        f1 += w[k] * x.y;
    }
    return pack2(f0, f1);
}
// grid levels l0 .. l0+7 as 8 FP16 pairs
__device__ __forceinline__ void encode_levels8(const NrcGeom& g, const __half2* __restrict__ grid, int l0, float px,
                                               float py, float pz, uint32_t (&a)[8])
{
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        float w0[8];
        uint32_t v0[8];
        level_fetch(g, grid, l0 + i, px, py, pz, w0, v0);
        a[i] = level_mix(w0, v0);
    }
}
// inputs 32..63: 16 SH coefficients, normal, roughness, the constant 1, zeros
__device__ __forceinline__ void encode_rest(const StrelkaNrcRecord& rec, uint32_t (&a)[16])
{
    float sh[16];
    sh16(rec.dir[0], rec.dir[1], rec.dir[2], sh);
#pragma unroll
    for (int i = 0; i < 8; ++i) a[i] = pack2(sh[2 * i], sh[2 * i + 1]);
    a[8] = pack2(rec.normal[0] * 0.5f + 0.5f, rec.normal[1] * 0.5f + 0.5f);
    a[9] = pack2(rec.normal[2] * 0.5f + 0.5f, rec.roughness);
    a[10] = pack2(1.0f, 0.0f);
#pragma unroll
    for (int i = 11; i < 16; ++i) a[i] = 0u;
}

// ReLU + FP16 of 16 accumulator columns into 8 packed pairs
__device__ __forceinline__ void relu_pack16(const uint32_t* d, uint32_t* a)
{
#pragma unroll
    for (int j = 0; j < 8; ++j)
        a[j] = pack2(fmaxf(__uint_as_float(d[2 * j]), 0.0f), fmaxf(__uint_as_float(d[2 * j + 1]), 0.0f));
}

// y for every record.  out != NULL: out[3*i + c] = y_c; otherwise
// col[slot] += throughput * max(y, 0) (the throughput rides in target[]).
// A tensor-core wait that runs out sets STRELKA_DEV_MMA_TIMEOUT in *status
// and ends the CTA after releasing its TMEM.
__global__ void __launch_bounds__(kTcThreads, kTcBlocksPerSM) k_nrc_infer(const StrelkaNrcRecord* __restrict__ recs, const uint32_t* countPtr,
                                                             uint32_t maxN, const __half* __restrict__ w,
                                                             const __half2* __restrict__ grid, NrcGeom g,
                                                             float* __restrict__ out, float4* __restrict__ col,
                                                             uint32_t* __restrict__ status)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* sW = smem;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kTcWeightBytes);
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + kTcWeightBytes + 8);
    const int tid = threadIdx.x, warp = tid >> 5, wg = tid >> 7, row = tid & (kTcTile - 1);
    // W0..W3 (64 rows) and W4 (16 rows) into the core-matrix layout, 16 B at a time
    for (int i = tid; i < kMatRows * (kIn / 8); i += kTcThreads) {
        const int r0 = i >> 3, c = i & 7;
        const int layer = r0 < 4 * kWidth ? r0 / kWidth : 4;
        const int r = r0 - layer * kWidth;
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(w + (size_t)r0 * kIn + c * 8));
        *reinterpret_cast<uint4*>(sW + layer * kTcLayerBytes + core_offset(r, c * 8)) = v;
    }
    if (warp == 0) {
        tc::tmem_alloc(slot, kTcCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) tc::mbar_init(bar, 1);
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tb = *slot;
    const uint32_t lane = tb + ((uint32_t)((warp & 3) * 32) << 16);  // this warp's 32 TMEM lanes
    const uint32_t sW0 = tc::smem_u32(sW);
    const uint32_t n = countPtr ? min(*countPtr, maxN) : maxN;
    const uint32_t tiles = (n + kTcTile - 1) / kTcTile;
    uint32_t phase = 0;
    bool timedOut = false;
    for (uint32_t t = blockIdx.x; t < tiles; t += gridDim.x) {
        const uint32_t q = t * kTcTile + (uint32_t)row;
        {
            // (tcgen05.st is warp-collective: every lane reaches the same stores)
            uint32_t a[8], b[16];
            if (q < n) {
                const StrelkaNrcRecord& rec = recs[q];
                float px, py, pz;
                normalized_position(g, rec, px, py, pz);
                encode_levels8(g, grid, 8 * wg, px, py, pz, a);
                if (wg == 0) encode_rest(rec, b);
            } else {
#pragma unroll
                for (int i = 0; i < 8; ++i) a[i] = 0u;
#pragma unroll
                for (int i = 0; i < 16; ++i) b[i] = 0u;
            }
            if (wg == 0) tc::tmem_st16(lane + kTcColA + 16, b);
            tc::tmem_st8(lane + kTcColA + 8 * wg, a);
            tc::tmem_wait_st();
        }
        bool abort = false;
#pragma unroll 1
        for (int l = 0; l < 5; ++l) {
            // this layer's A is in TMEM; thread 0 issues the MMAs and alone
            // waits for them, the others sleep on the CTA barrier meanwhile
            tc::fence_before_sync();
            __syncthreads();
            if (tid == 0) {
                tc::fence_after_sync();
                const uint32_t idesc = l < 4 ? tc::idesc_f16_f32(kTcTile, kWidth) : tc::idesc_f16_f32(kTcTile, kOutPad);
#pragma unroll
                for (int kb = 0; kb < 4; ++kb)
                    tc::mma_f16_ts(tb + kTcColD, tb + kTcColA + 8 * kb,
                                   tc::smem_desc(sW0 + l * kTcLayerBytes + 256 * kb, 128, 1024), idesc, kb > 0);
                tc::mma_commit(bar);
                if (!tc::mbar_wait_bounded(bar, phase, kTcWaitNs)) timedOut = true;
            }
            phase ^= 1;
            if (__syncthreads_or(timedOut)) {
                abort = true;
                break;
            }
            tc::fence_after_sync();
            if (l < 4) {
                // this warpgroup's outputs 32*wg .. +31 become inputs 32*wg .. +31
                uint32_t d[32], a[16];
                tc::tmem_ld16(lane + kTcColD + 32 * wg, d);
                tc::tmem_ld16(lane + kTcColD + 32 * wg + 16, d + 16);
                tc::tmem_wait_ld();
                relu_pack16(d, a);
                relu_pack16(d + 16, a + 8);
                tc::tmem_st16(lane + kTcColA + 16 * wg, a);
                tc::tmem_wait_st();
            } else if (wg == 0) {
                uint32_t y[4];
                tc::tmem_ld4(lane + kTcColD, y);
                tc::tmem_wait_ld();
                if (q < n && !timedOut) {
                    const float y0 = __uint_as_float(y[0]), y1 = __uint_as_float(y[1]), y2 = __uint_as_float(y[2]);
                    if (out) {
                        out[3 * (size_t)q + 0] = y0;
                        out[3 * (size_t)q + 1] = y1;
                        out[3 * (size_t)q + 2] = y2;
                    } else {
                        const StrelkaNrcRecord& r = recs[q];
                        float* c = reinterpret_cast<float*>(&col[r.slot]);
                        c[0] += r.target[0] * fmaxf(y0, 0.0f);
                        c[1] += r.target[1] * fmaxf(y1, 0.0f);
                        c[2] += r.target[2] * fmaxf(y2, 0.0f);
                    }
                }
            }
        }
        if (abort) break;
    }
    if (timedOut) atomicOr(status, STRELKA_DEV_MMA_TIMEOUT);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tb, kTcCols);
    }
}

// ---------------------------------------------------------------------------
// Training on the tcgen05 tensor cores: forward + backward for every record,
// summing weight gradients (dW, kParams floats), hash-grid gradients
// (gridGrad) and the loss; gradients are of sum_i loss_i scaled by
// kGradScale.
//
// A CTA of 512 threads (four warpgroups) owns tiles of 128 records, record i
// of a tile in TMEM lane i and in row i of the shared-memory operands.
// Warpgroup g encodes grid levels 4g..4g+3 (warpgroup 0 also the direction /
// normal / roughness inputs) and handles accumulator columns 16g..16g+15 in
// every epilogue.  All operands are in shared memory in one core-matrix
// layout, (row, col) at (row/8)*1024 + (col/8)*128 + (row%8)*16 + (col%8)*2
// bytes, which the tensor core reads either way round: as a K-major
// [rows x K = cols] operand (LBO 128, SBO 1024) or as an MN-major
// [MN = cols x K = rows] operand (LBO 1024, SBO 128).  So:
//   forward   h_{l+1} = relu(h_l W_l^T): A = h_l (K-major), B = W_l (K-major);
//   input gradient d_in = d_l W_l: A = d_l (K-major), B = W_l as MN-major;
//   weight gradient dW_l += d_l^T h_l over the tile's 128 records (M = 64):
//     A = d_l as MN-major, B = h_l as MN-major.
// The five weight-gradient accumulators stay in TMEM for the CTA's lifetime
// and are added to dW once at the end.  Waits are bounded as in inference.
constexpr int kTrThreads = 512;
constexpr uint32_t kTrActBytes = kTcTile * kIn * 2;  // one 128 x 64 FP16 operand, 16 KB
constexpr uint32_t kTrActOff = kTcWeightBytes;      // x, h1..h4
constexpr uint32_t kTrDOff = kTrActOff + 5 * kTrActBytes;
constexpr uint32_t kTrBarOff = kTrDOff + kTrActBytes;
constexpr uint32_t kTrSmem = kTrBarOff + 64;        // 130 KB: one CTA per SM
constexpr uint32_t kTrCols = 512;                   // TMEM: D (64) + dW_0..dW_4 (64 each)
constexpr uint32_t kTrColW = 64;

__device__ __forceinline__ void st_chunk(unsigned char* buf, int row, int chunk, const uint32_t* v)
{
    *reinterpret_cast<uint4*>(buf + core_offset(row, 8 * chunk)) = make_uint4(v[0], v[1], v[2], v[3]);
}
__device__ __forceinline__ uint4 ld_chunk(const unsigned char* buf, int row, int chunk)
{
    return *reinterpret_cast<const uint4*>(buf + core_offset(row, 8 * chunk));
}

// grid levels l0 .. l0+3 as 4 FP16 pairs
__device__ __forceinline__ void encode_levels4(const NrcGeom& g, const __half2* __restrict__ grid, int l0, float px,
                                               float py, float pz, uint32_t (&a)[4])
{
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        float w0[8];
        uint32_t v0[8];
        level_fetch(g, grid, l0 + i, px, py, pz, w0, v0);
        a[i] = level_mix(w0, v0);
    }
}

__global__ void __launch_bounds__(kTrThreads, 1) k_nrc_train(const StrelkaNrcRecord* __restrict__ recs, const uint32_t* countPtr,
                                                             uint32_t maxN, const __half* __restrict__ w,
                                                             const __half2* __restrict__ grid, NrcGeom g,
                                                             float* __restrict__ dW, float* __restrict__ gridGrad,
                                                             float* __restrict__ lossSum, uint32_t* __restrict__ status)
{
    extern __shared__ __align__(1024) unsigned char smem[];
    unsigned char* sW = smem;
    unsigned char* sAct = smem + kTrActOff;
    unsigned char* sD = smem + kTrDOff;
    uint64_t* bar = reinterpret_cast<uint64_t*>(smem + kTrBarOff);
    uint32_t* slot = reinterpret_cast<uint32_t*>(smem + kTrBarOff + 8);
    const int tid = threadIdx.x, warp = tid >> 5, wg = tid >> 7, row = tid & (kTcTile - 1);
    for (int i = tid; i < kMatRows * (kIn / 8); i += kTrThreads) {
        const int r0 = i >> 3, c = i & 7;
        const int layer = r0 < 4 * kWidth ? r0 / kWidth : 4;
        const int r = r0 - layer * kWidth;
        const uint4 v = __ldg(reinterpret_cast<const uint4*>(w + (size_t)r0 * kIn + c * 8));
        *reinterpret_cast<uint4*>(sW + layer * kTcLayerBytes + core_offset(r, c * 8)) = v;
    }
    if (warp == 0) {
        tc::tmem_alloc(slot, kTrCols);
        tc::tmem_relinquish();
    }
    if (tid == 0) tc::mbar_init(bar, 1);
    tc::fence_proxy_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    const uint32_t tb = *slot;
    const uint32_t lane = tb + ((uint32_t)((warp & 3) * 32) << 16);
    const uint32_t sW0 = tc::smem_u32(sW), sA0 = tc::smem_u32(sAct), sD0 = tc::smem_u32(sD);
    const uint32_t n = countPtr ? min(*countPtr, maxN) : maxN;
    const uint32_t tiles = (n + kTcTile - 1) / kTcTile;
    uint32_t phase = 0;
    bool timedOut = false, abort = false;
    float lossAcc = 0.0f;
    // one MMA batch: thread 0 waits for it, the others sleep on the barrier
    auto run = [&](auto issue) -> bool {
        tc::fence_before_sync();
        __syncthreads();
        if (tid == 0) {
            tc::fence_after_sync();
            issue();
            tc::mma_commit(bar);
            if (!tc::mbar_wait_bounded(bar, phase, kTcWaitNs)) timedOut = true;
        }
        phase ^= 1;
        const bool bad = __syncthreads_or(timedOut);
        tc::fence_after_sync();
        return !bad;
    };
    for (uint32_t t = blockIdx.x; t < tiles && !abort; t += gridDim.x) {
        const bool firstTile = t == blockIdx.x;
        const uint32_t q = t * kTcTile + (uint32_t)row;
        const bool valid = q < n;
        float px = 0.0f, py = 0.0f, pz = 0.0f;
        // ---- encode: x into sAct[0] ----
        {
            uint32_t a[4] = {0u, 0u, 0u, 0u};
            if (valid) {
                normalized_position(g, recs[q], px, py, pz);
                encode_levels4(g, grid, 4 * wg, px, py, pz, a);
            }
            st_chunk(sAct, row, wg, a);
            if (wg == 0) {
                uint32_t b[16];
                if (valid) {
                    encode_rest(recs[q], b);
                } else {
#pragma unroll
                    for (int i = 0; i < 16; ++i) b[i] = 0u;
                }
#pragma unroll
                for (int c = 0; c < 4; ++c) st_chunk(sAct, row, 4 + c, b + 4 * c);
            }
            tc::fence_proxy_async_smem();
        }
        // ---- forward ----
        for (int l = 0; l < 5 && !abort; ++l) {
            const bool ok = run([&] {
                const uint32_t idesc = l < 4 ? tc::idesc_f16_f32(kTcTile, kWidth) : tc::idesc_f16_f32(kTcTile, kOutPad);
#pragma unroll
                for (int kb = 0; kb < 4; ++kb)
                    tc::mma_f16_ss(tb + kTcColD, tc::smem_desc(sA0 + l * kTrActBytes + 256 * kb, 128, 1024),
                                   tc::smem_desc(sW0 + l * kTcLayerBytes + 256 * kb, 128, 1024), idesc, kb > 0);
            });
            if (!ok) {
                abort = true;
                break;
            }
            if (l < 4) {
                uint32_t d[16], a[8];
                tc::tmem_ld16(lane + kTcColD + 16 * wg, d);
                tc::tmem_wait_ld();
                relu_pack16(d, a);
                st_chunk(sAct + (l + 1) * kTrActBytes, row, 2 * wg, a);
                st_chunk(sAct + (l + 1) * kTrActBytes, row, 2 * wg + 1, a + 4);
                tc::fence_proxy_async_smem();
            } else if (wg == 0) {
                // dL/dy of the relative L2 loss, clamped and scaled, as row q of d_4
                uint32_t y[4];
                tc::tmem_ld4(lane + kTcColD, y);
                tc::tmem_wait_ld();
                float gv[3] = {0.0f, 0.0f, 0.0f};
                if (valid) {
#pragma unroll
                    for (int c = 0; c < 3; ++c) {
                        const float yy = __uint_as_float(y[c]);
                        const float tt = recs[q].target[c];
                        const float den = yy * yy + 0.01f;
                        const float diff = yy - tt;
                        lossAcc += diff * diff / den;
                        gv[c] = fminf(fmaxf(2.0f * diff / den, -kGradClamp), kGradClamp) * kGradScale;
                    }
                }
                const uint32_t c0[4] = {pack2(gv[0], gv[1]), pack2(gv[2], 0.0f), 0u, 0u};
                const uint32_t z[4] = {0u, 0u, 0u, 0u};
                st_chunk(sD, row, 0, c0);
#pragma unroll
                for (int c = 1; c < 8; ++c) st_chunk(sD, row, c, z);
                tc::fence_proxy_async_smem();
            }
        }
        // ---- backward through W4 .. W0 ----
        for (int l = 4; l >= 0 && !abort; --l) {
            const bool ok = run([&] {
                // dW_l += d_l^T h_l: M = 64 outputs, N = 64 inputs, K = the 128 records
#pragma unroll
                for (int ks = 0; ks < 8; ++ks)
                    tc::mma_f16_ss(tb + kTrColW + 64 * l, tc::smem_desc(sD0 + 2048 * ks, 1024, 128),
                                   tc::smem_desc(sA0 + l * kTrActBytes + 2048 * ks, 1024, 128),
                                   tc::idesc_f16_f32(64, kIn, true, true), (!firstTile || ks > 0) ? 1u : 0u);
                // d_in = d_l W_l: M = 128 records, N = 64 inputs, K = the layer's outputs
                const int ksteps = l == 4 ? kOutPad / 16 : kWidth / 16;
                for (int kb = 0; kb < ksteps; ++kb)
                    tc::mma_f16_ss(tb + kTcColD, tc::smem_desc(sD0 + 256 * kb, 128, 1024),
                                   tc::smem_desc(sW0 + l * kTcLayerBytes + 2048 * kb, 1024, 128),
                                   tc::idesc_f16_f32(kTcTile, kIn, false, true), kb > 0 ? 1u : 0u);
            });
            if (!ok) {
                abort = true;
                break;
            }
            if (l > 0) {
                // ReLU mask of this layer's input (h_l > 0), FP16 into d_{l-1}
                uint32_t d[16], a[8];
                tc::tmem_ld16(lane + kTcColD + 16 * wg, d);
                tc::tmem_wait_ld();
                const unsigned char* hl = sAct + l * kTrActBytes;
#pragma unroll
                for (int c = 0; c < 2; ++c) {
                    const uint4 hv = ld_chunk(hl, row, 2 * wg + c);
                    const uint32_t hw[4] = {hv.x, hv.y, hv.z, hv.w};
#pragma unroll
                    for (int j = 0; j < 4; ++j) {
                        const float2 h2 = __half22float2(*reinterpret_cast<const __half2*>(&hw[j]));
                        const float g0 = h2.x > 0.0f ? __uint_as_float(d[8 * c + 2 * j]) : 0.0f;
                        const float g1 = h2.y > 0.0f ? __uint_as_float(d[8 * c + 2 * j + 1]) : 0.0f;
                        a[4 * c + j] = pack2(g0, g1);
                    }
                }
                st_chunk(sD, row, 2 * wg, a);
                st_chunk(sD, row, 2 * wg + 1, a + 4);
                tc::fence_proxy_async_smem();
            } else {
                // gradients of this warpgroup's grid features (levels 4g..4g+3),
                // scattered through the trilinear weights
                uint32_t d[8];
                tc::tmem_ld8(lane + kTcColD + 8 * wg, d);
                tc::tmem_wait_ld();
                if (valid) {
#pragma unroll
                    for (int i = 0; i < 4; ++i) {
                        Corner c;
                        level_corners(g, 4 * wg + i, px, py, pz, c);
                        const float g0 = __uint_as_float(d[2 * i]), g1 = __uint_as_float(d[2 * i + 1]);
#pragma unroll
                        for (int k = 0; k < 8; ++k)
                            atomicAdd(reinterpret_cast<float2*>(gridGrad) + c.idx[k], make_float2(c.w[k] * g0, c.w[k] * g1));
                    }
                }
            }
        }
    }
    // loss, and the weight gradients accumulated in TMEM (row r of an M = 64
    // accumulator sits in lane (r % 16) + 32 (r / 16))
    for (int off = 16; off > 0; off >>= 1) lossAcc += __shfl_xor_sync(0xffffffffu, lossAcc, off);
    if ((tid & 31) == 0 && lossSum && lossAcc != 0.0f) atomicAdd(lossSum, lossAcc);
    tc::fence_before_sync();
    __syncthreads();
    tc::fence_after_sync();
    if (blockIdx.x < tiles && !abort) {
        const int sub = warp & 3;
        for (int l = warp >> 2; l < 5; l += kTrThreads / 128) {
            const int rows = l == 4 ? kOutPad : kWidth;
            const int r = 16 * sub + (tid & 15);
            for (int c0 = 0; c0 < kIn; c0 += 16) {
                uint32_t d[16];
                tc::tmem_ld16(tb + ((uint32_t)(sub * 32) << 16) + kTrColW + 64 * l + c0, d);
                tc::tmem_wait_ld();
                if ((tid & 31) < 16 && r < rows) {
                    float* dst = dW + (size_t)l * kWidth * kIn + (size_t)r * kIn + c0;
#pragma unroll
                    for (int c = 0; c < 16; ++c) {
                        const float v = __uint_as_float(d[c]);
                        if (v != 0.0f) atomicAdd(dst + c, v);
                    }
                }
            }
        }
    }
    if (timedOut) atomicOr(status, STRELKA_DEV_MMA_TIMEOUT);
    tc::fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tc::fence_after_sync();
        tc::tmem_dealloc(tb, kTrCols);
    }
}

__global__ void k_nrc_adam(float* __restrict__ p, float* __restrict__ m, float* __restrict__ v, const float* __restrict__ grad,
                           __half* __restrict__ ph, size_t n, float lr, float gscale, float b1, float b2, float eps,
                           float c1, float c2, const uint32_t* countPtr)
{
    if (countPtr) gscale = 1.0f / (kGradScale * fmaxf((float)*countPtr, 1.0f) * 3.0f);
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        const float gr = grad[i] * gscale;
        const float mi = b1 * m[i] + (1.0f - b1) * gr;
        const float vi = b2 * v[i] + (1.0f - b2) * gr * gr;
        m[i] = mi;
        v[i] = vi;
        const float pi = p[i] - lr * (mi / c1) / (sqrtf(vi / c2) + eps);
        p[i] = pi;
        ph[i] = __float2half(pi);
    }
}

__global__ void k_to_half(const float* __restrict__ p, __half* __restrict__ ph, size_t n)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        ph[i] = __float2half(p[i]);
}


}  // namespace

struct StrelkaNrc {
    StrelkaNrcConfig cfg{};
    NrcGeom geom{};
    int numSMs = 148;
    size_t gridN = 0;  // halves in the grid (levels * T * 2)
    float* mlp = nullptr;
    float* mlpM = nullptr;
    float* mlpV = nullptr;
    float* mlpGrad = nullptr;
    __half* mlpHalf = nullptr;
    float* grid = nullptr;
    float* gridM = nullptr;
    float* gridV = nullptr;
    float* gridGrad = nullptr;
    __half* gridHalf = nullptr;
    float* loss = nullptr;
    uint32_t* status = nullptr;  // device status word (STRELKA_DEV_* bits)
    uint64_t step = 0;
};

namespace {
void nrc_free(StrelkaNrc* n)
{
    void* ptrs[] = {n->mlp, n->mlpM, n->mlpV, n->mlpGrad, n->mlpHalf, n->grid, n->gridM, n->gridV, n->gridGrad,
                    n->gridHalf, n->loss, n->status};
    for (void* p : ptrs)
        if (p) cudaFree(p);
}
int grid_blocks(StrelkaNrc* nrc, size_t n, int block)
{
    size_t b = (n + block - 1) / block;
    size_t cap = (size_t)nrc->numSMs * 16;
    return (int)std::max<size_t>(1, std::min(b, cap));
}
}  // namespace

extern "C" int strelka_nrc_create(const StrelkaNrcConfig* cfg, StrelkaNrc** out)
{
    if (!cfg || !out) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (cfg->log2TableSize < 8 || cfg->log2TableSize > 24)
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "log2TableSize must be in [8, 24]");
    auto* nrc = new StrelkaNrc();
    nrc->cfg = *cfg;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nrc->numSMs, cudaDevAttrMultiProcessorCount, dev);
    NrcGeom& g = nrc->geom;
    for (int a = 0; a < 3; ++a) {
        g.bmin[a] = cfg->sceneMin[a];
        float ext = cfg->sceneMax[a] - cfg->sceneMin[a];
        g.binv[a] = ext > 0 ? 1.0f / ext : 0.0f;
    }
    g.T = 1u << cfg->log2TableSize;
    for (int l = 0; l < kLevels; ++l) {
        // res_l = floor(16 * 1.5^l)
        g.res[l] = (int)std::floor(16.0 * std::pow(1.5, (double)l));
        const double cells = std::pow((double)g.res[l] + 1.0, 3.0);
        g.dense[l] = cells <= (double)g.T ? 1 : 0;
    }
    nrc->gridN = (size_t)kLevels * g.T * 2;
    bool ok = cudaMalloc(&nrc->mlp, kParams * 4) == cudaSuccess && cudaMalloc(&nrc->mlpM, kParams * 4) == cudaSuccess &&
              cudaMalloc(&nrc->mlpV, kParams * 4) == cudaSuccess && cudaMalloc(&nrc->mlpGrad, kParams * 4) == cudaSuccess &&
              cudaMalloc(&nrc->mlpHalf, kParams * 2) == cudaSuccess &&
              cudaMalloc(&nrc->grid, nrc->gridN * 4) == cudaSuccess && cudaMalloc(&nrc->gridM, nrc->gridN * 4) == cudaSuccess &&
              cudaMalloc(&nrc->gridV, nrc->gridN * 4) == cudaSuccess &&
              cudaMalloc(&nrc->gridGrad, nrc->gridN * 4) == cudaSuccess &&
              cudaMalloc(&nrc->gridHalf, nrc->gridN * 2) == cudaSuccess && cudaMalloc(&nrc->loss, 4) == cudaSuccess &&
              cudaMalloc(&nrc->status, 4) == cudaSuccess;
    if (!ok) {
        nrc_free(nrc);
        delete nrc;
        return fail(STRELKA_ERR_OUT_OF_MEMORY, "cudaMalloc failed for the radiance cache");
    }
    // initial parameters: uniform +-sqrt(6/(fan_in+fan_out)) weights, +-1e-4 grid
    std::mt19937_64 rng(cfg->seed);
    auto u01 = [&]() { return (double)(rng() >> 11) * (1.0 / 9007199254740992.0); };
    std::vector<float> w(kParams);
    for (int l = 0; l < 5; ++l) {
        const int rows = l == 4 ? kOutPad : kWidth;
        const int fanOut = l == 4 ? 3 : kWidth;
        const double s = std::sqrt(6.0 / (double)(kIn + fanOut));
        for (int r = 0; r < rows; ++r)
            for (int c = 0; c < kIn; ++c) {
                float v = (float)((2.0 * u01() - 1.0) * s);
                if (l == 4 && r >= 3) v = 0.0f;  // padded outputs
                w[(size_t)l * kWidth * kIn + (size_t)r * kIn + c] = v;
            }
    }
    std::vector<float> gr(nrc->gridN);
    for (auto& v : gr) v = (float)((2.0 * u01() - 1.0) * 1e-4);
    cudaMemcpy(nrc->mlp, w.data(), kParams * 4, cudaMemcpyHostToDevice);
    cudaMemcpy(nrc->grid, gr.data(), nrc->gridN * 4, cudaMemcpyHostToDevice);
    cudaMemset(nrc->status, 0, 4);
    cudaMemset(nrc->mlpM, 0, kParams * 4);
    cudaMemset(nrc->mlpV, 0, kParams * 4);
    cudaMemset(nrc->gridM, 0, nrc->gridN * 4);
    cudaMemset(nrc->gridV, 0, nrc->gridN * 4);
    k_to_half<<<64, 256>>>(nrc->mlp, nrc->mlpHalf, kParams);
    k_to_half<<<grid_blocks(nrc, nrc->gridN, 256), 256>>>(nrc->grid, nrc->gridHalf, nrc->gridN);
    cudaFuncSetAttribute(k_nrc_infer, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem);
    cudaFuncSetAttribute(k_nrc_infer, cudaFuncAttributePreferredSharedMemoryCarveout, kTcCarveoutPercent);
    cudaFuncSetAttribute(k_nrc_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrSmem);
    cudaFuncSetAttribute(k_nrc_train, cudaFuncAttributePreferredSharedMemoryCarveout, kTcCarveoutPercent);
    cudaError_t e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        nrc_free(nrc);
        delete nrc;
        return sb::cuda_fail(e, "radiance cache initialisation");
    }
    *out = nrc;
    return STRELKA_OK;
}

extern "C" int strelka_nrc_destroy(StrelkaNrc* nrc)
{
    if (!nrc) return STRELKA_OK;
    nrc_free(nrc);
    delete nrc;
    return STRELKA_OK;
}

// internal entry points shared with the path tracer (device-side counts)
int nrc_infer_device(StrelkaNrc* nrc, const StrelkaNrcRecord* recs, const uint32_t* countPtr, uint32_t maxN, float* out,
                     float4* col, uint32_t* status, cudaStream_t st)
{
    if (maxN == 0) return STRELKA_OK;
    const int tiles = (int)((maxN + kTcTile - 1) / kTcTile);
    const int blocks = std::max(1, std::min(tiles, nrc->numSMs * kTcBlocksPerSM));
    k_nrc_infer<<<blocks, kTcThreads, kTcSmem, st>>>(recs, countPtr, maxN, nrc->mlpHalf,
                                                 reinterpret_cast<const __half2*>(nrc->gridHalf), nrc->geom, out, col,
                                                 status ? status : nrc->status);
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}

int nrc_gradients_device(StrelkaNrc* nrc, const StrelkaNrcRecord* recs, const uint32_t* countPtr, uint32_t maxN,
                         cudaStream_t st)
{
    SB_CUDA_TRY(cudaMemsetAsync(nrc->mlpGrad, 0, kParams * 4, st));
    SB_CUDA_TRY(cudaMemsetAsync(nrc->gridGrad, 0, nrc->gridN * 4, st));
    SB_CUDA_TRY(cudaMemsetAsync(nrc->loss, 0, 4, st));
    if (maxN == 0) return STRELKA_OK;
    const int tiles = (int)((maxN + kTcTile - 1) / kTcTile);
    const int blocks = std::max(1, std::min(tiles, nrc->numSMs));
    k_nrc_train<<<blocks, kTrThreads, kTrSmem, st>>>(recs, countPtr, maxN, nrc->mlpHalf,
                                                    reinterpret_cast<const __half2*>(nrc->gridHalf), nrc->geom,
                                                    nrc->mlpGrad, nrc->gridGrad, nrc->loss, nrc->status);
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}

int nrc_adam_device(StrelkaNrc* nrc, float batch, cudaStream_t st) { return nrc_adam_device_count(nrc, batch, nullptr, st); }

int nrc_adam_device_count(StrelkaNrc* nrc, float batch, const uint32_t* countPtr, cudaStream_t st)
{
    const float b1 = 0.9f, b2 = 0.99f, eps = 1e-8f;
    nrc->step += 1;
    const float c1 = 1.0f - (float)std::pow((double)b1, (double)nrc->step);
    const float c2 = 1.0f - (float)std::pow((double)b2, (double)nrc->step);
    // mean loss gradient: undo the FP16 scale, divide by the batch (x3 channels)
    const float gscale = 1.0f / (kGradScale * std::max(batch, 1.0f) * 3.0f);
    const float lr = nrc->cfg.learningRate;
    k_nrc_adam<<<64, 256, 0, st>>>(nrc->mlp, nrc->mlpM, nrc->mlpV, nrc->mlpGrad, nrc->mlpHalf, kParams, lr, gscale, b1,
                                   b2, eps, c1, c2, countPtr);
    k_nrc_adam<<<grid_blocks(nrc, nrc->gridN, 256), 256, 0, st>>>(nrc->grid, nrc->gridM, nrc->gridV, nrc->gridGrad,
                                                                  nrc->gridHalf, nrc->gridN, lr, gscale, b1, b2, eps, c1,
                                                                  c2, countPtr);
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}

extern "C" int strelka_nrc_infer(StrelkaNrc* nrc, const StrelkaNrcRecord* records, uint32_t n, float* outRGB, void* stream)
{
    if (!nrc || (n && (!records || !outRGB))) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    return nrc_infer_device(nrc, records, nullptr, n, outRGB, nullptr, nullptr, static_cast<cudaStream_t>(stream));
}

extern "C" int strelka_nrc_gradients(StrelkaNrc* nrc, const StrelkaNrcRecord* samples, uint32_t n, float* mlpGrad,
                                     float* gridGrad, float* lossSum, void* stream)
{
    if (!nrc || (n && !samples)) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = nrc_gradients_device(nrc, samples, nullptr, n, st);
    if (rc) return rc;
    // raw gradients of sum_i sum_c loss, undoing the FP16 scale
    const float inv = 1.0f / kGradScale;
    if (mlpGrad) {
        std::vector<float> h(kParams);
        SB_CUDA_TRY(cudaMemcpyAsync(h.data(), nrc->mlpGrad, kParams * 4, cudaMemcpyDeviceToHost, st));
        SB_CUDA_TRY(cudaStreamSynchronize(st));
        for (auto& v : h) v *= inv;
        memcpy(mlpGrad, h.data(), kParams * 4);
    }
    if (gridGrad) {
        std::vector<float> h(nrc->gridN);
        SB_CUDA_TRY(cudaMemcpyAsync(h.data(), nrc->gridGrad, nrc->gridN * 4, cudaMemcpyDeviceToHost, st));
        SB_CUDA_TRY(cudaStreamSynchronize(st));
        for (auto& v : h) v *= inv;
        memcpy(gridGrad, h.data(), nrc->gridN * 4);
    }
    if (lossSum) {
        SB_CUDA_TRY(cudaMemcpyAsync(lossSum, nrc->loss, 4, cudaMemcpyDeviceToHost, st));
        SB_CUDA_TRY(cudaStreamSynchronize(st));
    }
    return STRELKA_OK;
}

extern "C" int strelka_nrc_train(StrelkaNrc* nrc, const StrelkaNrcRecord* samples, uint32_t n, float* lossOut, void* stream)
{
    if (!nrc || (n && !samples)) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int rc = nrc_gradients_device(nrc, samples, nullptr, n, st);
    if (rc) return rc;
    rc = nrc_adam_device(nrc, (float)n, st);
    if (rc) return rc;
    if (lossOut) {
        SB_CUDA_TRY(cudaMemcpyAsync(lossOut, nrc->loss, 4, cudaMemcpyDeviceToHost, st));
        SB_CUDA_TRY(cudaStreamSynchronize(st));
        *lossOut /= (float)std::max<uint32_t>(n, 1) * 3.0f;
    }
    return STRELKA_OK;
}

extern "C" int strelka_nrc_get_params(StrelkaNrc* nrc, float* mlp, float* grid)
{
    if (!nrc) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    if (mlp) SB_CUDA_TRY(cudaMemcpy(mlp, nrc->mlp, kParams * 4, cudaMemcpyDeviceToHost));
    if (grid) SB_CUDA_TRY(cudaMemcpy(grid, nrc->grid, nrc->gridN * 4, cudaMemcpyDeviceToHost));
    return STRELKA_OK;
}

extern "C" int strelka_nrc_set_params(StrelkaNrc* nrc, const float* mlp, const float* grid)
{
    if (!nrc) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    if (mlp) {
        SB_CUDA_TRY(cudaMemcpy(nrc->mlp, mlp, kParams * 4, cudaMemcpyHostToDevice));
        k_to_half<<<64, 256>>>(nrc->mlp, nrc->mlpHalf, kParams);
    }
    if (grid) {
        SB_CUDA_TRY(cudaMemcpy(nrc->grid, grid, nrc->gridN * 4, cudaMemcpyHostToDevice));
        k_to_half<<<grid_blocks(nrc, nrc->gridN, 256), 256>>>(nrc->grid, nrc->gridHalf, nrc->gridN);
    }
    SB_CUDA_TRY(cudaDeviceSynchronize());
    return STRELKA_OK;
}

namespace {
// One thread waits, with the bounded wait of the tensor-core kernels, for the
// first phase of an mbarrier; unless `arrive`, nothing completes that phase.
__global__ void k_selftest_wait(uint64_t limitNs, int arrive, uint32_t* status)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        tc::mbar_init(&bar, 1);
        if (arrive) tc::mbar_arrive(&bar);
        if (!tc::mbar_wait_bounded(&bar, 0, limitNs)) atomicOr(status, STRELKA_DEV_MMA_TIMEOUT);
    }
}
}  // namespace

extern "C" int strelka_selftest_wait_timeout(uint64_t limitNs, int arrive, uint32_t* deviceStatus, void* stream)
{
    if (!deviceStatus) return fail(STRELKA_ERR_INVALID_ARGUMENT, "deviceStatus is NULL");
    if (limitNs > 1000000000ull) return fail(STRELKA_ERR_INVALID_ARGUMENT, "limitNs above 1 s");
    k_selftest_wait<<<1, 32, 0, static_cast<cudaStream_t>(stream)>>>(limitNs, arrive, deviceStatus);
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}

extern "C" int strelka_nrc_get_device_status(StrelkaNrc* nrc, void* stream, uint32_t* status)
{
    if (!nrc || !status) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    SB_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    SB_CUDA_TRY(cudaMemcpy(status, nrc->status, sizeof(uint32_t), cudaMemcpyDeviceToHost));
    SB_CUDA_TRY(cudaMemset(nrc->status, 0, sizeof(uint32_t)));
    return STRELKA_OK;
}

extern "C" int strelka_nrc_info(StrelkaNrc* nrc, uint32_t* numMlpParams, uint64_t* numGridParams, int32_t* levelRes)
{
    if (!nrc) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    if (numMlpParams) *numMlpParams = kParams;
    if (numGridParams) *numGridParams = nrc->gridN;
    if (levelRes)
        for (int l = 0; l < kLevels; ++l) levelRes[l] = nrc->geom.res[l] * (nrc->geom.dense[l] ? 1 : -1);
    return STRELKA_OK;
}
