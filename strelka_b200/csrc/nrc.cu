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
// Inference runs on the tcgen05 tensor cores (k_nrc_infer): 128-record
// tiles, activations resident in tensor memory between layers, weights read
// by the tensor core from shared memory (details at the kernel).
//
// Training (k_nrc_train) uses mma.sync m16n8k16: each warp owns a tile of 16
// records.  For a layer out = W * in, the 16x64 activation tile is the A
// operand (row-major) and W (out x in, row-major in shared memory with a
// 72-half row stride, which keeps the fragment loads bank-conflict free) is
// the column-major B operand; the m16n8k16 accumulator layout of one layer is
// exactly the A-fragment layout of the next layer's k-steps, so activations
// stay in registers between layers.  Backward uses the same instruction with
// W^T (fragments gathered from the same shared copy) and accumulates weight
// gradients d^T * a over each tile with a third mma shape, reduced in shared
// memory.
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
constexpr int kRow = 72;                       // shared-memory row stride (halves)
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
__device__ __forceinline__ void mma16816(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1)
{
    asm volatile(
        "mma.sync.aligned.m16n8k16.row.col.f32.f16.f16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, {%0,%1,%2,%3};\n"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}
__device__ __forceinline__ uint32_t pack2(float x, float y)
{
    __half2 h = __floats2half2_rn(x, y);
    return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ uint32_t pack2h(__half x, __half y)
{
    __half2 h = __halves2half2(x, y);
    return *reinterpret_cast<uint32_t*>(&h);
}
__device__ __forceinline__ uint32_t lds32(const __half* p) { return *reinterpret_cast<const uint32_t*>(p); }

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

// Encodes rows [0,16) of a tile into sx (16 x kRow halves): lane (r, half)
// handles row r = lane & 15 and levels 8*(lane >> 4) .. +7; lanes 0..15 also
// write the direction / normal / roughness / constant inputs.
__device__ __forceinline__ void encode_tile(const NrcGeom& g, const __half2* __restrict__ grid,
                                            const StrelkaNrcRecord* __restrict__ recs, uint32_t base, uint32_t n, __half* sx)
{
    const int lane = threadIdx.x & 31;
    const int r = lane & 15;
    const uint32_t q = base + (uint32_t)r;
    __half* row = sx + r * kRow;
    if (q >= n) {
        for (int c = (lane >> 4) * 32; c < (lane >> 4) * 32 + 32; ++c) row[c] = __float2half(0.0f);
        return;
    }
    const StrelkaNrcRecord rec = recs[q];
    float px, py, pz;
    normalized_position(g, rec, px, py, pz);
    const int l0 = (lane >> 4) * 8;
    for (int l = l0; l < l0 + 8; ++l) {
        Corner c;
        level_corners(g, l, px, py, pz, c);
        float f0 = 0.0f, f1 = 0.0f;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const float2 v = __half22float2(__ldg(&grid[c.idx[k]]));
            f0 += c.w[k] * v.x;
            f1 += c.w[k] * v.y;
        }
        row[2 * l] = __float2half(f0);
        row[2 * l + 1] = __float2half(f1);
    }
    if (lane < 16) {
        float sh[16];
        sh16(rec.dir[0], rec.dir[1], rec.dir[2], sh);
#pragma unroll
        for (int i = 0; i < 16; ++i) row[32 + i] = __float2half(sh[i]);
        row[48] = __float2half(rec.normal[0] * 0.5f + 0.5f);
        row[49] = __float2half(rec.normal[1] * 0.5f + 0.5f);
        row[50] = __float2half(rec.normal[2] * 0.5f + 0.5f);
        row[51] = __float2half(rec.roughness);
        row[52] = __float2half(1.0f);
#pragma unroll
        for (int i = 53; i < 64; ++i) row[i] = __float2half(0.0f);
    }
}

__device__ __forceinline__ void load_weights(const __half* __restrict__ w, __half* sW)
{
    for (int i = threadIdx.x; i < kMatRows * kIn; i += blockDim.x) {
        const int row = i / kIn, col = i - row * kIn;
        sW[row * kRow + col] = w[i];
    }
}

// A fragments of a 16 x 64 tile stored row-major (stride kRow) in shared memory.
__device__ __forceinline__ void load_a(const __half* s, uint32_t (&a)[4][4])
{
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        a[k][0] = lds32(s + gid * kRow + 16 * k + 2 * tig);
        a[k][1] = lds32(s + (gid + 8) * kRow + 16 * k + 2 * tig);
        a[k][2] = lds32(s + gid * kRow + 16 * k + 8 + 2 * tig);
        a[k][3] = lds32(s + (gid + 8) * kRow + 16 * k + 8 + 2 * tig);
    }
}

// acc[j] = (tile) * W^T for a 64x64 W at sW (out rows, in cols)
__device__ __forceinline__ void layer64(const __half* sWl, const uint32_t (&a)[4][4], float (&acc)[8][4])
{
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[j][0] = acc[j][1] = acc[j][2] = acc[j][3] = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const __half* wr = sWl + (8 * j + gid) * kRow + 16 * k + 2 * tig;
            mma16816(acc[j], a[k], lds32(wr), lds32(wr + 8));
        }
    }
}

// ReLU + FP16 of an accumulator tile, as the next layer's A fragments
__device__ __forceinline__ void relu_to_a(const float (&acc)[8][4], uint32_t (&a)[4][4])
{
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        a[k][0] = pack2(fmaxf(acc[2 * k][0], 0.0f), fmaxf(acc[2 * k][1], 0.0f));
        a[k][1] = pack2(fmaxf(acc[2 * k][2], 0.0f), fmaxf(acc[2 * k][3], 0.0f));
        a[k][2] = pack2(fmaxf(acc[2 * k + 1][0], 0.0f), fmaxf(acc[2 * k + 1][1], 0.0f));
        a[k][3] = pack2(fmaxf(acc[2 * k + 1][2], 0.0f), fmaxf(acc[2 * k + 1][3], 0.0f));
    }
}

// writes A fragments back as a row-major 16 x 64 tile
__device__ __forceinline__ void store_a(__half* s, const uint32_t (&a)[4][4])
{
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        *reinterpret_cast<uint32_t*>(s + gid * kRow + 16 * k + 2 * tig) = a[k][0];
        *reinterpret_cast<uint32_t*>(s + (gid + 8) * kRow + 16 * k + 2 * tig) = a[k][1];
        *reinterpret_cast<uint32_t*>(s + gid * kRow + 16 * k + 8 + 2 * tig) = a[k][2];
        *reinterpret_cast<uint32_t*>(s + (gid + 8) * kRow + 16 * k + 8 + 2 * tig) = a[k][3];
    }
}

// y = W4 * h4: first 8 outputs (n-tile 0; outputs 0..2 are used)
__device__ __forceinline__ void output_layer(const __half* sW4, const uint32_t (&a)[4][4], float (&y)[4])
{
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    y[0] = y[1] = y[2] = y[3] = 0.0f;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const __half* wr = sW4 + gid * kRow + 16 * k + 2 * tig;
        mma16816(y, a[k], lds32(wr), lds32(wr + 8));
    }
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
                                   tc::desc_kmajor(sW0 + l * kTcLayerBytes + 256 * kb, 128, 1024), idesc, kb > 0);
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
// Training: forward + backward for every record, summing weight gradients
// (dW, 17408 floats) and hash-grid gradients (gridGrad) and the loss.
// Gradients are of sum_i loss_i scaled by kGradScale.
__global__ void __launch_bounds__(256) k_nrc_train(const StrelkaNrcRecord* __restrict__ recs, const uint32_t* countPtr,
                                                   uint32_t maxN, const __half* __restrict__ w,
                                                   const __half2* __restrict__ grid, NrcGeom g, float* __restrict__ dW,
                                                   float* __restrict__ gridGrad, float* __restrict__ lossSum)
{
    extern __shared__ __align__(16) unsigned char smem[];
    __half* sW = reinterpret_cast<__half*>(smem);
    const int warp = threadIdx.x >> 5;
    __half* sAct = sW + kMatRows * kRow + warp * 5 * 16 * kRow;  // x, h1..h4
    __half* sD = sW + kMatRows * kRow + 8 * 5 * 16 * kRow + warp * 16 * kRow;
    float* sDW = reinterpret_cast<float*>(sW + kMatRows * kRow + 8 * 6 * 16 * kRow);
    load_weights(w, sW);
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) sDW[i] = 0.0f;
    __syncthreads();
    const uint32_t n = countPtr ? min(*countPtr, maxN) : maxN;
    const int lane = threadIdx.x & 31, gid = lane >> 2, tig = lane & 3;
    const uint32_t warpsTotal = gridDim.x * (blockDim.x >> 5);
    const uint32_t tiles = (n + 15) / 16;
    float lossAcc = 0.0f;
    for (uint32_t t = blockIdx.x * (blockDim.x >> 5) + warp; t < tiles; t += warpsTotal) {
        const uint32_t base = t * 16;
        // forward, keeping x, h1..h4 in shared memory
        encode_tile(g, grid, recs, base, n, sAct);
        __syncwarp();
        uint32_t a[4][4];
        load_a(sAct, a);
        float acc[8][4];
#pragma unroll
        for (int l = 0; l < 4; ++l) {
            layer64(sW + l * kWidth * kRow, a, acc);
            relu_to_a(acc, a);
            store_a(sAct + (l + 1) * 16 * kRow, a);
        }
        float y[4];
        output_layer(sW + 4 * kWidth * kRow, a, y);
        // dL/dy of the relative L2 loss, clamped and scaled, as FP16 rows of sD
        // (16 rows x 16 cols, outputs 3..15 zero)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int r = gid + 8 * h;
            const uint32_t q = base + (uint32_t)r;
            float gv[2] = {0.0f, 0.0f};
            if (q < n) {
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int c = 2 * tig + e;
                    if (c < 3) {
                        const float yy = y[2 * h + e];
                        const float tt = recs[q].target[c];
                        const float den = yy * yy + 0.01f;
                        const float diff = yy - tt;
                        lossAcc += diff * diff / den;
                        gv[e] = fminf(fmaxf(2.0f * diff / den, -kGradClamp), kGradClamp) * kGradScale;
                    }
                }
            }
            *reinterpret_cast<uint32_t*>(sD + r * kRow + 2 * tig) = pack2(gv[0], gv[1]);
            *reinterpret_cast<uint32_t*>(sD + r * kRow + 8 + 2 * tig) = 0u;
        }
        __syncwarp();

        // backward through W4 .. W0
        for (int l = 4; l >= 0; --l) {
            const int outDim = l == 4 ? kOutPad : kWidth;
            const __half* sWl = sW + l * kWidth * kRow;
            const __half* sIn = sAct + l * 16 * kRow;  // this layer's input activation
            float* gW = sDW + l * kWidth * kIn;
            // weight gradient dW_l += d^T * in  (M = outDim, N = 64, K = 16 rows)
            for (int mt = 0; mt < outDim / 16; ++mt) {
                uint32_t ad[4];
                {
                    const int m0 = 16 * mt + gid, m1 = m0 + 8;
                    ad[0] = pack2h(sD[(2 * tig) * kRow + m0], sD[(2 * tig + 1) * kRow + m0]);
                    ad[1] = pack2h(sD[(2 * tig) * kRow + m1], sD[(2 * tig + 1) * kRow + m1]);
                    ad[2] = pack2h(sD[(2 * tig + 8) * kRow + m0], sD[(2 * tig + 9) * kRow + m0]);
                    ad[3] = pack2h(sD[(2 * tig + 8) * kRow + m1], sD[(2 * tig + 9) * kRow + m1]);
                }
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int nn = 8 * j + gid;
                    const uint32_t b0 = pack2h(sIn[(2 * tig) * kRow + nn], sIn[(2 * tig + 1) * kRow + nn]);
                    const uint32_t b1 = pack2h(sIn[(2 * tig + 8) * kRow + nn], sIn[(2 * tig + 9) * kRow + nn]);
                    float c[4] = {0.0f, 0.0f, 0.0f, 0.0f};
                    mma16816(c, ad, b0, b1);
                    const int row0 = 16 * mt + gid, col0 = 8 * j + 2 * tig;
                    atomicAdd(&gW[row0 * kIn + col0], c[0]);
                    atomicAdd(&gW[row0 * kIn + col0 + 1], c[1]);
                    atomicAdd(&gW[(row0 + 8) * kIn + col0], c[2]);
                    atomicAdd(&gW[(row0 + 8) * kIn + col0 + 1], c[3]);
                }
            }
            // input gradient d_in = W_l^T * d  (N = 64 in-dims, K = outDim)
            float dacc[8][4];
#pragma unroll
            for (int j = 0; j < 8; ++j) dacc[j][0] = dacc[j][1] = dacc[j][2] = dacc[j][3] = 0.0f;
            for (int k = 0; k < outDim / 16; ++k) {
                uint32_t ak[4];
                ak[0] = lds32(sD + gid * kRow + 16 * k + 2 * tig);
                ak[1] = lds32(sD + (gid + 8) * kRow + 16 * k + 2 * tig);
                ak[2] = lds32(sD + gid * kRow + 16 * k + 8 + 2 * tig);
                ak[3] = lds32(sD + (gid + 8) * kRow + 16 * k + 8 + 2 * tig);
#pragma unroll
                for (int j = 0; j < 8; ++j) {
                    const int nn = 8 * j + gid;
                    const int k0 = 16 * k + 2 * tig;
                    const uint32_t b0 = pack2h(sWl[k0 * kRow + nn], sWl[(k0 + 1) * kRow + nn]);
                    const uint32_t b1 = pack2h(sWl[(k0 + 8) * kRow + nn], sWl[(k0 + 9) * kRow + nn]);
                    mma16816(dacc[j], ak, b0, b1);
                }
            }
            __syncwarp();
            if (l > 0) {
                // ReLU mask of the input activation (h_l > 0), then FP16 into sD
#pragma unroll
                for (int j = 0; j < 8; ++j) {
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int r = gid + 8 * h, c0 = 8 * j + 2 * tig;
                        const float m0 = __half2float(sIn[r * kRow + c0]) > 0.0f ? 1.0f : 0.0f;
                        const float m1 = __half2float(sIn[r * kRow + c0 + 1]) > 0.0f ? 1.0f : 0.0f;
                        *reinterpret_cast<uint32_t*>(sD + r * kRow + c0) =
                            pack2(dacc[j][2 * h] * m0, dacc[j][2 * h + 1] * m1);
                    }
                }
                __syncwarp();
            } else {
                // input gradient of the grid features (columns 0..31) as FP32
                float* sG = reinterpret_cast<float*>(sD);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
#pragma unroll
                    for (int h = 0; h < 2; ++h) {
                        const int r = gid + 8 * h, c0 = 8 * j + 2 * tig;
                        sG[r * 32 + c0] = dacc[j][2 * h];
                        sG[r * 32 + c0 + 1] = dacc[j][2 * h + 1];
                    }
                }
                __syncwarp();
            }
        }
        // scatter the grid gradients through the trilinear weights
        {
            const float* sG = reinterpret_cast<const float*>(sD);
            const int r = lane & 15;
            const uint32_t q = base + (uint32_t)r;
            if (q < n) {
                const StrelkaNrcRecord rec = recs[q];
                float px, py, pz;
                normalized_position(g, rec, px, py, pz);
                const int l0 = (lane >> 4) * 8;
                for (int l = l0; l < l0 + 8; ++l) {
                    Corner c;
                    level_corners(g, l, px, py, pz, c);
                    const float g0 = sG[r * 32 + 2 * l], g1 = sG[r * 32 + 2 * l + 1];
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        atomicAdd(&gridGrad[2 * (size_t)c.idx[k]], c.w[k] * g0);
                        atomicAdd(&gridGrad[2 * (size_t)c.idx[k] + 1], c.w[k] * g1);
                    }
                }
            }
        }
        __syncwarp();
    }
    // reduce the block's weight gradients and loss
    for (int off = 16; off > 0; off >>= 1) lossAcc += __shfl_xor_sync(0xffffffffu, lossAcc, off);
    if (lane == 0 && lossSum) atomicAdd(lossSum, lossAcc);
    __syncthreads();
    for (int i = threadIdx.x; i < kParams; i += blockDim.x) {
        const float v = sDW[i];
        if (v != 0.0f) atomicAdd(&dW[i], v);
    }
}

// Adam over a parameter array (FP32 master + FP16 copy).
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

size_t train_smem() { return (size_t)(kMatRows * kRow + 8 * 6 * 16 * kRow) * sizeof(__half) + kParams * sizeof(float); }

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
    cudaFuncSetAttribute(k_nrc_train, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)train_smem());
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
    const int tiles = (int)((maxN + 15) / 16);
    const int blocks = std::max(1, std::min((tiles + 7) / 8, nrc->numSMs));
    k_nrc_train<<<blocks, 256, train_smem(), st>>>(recs, countPtr, maxN, nrc->mlpHalf,
                                                  reinterpret_cast<const __half2*>(nrc->gridHalf), nrc->geom,
                                                  nrc->mlpGrad, nrc->gridGrad, nrc->loss);
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
