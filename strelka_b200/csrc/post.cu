// post.cu — reduction, accumulation and tonemap passes, sm_100a.
//
// ReductionPass   shaders/reduction.hlsl:9-32     (mean of spp samples)
// Accumulation    shaders/accumulation.hlsl:86-97 (progressive running mean)
// Tonemap         shaders/tonemap.hlsl:9-88       (Reinhard / ACESFitted / ACESFilm)
// and strelka_resolve_execute, which runs the three as one pass over the
// sample buffer with the same per-pixel arithmetic (so its output equals the
// three passes run in sequence) and optionally also writes RGBA8.
#include <cstdint>

#include "common.h"
#include "mdl_runtime.cuh"
#include "device_math.cuh"

using namespace sb;

namespace {

__device__ __forceinline__ v3 reduce_pixel(const float* __restrict__ sb, uint64_t pixel, int spp, float invSpp)
{
    float r = 0.0f, g = 0.0f, b = 0.0f;
    const float* p = sb + pixel * (uint64_t)spp * 3;
    for (int s = 0; s < spp; ++s) {
        r += invSpp * __ldg(p + 3 * s + 0);
        g += invSpp * __ldg(p + 3 * s + 1);
        b += invSpp * __ldg(p + 3 * s + 2);
    }
    return V(r, g, b);
}

__device__ __forceinline__ v3 accumulate_pixel(v3 cur, v3 prev, float wHistory, float wNew)
{
    return V(prev.x * wHistory + cur.x * wNew, prev.y * wHistory + cur.y * wNew, prev.z * wHistory + cur.z * wNew);
}

// tonemap.hlsl:9-64
__device__ __forceinline__ v3 aces_fitted(v3 c)
{
    v3 a = V((0.59719f * c.x + 0.35458f * c.y) + 0.04823f * c.z, (0.07600f * c.x + 0.90834f * c.y) + 0.01566f * c.z,
             (0.02840f * c.x + 0.13383f * c.y) + 0.83777f * c.z);
    float v[3] = {a.x, a.y, a.z}, r[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        float aa = v[i] * (v[i] + 0.0245786f) - 0.000090537f;
        float bb = v[i] * (0.983729f * v[i] + 0.4329510f) + 0.238081f;
        r[i] = aa / bb;
    }
    v3 o = V((1.60475f * r[0] + -0.53108f * r[1]) + -0.07367f * r[2], (-0.10208f * r[0] + 1.10813f * r[1]) + -0.00605f * r[2],
             (-0.00327f * r[0] + -0.07276f * r[1]) + 1.07602f * r[2]);
    return V(fsat(o.x), fsat(o.y), fsat(o.z));
}
__device__ __forceinline__ float aces_film1(float x)
{
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    return fsat((x * (a * x + b)) / (x * (c * x + d) + e));
}
__device__ __forceinline__ v3 reinhard(v3 c)
{
    float lum = (c.x * 0.299f + c.y * 0.587f) + c.z * 0.114f;
    float r = lum / (lum + 1.0f);
    float k = r / lum;
    return V(c.x * k, c.y * k, c.z * k);
}
__device__ __forceinline__ bool tonemap_pixel(uint32_t type, v3 c, v3& out)
{
    if (type == 0) out = reinhard(c);
    else if (type == 1) out = aces_fitted(c);
    else if (type == 2) out = V(aces_film1(c.x), aces_film1(c.y), aces_film1(c.z));
    else return false;
    return true;
}

__device__ __forceinline__ uint8_t to_u8(float x)
{
    float s = fsat(x) * 255.0f + 0.5f;
    return (uint8_t)(int)s;
}

__global__ void k_reduce(const float* __restrict__ sb, float4* __restrict__ out, uint32_t npix, int spp)
{
    const float invSpp = 1.0f / (float)spp;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        v3 c = reduce_pixel(sb, i, spp, invSpp);
        out[i] = make_float4(c.x, c.y, c.z, 1.0f);
    }
}

__global__ void k_accumulate(const float4* __restrict__ in, const float4* __restrict__ hist, float4* __restrict__ out,
                             uint32_t npix, float wHistory, float wNew)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        v3 r = accumulate_pixel(xyz(in[i]), xyz(hist[i]), wHistory, wNew);
        out[i] = make_float4(r.x, r.y, r.z, 1.0f);
    }
}

__global__ void k_tonemap(const float4* __restrict__ in, float4* __restrict__ out, uint32_t npix, uint32_t type)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        v3 r;
        if (tonemap_pixel(type, xyz(in[i]), r)) out[i] = make_float4(r.x, r.y, r.z, 1.0f);
    }
}

__global__ void k_resolve(const float* __restrict__ sb, int spp, uint32_t npix, int accumulate, const float4* __restrict__ hist,
                          float wHistory, float wNew, float4* __restrict__ accOut, uint32_t tmType, float4* __restrict__ tmOut,
                          uchar4* __restrict__ tm8)
{
    const float invSpp = 1.0f / (float)spp;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += gridDim.x * blockDim.x) {
        v3 c = reduce_pixel(sb, i, spp, invSpp);
        if (accumulate) c = accumulate_pixel(c, xyz(hist[i]), wHistory, wNew);
        if (accOut) accOut[i] = make_float4(c.x, c.y, c.z, 1.0f);
        v3 t;
        if (tonemap_pixel(tmType, c, t)) {
            if (tmOut) tmOut[i] = make_float4(t.x, t.y, t.z, 1.0f);
            if (tm8) tm8[i] = make_uchar4(to_u8(t.x), to_u8(t.y), to_u8(t.z), 255);
        }
    }
}

// Bilinear taps of the upscale pass (upscalepass.hlsl:17-19 with the
// clamp-to-edge linear sampler of upscalepass.cpp:12-38): the output pixel's
// uv in the input's texel space, the four clamped texel indices and the
// fractional weights.
struct Taps {
    uint32_t i00, i10, i01, i11;
    float w00, w10, w01, w11;
};

__device__ __forceinline__ Taps upscale_taps(uint32_t px, uint32_t py, float invW, float invH, int inW, int inH)
{
    const float u = ((float)px + 0.5f) * invW;
    const float v = ((float)py + 0.5f) * invH;
    const float fx = u * (float)inW - 0.5f;
    const float fy = v * (float)inH - 0.5f;
    const float flx = floorf(fx), fly = floorf(fy);
    const float a = fx - flx, b = fy - fly;
    const int x0 = min(max((int)flx, 0), inW - 1), x1 = min(max((int)flx + 1, 0), inW - 1);
    const int y0 = min(max((int)fly, 0), inH - 1), y1 = min(max((int)fly + 1, 0), inH - 1);
    Taps t;
    t.i00 = (uint32_t)y0 * (uint32_t)inW + (uint32_t)x0;
    t.i10 = (uint32_t)y0 * (uint32_t)inW + (uint32_t)x1;
    t.i01 = (uint32_t)y1 * (uint32_t)inW + (uint32_t)x0;
    t.i11 = (uint32_t)y1 * (uint32_t)inW + (uint32_t)x1;
    t.w00 = (1.0f - a) * (1.0f - b);
    t.w10 = a * (1.0f - b);
    t.w01 = (1.0f - a) * b;
    t.w11 = a * b;
    return t;
}

__device__ __forceinline__ v3 blend(const Taps& t, v3 c00, v3 c10, v3 c01, v3 c11)
{
    return V(((c00.x * t.w00 + c10.x * t.w10) + c01.x * t.w01) + c11.x * t.w11,
             ((c00.y * t.w00 + c10.y * t.w10) + c01.y * t.w01) + c11.y * t.w11,
             ((c00.z * t.w00 + c10.z * t.w10) + c01.z * t.w01) + c11.z * t.w11);
}

__global__ void k_upscale(const float4* __restrict__ in, int inW, int inH, float4* __restrict__ out, uint32_t outW,
                          uint32_t outH, float invW, float invH)
{
    const uint32_t n = outW * outH;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Taps t = upscale_taps(i % outW, i / outW, invW, invH, inW, inH);
        const v3 c = blend(t, xyz(__ldg(&in[t.i00])), xyz(__ldg(&in[t.i10])), xyz(__ldg(&in[t.i01])), xyz(__ldg(&in[t.i11])));
        out[i] = make_float4(c.x, c.y, c.z, 1.0f);
    }
}

// Tonemap of each tap (as k_tonemap computes it) then the upscale blend.
__global__ void k_tonemap_upscale(const float4* __restrict__ in, int inW, int inH, uint32_t tmType, float4* __restrict__ out,
                                  uchar4* __restrict__ out8, uint32_t outW, uint32_t outH, float invW, float invH)
{
    const uint32_t n = outW * outH;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const Taps t = upscale_taps(i % outW, i / outW, invW, invH, inW, inH);
        v3 c00, c10, c01, c11;
        tonemap_pixel(tmType, xyz(__ldg(&in[t.i00])), c00);
        tonemap_pixel(tmType, xyz(__ldg(&in[t.i10])), c10);
        tonemap_pixel(tmType, xyz(__ldg(&in[t.i01])), c01);
        tonemap_pixel(tmType, xyz(__ldg(&in[t.i11])), c11);
        const v3 c = blend(t, c00, c10, c01, c11);
        if (out) out[i] = make_float4(c.x, c.y, c.z, 1.0f);
        if (out8) out8[i] = make_uchar4(to_u8(c.x), to_u8(c.y), to_u8(c.z), 255);
    }
}

int grid_for(uint32_t n)
{
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    uint32_t blocks = (n + 255) / 256;
    uint32_t cap = (uint32_t)sms * 16;
    return (int)(blocks < cap ? (blocks ? blocks : 1) : cap);
}

bool aligned16(const void* p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

}  // namespace

extern "C" int strelka_reduction_execute(const ReductionDesc* d, uint32_t w, uint32_t h, uint64_t frameIndex, void* stream)
{
    (void)frameIndex;
    if (!d || !d->sampleBuffer || !d->result) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    const PathTracerParam& p = d->constants;
    if (p.dimension[0] <= 0 || p.dimension[1] <= 0 || p.spp <= 0) return fail(STRELKA_ERR_INVALID_ARGUMENT, "bad dimension/spp");
    const uint64_t npix = (uint64_t)p.dimension[0] * (uint64_t)p.dimension[1];
    if ((uint64_t)w * (h ? h : 1) != npix) return fail(STRELKA_ERR_INVALID_ARGUMENT, "w*h must equal W*H");
    if (!aligned16(d->result)) return fail(STRELKA_ERR_INVALID_ARGUMENT, "result must be 16-byte aligned");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_reduce<<<grid_for((uint32_t)npix), 256, 0, st>>>(d->sampleBuffer, reinterpret_cast<float4*>(d->result), (uint32_t)npix,
                                                      p.spp);
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}

extern "C" int strelka_accumulation_execute(const AccumulationDesc* d, uint32_t w, uint32_t h, uint64_t frameIndex, void* stream)
{
    (void)frameIndex;
    if (!d || !d->input || !d->history || !d->output) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    const AccumulationParam& p = d->constants;
    if (p.dimension[0] <= 0 || p.dimension[1] <= 0) return fail(STRELKA_ERR_INVALID_ARGUMENT, "bad dimension");
    if ((int64_t)w != p.dimension[0] || (int64_t)h != p.dimension[1])
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "w,h must equal the dimension");
    if (!aligned16(d->input) || !aligned16(d->history) || !aligned16(d->output))
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "images must be 16-byte aligned");
    const uint32_t npix = (uint32_t)p.dimension[0] * (uint32_t)p.dimension[1];
    // accumulation.hlsl:88-89
    const float wHistory = (float)p.iteration / (float)(p.iteration + 1u);
    const float wNew = 1.0f / (float)(p.iteration + 1u);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_accumulate<<<grid_for(npix), 256, 0, st>>>(reinterpret_cast<const float4*>(d->input),
                                                 reinterpret_cast<const float4*>(d->history),
                                                 reinterpret_cast<float4*>(d->output), npix, wHistory, wNew);
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}

extern "C" int strelka_tonemap_execute(const TonemapDesc* d, uint32_t w, uint32_t h, uint64_t frameIndex, void* stream)
{
    (void)frameIndex;
    if (!d || !d->input || !d->output) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    const Tonemapparam& p = d->constants;
    if (p.dimension[0] <= 0 || p.dimension[1] <= 0) return fail(STRELKA_ERR_INVALID_ARGUMENT, "bad dimension");
    if ((int64_t)w != p.dimension[0] || (int64_t)h != p.dimension[1])
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "w,h must equal the dimension");
    if (!aligned16(d->input) || !aligned16(d->output)) return fail(STRELKA_ERR_INVALID_ARGUMENT, "images must be 16-byte aligned");
    const uint32_t npix = (uint32_t)p.dimension[0] * (uint32_t)p.dimension[1];
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_tonemap<<<grid_for(npix), 256, 0, st>>>(reinterpret_cast<const float4*>(d->input), reinterpret_cast<float4*>(d->output),
                                              npix, p.tonemapperType);
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}

extern "C" int strelka_resolve_execute(const PathTracerParam* pp, const float* sampleBuffer, int accumulate,
                                       const AccumulationParam* ap, const float* history, float* accOutput,
                                       const Tonemapparam* tp, float* tonemapOutput, uint8_t* tonemapRGBA8, void* stream)
{
    if (!pp || !sampleBuffer || !tp) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    if (pp->dimension[0] <= 0 || pp->dimension[1] <= 0 || pp->spp <= 0)
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "bad dimension/spp");
    if (accumulate && (!ap || !history)) return fail(STRELKA_ERR_INVALID_ARGUMENT, "accumulation needs param and history");
    if (tp->dimension[0] != pp->dimension[0] || tp->dimension[1] != pp->dimension[1])
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "tonemap dimension mismatch");
    if ((accOutput && !aligned16(accOutput)) || (tonemapOutput && !aligned16(tonemapOutput)) ||
        (history && !aligned16(history)) || (tonemapRGBA8 && (reinterpret_cast<uintptr_t>(tonemapRGBA8) & 3)))
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "misaligned image");
    const uint32_t npix = (uint32_t)pp->dimension[0] * (uint32_t)pp->dimension[1];
    float wH = 0.0f, wN = 1.0f;
    if (accumulate) {
        wH = (float)ap->iteration / (float)(ap->iteration + 1u);
        wN = 1.0f / (float)(ap->iteration + 1u);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    k_resolve<<<grid_for(npix), 256, 0, st>>>(sampleBuffer, pp->spp, npix, accumulate, reinterpret_cast<const float4*>(history),
                                              wH, wN, reinterpret_cast<float4*>(accOutput), tp->tonemapperType,
                                              reinterpret_cast<float4*>(tonemapOutput),
                                              reinterpret_cast<uchar4*>(tonemapRGBA8));
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}

extern "C" int strelka_upscale_execute(const UpscaleDesc* d, uint32_t w, uint32_t h, uint64_t frameIndex, void* stream)
{
    (void)frameIndex;
    if (!d || !d->input || !d->output) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    const Upscalepassparam& p = d->constants;
    if (p.dimension[0] <= 0 || p.dimension[1] <= 0 || d->inputWidth == 0 || d->inputHeight == 0)
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "bad dimension");
    if ((int64_t)w != p.dimension[0] || (int64_t)h != p.dimension[1])
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "w,h must equal the output dimension");
    if ((uint64_t)p.dimension[0] * (uint64_t)p.dimension[1] > 0xFFFFFFFFull ||
        (uint64_t)d->inputWidth * d->inputHeight > 0xFFFFFFFFull || d->inputWidth > 0x7FFFFFFFu || d->inputHeight > 0x7FFFFFFFu)
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "image too large");
    if (!aligned16(d->input) || !aligned16(d->output)) return fail(STRELKA_ERR_INVALID_ARGUMENT, "images must be 16-byte aligned");
    const uint32_t n = (uint32_t)p.dimension[0] * (uint32_t)p.dimension[1];
    k_upscale<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const float4*>(d->input), (int)d->inputWidth, (int)d->inputHeight,
        reinterpret_cast<float4*>(d->output), (uint32_t)p.dimension[0], (uint32_t)p.dimension[1], p.invDimension[0],
        p.invDimension[1]);
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}

extern "C" int strelka_tonemap_upscale_execute(const Tonemapparam* tm, const float* input, const Upscalepassparam* up,
                                               float* output, uint8_t* outputRGBA8, void* stream)
{
    if (!tm || !input || !up || (!output && !outputRGBA8)) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    if (tm->dimension[0] <= 0 || tm->dimension[1] <= 0 || up->dimension[0] <= 0 || up->dimension[1] <= 0)
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "bad dimension");
    if (tm->tonemapperType > 2) return fail(STRELKA_ERR_INVALID_ARGUMENT, "unknown tonemapper %u", tm->tonemapperType);
    if ((uint64_t)up->dimension[0] * (uint64_t)up->dimension[1] > 0xFFFFFFFFull ||
        (uint64_t)tm->dimension[0] * (uint64_t)tm->dimension[1] > 0xFFFFFFFFull)
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "image too large");
    if (!aligned16(input) || (output && !aligned16(output)) || (outputRGBA8 && (reinterpret_cast<uintptr_t>(outputRGBA8) & 3)))
        return fail(STRELKA_ERR_INVALID_ARGUMENT, "misaligned image");
    const uint32_t n = (uint32_t)up->dimension[0] * (uint32_t)up->dimension[1];
    k_tonemap_upscale<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(
        reinterpret_cast<const float4*>(input), tm->dimension[0], tm->dimension[1], tm->tonemapperType,
        reinterpret_cast<float4*>(output), reinterpret_cast<uchar4*>(outputRGBA8), (uint32_t)up->dimension[0],
        (uint32_t)up->dimension[1], up->invDimension[0], up->invDimension[1]);
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}

// ---------------------------------------------------------------------------
// MDL runtime readers over a buffer (mdl_runtime.hlsl:24-75), one read per
// (offset, kind) pair: kind 0 float, 1 double, 2 int, 3 uint, 4 bool; out[i]
// receives the value's bits (float/int/uint/bool zero-extended to 64 bits).
namespace {
__global__ void k_mdl_read(const uint8_t* base, uint64_t bytes, const uint32_t* __restrict__ offs,
                           const uint32_t* __restrict__ kinds, uint32_t n, uint64_t* out)
{
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const uint32_t o = offs[i];
        uint64_t r = 0;
        switch (kinds[i]) {
            case 0: r = __float_as_uint(sb::mdl_read_as_float(base, bytes, o)); break;
            case 1: r = (uint64_t)__double_as_longlong(sb::mdl_read_as_double(base, bytes, o)); break;
            case 2: r = (uint32_t)sb::mdl_read_as_int(base, bytes, o); break;
            case 3: r = sb::mdl_read_as_uint(base, bytes, o); break;
            case 4: r = sb::mdl_read_as_bool(base, bytes, o) ? 1u : 0u; break;
            default: r = 0; break;
        }
        out[i] = r;
    }
}
}  // namespace

extern "C" int strelka_mdl_read(const uint8_t* buffer, uint64_t bytes, const uint32_t* offsets, const uint32_t* kinds,
                                uint32_t n, uint64_t* out, void* stream)
{
    if (n == 0) return STRELKA_OK;
    if (!offsets || !kinds || !out) return fail(STRELKA_ERR_INVALID_ARGUMENT, "NULL argument");
    if (buffer && (reinterpret_cast<uintptr_t>(buffer) & 3)) return fail(STRELKA_ERR_INVALID_ARGUMENT, "buffer must be 4-byte aligned");
    k_mdl_read<<<grid_for(n), 256, 0, static_cast<cudaStream_t>(stream)>>>(buffer, bytes, offsets, kinds, n, out);
    SB_CUDA_TRY(cudaGetLastError());
    return STRELKA_OK;
}
