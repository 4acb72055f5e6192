// post.cpp -- the reference's reduction, accumulation, tonemap and upscale
// shaders, compiled on the host.
//
// TEST INFRASTRUCTURE (oracle/build_ref.sh builds it into oracle/_ref/): the
// reference's own shaders/reduction.hlsl, accumulation.hlsl, tonemap.hlsl
// and upscalepass.hlsl, rewritten only syntactically by oracle/hlsl2cpp.py,
// over the HLSL shim of shim.h; each pass in a namespace of its own, as each
// is a separate shader with its own globals.
#include <cstring>

#include "shim.h"

#include "../oracle.h"

namespace ref_red {
#include "reduction.hlsl"
}
namespace ref_acc {
#include "accumulation.hlsl"
}
namespace ref_tm {
#include "tonemap.hlsl"
}
namespace ref_up {
#include "upscalepass.hlsl"
}

static_assert(sizeof(ref_red::PathTracerParam) == sizeof(::PathTracerParam) &&
                  sizeof(ref_acc::AccumulationParam) == sizeof(::AccumulationParam) &&
                  sizeof(ref_tm::Tonemapparam) == sizeof(::Tonemapparam) &&
                  sizeof(ref_up::Upscalepassparam) == sizeof(::Upscalepassparam),
              "the reference's parameter structs as compiled here must match the C ABI's");

template <class Dst, class Src> static void set_ubo(Dst& ubo, const Src* p)
{
    static_assert(sizeof(Src) <= sizeof(Dst), "size");
    memcpy(static_cast<void*>(&ubo), p, sizeof(Src));
}

extern "C" {

/* reduction.hlsl:9-32 over the W*H pixels of p->dimension: out RGBA32F. */
int strelka_ref_reduce(const ::PathTracerParam* p, const float* sampleBuffer, float* out)
{
    using namespace ref_red;
    set_ubo(ubo, p);
    const uint W = (uint)p->dimension[0], H = (uint)p->dimension[1];
    ref_red::sampleBuffer.p = sampleBuffer;
    ref_red::sampleBuffer.n = (uint64_t)W * H * (uint64_t)p->spp * 3;
    output.p = reinterpret_cast<float4*>(out);
    output.w = W;
    output.h = H;
    for (uint i = 0; i < W * H; ++i) computeMain(uint2(i, 0u));
    return 0;
}

/* accumulation.hlsl:86-108 over p->dimension: in, history and out RGBA32F. */
int strelka_ref_accumulate(const ::AccumulationParam* p, const float* in, const float* history, float* out)
{
    using namespace ref_acc;
    set_ubo(ubo, p);
    const uint W = (uint)p->dimension[0], H = (uint)p->dimension[1];
    input.p = reinterpret_cast<const float4*>(in);
    input.w = W;
    input.h = H;
    ref_acc::history.p = reinterpret_cast<const float4*>(history);
    ref_acc::history.w = W;
    ref_acc::history.h = H;
    output.p = reinterpret_cast<float4*>(out);
    output.w = W;
    output.h = H;
    for (uint y = 0; y < H; ++y)
        for (uint x = 0; x < W; ++x) computeMain(uint2(x, y));
    return 0;
}

/* tonemap.hlsl:66-88 over p->dimension: in and out RGBA32F. */
int strelka_ref_tonemap(const ::Tonemapparam* p, const float* in, float* out)
{
    using namespace ref_tm;
    set_ubo(ubo, p);
    const uint W = (uint)p->dimension[0], H = (uint)p->dimension[1];
    input.p = reinterpret_cast<const float4*>(in);
    input.w = W;
    input.h = H;
    output.p = reinterpret_cast<float4*>(out);
    output.w = W;
    output.h = H;
    for (uint y = 0; y < H; ++y)
        for (uint x = 0; x < W; ++x) computeMain(uint2(x, y));
    return 0;
}

/* upscalepass.hlsl:9-21: in RGBA32F inW x inH, out RGBA32F p->dimension. */
int strelka_ref_upscale(const ::Upscalepassparam* p, const float* in, uint32_t inW, uint32_t inH, float* out)
{
    using namespace ref_up;
    set_ubo(ubo, p);
    const uint W = (uint)p->dimension[0], H = (uint)p->dimension[1];
    input.p = reinterpret_cast<const float4*>(in);
    input.w = inW;
    input.h = inH;
    output.p = reinterpret_cast<float4*>(out);
    output.w = W;
    output.h = H;
    for (uint y = 0; y < H; ++y)
        for (uint x = 0; x < W; ++x) computeMain(uint2(x, y));
    return 0;
}
}
