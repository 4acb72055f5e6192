// device_math.cuh — scalar/vector math of the path-tracing hot path, sm_100a.
//
// The kernels are compiled with -fmad=false: every expression below rounds
// once per operation in source order, so results are reproducible on the
// host.  Reductions follow the reference HLSL expressions:
//   dot(a,b) = (a.x*b.x + a.y*b.y) + a.z*b.z; cross is the textbook formula;
//   normalize(v) = v * (1/sqrt(dot(v,v))); HLSL min/max = fminf/fmaxf;
//   saturate(x) = fminf(fmaxf(x, 0), 1); mul(M, v) over a column-major
//   (glm) float4x4 sums the four products of a row left to right.
// sin/cos/acos are the project's own: Cody–Waite reduction by pi/2 with a
// three-part split, Taylor polynomials of sin (to r^11) and cos (to r^12),
// and the arcsine Maclaurin series to x^23 with acos(x) = 2 asin(sqrt((1-x)/2))
// for |x| > 1/2.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

#include "../../include/strelka_b200.h"

#define SB_INVALID 0xFFFFFFFFu
// helper.h:3-7: PI is the literal 3.1415926535897, folded then rounded to float
#define SB_PI_F ((float)3.1415926535897)
#define SB_TWO_PI_F ((float)(2.0 * 3.1415926535897))
#define SB_FOUR_PI_F ((float)(4.0 * 3.1415926535897))
#define SB_INV_PI_F ((float)(1.0 / 3.1415926535897))
#define SB_PI_OVER_2_F ((float)1.57079632679489661923)
#define SB_PI_OVER_4_F ((float)0.78539816339744830961)

// MDL event flags, shaders/mdl_types.hlsl:188-201
#define SB_EV_ABSORB 0
#define SB_EV_DIFFUSE 1
#define SB_EV_GLOSSY 2
#define SB_EV_SPECULAR 4
#define SB_EV_REFLECTION 8
#define SB_EV_TRANSMISSION 16

namespace sb {

struct v3 {
    float x, y, z;
};

__device__ __forceinline__ v3 V(float x, float y, float z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
__device__ __forceinline__ v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
__device__ __forceinline__ v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
__device__ __forceinline__ v3 vmul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
__device__ __forceinline__ v3 vscale(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
__device__ __forceinline__ v3 vdivs(v3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }
__device__ __forceinline__ v3 vneg(v3 a) { return V(-a.x, -a.y, -a.z); }
__device__ __forceinline__ float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ v3 vcross(v3 a, v3 b)
{
    return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ float vlength(v3 a) { return sqrtf(vdot(a, a)); }
__device__ __forceinline__ v3 vnormalize(v3 a)
{
    float inv = 1.0f / sqrtf(vdot(a, a));
    return vscale(a, inv);
}
__device__ __forceinline__ float fsat(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
__device__ __forceinline__ bool vhasnan(v3 a) { return isnan(a.x) || isnan(a.y) || isnan(a.z); }
__device__ __forceinline__ v3 xyz(float4 a) { return V(a.x, a.y, a.z); }
__device__ __forceinline__ float4 f4(v3 a, float w) { return make_float4(a.x, a.y, a.z, w); }

// ---------------------------------------------------------------------------
// Own sin/cos/acos (identical operation sequence on the host checker).
__device__ __forceinline__ void own_sincos(float x, float* s, float* c)
{
    if (!(fabsf(x) <= 1.0e30f)) {
        *s = __int_as_float(0x7fc00000);
        *c = __int_as_float(0x7fc00000);
        return;
    }
    const float PIO2_1 = 0x1.921fb6p+0f;
    const float PIO2_2 = -0x1.777a5cp-25f;
    const float PIO2_3 = -0x1.ee59dap-50f;
    const float TWO_OVER_PI = 0x1.45f306p-1f;
    float k = rintf(x * TWO_OVER_PI);
    float r = fmaf(-k, PIO2_1, x);
    r = fmaf(-k, PIO2_2, r);
    r = fmaf(-k, PIO2_3, r);
    float r2 = r * r;
    float ps = fmaf(r2, -2.5052108385441720e-8f, 2.7557319223985893e-6f);
    ps = fmaf(r2, ps, -1.9841269841269841e-4f);
    ps = fmaf(r2, ps, 8.3333333333333333e-3f);
    ps = fmaf(r2, ps, -1.6666666666666667e-1f);
    float sr = fmaf(r * r2, ps, r);
    float pc = fmaf(r2, 2.0876756987868099e-9f, -2.7557319223985891e-7f);
    pc = fmaf(r2, pc, 2.4801587301587302e-5f);
    pc = fmaf(r2, pc, -1.3888888888888889e-3f);
    pc = fmaf(r2, pc, 4.1666666666666667e-2f);
    pc = fmaf(r2, pc, -0.5f);
    float cr = fmaf(r2, pc, 1.0f);
    int q = (int)(k - 4.0f * floorf(k * 0.25f));
    if (q == 0) { *s = sr; *c = cr; }
    else if (q == 1) { *s = cr; *c = -sr; }
    else if (q == 2) { *s = -sr; *c = -cr; }
    else { *s = -cr; *c = sr; }
}

__device__ __forceinline__ float own_asin_small(float x)
{
    float z = x * x;
    float p = fmaf(z, 6.4472103118896484e-3f, 7.3125258735988454e-3f);
    p = fmaf(z, p, 8.3903358096168155e-3f);
    p = fmaf(z, p, 9.7616095291940789e-3f);
    p = fmaf(z, p, 1.1551800896139705e-2f);
    p = fmaf(z, p, 1.3964843750000000e-2f);
    p = fmaf(z, p, 1.7352764423076924e-2f);
    p = fmaf(z, p, 2.2372159090909092e-2f);
    p = fmaf(z, p, 3.0381944444444444e-2f);
    p = fmaf(z, p, 4.4642857142857144e-2f);
    p = fmaf(z, p, 7.5000000000000000e-2f);
    p = fmaf(z, p, 1.6666666666666667e-1f);
    return fmaf(x * z, p, x);
}

__device__ __forceinline__ float own_acosf(float x)
{
    const float PIO2_1 = 0x1.921fb6p+0f;
    const float PIO2_2 = -0x1.777a5cp-25f;
    const float PI_HI = 0x1.921fb6p+1f;
    const float PI_LO = -0x1.777a5cp-24f;
    if (fabsf(x) <= 0.5f) return PIO2_1 - (own_asin_small(x) - PIO2_2);
    if (x > 0.5f) return 2.0f * own_asin_small(sqrtf((1.0f - x) * 0.5f));
    return PI_HI - (2.0f * own_asin_small(sqrtf((1.0f + x) * 0.5f)) - PI_LO);
}

__device__ __forceinline__ float own_sinf(float x) { float s, c; own_sincos(x, &s, &c); return s; }
__device__ __forceinline__ float own_cosf(float x) { float s, c; own_sincos(x, &s, &c); return c; }

// ---------------------------------------------------------------------------
// random.h:14-48
__device__ __forceinline__ uint32_t jenkins_hash(uint32_t x)
{
    x += x << 10;
    x ^= x >> 6;
    x += x << 3;
    x ^= x >> 11;
    x += x << 15;
    return x;
}
__device__ __forceinline__ uint32_t init_rng(uint32_t px, uint32_t py, uint32_t width, uint32_t frame)
{
    uint32_t seed = (px * 1u + py * width) ^ jenkins_hash(frame);
    return jenkins_hash(seed);
}
__device__ __forceinline__ float rand01(uint32_t& s)
{
    uint32_t x = s;
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    s = x;
    return __uint_as_float(0x3f800000u | (x >> 9)) - 1.0f;
}

// helper.h:117-148
__device__ __forceinline__ uint32_t permute(uint32_t i, uint32_t l, uint32_t p)
{
    uint32_t w = l - 1;
    w |= w >> 1;
    w |= w >> 2;
    w |= w >> 4;
    w |= w >> 8;
    w |= w >> 16;
    do {
        i ^= p;
        i *= 0xe170893du;
        i ^= p >> 16;
        i ^= (i & w) >> 4;
        i ^= p >> 8;
        i *= 0x0929eb3fu;
        i ^= p >> 23;
        i ^= (i & w) >> 1;
        i *= 1u | p >> 27;
        i *= 0x6935fa69u;
        i ^= (i & w) >> 11;
        i *= 0x74dcb303u;
        i ^= (i & w) >> 2;
        i *= 0x9e501cc3u;
        i ^= (i & w) >> 2;
        i *= 0xc860a3dfu;
        i &= w;
        i ^= i >> 5;
    } while (i >= l);
    return (i + p) % l;
}
// helper.h:150-163
__device__ __forceinline__ float randfloat(uint32_t i, uint32_t p)
{
    i ^= p;
    i ^= i >> 17;
    i ^= i >> 10;
    i *= 0xb36534e5u;
    i ^= i >> 12;
    i ^= i >> 21;
    i *= 0x93fc4795u;
    i ^= 0xdf6e307fu;
    i ^= i >> 17;
    i *= 1u | p >> 18;
    return (float)i * (1.0f / 4294967808.0f);
}

// ---------------------------------------------------------------------------
// pack.h:4-24
__device__ __forceinline__ v3 unpack_normal(uint32_t val)
{
    v3 n;
    n.z = (float)((val & 0xfff00000u) >> 20) / 511.99999f * 2.0f - 1.0f;
    n.y = (float)((val & 0x000ffc00u) >> 10) / 511.99999f * 2.0f - 1.0f;
    n.x = (float)(val & 0x000003ffu) / 511.99999f * 2.0f - 1.0f;
    return n;
}
__device__ __forceinline__ void unpack_uv(uint32_t val, float& u, float& v)
{
    v = (float)((val & 0xffff0000u) >> 16) / 16383.99999f * 20.0f - 10.0f;
    u = (float)(val & 0x0000ffffu) / 16383.99999f * 20.0f - 10.0f;
}

// helper.h:12-28 (Ray Tracing Gems ch. 6)
__device__ __forceinline__ float offset_axis(float p, float n)
{
    const float origin = 1.0f / 32.0f;
    const float float_scale = 1.0f / 65536.0f;
    const float int_scale = 256.0f;
    int32_t of_i = (int32_t)(int_scale * n);
    uint32_t bits = __float_as_uint(p) + (uint32_t)((p < 0) ? -of_i : of_i);
    float p_i = __uint_as_float(bits);
    return fabsf(p) < origin ? p + float_scale * n : p_i;
}
__device__ __forceinline__ v3 offset_ray(v3 p, v3 n) { return V(offset_axis(p.x, n.x), offset_axis(p.y, n.y), offset_axis(p.z, n.z)); }

// helper.h:31-39
__device__ __forceinline__ v3 interp3(v3 a1, v3 a2, v3 a3, float bx, float by)
{
    float w = (1.0f - bx) - by;
    return V((a1.x * w + a2.x * bx) + a3.x * by, (a1.y * w + a2.y * bx) + a3.y * by,
             (a1.z * w + a2.z * bx) + a3.z * by);
}

// helper.h:41-50: columns tangent, binormal, normal
struct Frame {
    v3 t, b, n;
};
__device__ __forceinline__ Frame tangent_space(v3 normal)
{
    v3 helper = V(1.0f, 0.0f, 0.0f);
    if (fabsf(normal.x) > 0.99f) helper = V(0.0f, 0.0f, 1.0f);
    Frame f;
    f.t = vnormalize(vcross(normal, helper));
    f.b = vnormalize(vcross(normal, f.t));
    f.n = normal;
    return f;
}
__device__ __forceinline__ v3 frame_to_world(const Frame& f, v3 w)
{
    return V((f.t.x * w.x + f.b.x * w.y) + f.n.x * w.z, (f.t.y * w.x + f.b.y * w.y) + f.n.y * w.z,
             (f.t.z * w.x + f.b.z * w.y) + f.n.z * w.z);
}

// helper.h:73-79
__device__ __forceinline__ v3 sample_hemisphere_cosine(float ux, float uy)
{
    float cosTheta = sqrtf(fsat(ux));
    float sinTheta = sqrtf(fsat(1.0f - cosTheta * cosTheta));
    float phi = SB_TWO_PI_F * uy;
    float s, c;
    own_sincos(phi, &s, &c);
    return V(c * sinTheta, s * sinTheta, cosTheta + 1e-6f);
}

// mul(M, float4(v, w)).xyz over a column-major float4x4 in global memory
__device__ __forceinline__ v3 mat_mul_point(const float* m, v3 v, float w)
{
    float r[3];
#pragma unroll
    for (int i = 0; i < 3; ++i)
        r[i] = ((m[0 * 4 + i] * v.x + m[1 * 4 + i] * v.y) + m[2 * 4 + i] * v.z) + m[3 * 4 + i] * w;
    return V(r[0], r[1], r[2]);
}
__device__ __forceinline__ void mat_mul4(const float* m, const float v[4], float out[4])
{
#pragma unroll
    for (int i = 0; i < 4; ++i)
        out[i] = ((m[0 * 4 + i] * v[0] + m[1 * 4 + i] * v[1]) + m[2 * 4 + i] * v[2]) + m[3 * 4 + i] * v[3];
}
__device__ __forceinline__ v3 mat_mul_dir3(const float* m, v3 v)
{
    float r[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) r[i] = (m[0 * 4 + i] * v.x + m[1 * 4 + i] * v.y) + m[2 * 4 + i] * v.z;
    return V(r[0], r[1], r[2]);
}

}  // namespace sb
