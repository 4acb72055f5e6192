/*
 * own_math.h -- the project's own sin, cos and acos in single precision.
 *
 * TEST INFRASTRUCTURE (shared by oracle/oracle.c and the HLSL shim of
 * oracle/ref/): the CUDA kernels carry the same functions
 * (strelka_b200/csrc/device_math.cuh), so the three agree bit for bit.
 * The reference's sin/cos/acos are whatever the GPU driver compiles HLSL's
 * intrinsics to (implementation-defined precision); these stand in for them.
 *
 * sin/cos: Cody-Waite reduction by pi/2 (three-part split of pi/2, FMA
 * steps) and the Taylor polynomials of sin (to r^11) and cos (to r^12) on
 * |r| <= pi/4.  acos: the arcsine Maclaurin series to x^23 on |x| <= 1/2 and
 * acos(x) = 2 asin(sqrt((1-x)/2)) outside.  Builds as C11 and C++17.
 */
#ifndef STRELKA_OWN_MATH_H
#define STRELKA_OWN_MATH_H
#include <math.h>

static const float PIO2_1 = 0x1.921fb6p+0f;
static const float PIO2_2 = -0x1.777a5cp-25f;
static const float PIO2_3 = -0x1.ee59dap-50f;
static const float TWO_OVER_PI = 0x1.45f306p-1f;
static const float PI_HI = 0x1.921fb6p+1f;
static const float PI_LO = -0x1.777a5cp-24f;

static inline void own_sincos(float x, float* s, float* c)
{
    if (!(fabsf(x) <= 1.0e30f)) { *s = NAN; *c = NAN; return; }
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
    switch (q) {
    case 0: *s = sr; *c = cr; break;
    case 1: *s = cr; *c = -sr; break;
    case 2: *s = -sr; *c = -cr; break;
    default: *s = -cr; *c = sr; break;
    }
}
static inline float own_sinf(float x) { float s, c; own_sincos(x, &s, &c); return s; }
static inline float own_cosf(float x) { float s, c; own_sincos(x, &s, &c); return c; }

static inline float own_asin_small(float x) /* |x| <= 0.5 */
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
static inline float own_acosf(float x)
{
    if (fabsf(x) <= 0.5f) return PIO2_1 - (own_asin_small(x) - PIO2_2);
    if (x > 0.5f) return 2.0f * own_asin_small(sqrtf((1.0f - x) * 0.5f));
    return PI_HI - (2.0f * own_asin_small(sqrtf((1.0f + x) * 0.5f)) - PI_LO);
}

#endif
