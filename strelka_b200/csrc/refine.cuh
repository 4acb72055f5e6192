// refine.cuh — float-float recomputation of a closest hit's distance and
// barycentrics (validation aid; never used by the render path).
//
// The Möller–Trumbore formulas of raytracing.h:36-88 evaluated in
// double-float arithmetic (Dekker 1971, Knuth TAOCP vol. 2: TwoSum and an
// FMA-based TwoProduct), starting from the object-space vertices and the
// instance matrix, so the result is the correctly rounded float of a ~44-bit
// computation.  No FP64 instruction is used.
#pragma once
#include "traverse.cuh"

namespace sb {

struct ff {
    float h, l;
};

__device__ __forceinline__ ff ff_two_sum(float a, float b)
{
    float s = a + b;
    float bb = s - a;
    float e = (a - (s - bb)) + (b - bb);
    return {s, e};
}
__device__ __forceinline__ ff ff_quick(float a, float b)
{
    float s = a + b;
    float e = b - (s - a);
    return {s, e};
}
__device__ __forceinline__ ff ff_two_prod(float a, float b)
{
    float p = a * b;
    float e = fmaf(a, b, -p);
    return {p, e};
}
__device__ __forceinline__ ff ff_add(ff a, ff b)
{
    ff s = ff_two_sum(a.h, b.h);
    ff t = ff_two_sum(a.l, b.l);
    float e = s.l + t.h;
    s = ff_quick(s.h, e);
    e = s.l + t.l;
    return ff_quick(s.h, e);
}
__device__ __forceinline__ ff ff_neg(ff a) { return {-a.h, -a.l}; }
__device__ __forceinline__ ff ff_sub(ff a, ff b) { return ff_add(a, ff_neg(b)); }
__device__ __forceinline__ ff ff_mul(ff a, ff b)
{
    ff p = ff_two_prod(a.h, b.h);
    float e = p.l + (a.h * b.l + a.l * b.h);
    return ff_quick(p.h, e);
}
__device__ __forceinline__ ff ff_div(ff a, ff b)
{
    float q1 = a.h / b.h;
    ff r = ff_sub(a, ff_mul(ff{q1, 0.0f}, b));
    float q2 = r.h / b.h;
    r = ff_sub(r, ff_mul(ff{q2, 0.0f}, b));
    float q3 = r.h / b.h;
    ff q = ff_quick(q1, q2);
    return ff_add(q, ff{q3, 0.0f});
}

struct ff3 {
    ff x, y, z;
};
__device__ __forceinline__ ff3 ff3_sub(ff3 a, ff3 b) { return {ff_sub(a.x, b.x), ff_sub(a.y, b.y), ff_sub(a.z, b.z)}; }
__device__ __forceinline__ ff ff3_dot(ff3 a, ff3 b)
{
    return ff_add(ff_add(ff_mul(a.x, b.x), ff_mul(a.y, b.y)), ff_mul(a.z, b.z));
}
__device__ __forceinline__ ff3 ff3_cross(ff3 a, ff3 b)
{
    return {ff_sub(ff_mul(a.y, b.z), ff_mul(a.z, b.y)), ff_sub(ff_mul(a.z, b.x), ff_mul(a.x, b.z)),
            ff_sub(ff_mul(a.x, b.y), ff_mul(a.y, b.x))};
}
__device__ __forceinline__ ff3 ff3_from(v3 a) { return {{a.x, 0.0f}, {a.y, 0.0f}, {a.z, 0.0f}}; }

// object-space vertex through the column-major instance matrix
__device__ __forceinline__ ff3 ff_xform(const float* m, const float* p)
{
    ff r[3];
#pragma unroll
    for (int i = 0; i < 3; ++i) {
        ff acc = ff_two_prod(m[0 * 4 + i], p[0]);
        acc = ff_add(acc, ff_two_prod(m[1 * 4 + i], p[1]));
        acc = ff_add(acc, ff_two_prod(m[2 * 4 + i], p[2]));
        acc = ff_add(acc, ff{m[3 * 4 + i], 0.0f});
        r[i] = acc;
    }
    return {r[0], r[1], r[2]};
}

// Recomputes (t, u, v) of ray (o, d) against triangle (inst, prim).
__device__ __forceinline__ bool refine_hit(const DevScene& s, v3 o, v3 d, uint32_t inst, uint32_t prim, float& t, float& u,
                                           float& v)
{
    if (inst >= s.numInstances) return false;
    const InstanceConstants* ic = &s.inst[inst];
    const uint32_t base = (uint32_t)ic->indexOffset + prim * 3u;
    if ((uint64_t)base + 2 >= s.numIndices) return false;
    const uint32_t i0 = s.ib[base], i1 = s.ib[base + 1], i2 = s.ib[base + 2];
    if (i0 >= s.numVertices || i1 >= s.numVertices || i2 >= s.numVertices) return false;
    const float* m = ic->objectToWorld.m;
    ff3 P0 = ff_xform(m, s.vb[i0].position);
    ff3 P1 = ff_xform(m, s.vb[i1].position);
    ff3 P2 = ff_xform(m, s.vb[i2].position);
    ff3 D = ff3_from(d);
    ff3 e0 = ff3_sub(P1, P0), e1 = ff3_sub(P2, P0), tv = ff3_sub(ff3_from(o), P0);
    ff3 pv = ff3_cross(D, e1);
    ff det = ff3_dot(e0, pv);
    ff3 qv = ff3_cross(tv, e0);
    u = ff_div(ff3_dot(tv, pv), det).h;
    v = ff_div(ff3_dot(D, qv), det).h;
    t = ff_div(ff3_dot(e1, qv), det).h;
    return true;
}

}  // namespace sb
