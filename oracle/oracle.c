/*
 * oracle.c — CPU restatement of Strelka's path-tracing hot path.
 *
 * TEST INFRASTRUCTURE ONLY (see oracle.h): the checker for the CUDA kernels,
 * never part of the product.  Build: oracle/build.sh (gcc -O3
 * -ffp-contract=off -fopenmp).  Reference citations are paths inside the
 * ikryukov/Strelka source tree.
 *
 * Conventions that make this file and the kernels agree bit for bit:
 *  - every expression is evaluated in the order the HLSL source writes it,
 *    one IEEE single-precision rounding per operation, no FMA contraction;
 *  - dot(a,b) = (a.x*b.x + a.y*b.y) + a.z*b.z; cross is the textbook formula;
 *    normalize(v) = v * (1/sqrt(dot(v,v))); length = sqrt(dot(v,v));
 *  - HLSL min/max/clamp/saturate are fminf/fmaxf (a NaN operand yields the
 *    other operand); saturate(x) = fminf(fmaxf(x, 0), 1);
 *  - matrices are column-major (glm): M[r][c] = m[c*4 + r]; mul(M, v) sums
 *    the four products of a row left to right;
 *  - sin/cos/acos are the project's own polynomial versions below.
 */
#include "oracle.h"
#include "own_math.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define INVALID_INDEX 0xFFFFFFFFu
/* helper.h:3-7: PI is the double literal 3.1415926535897; in float context
 * HLSL folds constant expressions first and rounds once. */
#define PI_F ((float)3.1415926535897)
#define TWO_PI_F ((float)(2.0 * 3.1415926535897))
#define FOUR_PI_F ((float)(4.0 * 3.1415926535897))
#define INV_PI_F ((float)(1.0 / 3.1415926535897))
#define PI_OVER_2_F ((float)1.57079632679489661923)
#define PI_OVER_4_F ((float)0.78539816339744830961)

/* MDL event flags, shaders/mdl_types.hlsl:188-201 */
#define EV_ABSORB 0
#define EV_DIFFUSE 1
#define EV_GLOSSY 2
#define EV_SPECULAR 4
#define EV_REFLECTION 8
#define EV_TRANSMISSION 16

typedef struct { float x, y, z; } v3;

static inline v3 V(float x, float y, float z) { v3 r; r.x = x; r.y = y; r.z = z; return r; }
static inline v3 vadd(v3 a, v3 b) { return V(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vmul(v3 a, v3 b) { return V(a.x * b.x, a.y * b.y, a.z * b.z); }
static inline v3 vscale(v3 a, float s) { return V(a.x * s, a.y * s, a.z * s); }
static inline v3 vdivs(v3 a, float s) { return V(a.x / s, a.y / s, a.z / s); }
static inline v3 vdiv(v3 a, v3 b) { return V(a.x / b.x, a.y / b.y, a.z / b.z); }
static inline v3 vneg(v3 a) { return V(-a.x, -a.y, -a.z); }
static inline float vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 vcross(v3 a, v3 b)
{
    return V(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
static inline float vlength(v3 a) { return sqrtf(vdot(a, a)); }
static inline v3 vnormalize(v3 a)
{
    float inv = 1.0f / sqrtf(vdot(a, a));
    return vscale(a, inv);
}
static inline float fsat(float x) { return fminf(fmaxf(x, 0.0f), 1.0f); }
static inline v3 vload(const float* p) { return V(p[0], p[1], p[2]); }
static inline int vhasnan(v3 a) { return isnan(a.x) || isnan(a.y) || isnan(a.z); }

static inline float asfloat_u(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }
static inline uint32_t asuint_f(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }

/* mul(M, float4(v, w)).xyz for a column-major float4x4 */
static inline v3 mat_mul_point(const StrelkaFloat4x4* M, v3 v, float w)
{
    const float* m = M->m;
    float r[3];
    for (int i = 0; i < 3; ++i)
        r[i] = ((m[0 * 4 + i] * v.x + m[1 * 4 + i] * v.y) + m[2 * 4 + i] * v.z) + m[3 * 4 + i] * w;
    return V(r[0], r[1], r[2]);
}
/* mul(M, float4) full 4-vector */
static inline void mat_mul4(const StrelkaFloat4x4* M, const float v[4], float out[4])
{
    const float* m = M->m;
    for (int i = 0; i < 4; ++i)
        out[i] = ((m[0 * 4 + i] * v[0] + m[1 * 4 + i] * v[1]) + m[2 * 4 + i] * v[2]) + m[3 * 4 + i] * v[3];
}
/* mul((float3x3)M, v) */
static inline v3 mat_mul_dir3(const StrelkaFloat4x4* M, v3 v)
{
    const float* m = M->m;
    float r[3];
    for (int i = 0; i < 3; ++i)
        r[i] = (m[0 * 4 + i] * v.x + m[1 * 4 + i] * v.y) + m[2 * 4 + i] * v.z;
    return V(r[0], r[1], r[2]);
}

/* ------------------------------------------------------------------------- */
/* Own sin/cos/acos (own_math.h), exported for the tests. */
float oracle_sinf(float x) { return own_sinf(x); }
float oracle_cosf(float x) { return own_cosf(x); }
float oracle_acosf(float x) { return own_acosf(x); }
#define SINF oracle_sinf
#define COSF oracle_cosf
#define ACOSF oracle_acosf

/* ------------------------------------------------------------------------- */
/* random.h:14-48 */
uint32_t oracle_jenkins_hash(uint32_t x)
{
    x += x << 10;
    x ^= x >> 6;
    x += x << 3;
    x ^= x >> 11;
    x += x << 15;
    return x;
}
/* random.h:26-30: seed = dot(pixel, (1, W)) ^ hash(frame); state = hash(seed) */
uint32_t oracle_init_rng(uint32_t px, uint32_t py, uint32_t width, uint32_t frame)
{
    uint32_t seed = (px * 1u + py * width) ^ oracle_jenkins_hash(frame);
    return oracle_jenkins_hash(seed);
}
static inline float uint_to_float(uint32_t x) { return asfloat_u(0x3f800000u | (x >> 9)) - 1.0f; }
uint32_t oracle_xorshift(uint32_t* s)
{
    uint32_t x = *s;
    x ^= x << 13;
    x ^= x >> 17;
    x ^= x << 5;
    *s = x;
    return x;
}
float oracle_rand(uint32_t* s) { return uint_to_float(oracle_xorshift(s)); }

/* helper.h:117-148 (Kensler, correlated multi-jittered sampling) */
uint32_t oracle_permute(uint32_t i, uint32_t l, uint32_t p)
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
/* helper.h:150-163 */
float oracle_randfloat(uint32_t i, uint32_t p)
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

/* ------------------------------------------------------------------------- */
/* pack.h:4-14, 16-24 */
static v3 unpack_normal(uint32_t val)
{
    v3 n;
    n.z = (float)((val & 0xfff00000u) >> 20) / 511.99999f * 2.0f - 1.0f;
    n.y = (float)((val & 0x000ffc00u) >> 10) / 511.99999f * 2.0f - 1.0f;
    n.x = (float)(val & 0x000003ffu) / 511.99999f * 2.0f - 1.0f;
    return n;
}
void oracle_unpack_normal(uint32_t v, float out[3]) { v3 n = unpack_normal(v); out[0] = n.x; out[1] = n.y; out[2] = n.z; }
static void unpack_uv(uint32_t val, float* u, float* v)
{
    *v = (float)((val & 0xffff0000u) >> 16) / 16383.99999f * 20.0f - 10.0f;
    *u = (float)(val & 0x0000ffffu) / 16383.99999f * 20.0f - 10.0f;
}
void oracle_unpack_uv(uint32_t v, float out[2]) { unpack_uv(v, &out[0], &out[1]); }

/* helper.h:12-28 (Ray Tracing Gems ch. 6) */
static float offset_axis(float p, float n)
{
    const float origin = 1.0f / 32.0f;
    const float float_scale = 1.0f / 65536.0f;
    const float int_scale = 256.0f;
    int32_t of_i = (int32_t)(int_scale * n);
    uint32_t bits = asuint_f(p) + (uint32_t)((p < 0) ? -of_i : of_i);
    float p_i = asfloat_u(bits);
    return fabsf(p) < origin ? p + float_scale * n : p_i;
}
static v3 offset_ray(v3 p, v3 n) { return V(offset_axis(p.x, n.x), offset_axis(p.y, n.y), offset_axis(p.z, n.z)); }
void oracle_offset_ray(const float p[3], const float n[3], float out[3])
{
    v3 r = offset_ray(vload(p), vload(n));
    out[0] = r.x; out[1] = r.y; out[2] = r.z;
}

/* helper.h:31-39 */
static v3 interp3(v3 a1, v3 a2, v3 a3, float bx, float by)
{
    float w = (1.0f - bx) - by;
    return V((a1.x * w + a2.x * bx) + a3.x * by, (a1.y * w + a2.y * bx) + a3.y * by,
             (a1.z * w + a2.z * bx) + a3.z * by);
}

/* helper.h:41-50: columns tangent, binormal, normal */
typedef struct { v3 t, b, n; } Frame;
static Frame tangent_space(v3 normal)
{
    v3 helper = V(1.0f, 0.0f, 0.0f);
    if (fabsf(normal.x) > 0.99f) helper = V(0.0f, 0.0f, 1.0f);
    Frame f;
    f.t = vnormalize(vcross(normal, helper));
    f.b = vnormalize(vcross(normal, f.t));
    f.n = normal;
    return f;
}
static v3 frame_to_world(const Frame* f, v3 w)
{
    return V((f->t.x * w.x + f->b.x * w.y) + f->n.x * w.z, (f->t.y * w.x + f->b.y * w.y) + f->n.y * w.z,
             (f->t.z * w.x + f->b.z * w.y) + f->n.z * w.z);
}

/* helper.h:73-79 */
static v3 sample_hemisphere_cosine(float ux, float uy)
{
    float cosTheta = sqrtf(fsat(ux));
    float sinTheta = sqrtf(fsat(1.0f - cosTheta * cosTheta));
    float phi = TWO_PI_F * uy;
    float s, c;
    own_sincos(phi, &s, &c);
    return V(c * sinTheta, s * sinTheta, cosTheta + 1e-6f);
}

/* ------------------------------------------------------------------------- */
/* ray.h:19-33 (the C++ twin; HLSL min/max as fminf/fmaxf) */
int oracle_intersect_ray_box(const float o[3], const float inv[3], const float pmin[3],
                             const float pmax[3], float* t)
{
    float fx = (pmax[0] - o[0]) * inv[0], fy = (pmax[1] - o[1]) * inv[1], fz = (pmax[2] - o[2]) * inv[2];
    float nx = (pmin[0] - o[0]) * inv[0], ny = (pmin[1] - o[1]) * inv[1], nz = (pmin[2] - o[2]) * inv[2];
    float tmaxx = fmaxf(fx, nx), tmaxy = fmaxf(fy, ny), tmaxz = fmaxf(fz, nz);
    float tminx = fminf(fx, nx), tminy = fminf(fy, ny), tminz = fminf(fz, nz);
    float t1 = fminf(tmaxx, fminf(tmaxy, tmaxz));
    float t0 = fmaxf(fmaxf(tminx, fmaxf(tminy, tminz)), 0.0f);
    *t = t0;
    return t1 >= t0;
}

/* raytracing.h:36-88 (Möller–Trumbore with the reference's thresholds) */
static int ray_triangle(v3 orig, v3 dir, v3 v0, v3 e0, v3 e1, float* t, float* bu, float* bv)
{
    *t = 1e9f;
    v3 pvec = vcross(dir, e1);
    float det = vdot(e0, pvec);
    if (fabsf(det) < 1e-6f) return 0;
    float invDet = 1.0f / det;
    v3 tvec = vsub(orig, v0);
    float u = vdot(tvec, pvec) * invDet;
    if (u < 0.0f || u > 1.0f) return 0;
    v3 qvec = vcross(tvec, e0);
    float v = vdot(dir, qvec) * invDet;
    if (v < 0.0f || (u + v) > 1.0f) return 0;
    *t = vdot(e1, qvec) * invDet;
    if (*t < 1e-6f) return 0;
    *bu = u;
    *bv = v;
    return 1;
}
int oracle_ray_triangle(const float o[3], const float d[3], const float v0[3], const float e0[3],
                        const float e1[3], float* t, float* u, float* v)
{
    *u = 0.0f; *v = 0.0f;
    return ray_triangle(vload(o), vload(d), vload(v0), vload(e0), vload(e1), t, u, v);
}

/* raytracing.h:134-153 */
typedef struct { v3 v0, e0, e1; int ok; } Tri;
static Tri get_triangle(const OracleScene* s, uint32_t inst, uint32_t prim)
{
    Tri r;
    memset(&r, 0, sizeof(r));
    if (inst >= s->numInstances) return r;
    const InstanceConstants* ic = &s->instances[inst];
    uint32_t base = (uint32_t)ic->indexOffset + prim * 3u;
    if ((uint64_t)base + 2 >= s->numIndices) return r;
    uint32_t i0 = s->ib[base], i1 = s->ib[base + 1], i2 = s->ib[base + 2];
    if (i0 >= s->numVertices || i1 >= s->numVertices || i2 >= s->numVertices) return r;
    r.v0 = mat_mul_point(&ic->objectToWorld, vload(s->vb[i0].position), 1.0f);
    r.e0 = vsub(mat_mul_point(&ic->objectToWorld, vload(s->vb[i1].position), 1.0f), r.v0);
    r.e1 = vsub(mat_mul_point(&ic->objectToWorld, vload(s->vb[i2].position), 1.0f), r.v0);
    r.ok = 1;
    return r;
}

/* The pruning rule of the GPU closest-hit traversal: an inner node whose
 * entry distance exceeds the best hit by more than a relative 2^-12 is
 * skipped (it cannot hold a strictly closer triangle). */
#define PRUNE_SCALE (1.0f + 0x1p-12f)

/* raytracing.h:198-247 */
static int closest_hit(const OracleScene* s, v3 o, float tmax, v3 d, Hit* hit, int prune,
                       unsigned long long* nInner, unsigned long long* nLeaf)
{
    float inv[3] = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    float oo[3] = {o.x, o.y, o.z};
    float minHit = 1e9f;
    int found = 0;
    uint32_t node = 0;
    uint64_t cap = 2ull * s->numNodes + 2;
    uint64_t visits = 0;
    while (node != INVALID_INDEX) {
        if (node >= s->numNodes || ++visits > cap) break;
        const BVHNode* n = &s->nodes[node];
        uint32_t inst = (uint32_t)n->instId;
        float boxT = 1e9f;
        if (inst != INVALID_INDEX) {
            (*nLeaf)++;
            uint32_t prim = asuint_f(n->minBounds[0]);
            Tri tri = get_triangle(s, inst, prim);
            float t = 0.0f, bu = 0.0f, bv = 0.0f;
            int isect = tri.ok && ray_triangle(o, d, tri.v0, tri.e0, tri.e1, &t, &bu, &bv);
            if (isect && (t < tmax) && (t < minHit)) {
                minHit = t;
                hit->t = t;
                hit->bary[0] = bu;
                hit->bary[1] = bv;
                hit->instId = inst;
                hit->primId = prim;
                found = 1;
            }
            node = (uint32_t)n->nodeOffset;
            continue;
        }
        (*nInner)++;
        if (oracle_intersect_ray_box(oo, inv, n->minBounds, n->maxBounds, &boxT)) {
            if (boxT > tmax || (prune && boxT > minHit * PRUNE_SCALE)) {
                node = (uint32_t)n->nodeOffset;
                continue;
            }
            ++node;
            continue;
        }
        node = (uint32_t)n->nodeOffset;
    }
    return found;
}

/* raytracing.h:249-286 */
static int any_hit(const OracleScene* s, v3 o, float tmax, v3 d, Hit* hit, unsigned long long* nInner,
                   unsigned long long* nLeaf)
{
    float inv[3] = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    float oo[3] = {o.x, o.y, o.z};
    uint32_t node = 0;
    uint64_t cap = 2ull * s->numNodes + 2;
    uint64_t visits = 0;
    while (node != INVALID_INDEX) {
        if (node >= s->numNodes || ++visits > cap) break;
        const BVHNode* n = &s->nodes[node];
        uint32_t inst = (uint32_t)n->instId;
        float boxT = 1e9f;
        if (inst != INVALID_INDEX) {
            (*nLeaf)++;
            uint32_t prim = asuint_f(n->minBounds[0]);
            Tri tri = get_triangle(s, inst, prim);
            float t = 1e9f, bu, bv;
            int isect = tri.ok && ray_triangle(o, d, tri.v0, tri.e0, tri.e1, &t, &bu, &bv);
            hit->t = t;
            if (isect && (t < tmax)) {
                hit->instId = inst;
                hit->primId = prim;
                return 1;
            }
        } else {
            (*nInner)++;
            if (oracle_intersect_ray_box(oo, inv, n->minBounds, n->maxBounds, &boxT)) {
                if (boxT > tmax) {
                    node = (uint32_t)n->nodeOffset;
                    continue;
                }
                ++node;
                continue;
            }
        }
        node = (uint32_t)n->nodeOffset;
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Helpers of the GPU traversal replay below (not a reference algorithm): for
 * an inner node n the children are L = n+1 and R = escape(L), the implicit
 * tree of the depth-first layout.  A full stack falls back to the stackless
 * loops. */
#define WIDE_STACK 64
static int node_is_leaf(const OracleScene* s, uint32_t c) { return (uint32_t)s->nodes[c].instId != INVALID_INDEX; }

static void pair_children(const OracleScene* s, uint32_t n, uint32_t* L, uint32_t* R)
{
    *L = n + 1 < s->numNodes ? n + 1 : INVALID_INDEX;
    *R = INVALID_INDEX;
    if (*L != INVALID_INDEX) {
        uint32_t r = (uint32_t)s->nodes[*L].nodeOffset;
        *R = r < s->numNodes ? r : INVALID_INDEX;
    }
}

static int leaf_test(const OracleScene* s, uint32_t leaf, v3 o, v3 d, float* t, float* bu, float* bv, uint32_t* inst,
                     uint32_t* prim)
{
    const BVHNode* n = &s->nodes[leaf];
    *inst = (uint32_t)n->instId;
    *prim = asuint_f(n->minBounds[0]);
    Tri tri = get_triangle(s, *inst, *prim);
    *t = 1e9f;
    if (!tri.ok) {
        *t = NAN;
        return 0;
    }
    return ray_triangle(o, d, tri.v0, tri.e0, tri.e1, t, bu, bv);
}

static void stackless_closest_from(const OracleScene* s, v3 o, float tmax, v3 d, const float inv[3], uint32_t node, float* minHit,
                                   uint32_t* best, Hit* hit, int* found, unsigned long long* nI, unsigned long long* nL)
{
    float oo[3] = {o.x, o.y, o.z};
    uint64_t cap = 2ull * s->numNodes + 2, visits = 0;
    while (node != INVALID_INDEX) {
        if (node >= s->numNodes || ++visits > cap) break;
        const BVHNode* n = &s->nodes[node];
        if ((uint32_t)n->instId != INVALID_INDEX) {
            (*nL)++;
            float t, bu = 0, bv = 0;
            uint32_t iid, pid;
            if (leaf_test(s, node, o, d, &t, &bu, &bv, &iid, &pid) && t < tmax && (t < *minHit || (t == *minHit && node < *best))) {
                *minHit = t;
                *best = node;
                hit->t = t; hit->bary[0] = bu; hit->bary[1] = bv; hit->instId = iid; hit->primId = pid;
                *found = 1;
            }
            node = (uint32_t)n->nodeOffset;
            continue;
        }
        (*nI)++;
        float boxT;
        if (oracle_intersect_ray_box(oo, inv, n->minBounds, n->maxBounds, &boxT) && !(boxT > tmax) &&
            !(boxT > *minHit * PRUNE_SCALE)) {
            ++node;
            continue;
        }
        node = (uint32_t)n->nodeOffset;
    }
}

/* The GPU's 4-wide traversal (csrc/traverse.cuh), replayed over the binary
 * tree.  A 4-wide node is a binary inner node P at even depth; its entries, in
 * order, are for each binary child c of P: c itself when it is a leaf
 * (tested without a box, except at the root, whose box gates it), otherwise
 * c's two children, an inner one with its
 * own box and a leaf one gated by c's box.  One step processes a node: all
 * entry boxes first (pruned against the best hit at the node's entry), then
 * the leaves that passed in order; closest hit sorts the inner candidates by
 * entry distance with the GPU's compare-exchange network, continues with the
 * nearest and pushes the others farthest first; any hit keeps the
 * depth-first order.  Refs: W_LEAF marks a leaf (W_NOBOX: without a box);
 * inner refs are binary node indices here. */
#define W_LEAF 0x80000000u
#define W_NOBOX 0x40000000u

static void wide_entries(const OracleScene* s, uint32_t P, uint32_t ref[4], uint32_t gate[4])
{
    for (int k = 0; k < 4; ++k) {
        ref[k] = INVALID_INDEX;
        gate[k] = INVALID_INDEX;
    }
    int e = 0;
    uint32_t child[2];
    pair_children(s, P, &child[0], &child[1]);
    for (int k = 0; k < 2; ++k) {
        uint32_t c = child[k];
        if (c == INVALID_INDEX) continue;
        if (node_is_leaf(s, c)) {
            /* at the root, gated by the root's box (the reference tests it first) */
            if (P == 0) {
                ref[e] = c | W_LEAF;
                gate[e++] = 0;
            } else {
                ref[e++] = c | W_LEAF | W_NOBOX;
            }
            continue;
        }
        uint32_t g[2];
        pair_children(s, c, &g[0], &g[1]);
        for (int j = 0; j < 2; ++j) {
            if (g[j] == INVALID_INDEX) continue;
            if (node_is_leaf(s, g[j])) {
                ref[e] = g[j] | W_LEAF;
                gate[e] = c;
            } else {
                ref[e] = g[j];
                gate[e] = g[j];
            }
            ++e;
        }
    }
}

static void wide_cswap(float* t, uint32_t* r, int a, int b)
{
    if (t[b] < t[a]) {
        float x = t[a]; t[a] = t[b]; t[b] = x;
        uint32_t y = r[a]; r[a] = r[b]; r[b] = y;
    }
}

static int wide_closest(const OracleScene* s, v3 o, float tmax, v3 d, Hit* hit, unsigned long long* nI, unsigned long long* nL)
{
    float inv[3] = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    float oo[3] = {o.x, o.y, o.z};
    float minHit = 1e9f;
    uint32_t best = INVALID_INDEX; /* node index of the best hit's leaf: ties go to the first in depth-first order */
    int found = 0;
    if (s->numNodes == 0) return 0;
    uint32_t stackN[WIDE_STACK];
    float stackT[WIDE_STACK];
    int sp = 0;
    uint32_t cur = node_is_leaf(s, 0) ? (W_LEAF | W_NOBOX) : 0, steps = 0;
    for (;;) {
        if (cur != INVALID_INDEX) {
            if (++steps > s->numNodes + 1u) break;
            if (cur & W_LEAF) {
                (*nL)++;
                float t, bu = 0, bv = 0;
                uint32_t iid, pid, leaf = cur & ~(W_LEAF | W_NOBOX);
                if (leaf_test(s, leaf, o, d, &t, &bu, &bv, &iid, &pid) && t < tmax && (t < minHit || (t == minHit && leaf < best))) {
                    minHit = t;
                    best = leaf;
                    hit->t = t; hit->bary[0] = bu; hit->bary[1] = bv; hit->instId = iid; hit->primId = pid;
                    found = 1;
                }
                cur = INVALID_INDEX;
            } else {
                if (cur >= s->numNodes) break;
                (*nI)++;
                uint32_t ref[4], gate[4];
                wide_entries(s, cur, ref, gate);
                float bt[4];
                int pass[4];
                float lim0 = minHit * PRUNE_SCALE;
                for (int k = 0; k < 4; ++k) {
                    bt[k] = 0.0f;
                    pass[k] = 0;
                    if (ref[k] == INVALID_INDEX) continue;
                    if (ref[k] & W_NOBOX) {
                        pass[k] = 1;
                        continue;
                    }
                    const BVHNode* b = &s->nodes[gate[k]];
                    pass[k] = oracle_intersect_ray_box(oo, inv, b->minBounds, b->maxBounds, &bt[k]) && !(bt[k] > tmax) &&
                              !(bt[k] > lim0);
                }
                float ct[4];
                uint32_t cr[4];
                for (int k = 0; k < 4; ++k) {
                    ct[k] = INFINITY;
                    cr[k] = INVALID_INDEX;
                    if (!pass[k]) continue;
                    if (ref[k] & W_LEAF) {
                        (*nL)++;
                        float t, bu = 0, bv = 0;
                        uint32_t iid, pid, leaf = ref[k] & ~(W_LEAF | W_NOBOX);
                        if (leaf_test(s, leaf, o, d, &t, &bu, &bv, &iid, &pid) && t < tmax && (t < minHit || (t == minHit && leaf < best))) {
                            minHit = t;
                            best = leaf;
                            hit->t = t; hit->bary[0] = bu; hit->bary[1] = bv; hit->instId = iid; hit->primId = pid;
                            found = 1;
                        }
                    } else {
                        ct[k] = bt[k];
                        cr[k] = ref[k];
                    }
                }
                wide_cswap(ct, cr, 0, 1);
                wide_cswap(ct, cr, 2, 3);
                wide_cswap(ct, cr, 0, 2);
                wide_cswap(ct, cr, 1, 3);
                wide_cswap(ct, cr, 1, 2);
                float lim = minHit * PRUNE_SCALE;
                cur = (cr[0] != INVALID_INDEX && !(ct[0] > lim)) ? cr[0] : INVALID_INDEX;
                for (int k = 3; k >= 1; --k) {
                    if (cr[k] == INVALID_INDEX || ct[k] > lim) continue;
                    if (sp < WIDE_STACK) {
                        stackN[sp] = cr[k];
                        stackT[sp] = ct[k];
                        ++sp;
                    } else {
                        stackless_closest_from(s, o, tmax, d, inv, 0, &minHit, &best, hit, &found, nI, nL);
                        return found;
                    }
                }
            }
        }
        if (cur == INVALID_INDEX) {
            float lim = minHit * PRUNE_SCALE;
            while (sp > 0) {
                --sp;
                if (!(stackT[sp] > lim)) {
                    cur = stackN[sp];
                    break;
                }
            }
            if (cur == INVALID_INDEX) break;
        }
    }
    return found;
}

static int wide_any(const OracleScene* s, v3 o, float tmax, v3 d, Hit* hit, unsigned long long* nI, unsigned long long* nL)
{
    float inv[3] = {1.0f / d.x, 1.0f / d.y, 1.0f / d.z};
    float oo[3] = {o.x, o.y, o.z};
    if (s->numNodes == 0) return 0;
    uint32_t stackN[WIDE_STACK];
    int sp = 0;
    uint32_t cur = node_is_leaf(s, 0) ? (W_LEAF | W_NOBOX) : 0, steps = 0;
    for (;;) {
        if (cur != INVALID_INDEX && !(cur & W_LEAF)) {
            if (++steps > s->numNodes + 1u || cur >= s->numNodes) return 0;
            (*nI)++;
            uint32_t ref[4], gate[4];
            wide_entries(s, cur, ref, gate);
            int pass[4];
            for (int k = 0; k < 4; ++k) {
                pass[k] = 0;
                if (ref[k] == INVALID_INDEX) continue;
                if (ref[k] & W_NOBOX) {
                    pass[k] = 1;
                    continue;
                }
                const BVHNode* b = &s->nodes[gate[k]];
                float bt;
                pass[k] = oracle_intersect_ray_box(oo, inv, b->minBounds, b->maxBounds, &bt) && !(bt > tmax);
            }
            uint32_t first = INVALID_INDEX;
            for (int k = 3; k >= 0; --k) {
                if (!pass[k]) continue;
                if (first != INVALID_INDEX) {
                    if (sp < WIDE_STACK) {
                        stackN[sp++] = first;
                    } else {
                        /* the reference's stackless loop from the root */
                        uint32_t node = 0;
                        uint64_t cap = 2ull * s->numNodes + 2, visits = 0;
                        while (node != INVALID_INDEX) {
                            if (node >= s->numNodes || ++visits > cap) break;
                            const BVHNode* n = &s->nodes[node];
                            if ((uint32_t)n->instId != INVALID_INDEX) {
                                (*nL)++;
                                float t, bu, bv;
                                uint32_t iid, pid;
                                int is = leaf_test(s, node, o, d, &t, &bu, &bv, &iid, &pid);
                                hit->t = t;
                                if (is && t < tmax) {
                                    hit->instId = iid;
                                    hit->primId = pid;
                                    return 1;
                                }
                            } else {
                                (*nI)++;
                                float bt;
                                if (oracle_intersect_ray_box(oo, inv, n->minBounds, n->maxBounds, &bt) && !(bt > tmax)) {
                                    ++node;
                                    continue;
                                }
                            }
                            node = (uint32_t)n->nodeOffset;
                        }
                        return 0;
                    }
                }
                first = ref[k];
            }
            cur = first;
        }
        for (;;) {
            if (cur == INVALID_INDEX) {
                if (sp == 0) return 0;
                cur = stackN[--sp];
            }
            if (!(cur & W_LEAF)) break;
            (*nL)++;
            float t, bu, bv;
            uint32_t iid, pid;
            int is = leaf_test(s, cur & ~(W_LEAF | W_NOBOX), o, d, &t, &bu, &bv, &iid, &pid);
            hit->t = t;
            if (is && t < tmax) {
                hit->instId = iid;
                hit->primId = pid;
                return 1;
            }
            cur = INVALID_INDEX;
        }
    }
}

/* The GPU's closest-hit kernels with deferred leaf tests (csrc/traverse.cuh:
 * closest_defer_*), replayed for ONE warp of 32 lanes that takes every ray of
 * [0, n) from one work chunk, as the kernels do when the queue chunk is at
 * least n.  Per warp iteration:
 *   1. lanes without a query take the next rays in lane order;
 *   2. when at least DEFER_LANES lanes have pending leaves, or a lane with
 *      pending leaves has nothing current or fewer than 4 free slots, every
 *      lane with pending leaves tests its latest one;
 *   3. each lane with a query processes its current node when it has room
 *      for four more pending leaves (passing leaves join the list, inner
 *      candidates as in wide_closest), then pops when nothing is current,
 *      and finishes when nothing is current and no leaf is pending.
 * Results equal wide_closest's; the node and test counts are the warp's. */
#define DEFER_CAP 12
#define DEFER_LANES 16
typedef struct {
    int have, done;
    uint32_t ray;
    v3 o, d;
    float inv[3], oo[3], tmax, minHit;
    uint32_t best, cur, steps;
    int sp, np, found;
    uint32_t stackN[WIDE_STACK];
    float stackT[WIDE_STACK];
    uint32_t pend[DEFER_CAP];
    Hit hit;
} WarpLane;

static void warp_leaf(const OracleScene* s, WarpLane* L, uint32_t leaf)
{
    float t, bu = 0, bv = 0;
    uint32_t iid, pid;
    if (leaf_test(s, leaf, L->o, L->d, &t, &bu, &bv, &iid, &pid) && t < L->tmax &&
        (t < L->minHit || (t == L->minHit && leaf < L->best))) {
        L->minHit = t;
        L->best = leaf;
        L->hit.t = t; L->hit.bary[0] = bu; L->hit.bary[1] = bv; L->hit.instId = iid; L->hit.primId = pid;
        L->found = 1;
    }
}

/* closest_defer_node: returns 1 when the query ended early */
static int warp_node(const OracleScene* s, WarpLane* L, unsigned long long* nI, unsigned long long* nL)
{
    uint32_t cur = L->cur;
    if (++L->steps > s->numNodes + 1u) return 1;
    if (cur & W_LEAF) {
        L->pend[L->np++] = cur & ~(W_LEAF | W_NOBOX);
        L->cur = INVALID_INDEX;
        return 0;
    }
    if (cur >= s->numNodes) return 1;
    (*nI)++;
    uint32_t ref[4], gate[4];
    wide_entries(s, cur, ref, gate);
    float lim0 = L->minHit * PRUNE_SCALE, ct[4];
    uint32_t cr[4];
    for (int k = 0; k < 4; ++k) {
        ct[k] = INFINITY;
        cr[k] = INVALID_INDEX;
        if (ref[k] == INVALID_INDEX) continue;
        float bt = 0.0f;
        int pass = 1;
        if (!(ref[k] & W_NOBOX)) {
            const BVHNode* b = &s->nodes[gate[k]];
            pass = oracle_intersect_ray_box(L->oo, L->inv, b->minBounds, b->maxBounds, &bt) && !(bt > L->tmax) && !(bt > lim0);
        }
        if (!pass) continue;
        if (ref[k] & W_LEAF) {
            L->pend[L->np++] = ref[k] & ~(W_LEAF | W_NOBOX);
        } else {
            ct[k] = bt;
            cr[k] = ref[k];
        }
    }
    wide_cswap(ct, cr, 0, 1);
    wide_cswap(ct, cr, 2, 3);
    wide_cswap(ct, cr, 0, 2);
    wide_cswap(ct, cr, 1, 3);
    wide_cswap(ct, cr, 1, 2);
    L->cur = cr[0];
    for (int k = 3; k >= 1; --k) {
        if (cr[k] == INVALID_INDEX) continue;
        if (L->sp < WIDE_STACK) {
            L->stackN[L->sp] = cr[k];
            L->stackT[L->sp] = ct[k];
            L->sp++;
        } else {
            stackless_closest_from(s, L->o, L->tmax, L->d, L->inv, 0, &L->minHit, &L->best, &L->hit, &L->found, nI, nL);
            L->cur = INVALID_INDEX;
            L->sp = 0;
            return 1;
        }
    }
    return 0;
}

int oracle_trace_warp(const OracleScene* s, const Ray* rays, uint32_t n, Hit* hits, uint8_t* found,
                      unsigned long long* counters)
{
    WarpLane* lane = (WarpLane*)calloc(32, sizeof(WarpLane));
    if (!lane) return -1;
    unsigned long long nI = 0, nL = 0;
    const uint32_t root = s->numNodes == 0 ? INVALID_INDEX : node_is_leaf(s, 0) ? (W_LEAF | W_NOBOX) : 0;
    uint32_t next = 0;
    for (;;) {
        /* 1. new queries, in lane order */
        for (int l = 0; l < 32; ++l) {
            WarpLane* L = &lane[l];
            if (L->have || next >= n) continue;
            const Ray* r = &rays[next];
            memset(L, 0, sizeof(*L));
            L->have = 1;
            L->ray = next++;
            L->o = V(r->o.x, r->o.y, r->o.z);
            L->d = V(r->d.x, r->d.y, r->d.z);
            L->oo[0] = r->o.x; L->oo[1] = r->o.y; L->oo[2] = r->o.z;
            L->inv[0] = 1.0f / r->d.x; L->inv[1] = 1.0f / r->d.y; L->inv[2] = 1.0f / r->d.z;
            L->tmax = r->o.w;
            L->minHit = 1e9f;
            L->best = INVALID_INDEX;
            L->cur = root;
            L->hit.t = 1e9f;
            L->hit.instId = INVALID_INDEX;
            L->hit.primId = INVALID_INDEX;
        }
        int any = 0;
        for (int l = 0; l < 32; ++l) any |= lane[l].have;
        if (!any) break;
        /* 2. deferred leaf tests */
        int waiting = 0, stuck = 0;
        for (int l = 0; l < 32; ++l) {
            WarpLane* L = &lane[l];
            if (!L->have || !L->np) continue;
            waiting++;
            if (L->cur == INVALID_INDEX || L->np > DEFER_CAP - 4) stuck = 1;
        }
        if (waiting && (waiting >= DEFER_LANES || stuck)) {
            for (int l = 0; l < 32; ++l) {
                WarpLane* L = &lane[l];
                if (!L->have || !L->np) continue;
                L->np--;
                nL++;
                warp_leaf(s, L, L->pend[L->np]);
            }
        }
        /* 3. node step, pop, finish */
        for (int l = 0; l < 32; ++l) {
            WarpLane* L = &lane[l];
            if (!L->have) continue;
            int fin = 0;
            if (L->cur != INVALID_INDEX && L->np <= DEFER_CAP - 4) {
                fin = warp_node(s, L, &nI, &nL);
                if (fin) L->np = 0;
            }
            if (!fin && L->cur == INVALID_INDEX) {
                float lim = L->minHit * PRUNE_SCALE;
                while (L->sp > 0) {
                    --L->sp;
                    if (!(L->stackT[L->sp] > lim)) {
                        L->cur = L->stackN[L->sp];
                        break;
                    }
                }
            }
            if (!fin && !(L->cur == INVALID_INDEX && L->np == 0)) continue;
            Hit h = L->hit;
            if (!L->found) {
                h.instId = INVALID_INDEX;
                h.primId = INVALID_INDEX;
                h.t = 1e9f;
                h.bary[0] = 0.0f;
                h.bary[1] = 0.0f;
            }
            hits[L->ray] = h;
            if (found) found[L->ray] = (uint8_t)L->found;
            L->have = 0;
        }
    }
    free(lane);
    counters[0] = nI;
    counters[1] = nL;
    return 0;
}

int oracle_trace(const OracleScene* s, const Ray* rays, uint32_t n, Hit* hits, uint8_t* found, int mode,
                 int prune, unsigned long long* counters, int nthreads)
{
    unsigned long long totInner = 0, totLeaf = 0;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 1024) reduction(+ : totInner, totLeaf)
#endif
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        const Ray* r = &rays[i];
        v3 o = V(r->o.x, r->o.y, r->o.z), d = V(r->d.x, r->d.y, r->d.z);
        Hit h;
        memset(&h, 0, sizeof(h));
        h.instId = INVALID_INDEX;
        h.primId = INVALID_INDEX;
        unsigned long long ni = 0, nl = 0;
        int f;
        if (prune == 2) f = mode == 1 ? wide_any(s, o, r->o.w, d, &h, &ni, &nl) : wide_closest(s, o, r->o.w, d, &h, &ni, &nl);
        else f = mode == 1 ? any_hit(s, o, r->o.w, d, &h, &ni, &nl) : closest_hit(s, o, r->o.w, d, &h, prune, &ni, &nl);
        if (!f) {
            h.instId = INVALID_INDEX;
            h.primId = INVALID_INDEX;
            if (mode != 1) h.t = 1e9f;
        }
        hits[i] = h;
        if (found) found[i] = (uint8_t)f;
        totInner += ni;
        totLeaf += nl;
    }
    if (counters) {
        counters[0] = totInner;
        counters[1] = totLeaf;
    }
    return 0;
}

int oracle_intersect_fp64(const OracleScene* s, const Ray* rays, const uint32_t* instIds, const uint32_t* primIds,
                          uint32_t n, double* tout, double* uout, double* vout)
{
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        tout[i] = NAN; uout[i] = NAN; vout[i] = NAN;
        uint32_t inst = instIds[i], prim = primIds[i];
        if (inst >= s->numInstances) continue;
        const InstanceConstants* ic = &s->instances[inst];
        uint32_t base = (uint32_t)ic->indexOffset + prim * 3u;
        if ((uint64_t)base + 2 >= s->numIndices) continue;
        double P[3][3];
        for (int k = 0; k < 3; ++k) {
            uint32_t vi = s->ib[base + k];
            const float* p = s->vb[vi].position;
            const float* m = ic->objectToWorld.m;
            for (int a = 0; a < 3; ++a)
                P[k][a] = (double)m[0 * 4 + a] * p[0] + (double)m[1 * 4 + a] * p[1] + (double)m[2 * 4 + a] * p[2] +
                          (double)m[3 * 4 + a];
        }
        double o[3] = {rays[i].o.x, rays[i].o.y, rays[i].o.z}, d[3] = {rays[i].d.x, rays[i].d.y, rays[i].d.z};
        double e0[3], e1[3], tv[3];
        for (int a = 0; a < 3; ++a) { e0[a] = P[1][a] - P[0][a]; e1[a] = P[2][a] - P[0][a]; tv[a] = o[a] - P[0][a]; }
        double pv[3] = {d[1] * e1[2] - d[2] * e1[1], d[2] * e1[0] - d[0] * e1[2], d[0] * e1[1] - d[1] * e1[0]};
        double det = e0[0] * pv[0] + e0[1] * pv[1] + e0[2] * pv[2];
        double qv[3] = {tv[1] * e0[2] - tv[2] * e0[1], tv[2] * e0[0] - tv[0] * e0[2], tv[0] * e0[1] - tv[1] * e0[0]};
        uout[i] = (tv[0] * pv[0] + tv[1] * pv[1] + tv[2] * pv[2]) / det;
        vout[i] = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) / det;
        tout[i] = (e1[0] * qv[0] + e1[1] * qv[1] + e1[2] * qv[2]) / det;
    }
    return 0;
}

/* Conditioning of the same formula: for each ray, the magnitude scale of
 * u, v and t, (sum of |terms| of the numerator + |value| x sum of |terms| of
 * det) / |det|, where the terms are the products the triple products
 * expand into.  A rounding error of relative size e in each product shifts
 * the value by at most about e x scale, so scale x 2^-52 bounds what FP64
 * itself resolves and scale x 2^-44 what a double-float evaluation does. */
int oracle_intersect_terms_fp64(const OracleScene* s, const Ray* rays, const uint32_t* instIds, const uint32_t* primIds,
                                uint32_t n, double* scale3)
{
#ifdef _OPENMP
#pragma omp parallel for schedule(static)
#endif
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        scale3[3 * i + 0] = NAN; scale3[3 * i + 1] = NAN; scale3[3 * i + 2] = NAN;
        uint32_t inst = instIds[i], prim = primIds[i];
        if (inst >= s->numInstances) continue;
        const InstanceConstants* ic = &s->instances[inst];
        uint32_t base = (uint32_t)ic->indexOffset + prim * 3u;
        if ((uint64_t)base + 2 >= s->numIndices) continue;
        double P[3][3];
        for (int k = 0; k < 3; ++k) {
            const float* p = s->vb[s->ib[base + k]].position;
            const float* m = ic->objectToWorld.m;
            for (int a = 0; a < 3; ++a)
                P[k][a] = (double)m[0 * 4 + a] * p[0] + (double)m[1 * 4 + a] * p[1] + (double)m[2 * 4 + a] * p[2] +
                          (double)m[3 * 4 + a];
        }
        double o[3] = {rays[i].o.x, rays[i].o.y, rays[i].o.z}, d[3] = {rays[i].d.x, rays[i].d.y, rays[i].d.z};
        double e0[3], e1[3], tv[3];
        for (int a = 0; a < 3; ++a) { e0[a] = P[1][a] - P[0][a]; e1[a] = P[2][a] - P[0][a]; tv[a] = o[a] - P[0][a]; }
        double pv[3] = {d[1] * e1[2] - d[2] * e1[1], d[2] * e1[0] - d[0] * e1[2], d[0] * e1[1] - d[1] * e1[0]};
        double qv[3] = {tv[1] * e0[2] - tv[2] * e0[1], tv[2] * e0[0] - tv[0] * e0[2], tv[0] * e0[1] - tv[1] * e0[0]};
        double apv[3] = {fabs(d[1] * e1[2]) + fabs(d[2] * e1[1]), fabs(d[2] * e1[0]) + fabs(d[0] * e1[2]),
                         fabs(d[0] * e1[1]) + fabs(d[1] * e1[0])};
        double aqv[3] = {fabs(tv[1] * e0[2]) + fabs(tv[2] * e0[1]), fabs(tv[2] * e0[0]) + fabs(tv[0] * e0[2]),
                         fabs(tv[0] * e0[1]) + fabs(tv[1] * e0[0])};
        double det = e0[0] * pv[0] + e0[1] * pv[1] + e0[2] * pv[2];
        double nDet = fabs(e0[0]) * apv[0] + fabs(e0[1]) * apv[1] + fabs(e0[2]) * apv[2];
        double nU = fabs(tv[0]) * apv[0] + fabs(tv[1]) * apv[1] + fabs(tv[2]) * apv[2];
        double nV = fabs(d[0]) * aqv[0] + fabs(d[1]) * aqv[1] + fabs(d[2]) * aqv[2];
        double nT = fabs(e1[0]) * aqv[0] + fabs(e1[1]) * aqv[1] + fabs(e1[2]) * aqv[2];
        double u = (tv[0] * pv[0] + tv[1] * pv[1] + tv[2] * pv[2]) / det;
        double v = (d[0] * qv[0] + d[1] * qv[1] + d[2] * qv[2]) / det;
        double t = (e1[0] * qv[0] + e1[1] * qv[1] + e1[2] * qv[2]) / det;
        double ad = fabs(det);
        scale3[3 * i + 0] = (nU + fabs(u) * nDet) / ad;
        scale3[3 * i + 1] = (nV + fabs(v) * nDet) / ad;
        scale3[3 * i + 2] = (nT + fabs(t) * nDet) / ad;
    }
    return 0;
}

/* ------------------------------------------------------------------------- */
/* lights.h */
typedef struct {
    v3 pointOnLight; float pdf;
    v3 normal; float area;
    v3 L; float distToLight;
} LightSample;

/* lights.h:34-46 */
static void frisvad(v3 n, v3* b1, v3* b2)
{
    if (n.z < -0.9999999f) {
        *b1 = V(0.0f, -1.0f, 0.0f);
        *b2 = V(-1.0f, 0.0f, 0.0f);
        return;
    }
    const float a = 1.0f / (1.0f + n.z);
    const float b = -n.x * n.y * a;
    *b1 = V(1.0f - n.x * n.x * a, b, -n.x);
    *b2 = V(b, 1.0f - n.y * n.y * a, -n.y);
}

/* lights.h:59-89.  As in the reference, the local 'u' (the second frisvad
 * axis) shadows the random sample, and the result is the rotated local
 * vector without the sphere centre. */
static v3 sample_sphere_solid_angle(const UniformLight* l, v3 hitPoint)
{
    v3 c = V(l->points[1].x, l->points[1].y, l->points[1].z);
    float r = l->points[0].x;
    v3 w = vsub(c, hitPoint);
    float distanceToCenter = vlength(w);
    w = vscale(w, 1.0f / distanceToCenter);
    float q = sqrtf(1.0f - (r / distanceToCenter) * (r / distanceToCenter));
    v3 v, u;
    frisvad(w, &v, &u);
    float r0 = u.x;
    float r1 = u.y;
    float theta = ACOSF(1.0f - r0 + r0 * q);
    float phi = TWO_PI_F * r1;
    float st, ct, sp, cp;
    own_sincos(theta, &st, &ct);
    own_sincos(phi, &sp, &cp);
    /* lights.h:48-56 */
    v3 local;
    local.x = 5.0f * sp * st;
    local.z = -5.0f * sp * ct;
    local.y = 5.0f * cp;
    /* mul(local, float3x3(u, w, v)) */
    return V((local.x * u.x + local.y * w.x) + local.z * v.x, (local.x * u.y + local.y * w.y) + local.z * v.y,
             (local.x * u.z + local.y * w.z) + local.z * v.z);
}

typedef struct {
    v3 o, x, y, z;
    float z0, z0sq, x0, y0, y0sq, x1, y1, y1sq, b0, b1, b0sq, k, S;
} SphQuad;

/* lights.h:102-166 */
static SphQuad sphquad_init(const UniformLight* l, v3 o)
{
    SphQuad q;
    v3 p0 = V(l->points[0].x, l->points[0].y, l->points[0].z);
    v3 p1 = V(l->points[1].x, l->points[1].y, l->points[1].z);
    v3 p3 = V(l->points[3].x, l->points[3].y, l->points[3].z);
    v3 ex = vsub(p1, p0);
    v3 ey = vsub(p3, p0);
    v3 s = p0;
    float exl = vlength(ex);
    float eyl = vlength(ey);
    q.o = o;
    q.x = vdivs(ex, exl);
    q.y = vdivs(ey, eyl);
    q.z = vcross(q.x, q.y);
    v3 d = vsub(s, o);
    q.z0 = vdot(d, q.z);
    if (q.z0 > 0) {
        q.z = vscale(q.z, -1.0f);
        q.z0 *= -1.0f;
    }
    q.z0sq = q.z0 * q.z0;
    q.x0 = vdot(d, q.x);
    q.y0 = vdot(d, q.y);
    q.x1 = q.x0 + exl;
    q.y1 = q.y0 + eyl;
    q.y0sq = q.y0 * q.y0;
    q.y1sq = q.y1 * q.y1;
    v3 v00 = V(q.x0, q.y0, q.z0), v01 = V(q.x0, q.y1, q.z0), v10 = V(q.x1, q.y0, q.z0), v11 = V(q.x1, q.y1, q.z0);
    v3 n0 = vnormalize(vcross(v00, v10));
    v3 n1 = vnormalize(vcross(v10, v11));
    v3 n2 = vnormalize(vcross(v11, v01));
    v3 n3 = vnormalize(vcross(v01, v00));
    float g0 = ACOSF(-vdot(n0, n1));
    float g1 = ACOSF(-vdot(n1, n2));
    float g2 = ACOSF(-vdot(n2, n3));
    float g3 = ACOSF(-vdot(n3, n0));
    q.b0 = n0.z;
    q.b1 = n2.z;
    q.b0sq = q.b0 * q.b0;
    q.k = TWO_PI_F - g2 - g3;
    q.S = g0 + g1 - q.k;
    return q;
}

/* lights.h:168-194 */
static v3 sphquad_sample(const SphQuad* q, float u, float v)
{
    float au = u * q->S + q->k;
    float sau, cau;
    own_sincos(au, &sau, &cau);
    float fu = (cau * q->b0 - q->b1) / sau;
    float cu = 1.0f / sqrtf(fu * fu + q->b0sq) * (fu > 0 ? 1.0f : -1.0f);
    cu = fminf(fmaxf(cu, -1.0f), 1.0f);
    float xu = -(cu * q->z0) / sqrtf(1.0f - cu * cu);
    xu = fminf(fmaxf(xu, q->x0), q->x1);
    float d = sqrtf(xu * xu + q->z0sq);
    float h0 = q->y0 / sqrtf(d * d + q->y0sq);
    float h1 = q->y1 / sqrtf(d * d + q->y1sq);
    float hv = h0 + v * (h1 - h0);
    float hv2 = hv * hv;
    float eps = 1e-5f;
    float yv = (hv < 1.0f - eps) ? (hv * d) / sqrtf(1.0f - hv2) : q->y1;
    return vadd(vadd(vadd(q->o, vscale(q->x, xu)), vscale(q->y, yv)), vscale(q->z, q->z0));
}

/* lights.h:196-219 */
static void concentric_sample_disk(float ux, float uy, float* ox, float* oy)
{
    float x = 2.0f * ux - 1.0f;
    float y = 2.0f * uy - 1.0f;
    if (x == 0 && y == 0) { *ox = 0.0f; *oy = 0.0f; return; }
    float theta, r;
    if (fabsf(x) > fabsf(y)) {
        r = x;
        theta = PI_OVER_4_F * (y / x);
    } else {
        r = y;
        theta = PI_OVER_2_F - PI_OVER_4_F * (x / y);
    }
    float s, c;
    own_sincos(theta, &s, &c);
    *ox = r * c;
    *oy = r * s;
}

/* lights.h:230-282 */
static v3 light_normal(const UniformLight* l, v3 hitPoint)
{
    v3 norm = V(0.0f, 0.0f, 0.0f);
    if (l->type == 0) {
        v3 e1 = V(l->points[1].x - l->points[0].x, l->points[1].y - l->points[0].y, l->points[1].z - l->points[0].z);
        v3 e2 = V(l->points[3].x - l->points[0].x, l->points[3].y - l->points[0].y, l->points[3].z - l->points[0].z);
        norm = vneg(vnormalize(vcross(e1, e2)));
    } else if (l->type == 1) {
        norm = V(l->normal.x, l->normal.y, l->normal.z);
    } else if (l->type == 2) {
        norm = vnormalize(vsub(hitPoint, V(l->points[1].x, l->points[1].y, l->points[1].z)));
    }
    return norm;
}
static float light_area(const UniformLight* l)
{
    float area = 0.0f;
    if (l->type == 0) {
        v3 e1 = V(l->points[1].x - l->points[0].x, l->points[1].y - l->points[0].y, l->points[1].z - l->points[0].z);
        v3 e2 = V(l->points[3].x - l->points[0].x, l->points[3].y - l->points[0].y, l->points[3].z - l->points[0].z);
        area = vlength(vcross(e1, e2));
    } else if (l->type == 1) {
        area = PI_F * l->points[0].x * l->points[0].x;
    } else if (l->type == 2) {
        area = FOUR_PI_F * l->points[0].x * l->points[0].x;
    }
    return area;
}
static void fill_light_data(const UniformLight* l, v3 hitPoint, LightSample* ls)
{
    ls->area = light_area(l);
    ls->normal = light_normal(l, hitPoint);
    v3 toLight = vsub(ls->pointOnLight, hitPoint);
    float len = vlength(toLight);
    ls->L = vdivs(toLight, len);
    ls->distToLight = len;
}

/* lights.h:284-340 */
static LightSample sample_light(const UniformLight* l, v3 hitPoint, float ux, float uy)
{
    LightSample ls;
    memset(&ls, 0, sizeof(ls));
    if (l->type == 0) {
        SphQuad q = sphquad_init(l, hitPoint);
        ls.pointOnLight = sphquad_sample(&q, ux, uy);
        fill_light_data(l, hitPoint, &ls);
        ls.pdf = ls.distToLight * ls.distToLight / (-vdot(ls.L, ls.normal) * ls.area);
    } else if (l->type == 1) {
        float pdx, pdy;
        concentric_sample_disk(ux, uy, &pdx, &pdy);
        float x = l->points[0].x * pdx;
        float y = l->points[0].x * pdy;
        v3 c = V(l->points[1].x, l->points[1].y, l->points[1].z);
        v3 ax = V(l->points[2].x, l->points[2].y, l->points[2].z);
        v3 ay = V(l->points[3].x, l->points[3].y, l->points[3].z);
        ls.pointOnLight = vadd(vadd(c, vscale(ax, x)), vscale(ay, y));
        fill_light_data(l, hitPoint, &ls);
        ls.pdf = ls.distToLight * ls.distToLight / (-vdot(ls.L, ls.normal) * ls.area);
    } else if (l->type == 2) {
        ls.pointOnLight = sample_sphere_solid_angle(l, hitPoint);
        fill_light_data(l, hitPoint, &ls);
        v3 c = V(l->points[1].x, l->points[1].y, l->points[1].z);
        float distanceToCenter = vlength(vsub(c, hitPoint));
        float sinThetaMax2 = l->points[0].x * l->points[0].x / (distanceToCenter * distanceToCenter);
        float cosThetaMax = sqrtf(fmaxf(0.0f, 1.0f - sinThetaMax2));
        ls.pdf = 1.0f / (TWO_PI_F * (1.0f - cosThetaMax));
    }
    return ls;
}

/* lights.h:284-340 for one light, exported for function-level checks:
 * out = {pointOnLight[3], pdf, normal[3], area, L[3], distToLight}. */
void oracle_sample_light(const UniformLight* l, const float hitPoint[3], float u0, float u1, float out[12])
{
    LightSample ls = sample_light(l, V(hitPoint[0], hitPoint[1], hitPoint[2]), u0, u1);
    out[0] = ls.pointOnLight.x; out[1] = ls.pointOnLight.y; out[2] = ls.pointOnLight.z; out[3] = ls.pdf;
    out[4] = ls.normal.x; out[5] = ls.normal.y; out[6] = ls.normal.z; out[7] = ls.area;
    out[8] = ls.L.x; out[9] = ls.L.y; out[10] = ls.L.z; out[11] = ls.distToLight;
}

/* ------------------------------------------------------------------------- */
/* Native materials (project-defined argument record StrelkaMaterialArgs). */
typedef struct {
    v3 normal, geom_normal, position;
    float u, v; /* text_coords[0].xy */
} ShadeState;

typedef struct {
    v3 base;
    float roughness;
    v3 emission;
    float ior;
    uint32_t tex;
    int fn;
} Mat;

static float srgb_to_linear(uint8_t c)
{
    float x = (float)c / 255.0f;
    return x <= 0.04045f ? x / 12.92f : powf((x + 0.055f) / 1.055f, 2.4f);
}

/* mdl_runtime.hlsl:125-140 then a bilinear REPEAT fetch of the sRGB texels
 * decoded to linear (the sampler of texturemanager.h:24-44 on an
 * R8G8B8A8_SRGB image, texturemanager.cpp:79). */
static float g_srgb_lut[256];
static int g_srgb_init = 0;
static void srgb_lut_init(void)
{
    if (g_srgb_init) return;
    for (int i = 0; i < 256; ++i) g_srgb_lut[i] = srgb_to_linear((uint8_t)i);
    g_srgb_init = 1;
}
static inline int wrapi(int i, int n) { int r = i % n; return r < 0 ? r + n : r; }
void oracle_tex_lookup(const OracleTexture* t, float u, float v, float out[4])
{
    srgb_lut_init();
    float W = (float)t->width, H = (float)t->height;
    /* apply_smootherstep_filter */
    float rx = u * W + 0.5f, ry = v * H + 0.5f;
    float ui = floorf(rx), vi = floorf(ry);
    float uf = rx - ui, vf = ry - vi;
    uf = uf * uf * uf * (uf * (uf * 6.0f - 15.0f) + 10.0f);
    vf = vf * vf * vf * (vf * (vf * 6.0f - 15.0f) + 10.0f);
    rx = ui + uf;
    ry = vi + vf;
    float cu = (rx - 0.5f) / W, cv = (ry - 0.5f) / H;
    /* bilinear, REPEAT */
    float x = cu * W - 0.5f, y = cv * H - 0.5f;
    float x0f = floorf(x), y0f = floorf(y);
    float fx = x - x0f, fy = y - y0f;
    int x0 = wrapi((int)x0f, (int)t->width), y0 = wrapi((int)y0f, (int)t->height);
    int x1 = wrapi(x0 + 1, (int)t->width), y1 = wrapi(y0 + 1, (int)t->height);
    const uint8_t* p00 = t->rgba8 + 4 * ((size_t)y0 * t->width + x0);
    const uint8_t* p10 = t->rgba8 + 4 * ((size_t)y0 * t->width + x1);
    const uint8_t* p01 = t->rgba8 + 4 * ((size_t)y1 * t->width + x0);
    const uint8_t* p11 = t->rgba8 + 4 * ((size_t)y1 * t->width + x1);
    for (int c = 0; c < 4; ++c) {
        float a00 = c < 3 ? g_srgb_lut[p00[c]] : (float)p00[c] / 255.0f;
        float a10 = c < 3 ? g_srgb_lut[p10[c]] : (float)p10[c] / 255.0f;
        float a01 = c < 3 ? g_srgb_lut[p01[c]] : (float)p01[c] / 255.0f;
        float a11 = c < 3 ? g_srgb_lut[p11[c]] : (float)p11[c] / 255.0f;
        float top = a00 + fx * (a10 - a00);
        float bot = a01 + fx * (a11 - a01);
        out[c] = top + fy * (bot - top);
    }
}

/* The native material at argument-block offset argOffset with function id
 * fn, its base colour textured at the shading state's (u, v). */
static int load_material_args(const OracleScene* s, int32_t argOffset, int32_t fn, const ShadeState* st, Mat* m)
{
    if (argOffset < 0 || (uint64_t)argOffset + sizeof(StrelkaMaterialArgs) > s->argBlockBytes) return 0;
    if (fn < 0 || fn >= STRELKA_FN_COUNT) return 0;
    StrelkaMaterialArgs a;
    memcpy(&a, s->argBlock + argOffset, sizeof(a));
    m->base = V(a.base_color[0], a.base_color[1], a.base_color[2]);
    m->roughness = a.roughness;
    m->emission = V(a.emission[0], a.emission[1], a.emission[2]);
    m->ior = a.ior;
    m->tex = a.base_color_texture;
    m->fn = fn;
    if (m->tex != 0) {
        if (m->tex - 1 >= s->numResourceInfos) return 0;
        uint32_t slot = s->resourceInfos[m->tex - 1].gpu_resource_array_start;
        if (slot >= s->numTextures) return 0;
        float texel[4];
        oracle_tex_lookup(&s->textures[slot], st->u, st->v, texel);
        m->base = V(m->base.x * texel[0], m->base.y * texel[1], m->base.z * texel[2]);
    }
    return 1;
}
static int load_material(const OracleScene* s, int32_t materialId, const ShadeState* st, Mat* m)
{
    if (materialId < 0 || (uint32_t)materialId >= s->numMaterials) return 0;
    const MdlMaterial* mm = &s->materials[materialId];
    return load_material_args(s, mm->arg_block_offset, mm->functionId, st, m);
}

/* GGX helpers (Walter et al. 2007) */
static float ggx_d(float alpha, float noh)
{
    float a2 = alpha * alpha;
    float t = noh * noh * (a2 - 1.0f) + 1.0f;
    return a2 / (PI_F * t * t);
}
static float ggx_g1(float alpha, float nov)
{
    float a2 = alpha * alpha;
    return 2.0f * nov / (nov + sqrtf(a2 + (1.0f - a2) * nov * nov));
}
static float mat_alpha(float roughness) { return fmaxf(roughness * roughness, 1e-3f); }
static float schlick_weight(float c) { float m = fsat(1.0f - c); float m2 = m * m; return m2 * m2 * m; }
static float fresnel_dielectric(float cosi, float eta) /* eta = ior_i / ior_t */
{
    float sin2t = eta * eta * (1.0f - cosi * cosi);
    if (sin2t >= 1.0f) return 1.0f;
    float cost = sqrtf(fsat(1.0f - sin2t));
    float rs = (cosi - eta * cost) / (cosi + eta * cost);
    float rp = (eta * cosi - cost) / (eta * cosi + cost);
    return 0.5f * (rs * rs + rp * rp);
}

typedef struct { v3 bsdf_diffuse, bsdf_glossy; float pdf; } EvalOut;
typedef struct { v3 k2, bsdf_over_pdf; float pdf; int event; } SampleOut;

/* BSDF evaluate (mdl_bsdf_scattering_evaluate contract: values include the
 * cosine).  Lambert follows shaders/pathtracer.hlsl:176-185. */
static EvalOut bsdf_evaluate(const Mat* m, const ShadeState* st, v3 k1, v3 k2, float ior1, float ior2)
{
    EvalOut e;
    e.bsdf_diffuse = V(0.0f, 0.0f, 0.0f);
    e.bsdf_glossy = V(0.0f, 0.0f, 0.0f);
    e.pdf = 0.0f;
    v3 N = st->normal;
    if (m->fn == STRELKA_FN_LAMBERT) {
        float c = fsat(vdot(N, k2));
        e.bsdf_diffuse = vscale(m->base, INV_PI_F * c);
        e.pdf = INV_PI_F * (c + 1e-6f);
        return e;
    }
    float nol = vdot(N, k2), nov = vdot(N, k1);
    if (!(nol > 0.0f) || !(nov > 0.0f)) return e;
    v3 h = vnormalize(vadd(k1, k2));
    float noh = fsat(vdot(N, h)), voh = fsat(vdot(k1, h));
    float alpha = mat_alpha(m->roughness);
    float D = ggx_d(alpha, noh);
    float G = ggx_g1(alpha, nov) * ggx_g1(alpha, nol);
    if (m->fn == STRELKA_FN_GGX_CONDUCTOR) {
        float w = schlick_weight(voh);
        v3 F = V(m->base.x + (1.0f - m->base.x) * w, m->base.y + (1.0f - m->base.y) * w, m->base.z + (1.0f - m->base.z) * w);
        float k = D * G / (4.0f * nov);
        e.bsdf_glossy = vscale(F, k);
        e.pdf = D * noh / (4.0f * voh);
    } else {
        float i1 = ior1 < 0.0f ? m->ior : ior1;
        float i2 = ior2 < 0.0f ? m->ior : ior2;
        float F = fresnel_dielectric(voh, i1 / i2);
        float k = F * D * G / (4.0f * nov);
        e.bsdf_glossy = V(k, k, k);
        e.pdf = F * D * noh / (4.0f * voh);
    }
    return e;
}

/* BSDF sample (mdl_bsdf_scattering_sample contract).  Lambert:
 * shaders/pathtracer.hlsl:208-234 with helper.h:41-50,73-79. */
static SampleOut bsdf_sample(const Mat* m, const ShadeState* st, v3 k1, const float xi[4], float ior1, float ior2)
{
    SampleOut so;
    so.k2 = V(0.0f, 0.0f, 0.0f);
    so.bsdf_over_pdf = V(0.0f, 0.0f, 0.0f);
    so.pdf = 0.0f;
    so.event = EV_ABSORB;
    v3 N = st->normal;
    Frame f = tangent_space(N);
    if (m->fn == STRELKA_FN_LAMBERT) {
        v3 w = sample_hemisphere_cosine(xi[0], xi[1]);
        so.k2 = frame_to_world(&f, w);
        so.pdf = INV_PI_F * (fsat(vdot(N, so.k2)) + 1e-6f);
        so.bsdf_over_pdf = m->base;
        so.event = EV_DIFFUSE | EV_REFLECTION;
        return so;
    }
    float nov = vdot(N, k1);
    if (!(nov > 0.0f)) return so;
    float alpha = mat_alpha(m->roughness);
    float a2 = alpha * alpha;
    float cosThetaH = sqrtf((1.0f - xi[0]) / (xi[0] * (a2 - 1.0f) + 1.0f));
    float sinThetaH = sqrtf(fsat(1.0f - cosThetaH * cosThetaH));
    float phi = TWO_PI_F * xi[1];
    float sp, cp;
    own_sincos(phi, &sp, &cp);
    v3 h = frame_to_world(&f, V(cp * sinThetaH, sp * sinThetaH, cosThetaH));
    float voh = vdot(k1, h);
    if (!(voh > 0.0f)) return so;
    float noh = fsat(vdot(N, h));
    float G1v = ggx_g1(alpha, nov);
    if (m->fn == STRELKA_FN_GGX_CONDUCTOR) {
        so.k2 = vsub(vscale(h, 2.0f * voh), k1);
        float nol = vdot(N, so.k2);
        if (!(nol > 0.0f)) return so;
        float w = schlick_weight(voh);
        v3 F = V(m->base.x + (1.0f - m->base.x) * w, m->base.y + (1.0f - m->base.y) * w, m->base.z + (1.0f - m->base.z) * w);
        float G = G1v * ggx_g1(alpha, nol);
        float k = G * voh / (nov * noh);
        so.bsdf_over_pdf = vscale(F, k);
        so.pdf = ggx_d(alpha, noh) * noh / (4.0f * voh);
        so.event = EV_GLOSSY | EV_REFLECTION;
        return so;
    }
    /* rough dielectric */
    float i1 = ior1 < 0.0f ? m->ior : ior1;
    float i2 = ior2 < 0.0f ? m->ior : ior2;
    float eta = i1 / i2;
    float F = fresnel_dielectric(voh, eta);
    float D = ggx_d(alpha, noh);
    if (xi[2] < F) {
        so.k2 = vsub(vscale(h, 2.0f * voh), k1);
        float nol = vdot(N, so.k2);
        if (!(nol > 0.0f)) return so;
        float G = G1v * ggx_g1(alpha, nol);
        float k = G * voh / (nov * noh);
        so.bsdf_over_pdf = V(k, k, k);
        so.pdf = F * D * noh / (4.0f * voh);
        so.event = EV_GLOSSY | EV_REFLECTION;
        return so;
    }
    /* refraction through the microfacet h: k2 = -eta*k1 + (eta*c1 - c2)*h */
    float sin2t = eta * eta * (1.0f - voh * voh);
    float c2 = sqrtf(fsat(1.0f - sin2t));
    float s = eta * voh - c2;
    so.k2 = vadd(vscale(k1, -eta), vscale(h, s));
    so.k2 = vnormalize(so.k2);
    float nol = vdot(N, so.k2);
    if (!(nol < 0.0f)) { so.event = EV_ABSORB; return so; }
    float G = G1v * ggx_g1(alpha, -nol);
    float k = G * voh / (nov * noh);
    so.bsdf_over_pdf = vscale(m->base, k);
    so.pdf = (1.0f - F) * D * noh;
    so.event = EV_GLOSSY | EV_TRANSMISSION;
    return so;
}

/* Exported native materials: the functions the MDL-generated dispatchers
 * (mdl_bsdf_scattering_sample / _evaluate, mdl_edf_emission_intensity,
 * src/materialmanager/mdlHlslCodeGen.cpp:32-81) stand for in this project.
 * state = {normal[3], geom_normal[3], position[3], u, v}. */
static void state_from(const float* st9uv, ShadeState* st)
{
    st->normal = V(st9uv[0], st9uv[1], st9uv[2]);
    st->geom_normal = V(st9uv[3], st9uv[4], st9uv[5]);
    st->position = V(st9uv[6], st9uv[7], st9uv[8]);
    st->u = st9uv[9];
    st->v = st9uv[10];
}
int oracle_material_sample(const OracleScene* s, int32_t argOffset, int32_t fn, const float* state, const float k1[3],
                           const float xi[4], float ior1, float ior2, float k2[3], float bsdfOverPdf[3], float* pdf,
                           int* event)
{
    ShadeState st;
    Mat m;
    state_from(state, &st);
    if (!load_material_args(s, argOffset, fn, &st, &m)) return 0;
    SampleOut so = bsdf_sample(&m, &st, V(k1[0], k1[1], k1[2]), xi, ior1, ior2);
    k2[0] = so.k2.x; k2[1] = so.k2.y; k2[2] = so.k2.z;
    bsdfOverPdf[0] = so.bsdf_over_pdf.x; bsdfOverPdf[1] = so.bsdf_over_pdf.y; bsdfOverPdf[2] = so.bsdf_over_pdf.z;
    *pdf = so.pdf;
    *event = so.event;
    return 1;
}
int oracle_material_evaluate(const OracleScene* s, int32_t argOffset, int32_t fn, const float* state,
                             const float k1[3], const float k2[3], float ior1, float ior2, float diffuse[3],
                             float glossy[3], float* pdf)
{
    ShadeState st;
    Mat m;
    state_from(state, &st);
    if (!load_material_args(s, argOffset, fn, &st, &m)) return 0;
    EvalOut e = bsdf_evaluate(&m, &st, V(k1[0], k1[1], k1[2]), V(k2[0], k2[1], k2[2]), ior1, ior2);
    diffuse[0] = e.bsdf_diffuse.x; diffuse[1] = e.bsdf_diffuse.y; diffuse[2] = e.bsdf_diffuse.z;
    glossy[0] = e.bsdf_glossy.x; glossy[1] = e.bsdf_glossy.y; glossy[2] = e.bsdf_glossy.z;
    *pdf = e.pdf;
    return 1;
}
int oracle_material_emission(const OracleScene* s, int32_t argOffset, int32_t fn, const float* state,
                             float intensity[3])
{
    ShadeState st;
    Mat m;
    state_from(state, &st);
    if (!load_material_args(s, argOffset, fn, &st, &m)) return 0;
    intensity[0] = m.emission.x; intensity[1] = m.emission.y; intensity[2] = m.emission.z;
    return 1;
}

/* ------------------------------------------------------------------------- */
/* Environment light (extension: the reference's miss adds zero).  Lat-long
 * map: u = (atan2(d.x, -d.z)/(2 pi)) + 0.5, v = acos(d.y)/pi; looked up
 * nearest-texel.  atan2 is computed from the own acos. */
static float own_atan2(float y, float x)
{
    float r = sqrtf(x * x + y * y);
    if (r == 0.0f) return 0.0f;
    float a = ACOSF(fminf(fmaxf(x / r, -1.0f), 1.0f));
    return y < 0.0f ? -a : a;
}
static v3 env_lookup(const OracleEnvMap* e, v3 d, int* texel)
{
    float phi = own_atan2(d.x, -d.z);
    float u = phi * (1.0f / TWO_PI_F) + 0.5f;
    float v = ACOSF(fminf(fmaxf(d.y, -1.0f), 1.0f)) * INV_PI_F;
    int x = (int)(u * (float)e->width);
    int y = (int)(v * (float)e->height);
    x = x < 0 ? 0 : (x >= (int)e->width ? (int)e->width - 1 : x);
    y = y < 0 ? 0 : (y >= (int)e->height ? (int)e->height - 1 : y);
    *texel = y * (int)e->width + x;
    const float* p = e->rgba32f + 4 * (size_t)(*texel);
    return V(p[0], p[1], p[2]);
}
/* solid-angle pdf of choosing direction d by sampling a texel proportional
 * to luminance*sin(theta) and a uniform point inside it */
static float env_pdf(const OracleEnvMap* e, int texel, v3 d)
{
    int y = texel / (int)e->width;
    int x = texel - y * (int)e->width;
    const float* mc = e->marginal_cdf;
    const float* cc = e->conditional_cdf + (size_t)y * (e->width + 1);
    float pRow = mc[y + 1] - mc[y];
    float pCol = cc[x + 1] - cc[x];
    float sinTheta = sqrtf(fmaxf(0.0f, 1.0f - d.y * d.y));
    if (!(sinTheta > 0.0f)) return 0.0f;
    float texelSolidAngle = (TWO_PI_F / (float)e->width) * (PI_F / (float)e->height) * sinTheta;
    return pRow * pCol / texelSolidAngle;
}
static int upper_bound_cdf(const float* cdf, int n, float u) /* returns i in [0,n) with cdf[i] <= u < cdf[i+1] */
{
    int lo = 0, hi = n;
    while (lo + 1 < hi) {
        int mid = (lo + hi) >> 1;
        if (cdf[mid] <= u) lo = mid; else hi = mid;
    }
    return lo;
}
static v3 env_sample(const OracleEnvMap* e, float u1, float u2, float* pdf, v3* radiance)
{
    int y = upper_bound_cdf(e->marginal_cdf, (int)e->height, u1);
    const float* cc = e->conditional_cdf + (size_t)y * (e->width + 1);
    int x = upper_bound_cdf(cc, (int)e->width, u2);
    /* position inside the texel from the remaining fractions */
    float fy = (u1 - e->marginal_cdf[y]) / fmaxf(e->marginal_cdf[y + 1] - e->marginal_cdf[y], 1e-30f);
    float fx = (u2 - cc[x]) / fmaxf(cc[x + 1] - cc[x], 1e-30f);
    float v = ((float)y + fsat(fy)) / (float)e->height;
    float u = ((float)x + fsat(fx)) / (float)e->width;
    float theta = v * PI_F;
    float phi = (u - 0.5f) * TWO_PI_F;
    float st, ct, sp, cp;
    own_sincos(theta, &st, &ct);
    own_sincos(phi, &sp, &cp);
    v3 d = V(st * sp, ct, -(st * cp));
    int texel = y * (int)e->width + x;
    const float* p = e->rgba32f + 4 * (size_t)texel;
    *radiance = V(p[0], p[1], p[2]);
    *pdf = env_pdf(e, texel, d);
    return d;
}

/* ------------------------------------------------------------------------- */
/* The path loop, shaders/pathtracerMdl.hlsl */

typedef struct {
    const PathTracerParam* ubo;
    const OracleScene* s;
} Ctx;

/* pathtracerMdl.hlsl:31-92 (+ the environment as one extra light) */
static v3 sample_lights(const Ctx* c, uint32_t* rng, const ShadeState* st, v3* toLight, float* lightPdf, int* valid)
{
    const OracleScene* s = c->s;
    uint32_t numLights = c->ubo->numLights;
    int hasEnv = s->envMap != NULL;
    uint32_t total = numLights + (hasEnv ? 1u : 0u);
    *valid = 1;
    *lightPdf = 0.0f;
    *toLight = V(0.0f, 0.0f, 0.0f);
    if (total == 0) {
        /* numLights == 0 and no environment: the reference reads the zeroed
         * lights[0], gets lightPdf = 0 * (1/0) = NaN and ends the path */
        *valid = 0;
        return V(0.0f, 0.0f, 0.0f);
    }
    uint32_t lightId = (uint32_t)((float)total * oracle_rand(rng));
    float lightSelectionPdf = 1.0f / (float)total;
    v3 result = V(0.0f, 0.0f, 0.0f);
    if (lightId >= numLights && hasEnv) {
        /* environment light */
        float r0 = oracle_rand(rng);
        float r1 = oracle_rand(rng);
        v3 Le;
        float pdf;
        v3 L = env_sample(s->envMap, r0, r1, &pdf, &Le);
        *toLight = L;
        if (vdot(st->normal, L) > 0.0f && pdf > 0.0f && (Le.x != 0 || Le.y != 0 || Le.z != 0)) {
            Ray sr;
            v3 o = offset_ray(st->position, st->geom_normal);
            sr.o.x = o.x; sr.o.y = o.y; sr.o.z = o.z; sr.o.w = 1e9f;
            (void)sr;
            Hit h;
            unsigned long long a = 0, b = 0;
            float vis = any_hit(s, o, 1e9f, L, &h, &a, &b) ? 0.0f : 1.0f;
            *lightPdf = pdf;
            float cs = fsat(vdot(st->normal, L));
            result = V(vis * Le.x * cs, vis * Le.y * cs, vis * Le.z * cs);
        }
        *lightPdf *= lightSelectionPdf;
        return result;
    }
    if (lightId >= s->lightCapacity) { *valid = 0; return result; }
    const UniformLight* light = &s->lights[lightId];
    LightSample ls;
    memset(&ls, 0, sizeof(ls));
    if (light->type >= 0 && light->type <= 2) {
        /* float2(rand(rngState), rand(rngState)) evaluates left to right */
        float r0 = oracle_rand(rng);
        float r1 = oracle_rand(rng);
        ls = sample_light(light, st->position, r0, r1);
    }
    *toLight = ls.L;
    v3 Li = V(light->color.x, light->color.y, light->color.z);
    if (vdot(st->normal, ls.L) > 0.0f && -vdot(ls.L, ls.normal) > 0.0f && (Li.x != 0 && Li.y != 0 && Li.z != 0)) {
        v3 o = offset_ray(st->position, st->geom_normal);
        Hit h;
        memset(&h, 0, sizeof(h));
        unsigned long long a = 0, b = 0;
        float visibility = any_hit(s, o, ls.distToLight, ls.L, &h, &a, &b) ? 0.0f : 1.0f;
        if (visibility == 0.0f) {
            if (h.instId < s->numInstances && s->instances[h.instId].lightId != -1) visibility = 1.0f;
        }
        *lightPdf = ls.pdf;
        float cs = fsat(vdot(st->normal, ls.L));
        result = V(visibility * Li.x * cs, visibility * Li.y * cs, visibility * Li.z * cs);
    }
    *lightPdf *= lightSelectionPdf;
    return result;
}

/* pathtracerMdl.hlsl:94-162 */
static void stratified_optimized(uint32_t sIn, float* rx, float* ry)
{
    const int N = 16, p = 16;
    int m = 4; /* int(sqrt(N * 1.0f)) */
    int n = (N + m - 1) / m;
    int s = (int)oracle_permute(sIn, (uint32_t)N, (uint32_t)p * 0x51633e2du);
    int sx = (int)oracle_permute((uint32_t)(s % m), (uint32_t)m, (uint32_t)p * 0x68bc21ebu);
    int sy = (int)oracle_permute((uint32_t)(s / m), (uint32_t)n, (uint32_t)p * 0x02e5be93u);
    float jx = oracle_randfloat((uint32_t)s, (uint32_t)p * 0x967a889bu);
    float jy = oracle_randfloat((uint32_t)s, (uint32_t)p * 0x368cc8b7u);
    *rx = ((float)sx + ((float)sy + jx) / (float)n) / (float)m;
    *ry = ((float)s + jy) / (float)N;
}
static void stratified1(uint32_t s, uint32_t* rng, float* jx, float* jy)
{
    const uint32_t N = 16;
    int m = 4; /* int(sqrt(N)) */
    int n = ((int)N + m - 1) / m;
    uint32_t x = (s / (uint32_t)n) % (uint32_t)n;
    uint32_t y = (s % (uint32_t)m) % (uint32_t)m;
    float r0 = oracle_rand(rng);
    *jx = ((float)x + ((float)y + r0) / (float)n) / (float)m;
    float r1 = oracle_rand(rng);
    *jy = ((float)y + ((float)x + r1) / (float)m) / (float)n;
}

/* pathtracerMdl.hlsl:165-202 */
static void camera_ray(const PathTracerParam* ubo, uint32_t px, uint32_t py, uint32_t* rng, uint32_t s, v3* o, v3* d)
{
    float ppx = 0.0f, ppy = 0.0f;
    if (ubo->stratifiedSamplingType == 0) {
        ppx = (float)px + 0.5f;
        ppy = (float)py + 0.5f;
    } else if (ubo->stratifiedSamplingType == 1) {
        ppx = (float)px + oracle_rand(rng);
        ppy = (float)py + oracle_rand(rng);
    } else if (ubo->stratifiedSamplingType == 2) {
        float jx, jy;
        stratified1(s, rng, &jx, &jy);
        ppx = (float)px + jx;
        ppy = (float)py + jy;
    } else if (ubo->stratifiedSamplingType == 3) {
        float jx, jy;
        stratified_optimized(s, &jx, &jy);
        ppx = (float)px + jx;
        ppy = (float)py + jy;
    }
    float ndcx = (ppx / (float)ubo->dimension[0]) * 2.0f - 1.0f;
    float ndcy = (ppy / (float)ubo->dimension[1]) * 2.0f - 1.0f;
    float clip[4] = {ndcx, ndcy, 1.0f, 1.0f};
    float view[4];
    mat_mul4(&ubo->clipToView, clip, view);
    float vdir[4] = {view[0], view[1], view[2], 0.0f};
    float wdir[4];
    mat_mul4(&ubo->viewToWorld, vdir, wdir);
    float orig[4] = {0.0f, 0.0f, 0.0f, 1.0f};
    float wo[4];
    mat_mul4(&ubo->viewToWorld, orig, wo);
    *o = V(wo[0], wo[1], wo[2]);
    *d = vnormalize(V(wdir[0], wdir[1], wdir[2]));
}

/* generateCameraRay exported for function-level checks: out = {o[3], d[3]}. */
void oracle_camera_ray(const PathTracerParam* p, uint32_t px, uint32_t py, uint32_t* rng, uint32_t s, float out[6])
{
    v3 o, d;
    camera_ray(p, px, py, rng, s, &o, &d);
    out[0] = o.x; out[1] = o.y; out[2] = o.z; out[3] = d.x; out[4] = d.y; out[5] = d.z;
}

/* pathtracerMdl.hlsl:204-404 */
static v3 path_trace(const Ctx* c, uint32_t px, uint32_t py, uint32_t* rng, uint32_t sIdx)
{
    const PathTracerParam* ubo = c->ubo;
    const OracleScene* s = c->s;
    v3 finalColor = V(0.0f, 0.0f, 0.0f);
    v3 throughput = V(1.0f, 1.0f, 1.0f);
    int depth = 0;
    const int maxDepth = (int)ubo->maxDepth;
    v3 ro, rd;
    camera_ray(ubo, px, py, rng, sIdx, &ro, &rd);
    float rtmax = 1e9f;
    int specularBounce = 0;
    int inside = 0;
    float lastBsdfPdf = 0.0f; /* environment MIS only */
    unsigned long long ci = 0, cl = 0;
    while (depth < maxDepth) {
        Hit hit;
        memset(&hit, 0, sizeof(hit));
        if (closest_hit(s, ro, rtmax, rd, &hit, 0, &ci, &cl)) {
            const InstanceConstants* ic = &s->instances[hit.instId];
            if (ic->lightId != -1 && (depth == 0 || specularBounce)) {
                if ((uint32_t)ic->lightId >= s->lightCapacity) break;
                const UniformLight* L = &s->lights[ic->lightId];
                finalColor = vadd(finalColor, vmul(throughput, V(L->color.x, L->color.y, L->color.z)));
                break;
            }
            if (ic->lightId != -1) {
                /* a diffuse bounce reached a light's emitter: the reference reads
                 * mdlMaterials[-1] here; this restatement ends the path */
                break;
            }
            uint32_t base = (uint32_t)ic->indexOffset + hit.primId * 3u;
            uint32_t i0 = s->ib[base + 0], i1 = s->ib[base + 1], i2 = s->ib[base + 2];
            v3 p0 = mat_mul_point(&ic->objectToWorld, vload(s->vb[i0].position), 1.0f);
            v3 p1 = mat_mul_point(&ic->objectToWorld, vload(s->vb[i1].position), 1.0f);
            v3 p2 = mat_mul_point(&ic->objectToWorld, vload(s->vb[i2].position), 1.0f);
            v3 geomNormal = vnormalize(vcross(vsub(p1, p0), vsub(p2, p0)));
            v3 n0 = mat_mul_dir3(&ic->normalMatrix, unpack_normal(s->vb[i0].normal));
            v3 n1 = mat_mul_dir3(&ic->normalMatrix, unpack_normal(s->vb[i1].normal));
            v3 n2 = mat_mul_dir3(&ic->normalMatrix, unpack_normal(s->vb[i2].normal));
            float bx = hit.bary[0], by = hit.bary[1];
            v3 worldPosition = interp3(p0, p1, p2, bx, by);
            v3 worldNormal = vnormalize(interp3(n0, n1, n2, bx, by));
            float sign = inside ? -1.0f : 1.0f;
            geomNormal = vscale(geomNormal, sign);
            worldNormal = vscale(worldNormal, sign);
            float uv0[2], uv1[2], uv2[2];
            unpack_uv(s->vb[i0].uv, &uv0[0], &uv0[1]);
            unpack_uv(s->vb[i1].uv, &uv1[0], &uv1[1]);
            unpack_uv(s->vb[i2].uv, &uv2[0], &uv2[1]);
            float w = (1.0f - bx) - by;
            ShadeState st;
            st.u = (uv0[0] * w + uv1[0] * bx) + uv2[0] * by;
            st.v = (uv0[1] * w + uv1[1] * bx) + uv2[1] * by;
            if (ubo->debug == 1) {
                return V((worldNormal.x + 1.0f) * 0.5f, (worldNormal.y + 1.0f) * 0.5f, (worldNormal.z + 1.0f) * 0.5f);
            }
            st.normal = worldNormal;
            st.geom_normal = geomNormal;
            st.position = worldPosition;
            Mat m;
            if (!load_material(s, ic->materialId, &st, &m)) break;
            const float ior1 = inside ? -1.0f : 1.0f; /* BSDF_USE_MATERIAL_IOR = -1 */
            const float ior2 = inside ? 1.0f : -1.0f;
            v3 k1 = vneg(rd);
            /* EDF: intensity * edf with edf = 1 */
            finalColor = vadd(finalColor, vmul(vmul(throughput, m.emission), V(1.0f, 1.0f, 1.0f)));
            v3 toLight;
            float lightPdf = 0.0f;
            int lvalid;
            v3 radiance = sample_lights(c, rng, &st, &toLight, &lightPdf, &lvalid);
            if (!lvalid) break;
            if (vhasnan(radiance) || isnan(lightPdf)) break;
            const int nextEventValid = ((vdot(toLight, st.geom_normal) > 0.0f) != (inside != 0)) && lightPdf != 0.0f;
            if (nextEventValid) {
                v3 radianceOverPdf = vdivs(radiance, lightPdf);
                EvalOut ev = bsdf_evaluate(&m, &st, k1, toLight, ior1, ior2);
                if (vhasnan(ev.bsdf_diffuse) || vhasnan(ev.bsdf_glossy)) break;
                if (ev.pdf > 0.0f) {
                    const float misWeight = (lightPdf == 0.0f) ? 1.0f : lightPdf / (lightPdf + ev.pdf);
                    v3 wgt = vscale(vmul(throughput, radianceOverPdf), misWeight);
                    finalColor = vadd(finalColor, vmul(wgt, ev.bsdf_diffuse));
                    finalColor = vadd(finalColor, vmul(wgt, ev.bsdf_glossy));
                }
            }
            float xi[4];
            xi[0] = oracle_rand(rng);
            xi[1] = oracle_rand(rng);
            xi[2] = oracle_rand(rng);
            xi[3] = oracle_rand(rng);
            SampleOut so = bsdf_sample(&m, &st, k1, xi, ior1, ior2);
            if (so.event == EV_ABSORB) break;
            specularBounce = (so.event & EV_SPECULAR) != 0;
            inside = (so.event & EV_TRANSMISSION) != 0;
            v3 rayDirectionNext = so.k2;
            v3 rayOriginNext = offset_ray(st.position, vscale(st.geom_normal, inside ? -1.0f : 1.0f));
            throughput = vmul(throughput, so.bsdf_over_pdf);
            lastBsdfPdf = so.pdf;
            if (depth > 3) {
                float p = fmaxf(throughput.x, fmaxf(throughput.y, throughput.z));
                if (oracle_rand(rng) > p) break;
                float sc = 1.0f / (p + 1e-5f);
                throughput = vscale(throughput, sc);
            }
            ro = rayOriginNext;
            rtmax = 1e9f;
            rd = rayDirectionNext;
        } else {
            /* miss: the reference adds throughput * 0 */
            if (s->envMap) {
                int texel;
                v3 Le = env_lookup(s->envMap, rd, &texel);
                float misW = 1.0f;
                if (depth > 0 && !specularBounce) {
                    uint32_t total = ubo->numLights + 1u;
                    float lp = env_pdf(s->envMap, texel, rd) * (1.0f / (float)total);
                    misW = lastBsdfPdf / (lastBsdfPdf + lp);
                }
                finalColor = vadd(finalColor, vscale(vmul(throughput, Le), misW));
            } else {
                finalColor = vadd(finalColor, vmul(throughput, V(0.0f, 0.0f, 0.0f)));
            }
            break;
        }
        ++depth;
    }
    return finalColor;
}

int oracle_pathtrace_range(const PathTracerParam* p, const OracleScene* s, float* sampleBuffer, uint64_t first,
                           uint64_t count, int nthreads)
{
    Ctx c;
    c.ubo = p;
    c.s = s;
    srgb_lut_init();
    uint64_t total = (uint64_t)(uint32_t)p->dimension[0] * (uint32_t)p->dimension[1] * (uint32_t)p->spp;
    uint64_t end = first + count;
    if (end > total) end = total;
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int64_t idx = (int64_t)first; idx < (int64_t)end; ++idx) {
        /* pathtracerMdl.hlsl:406-423 */
        uint32_t W = (uint32_t)p->dimension[0];
        uint32_t spp = (uint32_t)p->spp;
        uint32_t px = (uint32_t)idx / spp % W;
        uint32_t py = (uint32_t)idx / spp / W;
        uint32_t sampleNum = (uint32_t)idx % spp;
        uint32_t seedFrame = p->frameNumber * spp + sampleNum;
        uint32_t rng = oracle_init_rng(px, py, W, seedFrame);
        v3 color = path_trace(&c, px, py, &rng, seedFrame);
        sampleBuffer[(idx - first) * 3 + 0] = color.x;
        sampleBuffer[(idx - first) * 3 + 1] = color.y;
        sampleBuffer[(idx - first) * 3 + 2] = color.z;
    }
    return 0;
}

int oracle_pathtrace(const PathTracerParam* p, const OracleScene* s, float* sampleBuffer, int nthreads)
{
    uint64_t total = (uint64_t)(uint32_t)p->dimension[0] * (uint32_t)p->dimension[1] * (uint32_t)p->spp;
    return oracle_pathtrace_range(p, s, sampleBuffer, 0, total, nthreads);
}

/* ------------------------------------------------------------------------- */
/* reduction.hlsl:9-32 */
int oracle_reduce(const PathTracerParam* p, const float* sb, float* out)
{
    uint32_t n = (uint32_t)p->dimension[0] * (uint32_t)p->dimension[1];
    int spp = p->spp;
    float invSpp = 1.0f / (float)spp;
    for (uint32_t i = 0; i < n; ++i) {
        float r = 0.0f, g = 0.0f, b = 0.0f;
        for (int s = 0; s < spp; ++s) {
            size_t k = ((size_t)i * spp + s) * 3;
            r += invSpp * sb[k + 0];
            g += invSpp * sb[k + 1];
            b += invSpp * sb[k + 2];
        }
        out[4 * (size_t)i + 0] = r;
        out[4 * (size_t)i + 1] = g;
        out[4 * (size_t)i + 2] = b;
        out[4 * (size_t)i + 3] = 1.0f;
    }
    return 0;
}

/* accumulation.hlsl:86-97 */
int oracle_accumulate(const AccumulationParam* p, const float* in, const float* hist, float* out)
{
    size_t n = (size_t)(uint32_t)p->dimension[0] * (uint32_t)p->dimension[1];
    float wHistory = (float)p->iteration / (float)(p->iteration + 1u);
    float wNew = 1.0f / (float)(p->iteration + 1u);
    for (size_t i = 0; i < n; ++i) {
        for (int c = 0; c < 3; ++c) out[4 * i + c] = hist[4 * i + c] * wHistory + in[4 * i + c] * wNew;
        out[4 * i + 3] = 1.0f;
    }
    return 0;
}

/* tonemap.hlsl:9-64 */
static v3 aces_fitted(v3 c)
{
    /* ACESInputMat / ACESOutputMat rows, tonemap.hlsl:11-23 */
    v3 a = V((0.59719f * c.x + 0.35458f * c.y) + 0.04823f * c.z, (0.07600f * c.x + 0.90834f * c.y) + 0.01566f * c.z,
             (0.02840f * c.x + 0.13383f * c.y) + 0.83777f * c.z);
    float v[3] = {a.x, a.y, a.z}, r[3];
    for (int i = 0; i < 3; ++i) {
        float aa = v[i] * (v[i] + 0.0245786f) - 0.000090537f;
        float bb = v[i] * (0.983729f * v[i] + 0.4329510f) + 0.238081f;
        r[i] = aa / bb;
    }
    v3 o = V((1.60475f * r[0] + -0.53108f * r[1]) + -0.07367f * r[2], (-0.10208f * r[0] + 1.10813f * r[1]) + -0.00605f * r[2],
             (-0.00327f * r[0] + -0.07276f * r[1]) + 1.07602f * r[2]);
    return V(fsat(o.x), fsat(o.y), fsat(o.z));
}
static float aces_film1(float x)
{
    const float a = 2.51f, b = 0.03f, c = 2.43f, d = 0.59f, e = 0.14f;
    return fsat((x * (a * x + b)) / (x * (c * x + d) + e));
}
static v3 reinhard(v3 c)
{
    float lum = (c.x * 0.299f + c.y * 0.587f) + c.z * 0.114f;
    float r = lum / (lum + 1.0f);
    float k = r / lum;
    return V(c.x * k, c.y * k, c.z * k);
}
int oracle_tonemap(const Tonemapparam* p, const float* in, float* out)
{
    size_t n = (size_t)(uint32_t)p->dimension[0] * (uint32_t)p->dimension[1];
    for (size_t i = 0; i < n; ++i) {
        v3 c = V(in[4 * i], in[4 * i + 1], in[4 * i + 2]);
        v3 r;
        if (p->tonemapperType == 0) r = reinhard(c);
        else if (p->tonemapperType == 1) r = aces_fitted(c);
        else if (p->tonemapperType == 2) r = V(aces_film1(c.x), aces_film1(c.y), aces_film1(c.z));
        else continue; /* the reference leaves the output untouched */
        out[4 * i] = r.x;
        out[4 * i + 1] = r.y;
        out[4 * i + 2] = r.z;
        out[4 * i + 3] = 1.0f;
    }
    return 0;
}

/* upscalepass.hlsl:9-21: uv = (pixel + 0.5) * invDimension; SampleLevel with
 * a linear filter and clamp-to-edge addressing (upscalepass.cpp:12-38):
 * texel-space position uv * size - 0.5, the four clamped neighbours and the
 * fractional weights, blended in a fixed order; rgb kept, alpha 1. */
int oracle_upscale(const Upscalepassparam* p, const float* in, uint32_t inW, uint32_t inH, float* out)
{
    const uint32_t W = (uint32_t)p->dimension[0], H = (uint32_t)p->dimension[1];
    for (uint32_t py = 0; py < H; ++py)
        for (uint32_t px = 0; px < W; ++px) {
            const float u = ((float)px + 0.5f) * p->invDimension[0];
            const float v = ((float)py + 0.5f) * p->invDimension[1];
            const float fx = u * (float)inW - 0.5f;
            const float fy = v * (float)inH - 0.5f;
            const float flx = floorf(fx), fly = floorf(fy);
            const float a = fx - flx, b = fy - fly;
            int x0 = (int)flx, y0 = (int)fly, x1 = x0 + 1, y1 = y0 + 1;
            const int mx = (int)inW - 1, my = (int)inH - 1;
            x0 = x0 < 0 ? 0 : (x0 > mx ? mx : x0);
            x1 = x1 < 0 ? 0 : (x1 > mx ? mx : x1);
            y0 = y0 < 0 ? 0 : (y0 > my ? my : y0);
            y1 = y1 < 0 ? 0 : (y1 > my ? my : y1);
            const float w00 = (1.0f - a) * (1.0f - b), w10 = a * (1.0f - b), w01 = (1.0f - a) * b, w11 = a * b;
            const float* c00 = in + 4 * ((size_t)y0 * inW + x0);
            const float* c10 = in + 4 * ((size_t)y0 * inW + x1);
            const float* c01 = in + 4 * ((size_t)y1 * inW + x0);
            const float* c11 = in + 4 * ((size_t)y1 * inW + x1);
            float* o = out + 4 * ((size_t)py * W + px);
            for (int c = 0; c < 3; ++c) o[c] = ((c00[c] * w00 + c10[c] * w10) + c01[c] * w01) + c11[c] * w11;
            o[3] = 1.0f;
        }
    return 0;
}

/* mdl_runtime.hlsl:24-75.  Load(offs) of a ByteAddressBuffer reads the word
 * at offs with the two low bits ignored; past the end it reads 0 (robust
 * buffer access).  asdouble(lo, hi) puts the first word low; the bool reader
 * tests the byte at offs within its aligned word. */
static uint32_t mdl_word(const uint8_t* b, uint64_t bytes, uint32_t offs)
{
    uint64_t a = offs & ~3u;
    uint32_t w = 0;
    if (b && a + 4 <= bytes) memcpy(&w, b + a, 4);
    return w;
}

void oracle_mdl_read(const uint8_t* b, uint64_t bytes, const uint32_t* offs, const uint32_t* kinds, uint32_t n,
                     uint64_t* out)
{
    for (uint32_t i = 0; i < n; ++i) {
        const uint32_t o = offs[i];
        uint64_t r = 0;
        switch (kinds[i]) {
            case 0: case 2: case 3: r = mdl_word(b, bytes, o); break;
            case 1: r = (uint64_t)mdl_word(b, bytes, o) | ((uint64_t)mdl_word(b, bytes, o + 4u) << 32); break;
            case 4: r = (mdl_word(b, bytes, o & ~3u) & (0xffu << (8u * (o & 3u)))) != 0u; break;
            default: r = 0; break;
        }
        out[i] = r;
    }
}
