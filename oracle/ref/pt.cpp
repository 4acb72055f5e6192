// pt.cpp -- the reference's path-tracing shader, compiled on the host.
//
// TEST INFRASTRUCTURE (oracle/build_ref.sh builds it into oracle/_ref/): the
// reference's own shaders/pathtracerMdl.hlsl with raytracing.h, ray.h,
// random.h, helper.h, pack.h and lights.h, rewritten only syntactically by
// oracle/hlsl2cpp.py, over the HLSL shim of shim.h.  Its outputs check the
// oracle's restatement (oracle/oracle.c) function by function and image by
// image.
//
// The one part supplied here instead of taken from the reference is what the
// reference generates at run time with the MDL SDK (absent): the material
// dispatch functions mdl_bsdf_scattering_* / mdl_edf_emission_*
// (src/materialmanager/mdlHlslCodeGen.cpp:32-81).  They call the project's
// native materials in the oracle (oracle_material_*), so materials are not
// pinned by this library; everything else on the path is the reference's
// code.  The reference adds nothing on a miss, so scenes with an
// environment light are outside what this library can check.
#include <cstdio>
#include <cstring>
#ifdef _OPENMP
#include <omp.h>
#endif

#include "shim.h"

#include "../oracle.h"

thread_local int ref_ub = 0;

namespace ref_pt {
#include "pathtracerparam.h"
#include "random.h"
// Globals the reference's helpers name before pathtracerMdl.hlsl declares
// them (HLSL resolves global names regardless of order; C++ needs them
// declared first).
extern ConstantBuffer<PathTracerParam> ubo;
static Texture2D<float4> mdl_textures_2d[1];
static SamplerState mdl_sampler_tex;
#include "mdl_types.hlsl"

// ---- stand-ins for the MDL-generated dispatch functions -------------------
static const OracleScene* g_scene = nullptr;

static void state_array(const Shading_state_material& s, float st[11])
{
    st[0] = s.normal.x; st[1] = s.normal.y; st[2] = s.normal.z;
    st[3] = s.geom_normal.x; st[4] = s.geom_normal.y; st[5] = s.geom_normal.z;
    st[6] = s.position.x; st[7] = s.position.y; st[8] = s.position.z;
    st[9] = s.text_coords[0].x; st[10] = s.text_coords[0].y;
}
// The generated init functions take the state by value (`in`), so whatever
// they compute does not reach the caller's state.
static void mdl_edf_emission_init(int, Shading_state_material) {}
static void mdl_bsdf_scattering_init(int, Shading_state_material) {}
static void mdl_edf_emission_evaluate(int, Edf_evaluate_data& d, Shading_state_material)
{
    d.edf = float3(1.0f);
}
static float3 mdl_edf_emission_intensity(int fn, Shading_state_material s)
{
    float st[11], e[3] = {0.0f, 0.0f, 0.0f};
    state_array(s, st);
    if (!oracle_material_emission(g_scene, (int32_t)s.arg_block_offset, fn, st, e)) ref_ub = 1;
    return float3(e[0], e[1], e[2]);
}
static void mdl_bsdf_scattering_evaluate(int fn, Bsdf_evaluate_data& d, Shading_state_material s)
{
    float st[11], k1[3] = {d.k1.x, d.k1.y, d.k1.z}, k2[3] = {d.k2.x, d.k2.y, d.k2.z}, df[3], gl[3], pdf = 0.0f;
    state_array(s, st);
    if (!oracle_material_evaluate(g_scene, (int32_t)s.arg_block_offset, fn, st, k1, k2, d.ior1.x, d.ior2.x, df, gl,
                                  &pdf)) {
        ref_ub = 1;
        return;
    }
    d.bsdf_diffuse = float3(df[0], df[1], df[2]);
    d.bsdf_glossy = float3(gl[0], gl[1], gl[2]);
    d.pdf = pdf;
}
static void mdl_bsdf_scattering_sample(int fn, Bsdf_sample_data& d, Shading_state_material s)
{
    float st[11], k1[3] = {d.k1.x, d.k1.y, d.k1.z}, xi[4] = {d.xi.x, d.xi.y, d.xi.z, d.xi.w}, k2[3], bop[3], pdf;
    int ev = 0;
    state_array(s, st);
    if (!oracle_material_sample(g_scene, (int32_t)s.arg_block_offset, fn, st, k1, xi, d.ior1.x, d.ior2.x, k2, bop,
                                &pdf, &ev)) {
        ref_ub = 1;
        d.event_type = BSDF_EVENT_ABSORB;
        return;
    }
    d.k2 = float3(k2[0], k2[1], k2[2]);
    d.bsdf_over_pdf = float3(bop[0], bop[1], bop[2]);
    d.pdf = pdf;
    d.event_type = ev;
}

#include "pathtracerMdl.hlsl"

static_assert(sizeof(PathTracerParam) == 336 && sizeof(BVHNode) == 32 && sizeof(Vertex) == 32 &&
                  sizeof(InstanceConstants) == 208 && sizeof(UniformLight) == 112 && sizeof(MdlMaterial) == 16 &&
                  sizeof(Ray) == 32,
              "the reference's structs as compiled here must match the buffers' layout");

static void bind(const ::PathTracerParam* p, const OracleScene* s)
{
    memcpy(static_cast<void*>(static_cast<PathTracerParam*>(&ubo)), p, sizeof(PathTracerParam));
    bvhNodes.p = reinterpret_cast<const BVHNode*>(s->nodes);
    bvhNodes.n = s->numNodes;
    vb.p = reinterpret_cast<const Vertex*>(s->vb);
    vb.n = s->numVertices;
    ib.p = s->ib;
    ib.n = s->numIndices;
    instanceConstants.p = reinterpret_cast<const InstanceConstants*>(s->instances);
    instanceConstants.n = s->numInstances;
    mdlMaterials.p = reinterpret_cast<const MdlMaterial*>(s->materials);
    mdlMaterials.n = s->numMaterials;
    lights.p = reinterpret_cast<const UniformLight*>(s->lights);
    lights.n = s->lightCapacity;
    g_scene = s;
}

static Accel accel_of(const OracleScene* s)
{
    Accel a;
    a.bvhNodes.p = reinterpret_cast<const BVHNode*>(s->nodes);
    a.bvhNodes.n = s->numNodes;
    a.vb.p = reinterpret_cast<const Vertex*>(s->vb);
    a.vb.n = s->numVertices;
    a.ib.p = s->ib;
    a.ib.n = s->numIndices;
    a.instanceConstants.p = reinterpret_cast<const InstanceConstants*>(s->instances);
    a.instanceConstants.n = s->numInstances;
    return a;
}
}  // namespace ref_pt

extern "C" {

/* computeMain (pathtracerMdl.hlsl:406-423) over sample indices
 * [first, first + count): out[(idx - first)*3 + c].  ub[idx - first] = 1
 * where the sample went through an out-of-range buffer read (a result the
 * reference leaves undefined), else 0; ub may be NULL. */
int strelka_ref_pathtrace(const ::PathTracerParam* p, const OracleScene* s, float* out, uint64_t first, uint64_t count,
                          uint8_t* ub, int threads)
{
    ref_pt::bind(p, s);
    ref_pt::sampleBuffer.p = out;
    ref_pt::sampleBuffer.base = first * 3;
    ref_pt::sampleBuffer.n = count * 3;
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 64)
#endif
    for (int64_t k = 0; k < (int64_t)count; ++k) {
        ref_ub = 0;
        ref_pt::computeMain(uint2((uint)(first + (uint64_t)k), 0u));
        if (ub) ub[k] = (uint8_t)ref_ub;
    }
    return 0;
}

/* closestHit / anyHit (raytracing.h:198-286) for n rays: hits[i] as the
 * shader's Hit record, found[i] the return value.  On a miss the ids are
 * 0xFFFFFFFF; closest hit then reports t = 1e9 and zero barycentrics, any
 * hit the t its last triangle test wrote. */
int strelka_ref_trace(const OracleScene* s, const ::Ray* rays, uint32_t n, ::Hit* hits, uint8_t* found, int anyHitMode,
                      int threads)
{
    const ref_pt::Accel a = ref_pt::accel_of(s);
#ifdef _OPENMP
    if (threads > 0) omp_set_num_threads(threads);
#pragma omp parallel for schedule(dynamic, 256)
#endif
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        ref_pt::Ray r;
        memcpy(static_cast<void*>(&r), &rays[i], sizeof(r));
        ref_pt::Hit h;
        h.t = 0.0f;
        bool f = anyHitMode ? ref_pt::anyHit(a, r, h) : ref_pt::closestHit(a, r, h);
        if (!f) {
            // the shader leaves the ids of a miss unset; any hit's t is the
            // last triangle test's (its out parameter), closest hit's untouched
            h.instId = 0xFFFFFFFFu;
            h.primId = 0xFFFFFFFFu;
            if (!anyHitMode) {
                h.t = 1e9f;
                h.bary = float2(0.0f);
            }
        }
        memcpy(&hits[i], &h, sizeof(h));
        found[i] = f ? 1 : 0;
    }
    return 0;
}

uint32_t strelka_ref_jenkins_hash(uint32_t x) { return ref_pt::jenkinsHash(x); }
uint32_t strelka_ref_init_rng(uint32_t px, uint32_t py, uint32_t w, uint32_t h, uint32_t frame)
{
    return ref_pt::initRNG(uint2(px, py), uint2(w, h), frame);
}
uint32_t strelka_ref_xorshift(uint32_t* state) { return ref_pt::xorshift(*state); }
float strelka_ref_rand(uint32_t* state) { return ref_pt::rand(*state); }
uint32_t strelka_ref_permute(uint32_t i, uint32_t l, uint32_t p) { return ref_pt::permute(i, l, p); }
float strelka_ref_randfloat(uint32_t i, uint32_t p) { return ref_pt::randfloat(i, p); }

void strelka_ref_unpack_normal(uint32_t v, float out[3])
{
    float3 n = ref_pt::unpackNormal(v);
    out[0] = n.x; out[1] = n.y; out[2] = n.z;
}
void strelka_ref_unpack_uv(uint32_t v, float out[2])
{
    float2 uv = ref_pt::unpackUV(v);
    out[0] = uv.x; out[1] = uv.y;
}
void strelka_ref_unpack_tangent(uint32_t v, float out[3])
{
    float3 t = ref_pt::unpackTangent(v);
    out[0] = t.x; out[1] = t.y; out[2] = t.z;
}
void strelka_ref_offset_ray(const float p[3], const float n[3], float out[3])
{
    float3 o = ref_pt::offset_ray(float3(p[0], p[1], p[2]), float3(n[0], n[1], n[2]));
    out[0] = o.x; out[1] = o.y; out[2] = o.z;
}
int strelka_ref_intersect_ray_box(const float o[3], const float invdir[3], const float pmin[3], const float pmax[3],
                                  float* t)
{
    ref_pt::Ray r;
    r.o = float4(o[0], o[1], o[2], 0.0f);
    float tt = 0.0f;
    bool hit = ref_pt::intersectRayBox(r, float3(invdir[0], invdir[1], invdir[2]), float3(pmin[0], pmin[1], pmin[2]),
                               float3(pmax[0], pmax[1], pmax[2]), tt);
    *t = tt;
    return hit ? 1 : 0;
}
int strelka_ref_ray_triangle(const float o[3], const float d[3], const float v0[3], const float e0[3],
                             const float e1[3], float* t, float* u, float* v)
{
    float tt = 0.0f;
    float2 b(0.0f);
    bool hit = ref_pt::RayTriangleIntersect(float3(o[0], o[1], o[2]), float3(d[0], d[1], d[2]), float3(v0[0], v0[1], v0[2]),
                                    float3(e0[0], e0[1], e0[2]), float3(e1[0], e1[1], e1[2]), tt, b);
    *t = tt;
    *u = b.x;
    *v = b.y;
    return hit ? 1 : 0;
}
/* The light-type switch of estimateDirectLighting (pathtracerMdl.hlsl:31-50)
 * with the two samples given: out = {pointOnLight[3], pdf, normal[3], area,
 * L[3], distToLight}. */
void strelka_ref_sample_light(const ::UniformLight* light, const float hitPoint[3], const float normal[3], float u0,
                              float u1, float out[12])
{
    ref_pt::UniformLight l;
    memcpy(static_cast<void*>(&l), light, sizeof(l));
    const float3 p(hitPoint[0], hitPoint[1], hitPoint[2]);
    ref_pt::LightSampleData d;
    switch (l.type) {
    case 0: d = ref_pt::SampleRectLight(l, float2(u0, u1), p); break;
    case 1: d = ref_pt::SampleDiscLight(l, float2(u0, u1), p); break;
    case 2: d = ref_pt::SampleSphereLight(l, float3(normal[0], normal[1], normal[2]), p, float2(u0, u1)); break;
    }
    const float v[12] = {d.pointOnLight.x, d.pointOnLight.y, d.pointOnLight.z, d.pdf, d.normal.x, d.normal.y,
                         d.normal.z, d.area, d.L.x, d.L.y, d.L.z, d.distToLight};
    memcpy(out, v, sizeof(v));
}
/* generateCameraRay (pathtracerMdl.hlsl:165-202): out = {o[3], d[3]}. */
void strelka_ref_camera_ray(const ::PathTracerParam* p, uint32_t px, uint32_t py, uint32_t* rng, uint32_t s,
                            float out[6])
{
    memcpy(static_cast<void*>(static_cast<ref_pt::PathTracerParam*>(&ref_pt::ubo)), p, sizeof(ref_pt::PathTracerParam));
    ref_pt::Ray r = ref_pt::generateCameraRay(uint2(px, py), *rng, s);
    out[0] = r.o.x; out[1] = r.o.y; out[2] = r.o.z;
    out[3] = r.d.x; out[4] = r.d.y; out[5] = r.d.z;
}
}
