/*
 * oracle.h — CPU restatement of Strelka's path-tracing shader math.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA path:
 * only the tests, the smoke check and the CPU-baseline leg of the benchmark
 * may load it.  Nothing in the product links or calls it.
 *
 * Parity status: pinned to the reference's own shader source.
 * oracle/build_ref.sh compiles the reference's pathtracerMdl.hlsl (with
 * raytracing.h, ray.h, random.h, helper.h, pack.h, lights.h), reduction,
 * accumulation, tonemap and upscale shaders on the host (a syntax-only
 * rewrite, oracle/hlsl2cpp.py, over the HLSL shim oracle/ref/shim.h) into
 * oracle/_ref/; tests/test_ref_pin.py checks this file against it bit for
 * bit, function by function and sample by sample.  The reference's
 * material code is generated at run time by the MDL SDK, which is absent;
 * there both sides use the project's native materials below, unpinned.
 * Further pins: the slab-test known answers of tests/intersection/aabb.cpp,
 * hand-computed RNG states and analytic checks.
 *
 * Every function cites the reference lines it restates.  Floating-point
 * evaluation follows the source expressions left to right with no fused
 * multiply-add (build with -ffp-contract=off); sin/cos/acos are this
 * project's own correctly-reduced polynomial versions, which the CUDA kernels
 * implement identically, so the two sides agree bit for bit.
 */
#ifndef STRELKA_ORACLE_H
#define STRELKA_ORACLE_H

#include <stdint.h>
#include <stddef.h>
#include "../include/strelka_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct OracleTexture {
    const uint8_t* rgba8; /* host texels */
    uint32_t width, height;
} OracleTexture;

typedef struct OracleEnvMap {
    const float* rgba32f;
    const float* marginal_cdf;
    const float* conditional_cdf;
    uint32_t width, height;
    float integral;
} OracleEnvMap;

/* All pointers are host pointers. */
typedef struct OracleScene {
    const BVHNode* nodes; uint32_t numNodes;
    const Vertex* vb; uint32_t numVertices;
    const uint32_t* ib; uint32_t numIndices;
    const InstanceConstants* instances; uint32_t numInstances;
    const UniformLight* lights; uint32_t lightCapacity;
    const uint8_t* argBlock; uint64_t argBlockBytes;
    const MdlMaterial* materials; uint32_t numMaterials;
    const Mdl_resource_info* resourceInfos; uint32_t numResourceInfos;
    const OracleTexture* textures; uint32_t numTextures;
    const OracleEnvMap* envMap; /* NULL: black miss */
} OracleScene;

/* random.h:14-48 */
uint32_t oracle_jenkins_hash(uint32_t x);
uint32_t oracle_init_rng(uint32_t px, uint32_t py, uint32_t width, uint32_t frame);
uint32_t oracle_xorshift(uint32_t* state);
float oracle_rand(uint32_t* state);
/* helper.h:117-163 */
uint32_t oracle_permute(uint32_t i, uint32_t l, uint32_t p);
float oracle_randfloat(uint32_t i, uint32_t p);

/* own transcendental functions (shared definition with the kernels) */
float oracle_sinf(float x);
float oracle_cosf(float x);
float oracle_acosf(float x);

/* pack.h:4-33 */
void oracle_unpack_normal(uint32_t v, float out[3]);
void oracle_unpack_uv(uint32_t v, float out[2]);
/* helper.h:12-28 */
void oracle_offset_ray(const float p[3], const float n[3], float out[3]);
/* ray.h:19-33 */
int oracle_intersect_ray_box(const float o[3], const float invdir[3], const float pmin[3],
                             const float pmax[3], float* t);
/* raytracing.h:36-88 */
int oracle_ray_triangle(const float o[3], const float d[3], const float v0[3], const float e0[3],
                        const float e1[3], float* t, float* u, float* v);

/* raytracing.h:198-286 over n rays.  mode 0 closest, 1 any.  found[i] = 0/1.
 * prune = 0: the reference's stackless depth-first loop; 1: the same with
 * the GPU's closest-hit pruning rule; 2: the GPU's node-pair traversal (its
 * visit counts and its closest-hit tie order).  counters (may be NULL) gets
 * {inner visits, leaf visits} summed (for prune = 2: inner records
 * processed, triangle tests). */
int oracle_trace(const OracleScene* s, const Ray* rays, uint32_t n, Hit* hits, uint8_t* found,
                 int mode, int prune, unsigned long long* counters, int nthreads);

/* The GPU's closest-hit kernels with deferred leaf tests, replayed for one
 * warp that takes every ray of [0, n) from one work chunk (the kernels run
 * that way when their queue chunk is at least n).  Hits and found as
 * oracle_trace (equal to its results); counters gets the warp's {4-wide
 * nodes processed, triangle tests}. */
int oracle_trace_warp(const OracleScene* s, const Ray* rays, uint32_t n, Hit* hits, uint8_t* found,
                      unsigned long long* counters);

/* FP64 Möller–Trumbore of ray i against triangle (instId[i], primId[i]),
 * same formula as raytracing.h:36-88 evaluated in double (no thresholds). */
int oracle_intersect_fp64(const OracleScene* s, const Ray* rays, const uint32_t* instIds,
                          const uint32_t* primIds, uint32_t n, double* t, double* u, double* v);

/* Per ray, the conditioning scale of u, v and t in that formula (see
 * oracle.c): scale x 2^-52 bounds FP64's own error. */
int oracle_intersect_terms_fp64(const OracleScene* s, const Ray* rays, const uint32_t* instIds,
                                const uint32_t* primIds, uint32_t n, double* scale3);

/* lights.h:284-340 for one light: out = {pointOnLight[3], pdf, normal[3],
 * area, L[3], distToLight}. */
void oracle_sample_light(const UniformLight* l, const float hitPoint[3], float u0, float u1, float out[12]);
/* pathtracerMdl.hlsl:165-202: out = {origin[3], direction[3]}. */
void oracle_camera_ray(const PathTracerParam* p, uint32_t px, uint32_t py, uint32_t* rng, uint32_t s, float out[6]);

/* pathtracerMdl.hlsl:406-423 computeMain over idx in [0, W*H*spp):
 * writes sampleBuffer[(idx)*3 + c]. */
int oracle_pathtrace(const PathTracerParam* p, const OracleScene* s, float* sampleBuffer,
                     int nthreads);
/* Same, for the sub-range of sample indices [first, first+count). */
int oracle_pathtrace_range(const PathTracerParam* p, const OracleScene* s, float* sampleBuffer,
                           uint64_t first, uint64_t count, int nthreads);

/* reduction.hlsl:9-32 */
int oracle_reduce(const PathTracerParam* p, const float* sampleBuffer, float* rgba32f);
/* accumulation.hlsl:86-97 */
int oracle_accumulate(const AccumulationParam* p, const float* input, const float* history,
                      float* output);
/* tonemap.hlsl:9-88 */
int oracle_tonemap(const Tonemapparam* p, const float* input, float* output);
/* upscalepass.hlsl:9-21 with the pass's linear clamp-to-edge sampler
 * (upscalepass.cpp:12-38); input RGBA32F inW x inH, output p->dimension. */
/* mdl_runtime.hlsl:24-75: ByteAddressBuffer reads (kinds 0 float, 1 double,
 * 2 int, 3 uint, 4 bool); 0 past the end. */
void oracle_mdl_read(const uint8_t* buffer, uint64_t bytes, const uint32_t* offsets, const uint32_t* kinds, uint32_t n,
                     uint64_t* out);
int oracle_upscale(const Upscalepassparam* p, const float* input, uint32_t inW, uint32_t inH, float* output);

/* The project's native materials behind the MDL dispatch functions
 * (src/materialmanager/mdlHlslCodeGen.cpp:32-81), by argument-block offset
 * and function id; state = {normal[3], geom_normal[3], position[3], u, v}.
 * Return 0 when the material record is out of range.  Used by the HLSL shim
 * of oracle/ref/ in place of the MDL-generated code. */
int oracle_material_sample(const OracleScene* s, int32_t argOffset, int32_t fn, const float* state, const float k1[3],
                           const float xi[4], float ior1, float ior2, float k2[3], float bsdfOverPdf[3], float* pdf,
                           int* event);
int oracle_material_evaluate(const OracleScene* s, int32_t argOffset, int32_t fn, const float* state,
                             const float k1[3], const float k2[3], float ior1, float ior2, float diffuse[3],
                             float glossy[3], float* pdf);
int oracle_material_emission(const OracleScene* s, int32_t argOffset, int32_t fn, const float* state,
                             float intensity[3]);

/* texture lookup, mdl_runtime.hlsl:173-208 (REPEAT, no crop) */
void oracle_tex_lookup(const OracleTexture* t, float u, float v, float out[4]);

#ifdef __cplusplus
}
#endif
#endif
