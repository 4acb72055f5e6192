/*
 * strelka_b200_scenes.h — synthetic workload generators for the benchmark
 * configurations.  These have no counterpart in the reference's render-pass
 * API: they stand in for the scenes the reference loads through USD/glTF
 * (unavailable here), producing the same host buffers the reference uploads
 * at frame 0 (src/render/ptrender.cpp:412-639): vertices, indices, instance
 * constants, lights, the material tables and the flattened BVH built by
 * strelka_bvh_build over world-space triangles (ptrender.cpp:460-511).
 * All generators are seeded and deterministic.
 */
#ifndef STRELKA_B200_SCENES_H
#define STRELKA_B200_SCENES_H

#include "strelka_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct StrelkaHostScene {
    Vertex* vb;                  uint32_t numVertices;
    uint32_t* ib;                uint32_t numIndices;
    InstanceConstants* instances; uint32_t numInstances;
    UniformLight* lights;        uint32_t numLights;     /* lights[] has max(numLights,1) entries */
    MdlMaterial* materials;      uint32_t numMaterials;
    uint8_t* argBlock;           uint64_t argBlockBytes;
    Mdl_resource_info* resourceInfos; uint32_t numResourceInfos;
    uint32_t numTextures;
    uint8_t** textures;          /* numTextures RGBA8 sRGB images */
    uint32_t* texWidth;
    uint32_t* texHeight;
    float* envRGBA;              /* NULL when the scene has no environment light */
    uint32_t envWidth, envHeight;
    float* envMarginalCdf;       /* envHeight + 1 */
    float* envConditionalCdf;    /* envHeight * (envWidth + 1) */
    float envIntegral;
    BVHNode* nodes;              uint32_t numNodes;
    uint32_t numTriangles;
    PathTracerParam camera;      /* matrices, dimension, numLights, maxDepth, spp filled */
} StrelkaHostScene;

/* Cornell box: 5 axis-aligned walls (2 triangles each, inward normals), a
 * rect light of side `lightSide` with radiance `lightRadiance` and its
 * emitter quad (the reference's rect-light mesh, src/scene/scene.cpp:115-140),
 * two icospheres subdivided `sphereLevels` times (scene.cpp:142-208), fixed
 * Lambert albedos in [0.2, 0.8], a 40-degree pinhole camera. */
typedef struct StrelkaCornellConfig {
    uint32_t width, height;
    uint32_t sphereLevels;  /* 4 */
    float lightSide;        /* 0.25 */
    float lightRadiance;    /* 15 */
    uint32_t maxDepth;      /* 4 */
    uint32_t spp;           /* 1 */
    uint32_t tonemapper;    /* unused by the generator, kept for callers */
    /* Extra lights, a bit mask (0 = the rect light alone):
     *   1: a disc light (radius 0.12, radiance 10) facing down just under the
     *      ceiling light, so shadow rays toward the ceiling light often
     *      reach the disc's emitter first;
     *   2: a sphere light (radius 0.08, radiance 20) floating in the box.
     * Each is built as the reference builds it (src/scene/scene.cpp:
     * 210-361 meshes, 418-510 records) and gets an emitter instance. */
    uint32_t extraLights;
} StrelkaCornellConfig;
int strelka_scene_cornell(const StrelkaCornellConfig* cfg, StrelkaHostScene* out);

/* Triangle soup: numTris triangles with centroids uniform in [0,1]^3 and
 * vertices at centroid + dir * len, dir uniform on the sphere and len
 * log-normal(mu = ln 0.003, sigma = 0.5) per vertex; one identity instance. */
int strelka_scene_soup(uint32_t numTris, uint64_t seed, StrelkaHostScene* out);

/* Rays for the traversal microbenchmark: origins uniform in [-0.5,1.5]^3,
 * directions uniform on the sphere; tmax = 1e9 (closest) or uniform in
 * [0.1, 2] (shadow != 0). */
int strelka_rays_soup(uint32_t numRays, uint64_t seed, int shadow, Ray* out);

/* Large render: `instances` random affine instances (scale 0.5-2) of a
 * displaced geodesic sphere (frequency `frequency`, 20*f^2 triangles,
 * Perlin displacement 0.05) plus a ground quad, `numTextures` procedural
 * texSize^2 RGBA8 noise textures, a Lambert / GGX metal / GGX dielectric mix
 * with roughness in [0.05, 1], and an envW x envH RGBA32F environment with
 * one hot sun lobe. */
typedef struct StrelkaLargeConfig {
    uint32_t width, height;
    uint32_t instances;    /* 64 */
    uint32_t frequency;    /* 89: 158,420 triangles per sphere */
    uint32_t numTextures;  /* 8 */
    uint32_t texSize;      /* 2048 */
    uint32_t envWidth;     /* 1024 */
    uint32_t envHeight;    /* 512 */
    uint32_t maxDepth;     /* 8 */
    uint32_t spp;          /* 16 */
    uint64_t seed;
} StrelkaLargeConfig;
int strelka_scene_large(const StrelkaLargeConfig* cfg, StrelkaHostScene* out);

/* Environment importance tables on the host: weights luminance*sin(theta),
 * per-row conditional CDFs (envWidth+1 entries each) and the marginal CDF
 * (envHeight+1 entries), both normalised to end at 1. */
int strelka_envmap_build_cdf_host(const float* rgba32f, uint32_t width, uint32_t height, float* marginalCdf,
                                  float* conditionalCdf, float* integral);

void strelka_scene_free(StrelkaHostScene* scene);

/* Replaces the camera of a parameter block by a pinhole at `eye` looking at
 * `target` (y up) with a vertical field of view of fovDeg, rendering
 * width x height: the matrices Camera builds (src/scene/camera.cpp:61-131,
 * reverse Z) and the dimension fields; every other field is kept. */
int strelka_camera_lookat(PathTracerParam* param, uint32_t width, uint32_t height, const float eye[3],
                          const float target[3], float fovDeg);

#ifdef __cplusplus
}
#endif
#endif
