/*
 * strelka_b200.h — C ABI of the B200 (sm_100a) path-tracing hot path.
 *
 * This is the drop-in boundary for Strelka's render-pass API.  The reference
 * records four compute passes per frame, each through
 *     ComputePass<T>::execute(VkCommandBuffer&, const XDesc&, w, h, frameIndex)
 * (include/render/computepass.h:8-164, called from src/render/ptrender.cpp:735-862).
 * Here each pass is one extern "C" function taking the same constants struct,
 * the same buffers (as device pointers instead of Buffer and Image handles), the
 * same (w, h, frameIndex) triple and a cudaStream_t in place of the command
 * buffer.  Buffers stay owned by the caller, as they are owned by the
 * reference's ResourceManager; the passes only read and write them.
 *
 * Every entry point returns an int status: 0 = OK (STRELKA_OK), otherwise a
 * STRELKA_ERR_* code; strelka_get_last_error() returns the message of the most
 * recent failure on the calling thread.  Kernels never trap: out-of-range
 * indices and over-long traversals set a device status word that the host
 * reads with strelka_pathtracer_get_device_status().
 *
 * All structs below are byte-identical to the reference's shader structs; the
 * static asserts at the end of this file pin sizes and offsets.
 *
 * Matrices are column-major (the glm layout the reference uploads raw): the
 * element in row r, column c is m[c*4 + r], and a shader mul(M, v) is the
 * matrix-vector product M·v.
 */
#ifndef STRELKA_B200_H
#define STRELKA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------- */
/* Status codes (replace Result{eOk,eFail,eOutOfMemory}, include/render/common.h:338-343) */
enum {
    STRELKA_OK = 0,
    STRELKA_ERR_INVALID_ARGUMENT = 1,
    STRELKA_ERR_OUT_OF_MEMORY = 2,
    STRELKA_ERR_CUDA = 3,
    STRELKA_ERR_NO_DEVICE = 4,
    STRELKA_ERR_DEVICE_BOUNDS = 5,   /* a kernel saw an out-of-range index */
    STRELKA_ERR_TIMEOUT = 6,         /* a traversal or queue wait hit its iteration cap */
    STRELKA_ERR_UNSUPPORTED = 7
};

/* Device status bits (strelka_pathtracer_get_device_status). */
enum {
    STRELKA_DEV_OK = 0,
    STRELKA_DEV_NODE_OOB = 1u << 0,     /* node index >= numNodes */
    STRELKA_DEV_INSTANCE_OOB = 1u << 1, /* instance id >= numInstances */
    STRELKA_DEV_INDEX_OOB = 1u << 2,    /* ib offset or vertex index out of range */
    STRELKA_DEV_MATERIAL_OOB = 1u << 3, /* material id / arg block offset out of range */
    STRELKA_DEV_LIGHT_OOB = 1u << 4,    /* light id >= light capacity */
    STRELKA_DEV_TRAVERSAL_CAP = 1u << 5,/* traversal exceeded 2*numNodes+2 visits (cycle) */
    STRELKA_DEV_TEXTURE_OOB = 1u << 6,
    STRELKA_DEV_QUEUE_TIMEOUT = 1u << 7,
    STRELKA_DEV_MMA_TIMEOUT = 1u << 8   /* a tensor-core completion wait hit its time limit */
};

/* ------------------------------------------------------------------------- */
/* Shared shader structs                                                     */

typedef struct StrelkaFloat4 { float x, y, z, w; } StrelkaFloat4;
typedef struct StrelkaFloat4x4 { float m[16]; } StrelkaFloat4x4;

/* shaders/pathtracerparam.h:20-43 (336 bytes) */
typedef struct PathTracerParam {
    StrelkaFloat4x4 viewToWorld;
    StrelkaFloat4x4 clipToView;
    StrelkaFloat4x4 viewToClip;
    StrelkaFloat4x4 worldToView;
    StrelkaFloat4 camPos;
    int32_t dimension[2];
    float invDimension[2];
    uint32_t frameNumber;
    uint32_t maxDepth;
    uint32_t debug;
    uint32_t numLights;
    int32_t len;
    int32_t spp;
    int32_t iteration;
    uint32_t stratifiedSamplingType; /* 0 centre, 1 random, 2 stratified, 3 CMJ */
    StrelkaFloat4 pad0;
} PathTracerParam;

/* shaders/accumulationparam.h:19-34 (416 bytes) */
typedef struct AccumulationParam {
    StrelkaFloat4x4 prevViewToWorld;
    StrelkaFloat4x4 prevClipToView;
    StrelkaFloat4x4 prevWorldToView;
    StrelkaFloat4x4 prevViewToClip;
    StrelkaFloat4x4 viewToWorld;
    StrelkaFloat4x4 clipToView;
    int32_t dimension[2];
    uint32_t frameNumber;
    uint32_t iteration;
    float alpha;
    float isPt;
    float pad1;
    float pad2;
} AccumulationParam;

/* shaders/tonemapparam.h:17-22 (16 bytes) */
typedef struct Tonemapparam {
    int32_t dimension[2];
    uint32_t tonemapperType; /* 0 Reinhard, 1 ACESFitted, 2 ACESFilm */
    uint32_t pad0;
} Tonemapparam;

/* shaders/raytracing.h:27-33, include/render/bvh.h:18-24 (32 bytes).
 * Inner node: instId == -1, bounds valid, the left child is the next node,
 * nodeOffset is the escape index (next sibling or uncle, -1 at the end).
 * Leaf: instId = instance id, minBounds[0] holds the bits of the
 * per-instance triangle index, nodeOffset is the escape index. */
typedef struct BVHNode {
    float minBounds[3];
    int32_t instId;
    float maxBounds[3];
    int32_t nodeOffset;
} BVHNode;

/* shaders/raytracing.h:17-25, include/scene/scene.h:54-63 (32 bytes) */
typedef struct Vertex {
    float position[3];
    uint32_t tangent; /* 10/10/12-bit packed, shaders/pack.h:4-14 */
    uint32_t normal;  /* 10/10/12-bit packed */
    uint32_t uv;      /* 16/16-bit packed, shaders/pack.h:16-24 */
    float pad0;
    float pad1;
} Vertex;

/* shaders/instanceconstants.h:19-28 (208 bytes) */
typedef struct InstanceConstants {
    StrelkaFloat4x4 objectToWorld;
    StrelkaFloat4x4 worldToObject;
    StrelkaFloat4x4 normalMatrix;
    int32_t materialId; /* -1 for light emitter instances */
    int32_t indexOffset;
    int32_t indexCount;
    int32_t lightId; /* -1 unless the instance is a light's emitter mesh */
} InstanceConstants;

/* shaders/lights.h:10-19 (112 bytes).  type 0 rect (points = 4 corners),
 * 1 disc (points[0].x radius, [1] centre, [2..3] axes, normal),
 * 2 sphere (points[0].x radius, [1] centre). */
typedef struct UniformLight {
    StrelkaFloat4 points[4];
    StrelkaFloat4 color;
    StrelkaFloat4 normal;
    int32_t type;
    float pad0;
    float pad2;
    float pad3;
} UniformLight;

/* shaders/materials.h:17-23 (16 bytes) */
typedef struct MdlMaterial {
    int32_t arg_block_offset;       /* bytes into mdl_argument_block */
    int32_t ro_data_segment_offset; /* bytes into mdl_ro_data_segment */
    int32_t functionId;             /* STRELKA_FN_* */
    int32_t pad1;
} MdlMaterial;

/* shaders/materials.h:27-34 (16 bytes) */
typedef struct Mdl_resource_info {
    uint32_t gpu_resource_array_start; /* texture slot in matTextures */
    uint32_t pad0;
    uint32_t pad1;
    uint32_t pad2;
} Mdl_resource_info;

/* shaders/ray.h:12-16 (32 bytes): o.xyz origin, o.w max distance, d.xyz direction */
typedef struct Ray {
    StrelkaFloat4 o;
    StrelkaFloat4 d;
} Ray;

/* shaders/raytracing.h:90-96 (20 bytes) */
typedef struct Hit {
    float bary[2];
    float t;
    uint32_t instId;
    uint32_t primId;
} Hit;

/* include/render/bvh.h:31-36 (20 bytes): one world-space triangle corner */
typedef struct BVHInputPosition {
    float pos[3];
    uint32_t instId;
    uint32_t primId;
} BVHInputPosition;

/* ------------------------------------------------------------------------- */
/* Native material table.  The reference fills the MDL tables with code and
 * argument blocks generated by the MDL SDK (src/materialmanager/
 * mdlHlslCodeGen.cpp:32-81), which is not available.  The table ABI is kept
 * (MdlMaterial, argument block, ro-data, resource infos, texture array); the
 * functionId selects one of the native BSDFs below, and the argument block at
 * arg_block_offset holds one StrelkaMaterialArgs record (project-defined). */
enum {
    STRELKA_FN_LAMBERT = 0,        /* cosine-sampled Lambert, shaders/pathtracer.hlsl:176-234 */
    STRELKA_FN_GGX_CONDUCTOR = 1,  /* GGX microfacet metal, Schlick Fresnel */
    STRELKA_FN_GGX_DIELECTRIC = 2, /* GGX rough dielectric (reflect + refract) */
    STRELKA_FN_COUNT = 3
};

typedef struct StrelkaMaterialArgs {
    float base_color[3];          /* albedo / F0 / transmission tint (linear) */
    float roughness;              /* GGX alpha = roughness^2 */
    float emission[3];            /* EDF radiance; zero for non-emissive */
    float ior;                    /* dielectric index of refraction */
    uint32_t base_color_texture;  /* MDL resource id: 0 none, else mdl_resource_infos[id-1] */
    uint32_t pad[3];
} StrelkaMaterialArgs;            /* 48 bytes */

/* One bindless texture: RGBA8 sRGB texels in device memory, row-major,
 * sampled bilinearly with REPEAT wrapping at lod 0 (the reference's MDL
 * sampler, include/texturemanager/texturemanager.h:24-44). */
typedef struct StrelkaTexture {
    const uint8_t* rgba8;
    uint32_t width;
    uint32_t height;
    uint64_t pad;
} StrelkaTexture;

/* Optional environment light (the reference adds zero on a miss,
 * shaders/pathtracerMdl.hlsl:389-399).  Lat-long RGBA32F map with
 * importance-sampling tables from strelka_envmap_build_cdf_host(). */
typedef struct StrelkaEnvMap {
    const float* rgba32f;       /* width*height*4 floats */
    const float* marginal_cdf;  /* height+1 floats */
    const float* conditional_cdf; /* height*(width+1) floats */
    uint32_t width;
    uint32_t height;
    float integral;             /* sum of luminance*sin(theta) weights */
    float pad;
} StrelkaEnvMap;

/* ------------------------------------------------------------------------- */
/* Pass descriptors: include/render/pathtracer.h:9-31, reduction.h:10-16,
 * accumulation.h:9-15, tonemap.h:11-16.  Pointers are device pointers. */

typedef struct PathTracerDesc {
    PathTracerParam constants;
    const BVHNode* bvhNodes;      uint32_t numNodes;
    uint32_t numVertices;         const Vertex* vb;
    const uint32_t* ib;           uint32_t numIndices;
    uint32_t numInstances;        const InstanceConstants* instanceConst;
    const UniformLight* lights;   uint32_t lightCapacity;
    uint32_t pad0;
    float* sampleBuffer;          /* W*H*spp*3 floats, [(pixel*spp + s)*3 + c] */
    const uint8_t* mdl_ro_data_segment; uint64_t roDataBytes;
    const uint8_t* mdl_argument_block;  uint64_t argBlockBytes;
    const Mdl_resource_info* mdl_resource_infos; uint32_t numResourceInfos;
    uint32_t numMaterials;        const MdlMaterial* mdl_mdlMaterial;
    const StrelkaTexture* matTextures; /* device array of numTextures entries */
    uint32_t numTextures;         uint32_t pad1;
    const StrelkaEnvMap* envMap;  /* host pointer to a descriptor, or NULL: black miss */
    uint64_t sceneVersion;        /* bump when any scene buffer changes */
} PathTracerDesc;

typedef struct ReductionDesc {
    PathTracerParam constants;
    const float* sampleBuffer;    /* W*H*spp*3 */
    float* result;                /* W*H RGBA32F */
} ReductionDesc;

typedef struct AccumulationDesc {
    AccumulationParam constants;
    const float* input;           /* RGBA32F */
    const float* history;         /* RGBA32F */
    float* output;                /* RGBA32F */
} AccumulationDesc;

typedef struct TonemapDesc {
    Tonemapparam constants;
    const float* input;           /* RGBA32F */
    float* output;                /* RGBA32F */
} TonemapDesc;

/* shaders/upscalepassparam.h (16 bytes): the size of the OUTPUT image. */
typedef struct Upscalepassparam {
    int32_t dimension[2];
    float invDimension[2];
} Upscalepassparam;

/* UpscaleDesc (include/render/upscalepass.h:9-14).  The input image's size
 * is the render resolution, which the reference's Image handle carries. */
typedef struct UpscaleDesc {
    Upscalepassparam constants;
    const float* input;           /* RGBA32F, inputWidth x inputHeight */
    uint32_t inputWidth;
    uint32_t inputHeight;
    float* output;                /* RGBA32F, constants.dimension */
} UpscaleDesc;

/* ------------------------------------------------------------------------- */
/* Path tracer pass object (replaces PathTracer : ComputePass<PathTracerParam>,
 * include/render/pathtracer.h:33-50, src/render/pathtracer.cpp:1-94).  The
 * object caches scene-derived device data (a leaf triangle table of 48
 * bytes per leaf, a leaf shading table of 96 bytes per leaf, each node's
 * leaf index, a 4-wide BVH derived from bvhNodes and its build scratch:
 * about 156 bytes per BVH node allocated) keyed by
 * PathTracerDesc.sceneVersion and the buffer pointers, and owns the
 * wavefront path queues. */

enum {
    STRELKA_MODE_WAVEFRONT = 0,  /* generate / extend / shade / shadow kernels */
    STRELKA_MODE_MEGAKERNEL = 1  /* one thread per (pixel, sample), like computeMain */
};

typedef struct StrelkaPathTracerConfig {
    uint32_t mode;            /* STRELKA_MODE_* */
    uint32_t chunkPaths;      /* wavefront: paths in flight per chunk (0 = auto) */
    uint32_t blockSize;       /* threads per block (0 = auto) */
    uint32_t flags;           /* STRELKA_PT_* */
    uint32_t queueChunk;      /* wavefront: queue entries a warp takes at a time (0 = 32; a multiple of 32) */
    uint32_t tailDepth;       /* wavefront: bounces from this one on are finished by one persistent kernel per
                                 path (0 = 5; >= maxDepth: never); ignored with the radiance cache */
    uint32_t pad[2];
} StrelkaPathTracerConfig;

enum {
    STRELKA_PT_PROFILE = 1u << 0,       /* record per-kernel CUDA events (strelka_pathtracer_get_kernel_times) */
    STRELKA_PT_COUNT = 1u << 1,         /* count traversal visits (strelka_pathtracer_get_counters) */
    STRELKA_PT_NO_SHADE_SORT = 1u << 2, /* wavefront: shade paths in queue order, not sorted by material
                                           (frames with the radiance cache are never sorted, nor, unless
                                           STRELKA_PT_FORCE_SHADE_SORT is set, chunks of fewer than
                                           STRELKA_SHADE_SORT_MIN_PATHS paths) */
    /* wavefront traversal variants (default: by tree size, STRELKA_LARGE_SCENE_NODES): the large-scene
       variants keep the top of each traversal stack in shared memory and defer the leaf tests of
       bounces >= 1 across the warp; the small-scene ones leave L1 to the scene.  Same results. */
    STRELKA_PT_LARGE_SCENE_KERNELS = 1u << 3, /* always the large-scene variants */
    STRELKA_PT_SMALL_SCENE_KERNELS = 1u << 4, /* always the small-scene variants */
    STRELKA_PT_SERIAL_SHADOW = 1u << 5,       /* wavefront: each bounce's shadow queries run on the caller's
                                                 stream after its shading, not on a second stream beside the
                                                 next bounce's closest-hit queries (same results; lets the
                                                 shadow kernel be timed alone) */
    STRELKA_PT_FORCE_SHADE_SORT = 1u << 6     /* wavefront: sort by material whatever the chunk's size */
};

/* Paths in flight from which the wavefront sorts each bounce's shade queue
 * by material (below it the sort's three short launches per bounce cost more
 * than the coherence they buy).  The samples are the same either way. */
#define STRELKA_SHADE_SORT_MIN_PATHS (1u << 21)

/* BVH nodes from which the wavefront passes use their large-scene variants. */
#define STRELKA_LARGE_SCENE_NODES (1u << 21)

typedef struct StrelkaPathTracer StrelkaPathTracer;
typedef struct StrelkaNrc StrelkaNrc;

/* PathTracer::initialize (src/render/pathtracer.cpp:62-92). */
int strelka_pathtracer_create(const StrelkaPathTracerConfig* config, StrelkaPathTracer** out);
int strelka_pathtracer_destroy(StrelkaPathTracer* pt);

/* PathTracer::execute (src/render/pathtracer.cpp:50-59).  As in the reference,
 * w = W*H*spp threads of work and h = 1; writes desc->sampleBuffer.  The first
 * call for a scene version and frame size allocates the pass's tables and
 * path state; later calls allocate nothing and do not synchronise, so they
 * can be captured into a CUDA graph (the descriptor is read at capture). */
int strelka_pathtracer_execute(StrelkaPathTracer* pt, const PathTracerDesc* desc,
                               uint32_t w, uint32_t h, uint64_t frameIndex, void* stream);

/* Radiance-cache rendering (an extension; the reference has no cache).  With
 * enable != 0, each execute traces trainPaths short plain paths from random
 * samples of the frame and takes trainSteps Adam steps on their vertices (on
 * a stream of the pass's own, concurrently with the frame's paths), and
 * renders with every path ending at its first shading vertex after a
 * diffuse-ish bounce (a Lambert sample or roughness >= diffuseRoughness),
 * where the cache's prediction, taken after this frame's training, times the
 * path throughput is added.  Wavefront mode only.  The cache object stays
 * owned by the caller; pass NULL to detach it. */
typedef struct StrelkaNrcRenderConfig {
    uint32_t enable;
    uint32_t trainPaths;      /* e.g. 16384 (about 2^16 training vertices) */
    uint32_t trainSteps;      /* Adam steps per batch, >= 1 */
    float diffuseRoughness;   /* 0.25 */
    uint32_t pad[4];
} StrelkaNrcRenderConfig;

int strelka_pathtracer_set_nrc(StrelkaPathTracer* pt, StrelkaNrc* nrc, const StrelkaNrcRenderConfig* cfg);
/* Training without rendering: `batches` batches of trainPaths training paths
 * of the frame described by desc (sampleBuffer unused; each batch its own
 * random samples), traced in one launch, then trainSteps Adam steps per
 * batch in order, on `stream`.  Warms a fresh cache up cheaply. */
int strelka_pathtracer_train_nrc(StrelkaPathTracer* pt, const PathTracerDesc* desc, uint64_t frameIndex,
                                 uint32_t batches, void* stream);

/* Reads and clears the device status word (STRELKA_DEV_* bits); synchronises
 * the stream first. */
int strelka_pathtracer_get_device_status(StrelkaPathTracer* pt, void* stream, uint32_t* status);

/* Per-kernel timing when STRELKA_PT_PROFILE is set: for each kernel class
 * ("generate","extend","shade","shadow","finalize","megakernel","prep") the
 * CUDA-event milliseconds summed over every launch since the previous call,
 * and the launch count; clears the records.  Returns the number of classes. */
int strelka_pathtracer_get_kernel_times(StrelkaPathTracer* pt, void* stream, float* ms_out,
                                        uint32_t* launches_out, uint32_t capacity);

/* Traversal counters accumulated since the last call when STRELKA_PT_COUNT is
 * set: {extend inner-node visits, extend leaf visits, shadow inner visits,
 * shadow leaf visits, extend rays, shadow rays}.  Resets them.  Returns 6. */
int strelka_pathtracer_get_counters(StrelkaPathTracer* pt, void* stream, unsigned long long* out,
                                    uint32_t capacity);

/* ReductionPass::execute (src/render/reduction.cpp, shaders/reduction.hlsl:9-32); w = W*H. */
int strelka_reduction_execute(const ReductionDesc* desc, uint32_t w, uint32_t h,
                              uint64_t frameIndex, void* stream);

/* Accumulation::execute (src/render/accumulation.cpp, shaders/accumulation.hlsl:86-108); w = W, h = H. */
int strelka_accumulation_execute(const AccumulationDesc* desc, uint32_t w, uint32_t h,
                                 uint64_t frameIndex, void* stream);

/* Tonemap::execute (src/render/tonemap.cpp, shaders/tonemap.hlsl:66-88); w = W, h = H. */
int strelka_tonemap_execute(const TonemapDesc* desc, uint32_t w, uint32_t h,
                            uint64_t frameIndex, void* stream);

/* UpscalePass::execute (src/render/upscalepass.cpp:40-58, shaders/
 * upscalepass.hlsl:9-21): output[p] = (bilinear sample of the input at
 * uv = (p + 0.5) * invDimension, clamp to edge; rgb, 1), w x h = the output
 * dimension.  The reference's sampler is linear with clamp-to-edge
 * addressing (upscalepass.cpp:12-38); here the filter weights are exact FP32
 * (a hardware sampler rounds them to its sub-texel precision). */
int strelka_upscale_execute(const UpscaleDesc* desc, uint32_t w, uint32_t h, uint64_t frameIndex, void* stream);

/* Tonemap followed by the upscale pass and the final blit
 * (src/render/ptrender.cpp:850-896), fused: each output pixel tonemaps its
 * four bilinear taps of the render-resolution input and blends them, so the
 * tonemapped render-resolution image is never stored.  Bit-identical to
 * strelka_tonemap_execute then strelka_upscale_execute.  outputRGBA8 (may be
 * NULL) receives the same pixels quantised as the resolve pass does; output
 * (may be NULL) receives RGBA32F.  tm->dimension is the input size,
 * up->dimension the output size. */
int strelka_tonemap_upscale_execute(const Tonemapparam* tm, const float* input, const Upscalepassparam* up,
                                    float* output, uint8_t* outputRGBA8, void* stream);

/* Fused reduce + accumulate + tonemap in one pass over the sample buffer.
 * Equivalent, bit for bit, to the three passes above run in sequence
 * (src/render/ptrender.cpp:780-862); accumulation is applied when
 * accumulate != 0.  Writes the accumulated image (RGBA32F) to accOutput and the
 * tonemapped image to tonemapOutput (RGBA32F) and/or tonemapRGBA8 (either may be NULL). */
int strelka_resolve_execute(const PathTracerParam* ptParam, const float* sampleBuffer,
                            int accumulate, const AccumulationParam* accParam, const float* history,
                            float* accOutput, const Tonemapparam* tmParam, float* tonemapOutput,
                            uint8_t* tonemapRGBA8, void* stream);

/* ------------------------------------------------------------------------- */
/* Ray queries over the flattened BVH (the closestHit / anyHit functions of
 * shaders/raytracing.h:198-286, exposed for the traversal microbenchmark). */

enum {
    STRELKA_TRACE_CLOSEST = 0,
    STRELKA_TRACE_ANY = 1,          /* first hit in depth-first order with t < tmax */
    STRELKA_TRACE_COUNT = 1u << 4,  /* also count inner/leaf visits into counters[2] */
    STRELKA_TRACE_REFINE = 1u << 5  /* closest: recompute t/bary of the winner in float-float */
};

typedef struct TraceDesc {
    const BVHNode* bvhNodes;      uint32_t numNodes;
    uint32_t numVertices;         const Vertex* vb;
    const uint32_t* ib;           uint32_t numIndices;
    uint32_t numInstances;        const InstanceConstants* instanceConst;
    const Ray* rays;              /* device */
    Hit* hits;                    /* device */
    uint32_t numRays;
    uint32_t flags;               /* STRELKA_TRACE_* */
    unsigned long long* counters; /* device, 2 entries: inner visits, leaf visits (COUNT) */
    uint64_t sceneVersion;
} TraceDesc;

/* Uses the same scene cache as the path tracer object. */
int strelka_trace_execute(StrelkaPathTracer* pt, const TraceDesc* desc, void* stream);

/* Same query with host buffers for rays and hits: copies rays in, traces,
 * copies hits out on the given stream, and synchronises it. */
int strelka_trace_host(StrelkaPathTracer* pt, const TraceDesc* desc, const Ray* hostRays,
                       Hit* hostHits, void* stream);

/* Allocation-free variant of strelka_trace_execute; this entry point has no
 * counterpart in the reference.  For callers that cannot have the library
 * allocate device memory (an engine whose allocator owns the whole heap, a
 * real-time loop that cannot afford cudaMalloc's implicit synchronisation):
 * it needs no pass object and keeps its scratch (the derived leaf-triangle
 * table) in a fixed 12 MiB __device__ array.  Under CUDA's lazy module
 * loading (the default since 12.2) the runtime reserves that array on a
 * device at the first call there and holds it until exit, so a caller whose
 * allocator takes the whole heap should make one call per device first
 * (numNodes = 0 and numRays = 0 does only this set-up).  Scenes above
 * 262,144 BVH nodes (131,072 triangles) are rejected with
 * STRELKA_ERR_INVALID_ARGUMENT; flags other than STRELKA_TRACE_ANY are
 * rejected with STRELKA_ERR_UNSUPPORTED.  The first call on a device looks
 * up the scratch address for that device, so make it before starting any
 * stream capture.  All calls share the scratch: calls that overlap on the
 * GPU race.  deviceStatus (a device word, may be NULL) receives this call's
 * STRELKA_DEV_* bits. */
int strelka_trace_execute_noalloc(const TraceDesc* desc, uint32_t* deviceStatus, void* stream);

/* ------------------------------------------------------------------------- */
/* Neural radiance cache (no counterpart in the reference): a multiresolution
 * hash-grid encoding (16 levels x 2 FP16 features, 2^log2TableSize entries
 * per level, growth 1.5) of the position, degree-4 spherical harmonics of the
 * direction, the normal and the roughness, fed to a 64-wide MLP with 4 hidden
 * ReLU layers and 3 linear outputs (FP16 weights and activations, FP32
 * accumulation on tensor cores), trained online with Adam on the relative L2
 * loss.  Pointers to records are device pointers. */
typedef struct StrelkaNrcRecord {
    float pos[3];
    float dir[3];      /* outgoing direction (towards the previous vertex) */
    float normal[3];
    float roughness;
    float target[3];   /* training: radiance target; path-tracer queries: throughput */
    uint32_t slot;     /* path-tracer queries: wavefront slot */
    uint32_t pad[2];
} StrelkaNrcRecord;    /* 64 bytes */

typedef struct StrelkaNrcConfig {
    float sceneMin[3];
    float sceneMax[3];
    float learningRate;     /* Adam, 1e-2 */
    uint32_t seed;
    uint32_t log2TableSize; /* 19 */
    uint32_t pad[3];
} StrelkaNrcConfig;

int strelka_nrc_create(const StrelkaNrcConfig* config, StrelkaNrc** out);
int strelka_nrc_destroy(StrelkaNrc* nrc);
/* outRGB[3*i + c] = network output for records[i] (device pointers). */
int strelka_nrc_infer(StrelkaNrc* nrc, const StrelkaNrcRecord* records, uint32_t n, float* outRGB, void* stream);
/* One Adam step on the batch; *lossOut (host, may be NULL) receives the mean loss. */
int strelka_nrc_train(StrelkaNrc* nrc, const StrelkaNrcRecord* samples, uint32_t n, float* lossOut, void* stream);
/* Gradients of sum_i sum_c loss without updating (host outputs, may be NULL):
 * mlpGrad (numMlpParams floats), gridGrad (numGridParams floats), lossSum. */
int strelka_nrc_gradients(StrelkaNrc* nrc, const StrelkaNrcRecord* samples, uint32_t n, float* mlpGrad,
                          float* gridGrad, float* lossSum, void* stream);
/* FP32 master parameters, host arrays (numMlpParams and numGridParams floats). */
int strelka_nrc_get_params(StrelkaNrc* nrc, float* mlp, float* grid);
int strelka_nrc_set_params(StrelkaNrc* nrc, const float* mlp, const float* grid);
/* Sizes and the per-level grid resolution (negative when the level is hashed). */
/* Self-test of the bounded wait that guards every tensor-core completion wait
 * of the cache's kernels (no counterpart in the reference: test support).  One
 * thread waits for the first phase of an mbarrier, which nothing completes
 * unless `arrive` is nonzero; after limitNs nanoseconds (at most 1 s) it gives
 * up and sets STRELKA_DEV_MMA_TIMEOUT in *deviceStatus (a device pointer).
 * Asynchronous on `stream`. */
int strelka_selftest_wait_timeout(uint64_t limitNs, int arrive, uint32_t* deviceStatus, void* stream);
/* Reads and clears the cache's device status word (STRELKA_DEV_* bits);
 * synchronises the stream.  When STRELKA_DEV_MMA_TIMEOUT is set, every
 * output of the launches since the previous read (predictions, gradients,
 * the weights and grid after an Adam step) is undefined: a CTA that gave up
 * freed its tensor memory while its matrix multiply may still have been
 * writing it, which can corrupt another CTA's tile.  Discard them and
 * re-create the cache. */
int strelka_nrc_get_device_status(StrelkaNrc* nrc, void* stream, uint32_t* status);
int strelka_nrc_info(StrelkaNrc* nrc, uint32_t* numMlpParams, uint64_t* numGridParams, int32_t* levelRes);

/* ------------------------------------------------------------------------- */
/* BVH construction on the GPU (an extension: BvhBuilder::build,
 * src/render/bvh.cpp:107-254, runs Embree on the host).  Clustering over
 * 63-bit Morton codes of the triangle centroids (PLOC, or a linear BVH),
 * emitted in the same
 * flattened depth-first layout as strelka_bvh_build (one triangle per leaf,
 * 2n-1 nodes, escape indices, +1e-6 padding of the max corner), so every
 * traversal entry point reads it unchanged.  Faster to build than the host
 * SAH builder, slower to trace.  The builder object keeps its scratch
 * memory between builds; calls on one builder must not overlap. */
typedef struct StrelkaBvhBuilder StrelkaBvhBuilder;

enum {
    STRELKA_BVH_LBVH = 0, /* radix tree over the Morton order: fastest build */
    STRELKA_BVH_PLOC = 1  /* parallel locally-ordered clustering (default): SAH-like trees */
};

int strelka_bvh_builder_create(StrelkaBvhBuilder** out);
/* Tree construction of the builder: STRELKA_BVH_PLOC with a neighbour
 * search radius in [1, 32] (default 16), or STRELKA_BVH_LBVH (radius ignored). */
int strelka_bvh_builder_set_mode(StrelkaBvhBuilder* builder, uint32_t mode, uint32_t radius);
int strelka_bvh_builder_destroy(StrelkaBvhBuilder* builder);
/* positions: device array of numPositions corners, 3 per triangle, as
 * createBvhBuffer fills them (src/render/ptrender.cpp:460-511); nodes:
 * device array of nodeCapacity >= 2*numPositions/3 - 1 nodes.  Stream
 * ordered; *numNodes is set on return. */
int strelka_bvh_build_device(StrelkaBvhBuilder* builder, const BVHInputPosition* positions, uint32_t numPositions,
                             BVHNode* nodes, uint32_t nodeCapacity, uint32_t* numNodes, void* stream);
/* The same from the scene's own device buffers: every instance's triangles
 * (indexOffset, indexCount) transformed by objectToWorld on the device, as
 * createBvhBuffer does on the host.  Reads the instance table to the host
 * and synchronises the stream once. */
int strelka_bvh_build_scene_device(StrelkaBvhBuilder* builder, const Vertex* vb, uint32_t numVertices,
                                   const uint32_t* ib, uint32_t numIndices, const InstanceConstants* instances,
                                   uint32_t numInstances, BVHNode* nodes, uint32_t nodeCapacity, uint32_t* numNodes,
                                   void* stream);

/* ------------------------------------------------------------------------- */
/* Scene ingest: the formats on the host side of the path.  The reference
 * produces them in its Hydra render delegate; these functions reproduce that
 * arithmetic so that USD-derived scenes can be replayed here. */

/* packNormal (src/hdStrelka/RenderPass.cpp:50-56): components in [-1, 1]. */
uint32_t strelka_pack_normal(const float normal[3]);
/* packUV (src/hdStrelka/RenderPass.cpp:58-64): components in [-10, 10]. */
uint32_t strelka_pack_uv(const float uv[2]);
/* The vertex loop of HdStrelkaRenderPass::_BakeMeshInstance
 * (RenderPass.cpp:66-126): count points and normals (3 floats each), uvs
 * (2 floats each, may be NULL; v is flipped to 1 - v) into Vertex records;
 * massCenter (may be NULL) = the mean position. */
int strelka_bake_vertices(const float* points, const float* normals, const float* uvs, uint32_t count, Vertex* out,
                          float massCenter[3]);
/* _BlackbodyTemperatureAsRgb (src/hdStrelka/Light.cpp:59-98). */
int strelka_blackbody_rgb(float kelvin, float rgb[3]);

/* The USD light parameters HdStrelkaLight::Sync reads (Light.cpp:112-198). */
typedef struct StrelkaUsdLight {
    uint32_t type;                   /* 0 rect, 1 disk, 2 sphere */
    float color[3];
    uint32_t enableColorTemperature;
    float colorTemperature;          /* kelvin */
    float intensity;
    float exposure;
    float xform[16];                 /* column-major: xform[4*i + j] = GfMatrix4d[i][j] */
    float width, height;             /* rect */
    float radius;                    /* disk, sphere */
    uint32_t pad;
} StrelkaUsdLight;

/* HdStrelkaLight::Sync then Scene::updateLight (src/scene/scene.cpp:459-511). */
int strelka_light_from_usd(const StrelkaUsdLight* light, UniformLight* out);

/* The MDL runtime's buffer readers (shaders/mdl_runtime.hlsl:24-75), run on
 * the device over a device buffer (the argument block or the read-only data
 * segment of PathTracerDesc), one read per (offset, kind): kind 0 float,
 * 1 double, 2 int, 3 uint, 4 bool.  out[i] receives the value's bits
 * (zero-extended to 64).  Reads past `bytes` return 0; word reads ignore the
 * two low bits of the offset, as a ByteAddressBuffer does.  Device code reads
 * through the same functions (csrc/mdl_runtime.cuh). */
int strelka_mdl_read(const uint8_t* buffer, uint64_t bytes, const uint32_t* offsets, const uint32_t* kinds, uint32_t n,
                     uint64_t* out, void* stream);

/* ------------------------------------------------------------------------- */
/* Batched rendering (an extension; the reference renders one view per
 * PathTracer::execute, src/render/pathtracer.cpp:50-59).  Many scene/camera
 * jobs of uneven resolution, sample count, depth and triangle count are
 * rendered by one launch sequence captured once into a CUDA graph.  Each job
 * is a full PathTracerDesc with its own constants (dimension, spp, maxDepth,
 * frameNumber, camera) and its own sampleBuffer of W*H*spp*3 floats; its
 * samples are bit-identical to PathTracer::execute on the same descriptor. */
#define STRELKA_BATCH_MAX_JOBS 64

typedef struct StrelkaBatch StrelkaBatch;

enum {
    STRELKA_BATCH_PERSISTENT = 0, /* one persistent kernel tracing whole paths, fed by an atomic path queue */
    STRELKA_BATCH_WAVEFRONT = 1   /* job-aware wavefront kernels fed by atomic queues */
};

typedef struct StrelkaBatchConfig {
    uint32_t mode;          /* STRELKA_BATCH_* */
    uint32_t blockSize;     /* 64, 128 or 256 threads */
    uint32_t queueChunk;    /* queue items a warp takes at a time: a multiple of 32 in [32, 4096] */
    uint32_t materialSort;  /* wavefront: sort each bounce's shade queue by (job, material) */
    uint32_t useGraph;      /* 1: capture the launch sequence once and replay it with one cudaGraphLaunch */
    uint32_t pad[3];
} StrelkaBatchConfig;

typedef struct StrelkaBatchTuneEntry {
    StrelkaBatchConfig config;
    float ms;               /* median batch time over the repeats (CUDA events) */
    uint32_t pad[3];
} StrelkaBatchTuneEntry;

int strelka_batch_create(StrelkaBatch** out);
int strelka_batch_destroy(StrelkaBatch* batch);
/* Copies the job descriptors (at most STRELKA_BATCH_MAX_JOBS, at most 2^31
 * paths in all) and prepares each distinct scene's traversal records on
 * `stream`.  Device buffers stay owned by the caller.  Drops captured graphs
 * and the tuned configuration.  The batch runs its jobs smallest first (by
 * W*H*spp, ties in the given order) so that small jobs finish early; every
 * job's samples are the same whatever the order, and per-job results
 * (strelka_batch_job_latency) keep the caller's indexing. */
int strelka_batch_set_jobs(StrelkaBatch* batch, const PathTracerDesc* jobs, uint32_t numJobs, void* stream);
/* Sets every job's frameNumber to its descriptor's value + frameOffset
 * (synchronises the stream; captured graphs stay valid). */
int strelka_batch_set_frame(StrelkaBatch* batch, uint32_t frameOffset, void* stream);
/* Renders every job once.  config NULL: the tuned configuration when
 * strelka_batch_autotune has run, else wavefront / 128 / 256 / no sort /
 * graph. */
int strelka_batch_execute(StrelkaBatch* batch, const StrelkaBatchConfig* config, void* stream);
/* Coordinate-descent search over mode, block size {64,128,256}, queue chunk
 * {32..1024} and material sort, each candidate timed as the median of
 * `repeats` executions after one warm-up; keeps the fastest as the default
 * of strelka_batch_execute.  entries (may be NULL) receives every timed
 * candidate, *numEntries their count. */
int strelka_batch_autotune(StrelkaBatch* batch, uint32_t repeats, StrelkaBatchTuneEntry* entries, uint32_t capacity,
                           uint32_t* numEntries, StrelkaBatchConfig* best, void* stream);
/* Per-job latency of the last execution: ms from the batch's start to the
 * job's last sample (device timer); synchronises the stream.  Returns the
 * number of jobs. */
int strelka_batch_job_latency(StrelkaBatch* batch, void* stream, float* ms, uint32_t capacity);
/* Reads and clears the batch's device status word (STRELKA_DEV_* bits). */
int strelka_batch_get_device_status(StrelkaBatch* batch, void* stream, uint32_t* status);
int strelka_batch_info(StrelkaBatch* batch, uint64_t* totalPaths, uint32_t* numJobs, uint32_t* numSortKeys);

/* ------------------------------------------------------------------------- */
/* Host-side scene preparation (replaces BvhBuilder, include/render/bvh.h:38-46). */

/* SAH BVH over world-space triangles (3 consecutive positions per triangle),
 * emitting the reference's flattened depth-first layout with escape indices
 * (src/render/bvh.cpp:169-235).  *outNodes is allocated with malloc; free it
 * with strelka_host_free. */
int strelka_bvh_build(const BVHInputPosition* positions, uint32_t numPositions,
                      BVHNode** outNodes, uint32_t* outNumNodes);
void strelka_host_free(void* p);

/* ------------------------------------------------------------------------- */
/* Errors and versioning */
int strelka_get_last_error(char* buffer, size_t capacity);
int strelka_version(void);
/* Sizes of every struct above, for bindings to check their layouts:
 * returns sizeof for names "PathTracerParam", "BVHNode", ... or 0. */
size_t strelka_sizeof(const char* struct_name);

#ifdef __cplusplus
} /* extern "C" */
#endif

/* Layout pins. */
#ifdef __cplusplus
#define STRELKA_STATIC_ASSERT(c, m) static_assert(c, m)
#else
#define STRELKA_STATIC_ASSERT(c, m) _Static_assert(c, m)
#endif
STRELKA_STATIC_ASSERT(sizeof(PathTracerParam) == 336, "PathTracerParam size");
STRELKA_STATIC_ASSERT(offsetof(PathTracerParam, camPos) == 256, "camPos offset");
STRELKA_STATIC_ASSERT(offsetof(PathTracerParam, dimension) == 272, "dimension offset");
STRELKA_STATIC_ASSERT(offsetof(PathTracerParam, frameNumber) == 288, "frameNumber offset");
STRELKA_STATIC_ASSERT(offsetof(PathTracerParam, len) == 304, "len offset");
STRELKA_STATIC_ASSERT(offsetof(PathTracerParam, stratifiedSamplingType) == 316, "sst offset");
STRELKA_STATIC_ASSERT(sizeof(AccumulationParam) == 416, "AccumulationParam size");
STRELKA_STATIC_ASSERT(offsetof(AccumulationParam, dimension) == 384, "acc dimension offset");
STRELKA_STATIC_ASSERT(offsetof(AccumulationParam, alpha) == 400, "acc alpha offset");
STRELKA_STATIC_ASSERT(sizeof(Tonemapparam) == 16, "Tonemapparam size");
STRELKA_STATIC_ASSERT(sizeof(Upscalepassparam) == 16, "Upscalepassparam size");
STRELKA_STATIC_ASSERT(sizeof(StrelkaUsdLight) == 112, "StrelkaUsdLight size");
STRELKA_STATIC_ASSERT(sizeof(BVHNode) == 32, "BVHNode size");
STRELKA_STATIC_ASSERT(sizeof(Vertex) == 32, "Vertex size");
STRELKA_STATIC_ASSERT(sizeof(InstanceConstants) == 208, "InstanceConstants size");
STRELKA_STATIC_ASSERT(offsetof(InstanceConstants, materialId) == 192, "materialId offset");
STRELKA_STATIC_ASSERT(sizeof(UniformLight) == 112, "UniformLight size");
STRELKA_STATIC_ASSERT(offsetof(UniformLight, type) == 96, "light type offset");
STRELKA_STATIC_ASSERT(sizeof(MdlMaterial) == 16, "MdlMaterial size");
STRELKA_STATIC_ASSERT(sizeof(Mdl_resource_info) == 16, "Mdl_resource_info size");
STRELKA_STATIC_ASSERT(sizeof(Ray) == 32, "Ray size");
STRELKA_STATIC_ASSERT(sizeof(Hit) == 20, "Hit size");
STRELKA_STATIC_ASSERT(sizeof(BVHInputPosition) == 20, "BVHInputPosition size");
STRELKA_STATIC_ASSERT(sizeof(StrelkaMaterialArgs) == 48, "StrelkaMaterialArgs size");
STRELKA_STATIC_ASSERT(sizeof(StrelkaTexture) == 24, "StrelkaTexture size");
STRELKA_STATIC_ASSERT(sizeof(StrelkaNrcRecord) == 64, "StrelkaNrcRecord size");

#endif /* STRELKA_B200_H */
