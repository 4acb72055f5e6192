"""ctypes view of the C ABI in ``include/strelka_b200.h`` and
``include/strelka_b200_scenes.h``.

The structures here are checked field by field against the library's own
``strelka_sizeof`` when the library loads.  The library is required: there is
no Python or CPU fallback for any pass, and loading fails loudly when
``libstrelka_b200.so`` is missing.
"""
from __future__ import annotations

import ctypes as C
import os

_PKG = os.path.dirname(os.path.abspath(__file__))
# STRELKA_B200_LIB selects another build of the library (e.g. a tuning variant)
LIB_PATH = os.environ.get("STRELKA_B200_LIB", os.path.join(_PKG, "libstrelka_b200.so"))

# status codes
OK = 0
ERR_INVALID_ARGUMENT = 1
ERR_OUT_OF_MEMORY = 2
ERR_CUDA = 3
ERR_NO_DEVICE = 4
ERR_DEVICE_BOUNDS = 5
ERR_TIMEOUT = 6
ERR_UNSUPPORTED = 7

DEV_NODE_OOB = 1 << 0
DEV_INSTANCE_OOB = 1 << 1
DEV_INDEX_OOB = 1 << 2
DEV_MATERIAL_OOB = 1 << 3
DEV_LIGHT_OOB = 1 << 4
DEV_TRAVERSAL_CAP = 1 << 5
DEV_TEXTURE_OOB = 1 << 6
DEV_QUEUE_TIMEOUT = 1 << 7
DEV_MMA_TIMEOUT = 1 << 8

FN_LAMBERT = 0
FN_GGX_CONDUCTOR = 1
FN_GGX_DIELECTRIC = 2

BATCH_PERSISTENT = 0
BATCH_WAVEFRONT = 1
BATCH_MAX_JOBS = 64
BVH_LBVH = 0
BVH_PLOC = 1
MODE_WAVEFRONT = 0
MODE_MEGAKERNEL = 1
PT_PROFILE = 1
PT_COUNT = 2
PT_NO_SHADE_SORT = 4
PT_LARGE_SCENE_KERNELS = 8
PT_SMALL_SCENE_KERNELS = 16
PT_SERIAL_SHADOW = 32
PT_FORCE_SHADE_SORT = 64
SHADE_SORT_MIN_PATHS = 1 << 21
LARGE_SCENE_NODES = 1 << 21

TRACE_CLOSEST = 0
TRACE_ANY = 1
TRACE_COUNT = 1 << 4
TRACE_REFINE = 1 << 5

KERNEL_CLASSES = ["generate", "extend", "shade", "shadow", "finalize", "megakernel", "prep", "nrc_paths", "nrc_train",
                  "nrc_infer", "sort", "tail"]

vp = C.c_void_p
u8p = C.POINTER(C.c_uint8)


class Float4(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float), ("w", C.c_float)]


class Float4x4(C.Structure):
    _fields_ = [("m", C.c_float * 16)]


class PathTracerParam(C.Structure):
    _fields_ = [
        ("viewToWorld", Float4x4), ("clipToView", Float4x4), ("viewToClip", Float4x4), ("worldToView", Float4x4),
        ("camPos", Float4), ("dimension", C.c_int32 * 2), ("invDimension", C.c_float * 2),
        ("frameNumber", C.c_uint32), ("maxDepth", C.c_uint32), ("debug", C.c_uint32), ("numLights", C.c_uint32),
        ("len", C.c_int32), ("spp", C.c_int32), ("iteration", C.c_int32), ("stratifiedSamplingType", C.c_uint32),
        ("pad0", Float4),
    ]


class AccumulationParam(C.Structure):
    _fields_ = [
        ("prevViewToWorld", Float4x4), ("prevClipToView", Float4x4), ("prevWorldToView", Float4x4),
        ("prevViewToClip", Float4x4), ("viewToWorld", Float4x4), ("clipToView", Float4x4),
        ("dimension", C.c_int32 * 2), ("frameNumber", C.c_uint32), ("iteration", C.c_uint32),
        ("alpha", C.c_float), ("isPt", C.c_float), ("pad1", C.c_float), ("pad2", C.c_float),
    ]


class Tonemapparam(C.Structure):
    _fields_ = [("dimension", C.c_int32 * 2), ("tonemapperType", C.c_uint32), ("pad0", C.c_uint32)]


class BVHNode(C.Structure):
    _fields_ = [("minBounds", C.c_float * 3), ("instId", C.c_int32), ("maxBounds", C.c_float * 3),
                ("nodeOffset", C.c_int32)]


class Vertex(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("tangent", C.c_uint32), ("normal", C.c_uint32), ("uv", C.c_uint32),
                ("pad0", C.c_float), ("pad1", C.c_float)]


class InstanceConstants(C.Structure):
    _fields_ = [("objectToWorld", Float4x4), ("worldToObject", Float4x4), ("normalMatrix", Float4x4),
                ("materialId", C.c_int32), ("indexOffset", C.c_int32), ("indexCount", C.c_int32),
                ("lightId", C.c_int32)]


class UniformLight(C.Structure):
    _fields_ = [("points", Float4 * 4), ("color", Float4), ("normal", Float4), ("type", C.c_int32),
                ("pad0", C.c_float), ("pad2", C.c_float), ("pad3", C.c_float)]


class MdlMaterial(C.Structure):
    _fields_ = [("arg_block_offset", C.c_int32), ("ro_data_segment_offset", C.c_int32), ("functionId", C.c_int32),
                ("pad1", C.c_int32)]


class Mdl_resource_info(C.Structure):
    _fields_ = [("gpu_resource_array_start", C.c_uint32), ("pad0", C.c_uint32), ("pad1", C.c_uint32),
                ("pad2", C.c_uint32)]


class Ray(C.Structure):
    _fields_ = [("o", Float4), ("d", Float4)]


class Hit(C.Structure):
    _fields_ = [("bary", C.c_float * 2), ("t", C.c_float), ("instId", C.c_uint32), ("primId", C.c_uint32)]


class BVHInputPosition(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("instId", C.c_uint32), ("primId", C.c_uint32)]


class StrelkaMaterialArgs(C.Structure):
    _fields_ = [("base_color", C.c_float * 3), ("roughness", C.c_float), ("emission", C.c_float * 3),
                ("ior", C.c_float), ("base_color_texture", C.c_uint32), ("pad", C.c_uint32 * 3)]


class StrelkaTexture(C.Structure):
    _fields_ = [("rgba8", vp), ("width", C.c_uint32), ("height", C.c_uint32), ("pad", C.c_uint64)]


class StrelkaEnvMap(C.Structure):
    _fields_ = [("rgba32f", vp), ("marginal_cdf", vp), ("conditional_cdf", vp), ("width", C.c_uint32),
                ("height", C.c_uint32), ("integral", C.c_float), ("pad", C.c_float)]


class PathTracerDesc(C.Structure):
    _fields_ = [
        ("constants", PathTracerParam),
        ("bvhNodes", vp), ("numNodes", C.c_uint32),
        ("numVertices", C.c_uint32), ("vb", vp),
        ("ib", vp), ("numIndices", C.c_uint32),
        ("numInstances", C.c_uint32), ("instanceConst", vp),
        ("lights", vp), ("lightCapacity", C.c_uint32),
        ("pad0", C.c_uint32),
        ("sampleBuffer", vp),
        ("mdl_ro_data_segment", vp), ("roDataBytes", C.c_uint64),
        ("mdl_argument_block", vp), ("argBlockBytes", C.c_uint64),
        ("mdl_resource_infos", vp), ("numResourceInfos", C.c_uint32),
        ("numMaterials", C.c_uint32), ("mdl_mdlMaterial", vp),
        ("matTextures", vp),
        ("numTextures", C.c_uint32), ("pad1", C.c_uint32),
        ("envMap", vp),
        ("sceneVersion", C.c_uint64),
    ]


class ReductionDesc(C.Structure):
    _fields_ = [("constants", PathTracerParam), ("sampleBuffer", vp), ("result", vp)]


class AccumulationDesc(C.Structure):
    _fields_ = [("constants", AccumulationParam), ("input", vp), ("history", vp), ("output", vp)]


class TonemapDesc(C.Structure):
    _fields_ = [("constants", Tonemapparam), ("input", vp), ("output", vp)]


class Upscalepassparam(C.Structure):
    _fields_ = [("dimension", C.c_int32 * 2), ("invDimension", C.c_float * 2)]


class UpscaleDesc(C.Structure):
    _fields_ = [("constants", Upscalepassparam), ("input", vp), ("inputWidth", C.c_uint32), ("inputHeight", C.c_uint32),
                ("output", vp)]


class StrelkaUsdLight(C.Structure):
    _fields_ = [("type", C.c_uint32), ("color", C.c_float * 3), ("enableColorTemperature", C.c_uint32),
                ("colorTemperature", C.c_float), ("intensity", C.c_float), ("exposure", C.c_float),
                ("xform", C.c_float * 16), ("width", C.c_float), ("height", C.c_float), ("radius", C.c_float),
                ("pad", C.c_uint32)]


class StrelkaPathTracerConfig(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("chunkPaths", C.c_uint32), ("blockSize", C.c_uint32), ("flags", C.c_uint32),
                ("queueChunk", C.c_uint32), ("tailDepth", C.c_uint32), ("pad", C.c_uint32 * 2)]


class TraceDesc(C.Structure):
    _fields_ = [
        ("bvhNodes", vp), ("numNodes", C.c_uint32),
        ("numVertices", C.c_uint32), ("vb", vp),
        ("ib", vp), ("numIndices", C.c_uint32),
        ("numInstances", C.c_uint32), ("instanceConst", vp),
        ("rays", vp), ("hits", vp),
        ("numRays", C.c_uint32), ("flags", C.c_uint32),
        ("counters", vp),
        ("sceneVersion", C.c_uint64),
    ]


class StrelkaNrcRecord(C.Structure):
    _fields_ = [("pos", C.c_float * 3), ("dir", C.c_float * 3), ("normal", C.c_float * 3), ("roughness", C.c_float),
                ("target", C.c_float * 3), ("slot", C.c_uint32), ("pad", C.c_uint32 * 2)]


class StrelkaNrcConfig(C.Structure):
    _fields_ = [("sceneMin", C.c_float * 3), ("sceneMax", C.c_float * 3), ("learningRate", C.c_float),
                ("seed", C.c_uint32), ("log2TableSize", C.c_uint32), ("pad", C.c_uint32 * 3)]


class StrelkaNrcRenderConfig(C.Structure):
    _fields_ = [("enable", C.c_uint32), ("trainPaths", C.c_uint32), ("trainSteps", C.c_uint32),
                ("diffuseRoughness", C.c_float), ("pad", C.c_uint32 * 4)]


class StrelkaBatchConfig(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("blockSize", C.c_uint32), ("queueChunk", C.c_uint32),
                ("materialSort", C.c_uint32), ("useGraph", C.c_uint32), ("pad", C.c_uint32 * 3)]


class StrelkaBatchTuneEntry(C.Structure):
    _fields_ = [("config", StrelkaBatchConfig), ("ms", C.c_float), ("pad", C.c_uint32 * 3)]


class StrelkaHostScene(C.Structure):
    _fields_ = [
        ("vb", C.POINTER(Vertex)), ("numVertices", C.c_uint32),
        ("ib", C.POINTER(C.c_uint32)), ("numIndices", C.c_uint32),
        ("instances", C.POINTER(InstanceConstants)), ("numInstances", C.c_uint32),
        ("lights", C.POINTER(UniformLight)), ("numLights", C.c_uint32),
        ("materials", C.POINTER(MdlMaterial)), ("numMaterials", C.c_uint32),
        ("argBlock", u8p), ("argBlockBytes", C.c_uint64),
        ("resourceInfos", C.POINTER(Mdl_resource_info)), ("numResourceInfos", C.c_uint32),
        ("numTextures", C.c_uint32),
        ("textures", C.POINTER(u8p)),
        ("texWidth", C.POINTER(C.c_uint32)),
        ("texHeight", C.POINTER(C.c_uint32)),
        ("envRGBA", C.POINTER(C.c_float)),
        ("envWidth", C.c_uint32), ("envHeight", C.c_uint32),
        ("envMarginalCdf", C.POINTER(C.c_float)),
        ("envConditionalCdf", C.POINTER(C.c_float)),
        ("envIntegral", C.c_float),
        ("nodes", C.POINTER(BVHNode)), ("numNodes", C.c_uint32),
        ("numTriangles", C.c_uint32),
        ("camera", PathTracerParam),
    ]


class StrelkaCornellConfig(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("sphereLevels", C.c_uint32),
                ("lightSide", C.c_float), ("lightRadiance", C.c_float), ("maxDepth", C.c_uint32),
                ("spp", C.c_uint32), ("tonemapper", C.c_uint32), ("extraLights", C.c_uint32)]


class StrelkaLargeConfig(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("instances", C.c_uint32),
                ("frequency", C.c_uint32), ("numTextures", C.c_uint32), ("texSize", C.c_uint32),
                ("envWidth", C.c_uint32), ("envHeight", C.c_uint32), ("maxDepth", C.c_uint32),
                ("spp", C.c_uint32), ("seed", C.c_uint64)]


# every extern "C" entry point: name -> (restype, argtypes)
SIGNATURES = {
    "strelka_pathtracer_create": (C.c_int, [C.POINTER(StrelkaPathTracerConfig), C.POINTER(vp)]),
    "strelka_pathtracer_destroy": (C.c_int, [vp]),
    "strelka_pathtracer_execute": (C.c_int, [vp, C.POINTER(PathTracerDesc), C.c_uint32, C.c_uint32, C.c_uint64, vp]),
    "strelka_pathtracer_get_device_status": (C.c_int, [vp, vp, C.POINTER(C.c_uint32)]),
    "strelka_pathtracer_get_kernel_times": (C.c_int, [vp, vp, C.POINTER(C.c_float), C.POINTER(C.c_uint32), C.c_uint32]),
    "strelka_pathtracer_get_counters": (C.c_int, [vp, vp, C.POINTER(C.c_uint64), C.c_uint32]),
    "strelka_pathtracer_set_nrc": (C.c_int, [vp, vp, C.POINTER(StrelkaNrcRenderConfig)]),
    "strelka_pathtracer_train_nrc": (C.c_int, [vp, C.POINTER(PathTracerDesc), C.c_uint64, C.c_uint32, vp]),
    "strelka_reduction_execute": (C.c_int, [C.POINTER(ReductionDesc), C.c_uint32, C.c_uint32, C.c_uint64, vp]),
    "strelka_accumulation_execute": (C.c_int, [C.POINTER(AccumulationDesc), C.c_uint32, C.c_uint32, C.c_uint64, vp]),
    "strelka_tonemap_execute": (C.c_int, [C.POINTER(TonemapDesc), C.c_uint32, C.c_uint32, C.c_uint64, vp]),
    "strelka_upscale_execute": (C.c_int, [C.POINTER(UpscaleDesc), C.c_uint32, C.c_uint32, C.c_uint64, vp]),
    "strelka_tonemap_upscale_execute": (C.c_int, [C.POINTER(Tonemapparam), vp, C.POINTER(Upscalepassparam), vp, vp, vp]),
    "strelka_resolve_execute": (C.c_int, [C.POINTER(PathTracerParam), vp, C.c_int, C.POINTER(AccumulationParam), vp,
                                          vp, C.POINTER(Tonemapparam), vp, vp, vp]),
    "strelka_trace_execute": (C.c_int, [vp, C.POINTER(TraceDesc), vp]),
    "strelka_trace_host": (C.c_int, [vp, C.POINTER(TraceDesc), vp, vp, vp]),
    "strelka_trace_execute_noalloc": (C.c_int, [C.POINTER(TraceDesc), vp, vp]),
    "strelka_nrc_create": (C.c_int, [C.POINTER(StrelkaNrcConfig), C.POINTER(vp)]),
    "strelka_nrc_destroy": (C.c_int, [vp]),
    "strelka_nrc_infer": (C.c_int, [vp, vp, C.c_uint32, vp, vp]),
    "strelka_nrc_train": (C.c_int, [vp, vp, C.c_uint32, C.POINTER(C.c_float), vp]),
    "strelka_nrc_gradients": (C.c_int, [vp, vp, C.c_uint32, vp, vp, C.POINTER(C.c_float), vp]),
    "strelka_nrc_get_params": (C.c_int, [vp, vp, vp]),
    "strelka_nrc_set_params": (C.c_int, [vp, vp, vp]),
    "strelka_nrc_info": (C.c_int, [vp, C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), vp]),
    "strelka_nrc_get_device_status": (C.c_int, [vp, vp, C.POINTER(C.c_uint32)]),
    "strelka_selftest_wait_timeout": (C.c_int, [C.c_uint64, C.c_int, vp, vp]),
    "strelka_batch_create": (C.c_int, [C.POINTER(vp)]),
    "strelka_batch_destroy": (C.c_int, [vp]),
    "strelka_batch_set_jobs": (C.c_int, [vp, vp, C.c_uint32, vp]),
    "strelka_batch_set_frame": (C.c_int, [vp, C.c_uint32, vp]),
    "strelka_batch_execute": (C.c_int, [vp, C.POINTER(StrelkaBatchConfig), vp]),
    "strelka_batch_autotune": (C.c_int, [vp, C.c_uint32, C.POINTER(StrelkaBatchTuneEntry), C.c_uint32,
                                         C.POINTER(C.c_uint32), C.POINTER(StrelkaBatchConfig), vp]),
    "strelka_batch_job_latency": (C.c_int, [vp, vp, C.POINTER(C.c_float), C.c_uint32]),
    "strelka_batch_get_device_status": (C.c_int, [vp, vp, C.POINTER(C.c_uint32)]),
    "strelka_batch_info": (C.c_int, [vp, C.POINTER(C.c_uint64), C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]),
    "strelka_camera_lookat": (C.c_int, [C.POINTER(PathTracerParam), C.c_uint32, C.c_uint32, C.POINTER(C.c_float),
                                        C.POINTER(C.c_float), C.c_float]),
    "strelka_mdl_read": (C.c_int, [vp, C.c_uint64, vp, vp, C.c_uint32, vp, vp]),
    "strelka_pack_normal": (C.c_uint32, [C.POINTER(C.c_float)]),
    "strelka_pack_uv": (C.c_uint32, [C.POINTER(C.c_float)]),
    "strelka_bake_vertices": (C.c_int, [vp, vp, vp, C.c_uint32, vp, C.POINTER(C.c_float)]),
    "strelka_blackbody_rgb": (C.c_int, [C.c_float, C.POINTER(C.c_float)]),
    "strelka_light_from_usd": (C.c_int, [C.POINTER(StrelkaUsdLight), C.POINTER(UniformLight)]),
    "strelka_bvh_builder_create": (C.c_int, [C.POINTER(vp)]),
    "strelka_bvh_builder_destroy": (C.c_int, [vp]),
    "strelka_bvh_builder_set_mode": (C.c_int, [vp, C.c_uint32, C.c_uint32]),
    "strelka_bvh_build_device": (C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint32, C.POINTER(C.c_uint32), vp]),
    "strelka_bvh_build_scene_device": (C.c_int, [vp, vp, C.c_uint32, vp, C.c_uint32, vp, C.c_uint32, vp, C.c_uint32,
                                                 C.POINTER(C.c_uint32), vp]),
    "strelka_bvh_build": (C.c_int, [C.POINTER(BVHInputPosition), C.c_uint32, C.POINTER(C.POINTER(BVHNode)),
                                    C.POINTER(C.c_uint32)]),
    "strelka_host_free": (None, [vp]),
    "strelka_get_last_error": (C.c_int, [C.c_char_p, C.c_size_t]),
    "strelka_version": (C.c_int, []),
    "strelka_sizeof": (C.c_size_t, [C.c_char_p]),
    "strelka_scene_cornell": (C.c_int, [C.POINTER(StrelkaCornellConfig), C.POINTER(StrelkaHostScene)]),
    "strelka_scene_soup": (C.c_int, [C.c_uint32, C.c_uint64, C.POINTER(StrelkaHostScene)]),
    "strelka_rays_soup": (C.c_int, [C.c_uint32, C.c_uint64, C.c_int, vp]),
    "strelka_scene_large": (C.c_int, [C.POINTER(StrelkaLargeConfig), C.POINTER(StrelkaHostScene)]),
    "strelka_envmap_build_cdf_host": (C.c_int, [vp, C.c_uint32, C.c_uint32, vp, vp, C.POINTER(C.c_float)]),
    "strelka_scene_free": (None, [C.POINTER(StrelkaHostScene)]),
}

LAYOUT_CHECK = [PathTracerParam, AccumulationParam, Tonemapparam, BVHNode, Vertex, InstanceConstants, UniformLight,
                MdlMaterial, Mdl_resource_info, Ray, Hit, BVHInputPosition, StrelkaMaterialArgs, StrelkaTexture,
                StrelkaEnvMap, PathTracerDesc, ReductionDesc, AccumulationDesc, TonemapDesc, Upscalepassparam,
                UpscaleDesc, StrelkaUsdLight, TraceDesc,
                StrelkaPathTracerConfig, StrelkaNrcRecord, StrelkaNrcConfig, StrelkaNrcRenderConfig,
                StrelkaBatchConfig, StrelkaBatchTuneEntry]

_lib = None


class StrelkaError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"strelka error {code}: {message}")
        self.code = code


def load() -> C.CDLL:
    """Loads the in-tree library and checks every struct layout against it."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m strelka_b200.build`")
    lib = C.CDLL(LIB_PATH)
    for name, (res, args) in SIGNATURES.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    for st in LAYOUT_CHECK:
        n = lib.strelka_sizeof(st.__name__.encode())
        if n != C.sizeof(st):
            raise ImportError(f"layout mismatch for {st.__name__}: C {n} vs ctypes {C.sizeof(st)}")
    _lib = lib
    return lib


def last_error() -> str:
    lib = load()
    buf = C.create_string_buffer(1024)
    lib.strelka_get_last_error(buf, len(buf))
    return buf.value.decode(errors="replace")


def check(rc: int) -> None:
    if rc != OK:
        raise StrelkaError(rc, last_error())
