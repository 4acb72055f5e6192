"""Python bindings of the CPU oracle (``oracle/liboracle.so``).

TEST INFRASTRUCTURE ONLY: the checker for the CUDA path.  Only the tests,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import
this module; the product never does.

The oracle restates the reference's shader math in C (``oracle/oracle.c``,
each function citing the reference lines it follows).  Parity status: pinned
to the reference's own shader source.  oracle/build_ref.sh compiles the
reference's pathtracerMdl.hlsl (with its includes), reduction, accumulation,
tonemap and upscale shaders on the host into oracle/_ref/ (``oracle.ref``),
and tests/test_ref_pin.py checks this restatement against it bit for bit,
function by function and sample by sample.  Also: the reference's slab-test
known answers (tests/intersection/aabb.cpp), hand-computed RNG states,
analytic checks and the golden fixtures under ``tests/golden/``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_DIR, "liboracle.so")
FAST_LIB_PATH = os.path.join(_DIR, "liboracle_fast.so")
WORKLOAD_LIB_PATH = os.path.join(_DIR, "libworkload.so")

_libs: dict[str, C.CDLL] = {}


def build() -> None:
    """Builds the oracle's libraries, and oracle/_ref from the reference's
    own shader sources when the reference tree is present."""
    subprocess.run(["sh", os.path.join(_DIR, "build.sh")], check=True)
    subprocess.run(["sh", os.path.join(_DIR, "build_ref.sh")], check=True)


class OracleTexture(C.Structure):
    _fields_ = [("rgba8", C.c_void_p), ("width", C.c_uint32), ("height", C.c_uint32)]


class OracleEnvMap(C.Structure):
    _fields_ = [("rgba32f", C.c_void_p), ("marginal_cdf", C.c_void_p), ("conditional_cdf", C.c_void_p),
                ("width", C.c_uint32), ("height", C.c_uint32), ("integral", C.c_float)]


class OracleScene(C.Structure):
    _fields_ = [
        ("nodes", C.c_void_p), ("numNodes", C.c_uint32),
        ("vb", C.c_void_p), ("numVertices", C.c_uint32),
        ("ib", C.c_void_p), ("numIndices", C.c_uint32),
        ("instances", C.c_void_p), ("numInstances", C.c_uint32),
        ("lights", C.c_void_p), ("lightCapacity", C.c_uint32),
        ("argBlock", C.c_void_p), ("argBlockBytes", C.c_uint64),
        ("materials", C.c_void_p), ("numMaterials", C.c_uint32),
        ("resourceInfos", C.c_void_p), ("numResourceInfos", C.c_uint32),
        ("textures", C.c_void_p), ("numTextures", C.c_uint32),
        ("envMap", C.c_void_p),
    ]


def load(fast: bool = False) -> C.CDLL:
    path = FAST_LIB_PATH if fast else LIB_PATH
    if path in _libs:
        return _libs[path]
    if not os.path.exists(path):
        build()
    lib = C.CDLL(path)
    vp, u32, f32 = C.c_void_p, C.c_uint32, C.c_float
    sigs = {
        "oracle_jenkins_hash": (u32, [u32]),
        "oracle_init_rng": (u32, [u32, u32, u32, u32]),
        "oracle_xorshift": (u32, [C.POINTER(u32)]),
        "oracle_rand": (f32, [C.POINTER(u32)]),
        "oracle_permute": (u32, [u32, u32, u32]),
        "oracle_randfloat": (f32, [u32, u32]),
        "oracle_sinf": (f32, [f32]),
        "oracle_cosf": (f32, [f32]),
        "oracle_acosf": (f32, [f32]),
        "oracle_unpack_normal": (None, [u32, vp]),
        "oracle_unpack_uv": (None, [u32, vp]),
        "oracle_offset_ray": (None, [vp, vp, vp]),
        "oracle_intersect_ray_box": (C.c_int, [vp, vp, vp, vp, C.POINTER(f32)]),
        "oracle_ray_triangle": (C.c_int, [vp, vp, vp, vp, vp, C.POINTER(f32), C.POINTER(f32), C.POINTER(f32)]),
        "oracle_trace": (C.c_int, [C.POINTER(OracleScene), vp, u32, vp, vp, C.c_int, C.c_int, vp, C.c_int]),
        "oracle_trace_warp": (C.c_int, [C.POINTER(OracleScene), vp, u32, vp, vp, vp]),
        "oracle_intersect_fp64": (C.c_int, [C.POINTER(OracleScene), vp, vp, vp, u32, vp, vp, vp]),
        "oracle_intersect_terms_fp64": (C.c_int, [C.POINTER(OracleScene), vp, vp, vp, u32, vp]),
        "oracle_pathtrace": (C.c_int, [vp, C.POINTER(OracleScene), vp, C.c_int]),
        "oracle_pathtrace_range": (C.c_int, [vp, C.POINTER(OracleScene), vp, C.c_uint64, C.c_uint64, C.c_int]),
        "oracle_reduce": (C.c_int, [vp, vp, vp]),
        "oracle_accumulate": (C.c_int, [vp, vp, vp, vp]),
        "oracle_tonemap": (C.c_int, [vp, vp, vp]),
        "oracle_upscale": (C.c_int, [vp, vp, C.c_uint32, C.c_uint32, vp]),
        "oracle_mdl_read": (None, [vp, C.c_uint64, vp, vp, C.c_uint32, vp]),
        "oracle_tex_lookup": (None, [vp, f32, f32, vp]),
        "oracle_sample_light": (None, [vp, vp, f32, f32, vp]),
        "oracle_camera_ray": (None, [vp, u32, u32, C.POINTER(u32), u32, vp]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _libs[path] = lib
    return lib


def workload() -> C.CDLL:
    """The CPU-only build of the package's seeded scene generators and host
    SAH builder (oracle/libworkload.so), for processes that build workloads
    without loading the CUDA library: pass it to
    strelka_b200.scenes.use_generator_library."""
    if WORKLOAD_LIB_PATH in _libs:
        return _libs[WORKLOAD_LIB_PATH]
    if not os.path.exists(WORKLOAD_LIB_PATH):
        build()
    lib = C.CDLL(WORKLOAD_LIB_PATH)
    _libs[WORKLOAD_LIB_PATH] = lib
    return lib


def _ptr(a: np.ndarray) -> C.c_void_p:
    return C.c_void_p(a.ctypes.data) if a is not None and a.size else C.c_void_p(0)


class SceneView:
    """An OracleScene over a strelka_b200.scenes.HostScene (keeps arrays alive)."""

    def __init__(self, hs):
        self.hs = hs
        self._keep = []
        texs = (OracleTexture * max(len(hs.textures), 1))()
        for i, t in enumerate(hs.textures):
            t = np.ascontiguousarray(t)
            self._keep.append(t)
            texs[i] = OracleTexture(t.ctypes.data, t.shape[1], t.shape[0])
        self._texs = texs
        env = None
        if hs.env is not None:
            env = OracleEnvMap(hs.env.ctypes.data, hs.env_marginal.ctypes.data, hs.env_conditional.ctypes.data,
                               hs.env.shape[1], hs.env.shape[0], hs.env_integral)
        self._env = env
        self.scene = OracleScene(
            _ptr(hs.nodes), hs.num_nodes, _ptr(hs.vb), hs.num_vertices, _ptr(hs.ib), hs.ib.size,
            _ptr(hs.instances), hs.num_instances, _ptr(hs.lights), hs.lights.size // 112,
            _ptr(hs.arg_block), hs.arg_block.size, _ptr(hs.materials), hs.num_materials,
            _ptr(hs.resource_infos), hs.resource_infos.size // 16,
            C.cast(texs, C.c_void_p) if hs.textures else C.c_void_p(0), len(hs.textures),
            C.cast(C.pointer(env), C.c_void_p) if env is not None else C.c_void_p(0))


def trace(view: SceneView, rays: np.ndarray, any_hit: bool = False, prune: bool = False, threads: int = 0):
    """Returns (hits (n,5) uint32 raw Hit records, found (n,) bool, counters (2,) uint64)."""
    lib = load()
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[0]
    hits = np.zeros((n, 5), np.uint32)
    found = np.zeros(n, np.uint8)
    counters = np.zeros(2, np.uint64)
    lib.oracle_trace(C.byref(view.scene), _ptr(rays), n, _ptr(hits), _ptr(found), 1 if any_hit else 0,
                     int(prune), _ptr(counters), threads)
    return hits, found.astype(bool), counters


def trace_warp(view: SceneView, rays: np.ndarray):
    """The closest-hit kernels' deferred leaf tests replayed for one warp that
    takes all n rays from one work chunk: (hits (n,5) uint32, found (n,) bool,
    counters (2,) uint64 = 4-wide nodes processed, triangle tests)."""
    lib = load()
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[0]
    hits = np.zeros((n, 5), np.uint32)
    found = np.zeros(n, np.uint8)
    counters = np.zeros(2, np.uint64)
    if lib.oracle_trace_warp(C.byref(view.scene), _ptr(rays), n, _ptr(hits), _ptr(found), _ptr(counters)) != 0:
        raise MemoryError("oracle_trace_warp")
    return hits, found.astype(bool), counters


def intersect_fp64(view: SceneView, rays: np.ndarray, inst: np.ndarray, prim: np.ndarray):
    lib = load()
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[0]
    inst = np.ascontiguousarray(inst, np.uint32)
    prim = np.ascontiguousarray(prim, np.uint32)
    t = np.zeros(n, np.float64)
    u = np.zeros(n, np.float64)
    v = np.zeros(n, np.float64)
    lib.oracle_intersect_fp64(C.byref(view.scene), _ptr(rays), _ptr(inst), _ptr(prim), n, _ptr(t), _ptr(u), _ptr(v))
    return t, u, v


def intersect_terms_fp64(view: SceneView, rays: np.ndarray, inst: np.ndarray, prim: np.ndarray) -> np.ndarray:
    """(n, 3) conditioning scales of u, v, t (oracle_intersect_terms_fp64)."""
    lib = load()
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[0]
    out = np.zeros((n, 3), np.float64)
    lib.oracle_intersect_terms_fp64(C.byref(view.scene), _ptr(rays), _ptr(np.ascontiguousarray(inst, np.uint32)),
                                    _ptr(np.ascontiguousarray(prim, np.uint32)), n, _ptr(out))
    return out


def pathtrace(view: SceneView, param, threads: int = 0, first: int = 0, count: int | None = None,
              fast: bool = False) -> np.ndarray:
    """sampleBuffer (count*3 float32) for sample indices [first, first+count)."""
    lib = load(fast)
    total = param.dimension[0] * param.dimension[1] * param.spp
    if count is None:
        count = total - first
    out = np.zeros(count * 3, np.float32)
    lib.oracle_pathtrace_range(C.byref(param), C.byref(view.scene), _ptr(out), first, count, threads)
    return out


def reduce(param, sample_buffer: np.ndarray) -> np.ndarray:
    lib = load()
    out = np.zeros(param.dimension[0] * param.dimension[1] * 4, np.float32)
    lib.oracle_reduce(C.byref(param), _ptr(np.ascontiguousarray(sample_buffer, np.float32)), _ptr(out))
    return out


def accumulate(param, inp: np.ndarray, hist: np.ndarray) -> np.ndarray:
    lib = load()
    out = np.zeros_like(inp, dtype=np.float32)
    lib.oracle_accumulate(C.byref(param), _ptr(np.ascontiguousarray(inp, np.float32)),
                          _ptr(np.ascontiguousarray(hist, np.float32)), _ptr(out))
    return out


def mdl_read(buffer: np.ndarray, offsets: np.ndarray, kinds: np.ndarray) -> np.ndarray:
    """mdl_runtime.hlsl:24-75 readers over a byte buffer; uint64 bits per read."""
    lib = load()
    b = np.ascontiguousarray(buffer, np.uint8)
    o = np.ascontiguousarray(offsets, np.uint32)
    k = np.ascontiguousarray(kinds, np.uint32)
    out = np.zeros(o.size, np.uint64)
    lib.oracle_mdl_read(_ptr(b), b.size, _ptr(o), _ptr(k), o.size, _ptr(out))
    return out


def upscale(param, inp: np.ndarray, in_w: int, in_h: int) -> np.ndarray:
    """upscalepass.hlsl:9-21; inp is (in_h * in_w * 4) RGBA32F, param an
    Upscalepassparam with the output size."""
    lib = load()
    out = np.zeros(param.dimension[0] * param.dimension[1] * 4, np.float32)
    lib.oracle_upscale(C.byref(param), _ptr(np.ascontiguousarray(inp, np.float32)), in_w, in_h, _ptr(out))
    return out


def tonemap(param, inp: np.ndarray, init: np.ndarray | None = None) -> np.ndarray:
    lib = load()
    out = np.zeros_like(inp, dtype=np.float32) if init is None else init.copy()
    lib.oracle_tonemap(C.byref(param), _ptr(np.ascontiguousarray(inp, np.float32)), _ptr(out))
    return out
