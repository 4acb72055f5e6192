"""Host-side synthetic scenes (wrappers over ``strelka_scene_*``).

A :class:`HostScene` owns numpy copies of the buffers the reference uploads
at frame 0 (vertices, indices, instance constants, lights, MDL material
tables, textures, the environment map and the flattened BVH) plus a
``PathTracerParam`` template holding the camera.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import abi

# The library the generators are called from: the package's own by default.
# A CPU-only build of the same generator sources can stand in for it
# (use_generator_library), so that a process can build scenes without
# loading the CUDA library.
_gen_lib: C.CDLL | None = None


def use_generator_library(lib: C.CDLL | None) -> None:
    """Calls the scene generators through `lib` (a library exporting the
    strelka_scene_* / strelka_rays_soup / strelka_camera_lookat /
    strelka_bvh_build entry points of include/strelka_b200_scenes.h), or
    through the package's library again when `lib` is None."""
    global _gen_lib
    if lib is not None:
        for name, (res, args) in abi.SIGNATURES.items():
            fn = getattr(lib, name, None)
            if fn is not None:
                fn.restype = res
                fn.argtypes = args
    _gen_lib = lib


def _lib() -> C.CDLL:
    return _gen_lib if _gen_lib is not None else abi.load()


def _check(lib: C.CDLL, rc: int) -> None:
    if rc != abi.OK:
        buf = C.create_string_buffer(1024)
        lib.strelka_get_last_error(buf, len(buf))
        raise abi.StrelkaError(rc, buf.value.decode(errors="replace"))


def _np(ptr, count: int, ctype) -> np.ndarray:
    """Copies `count` elements of a ctypes array pointer into a uint8 numpy array."""
    nbytes = count * C.sizeof(ctype)
    if nbytes == 0 or not ptr:
        return np.zeros(0, np.uint8)
    buf = (C.c_uint8 * nbytes).from_address(C.addressof(ptr.contents))
    return np.frombuffer(buf, dtype=np.uint8).copy()


@dataclass
class HostScene:
    vb: np.ndarray            # uint8, numVertices * 32
    ib: np.ndarray            # uint32
    instances: np.ndarray     # uint8, numInstances * 208
    lights: np.ndarray        # uint8, max(numLights, 1) * 112
    num_lights: int
    materials: np.ndarray     # uint8, numMaterials * 16
    arg_block: np.ndarray     # uint8
    resource_infos: np.ndarray  # uint8, n * 16
    textures: list = field(default_factory=list)  # list of (H, W, 4) uint8
    env: np.ndarray | None = None           # (H, W, 4) float32
    env_marginal: np.ndarray | None = None  # float32 H+1
    env_conditional: np.ndarray | None = None  # float32 H*(W+1)
    env_integral: float = 0.0
    nodes: np.ndarray = None  # uint8, numNodes * 32
    num_triangles: int = 0
    camera: abi.PathTracerParam = None

    @property
    def num_vertices(self) -> int:
        return self.vb.size // 32

    @property
    def num_nodes(self) -> int:
        return self.nodes.size // 32

    @property
    def num_instances(self) -> int:
        return self.instances.size // 208

    @property
    def num_materials(self) -> int:
        return self.materials.size // 16

    def bounds(self) -> tuple[np.ndarray, np.ndarray]:
        """World-space box of the scene: the root node of the BVH (node 0 of
        the depth-first layout)."""
        if self.num_nodes == 0:
            return np.zeros(3, np.float32), np.ones(3, np.float32)
        root = self.nodes[:32].view(np.float32)
        return root[0:3].copy(), root[4:7].copy()

    def look_at(self, width: int, height: int, eye, target, fov_deg: float = 40.0, **kw) -> abi.PathTracerParam:
        """The parameter block with a pinhole camera at `eye` looking at
        `target` (strelka_camera_lookat), rendering width x height, and
        other fields overridden by `kw`."""
        p = self.param(**kw)
        e = (C.c_float * 3)(*[float(v) for v in eye])
        t = (C.c_float * 3)(*[float(v) for v in target])
        lib = _lib()
        _check(lib, lib.strelka_camera_lookat(C.byref(p), width, height, e, t, fov_deg))
        return p

    def param(self, **kw) -> abi.PathTracerParam:
        """A copy of the camera parameter block with fields overridden by `kw`."""
        p = abi.PathTracerParam()
        C.memmove(C.byref(p), C.byref(self.camera), C.sizeof(p))
        for k, v in kw.items():
            setattr(p, k, v)
        return p


def _from_c(hs: abi.StrelkaHostScene) -> HostScene:
    lib = _lib()
    try:
        textures = []
        for i in range(hs.numTextures):
            w, h = hs.texWidth[i], hs.texHeight[i]
            buf = (C.c_uint8 * (w * h * 4)).from_address(C.cast(hs.textures[i], C.c_void_p).value)
            textures.append(np.frombuffer(buf, np.uint8).reshape(h, w, 4).copy())
        env = marg = cond = None
        if hs.envRGBA:
            W, H = hs.envWidth, hs.envHeight
            env = np.ctypeslib.as_array(hs.envRGBA, shape=(H * W * 4,)).reshape(H, W, 4).copy()
            marg = np.ctypeslib.as_array(hs.envMarginalCdf, shape=(H + 1,)).copy()
            cond = np.ctypeslib.as_array(hs.envConditionalCdf, shape=(H * (W + 1),)).copy()
        cam = abi.PathTracerParam()
        C.memmove(C.byref(cam), C.byref(hs.camera), C.sizeof(cam))
        return HostScene(
            vb=_np(hs.vb, hs.numVertices, abi.Vertex),
            ib=_np(hs.ib, hs.numIndices, C.c_uint32).view(np.uint32),
            instances=_np(hs.instances, hs.numInstances, abi.InstanceConstants),
            lights=_np(hs.lights, max(hs.numLights, 1), abi.UniformLight),
            num_lights=hs.numLights,
            materials=_np(hs.materials, hs.numMaterials, abi.MdlMaterial),
            arg_block=_np(hs.argBlock, hs.argBlockBytes, C.c_uint8),
            resource_infos=_np(hs.resourceInfos, hs.numResourceInfos, abi.Mdl_resource_info),
            textures=textures,
            env=env, env_marginal=marg, env_conditional=cond, env_integral=hs.envIntegral,
            nodes=_np(hs.nodes, hs.numNodes, abi.BVHNode),
            num_triangles=hs.numTriangles,
            camera=cam,
        )
    finally:
        lib.strelka_scene_free(C.byref(hs))


CORNELL_DISC_LIGHT = 1
CORNELL_SPHERE_LIGHT = 2


def cornell(width: int = 512, height: int = 512, sphere_levels: int = 4, light_side: float = 0.25,
            light_radiance: float = 15.0, max_depth: int = 4, spp: int = 1, extra_lights: int = 0) -> HostScene:
    """The Cornell box; extra_lights adds a disc light under the ceiling light
    (CORNELL_DISC_LIGHT) and/or a sphere light (CORNELL_SPHERE_LIGHT)."""
    lib = _lib()
    cfg = abi.StrelkaCornellConfig(width, height, sphere_levels, light_side, light_radiance, max_depth, spp, 1,
                                   extra_lights)
    hs = abi.StrelkaHostScene()
    _check(lib, lib.strelka_scene_cornell(C.byref(cfg), C.byref(hs)))
    return _from_c(hs)


def soup(num_tris: int, seed: int = 0) -> HostScene:
    lib = _lib()
    hs = abi.StrelkaHostScene()
    _check(lib, lib.strelka_scene_soup(num_tris, seed, C.byref(hs)))
    return _from_c(hs)


def large(width: int = 1920, height: int = 1080, instances: int = 64, frequency: int = 89, num_textures: int = 8,
          tex_size: int = 2048, env_width: int = 1024, env_height: int = 512, max_depth: int = 8, spp: int = 16,
          seed: int = 0) -> HostScene:
    lib = _lib()
    cfg = abi.StrelkaLargeConfig(width, height, instances, frequency, num_textures, tex_size, env_width, env_height,
                                 max_depth, spp, seed)
    hs = abi.StrelkaHostScene()
    _check(lib, lib.strelka_scene_large(C.byref(cfg), C.byref(hs)))
    return _from_c(hs)


def rays_soup(n: int, seed: int = 1, shadow: bool = False) -> np.ndarray:
    """(n, 8) float32 rays: origin xyz, tmax, direction xyz, 0."""
    lib = _lib()
    out = np.zeros((n, 8), np.float32)
    _check(lib, lib.strelka_rays_soup(n, seed, 1 if shadow else 0, out.ctypes.data_as(C.c_void_p)))
    return out


def bvh_build(positions: np.ndarray, inst_ids: np.ndarray, prim_ids: np.ndarray) -> np.ndarray:
    """SAH BVH over world-space triangle corners (positions (3N, 3) float32);
    returns the flattened nodes as uint8 (numNodes * 32)."""
    lib = _lib()
    n = positions.shape[0]
    arr = (abi.BVHInputPosition * max(n, 1))()
    raw = np.frombuffer(arr, dtype=np.uint8).reshape(max(n, 1), 20)
    if n:
        raw[:n, 0:12] = np.ascontiguousarray(positions, np.float32).view(np.uint8).reshape(n, 12)
        raw[:n, 12:16] = np.ascontiguousarray(inst_ids, np.uint32).view(np.uint8).reshape(n, 4)
        raw[:n, 16:20] = np.ascontiguousarray(prim_ids, np.uint32).view(np.uint8).reshape(n, 4)
    out = C.POINTER(abi.BVHNode)()
    cnt = C.c_uint32(0)
    _check(lib, lib.strelka_bvh_build(arr, n, C.byref(out), C.byref(cnt)))
    if cnt.value == 0:
        return np.zeros(0, np.uint8)
    nodes = _np(out, cnt.value, abi.BVHNode)
    lib.strelka_host_free(C.cast(out, C.c_void_p))
    return nodes
