"""Python mirror of Strelka's render-pass API over the C ABI.

The reference records its passes as ``ComputePass<T>::execute(cmd, desc, w,
h, frameIndex)`` (include/render/computepass.h:8-164):

* ``PathTracer``     include/render/pathtracer.h:33-50, src/render/pathtracer.cpp
* ``ReductionPass``  include/render/reduction.h, src/render/reduction.cpp
* ``Accumulation``   include/render/accumulation.h, src/render/accumulation.cpp
* ``Tonemap``        include/render/tonemap.h, src/render/tonemap.cpp
* ``UpscalePass``    include/render/upscalepass.h, src/render/upscalepass.cpp

The classes below keep those names, descriptor contents and argument meaning;
a CUDA stream (an int handle, 0 = the legacy default stream) stands in for
the command buffer.  Device buffers are torch CUDA tensors (plumbing only);
all work runs in ``libstrelka_b200.so`` and raises :class:`abi.StrelkaError`
on any failure status.

:class:`DeviceScene` plays the role of the reference's ResourceManager for
the scene buffers created at frame 0 (src/render/ptrender.cpp:412-667).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import abi


def _torch():
    import torch

    return torch


def _stream_handle(stream) -> C.c_void_p:
    if stream is None:
        return C.c_void_p(0)
    if isinstance(stream, int):
        return C.c_void_p(stream)
    return C.c_void_p(stream.cuda_stream)


def to_device(arr: np.ndarray, device="cuda"):
    """Copies a numpy array to a uint8 CUDA tensor (16-byte aligned by the allocator)."""
    torch = _torch()
    a = np.ascontiguousarray(arr)
    t = torch.from_numpy(a.view(np.uint8).reshape(-1).copy())
    return t.to(device)


def ptr(t) -> int:
    return 0 if t is None else int(t.data_ptr())


class DeviceScene:
    """Device copies of a HostScene's buffers plus the descriptor fields."""

    _version = 1

    def __init__(self, hs, device="cuda", with_env: bool = True):
        torch = _torch()
        self.hs = hs
        self.device = device
        self.nodes = to_device(hs.nodes if hs.nodes.size else np.zeros(32, np.uint8), device)
        self.vb = to_device(hs.vb if hs.vb.size else np.zeros(32, np.uint8), device)
        self.ib = to_device(hs.ib if hs.ib.size else np.zeros(1, np.uint32), device)
        self.instances = to_device(hs.instances if hs.instances.size else np.zeros(208, np.uint8), device)
        self.lights = to_device(hs.lights, device)
        self.materials = to_device(hs.materials if hs.materials.size else np.zeros(16, np.uint8), device)
        self.args = to_device(hs.arg_block if hs.arg_block.size else np.zeros(48, np.uint8), device)
        self.resinfo = to_device(hs.resource_infos if hs.resource_infos.size else np.zeros(16, np.uint8), device)
        self.tex_data = [to_device(t, device) for t in hs.textures]
        texs = (abi.StrelkaTexture * max(len(hs.textures), 1))()
        for i, (t, d) in enumerate(zip(hs.textures, self.tex_data)):
            texs[i] = abi.StrelkaTexture(ptr(d), t.shape[1], t.shape[0], 0)
        self.tex_table = to_device(np.frombuffer(texs, np.uint8), device)
        self.env = None
        if with_env and hs.env is not None:
            self.env_rgba = to_device(hs.env, device)
            self.env_marg = to_device(hs.env_marginal, device)
            self.env_cond = to_device(hs.env_conditional, device)
            self.env = abi.StrelkaEnvMap(ptr(self.env_rgba), ptr(self.env_marg), ptr(self.env_cond), hs.env.shape[1],
                                         hs.env.shape[0], hs.env_integral, 0.0)
        self.version = DeviceScene._version
        DeviceScene._version += 1
        torch.cuda.synchronize()

    def desc(self, param, sample_buffer) -> abi.PathTracerDesc:
        hs = self.hs
        d = abi.PathTracerDesc()
        d.constants = param
        d.bvhNodes = ptr(self.nodes)
        d.numNodes = hs.num_nodes
        d.vb = ptr(self.vb)
        d.numVertices = hs.num_vertices
        d.ib = ptr(self.ib)
        d.numIndices = hs.ib.size
        d.instanceConst = ptr(self.instances)
        d.numInstances = hs.num_instances
        d.lights = ptr(self.lights)
        d.lightCapacity = hs.lights.size // 112
        d.sampleBuffer = ptr(sample_buffer)
        d.mdl_argument_block = ptr(self.args)
        d.argBlockBytes = hs.arg_block.size
        d.mdl_resource_infos = ptr(self.resinfo)
        d.numResourceInfos = hs.resource_infos.size // 16
        d.mdl_mdlMaterial = ptr(self.materials)
        d.numMaterials = hs.num_materials
        d.matTextures = ptr(self.tex_table) if hs.textures else 0
        d.numTextures = len(hs.textures)
        d.envMap = C.cast(C.pointer(self.env), C.c_void_p).value if self.env is not None else None
        d.sceneVersion = self.version
        return d

    def trace_desc(self, rays, hits, flags: int, counters=None) -> abi.TraceDesc:
        hs = self.hs
        d = abi.TraceDesc()
        d.bvhNodes = ptr(self.nodes)
        d.numNodes = hs.num_nodes
        d.vb = ptr(self.vb)
        d.numVertices = hs.num_vertices
        d.ib = ptr(self.ib)
        d.numIndices = hs.ib.size
        d.instanceConst = ptr(self.instances)
        d.numInstances = hs.num_instances
        d.rays = ptr(rays)
        d.hits = ptr(hits)
        d.numRays = 0 if rays is None else rays.numel() * rays.element_size() // 32
        d.flags = flags
        d.counters = ptr(counters)
        d.sceneVersion = self.version
        return d


class BvhBuilder:
    """BVH construction on the GPU (strelka_bvh_build_*_device): a linear BVH
    in the flattened depth-first layout of the host builder."""

    def __init__(self, mode: int = abi.BVH_PLOC, radius: int = 16):
        self.lib = abi.load()
        h = C.c_void_p()
        abi.check(self.lib.strelka_bvh_builder_create(C.byref(h)))
        self.handle = h
        abi.check(self.lib.strelka_bvh_builder_set_mode(h, mode, radius))

    def build_scene(self, ds: "DeviceScene", stream=None):
        """Nodes (a uint8 CUDA tensor, 32 bytes per node) over the scene's own
        device buffers: every instance's triangles in world space."""
        torch = _torch()
        hs = ds.hs
        counts = hs.instances.view(np.int32).reshape(-1, 52)[:, 50] if hs.instances.size else np.zeros(0, np.int32)
        tris = int(counts.astype(np.int64).sum()) // 3  # every instance's triangles
        cap = max(2 * tris - 1, 1)
        nodes = torch.empty(cap * 32, dtype=torch.uint8, device=ds.device)
        n = C.c_uint32()
        abi.check(self.lib.strelka_bvh_build_scene_device(self.handle, ptr(ds.vb), hs.num_vertices, ptr(ds.ib), hs.ib.size,
                                                          ptr(ds.instances), hs.num_instances, ptr(nodes), cap,
                                                          C.byref(n), _stream_handle(stream)))
        return nodes[:n.value * 32]

    def build(self, positions, num_positions: int, stream=None):
        """Nodes over a device array of BVHInputPosition (3 per triangle)."""
        torch = _torch()
        cap = max(2 * (num_positions // 3) - 1, 1)
        nodes = torch.empty(cap * 32, dtype=torch.uint8, device="cuda")
        n = C.c_uint32()
        abi.check(self.lib.strelka_bvh_build_device(self.handle, ptr(positions), num_positions, ptr(nodes), cap,
                                                    C.byref(n), _stream_handle(stream)))
        return nodes[:n.value * 32]

    def close(self) -> None:
        if self.handle:
            self.lib.strelka_bvh_builder_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class PathTracer:
    """PathTracer pass (include/render/pathtracer.h:33-50)."""

    def __init__(self, mode: int = abi.MODE_WAVEFRONT, chunk_paths: int = 0, profile: bool = False,
                 count: bool = False, queue_chunk: int = 0, shade_sort="auto", tail_depth: int = 0,
                 scene_kernels: str = "auto", serial_shadow: bool = False):
        """shade_sort: "auto" (by paths in flight, STRELKA_SHADE_SORT_MIN_PATHS), True (always,
        STRELKA_PT_FORCE_SHADE_SORT) or False (never, STRELKA_PT_NO_SHADE_SORT).
        scene_kernels: "auto" (by tree size), "large" or "small" (STRELKA_PT_*_SCENE_KERNELS).
        serial_shadow: shadow queries on the caller's stream after shading (STRELKA_PT_SERIAL_SHADOW)."""
        self.lib = abi.load()
        flags = ((abi.PT_PROFILE if profile else 0) | (abi.PT_COUNT if count else 0) |
                 {"auto": 0, True: abi.PT_FORCE_SHADE_SORT, False: abi.PT_NO_SHADE_SORT}[shade_sort] |
                 (abi.PT_SERIAL_SHADOW if serial_shadow else 0) |
                 {"auto": 0, "large": abi.PT_LARGE_SCENE_KERNELS, "small": abi.PT_SMALL_SCENE_KERNELS}[scene_kernels])
        cfg = abi.StrelkaPathTracerConfig(mode, chunk_paths, 0, flags, queue_chunk, tail_depth)
        h = C.c_void_p()
        abi.check(self.lib.strelka_pathtracer_create(C.byref(cfg), C.byref(h)))
        self.handle = h

    def execute(self, desc: abi.PathTracerDesc, w: int, h: int, frame_index: int = 0, stream=None) -> None:
        abi.check(self.lib.strelka_pathtracer_execute(self.handle, C.byref(desc), w, h, frame_index,
                                                      _stream_handle(stream)))

    def trace(self, desc: abi.TraceDesc, stream=None) -> None:
        abi.check(self.lib.strelka_trace_execute(self.handle, C.byref(desc), _stream_handle(stream)))

    def device_status(self, stream=None) -> int:
        st = C.c_uint32(0)
        abi.check(self.lib.strelka_pathtracer_get_device_status(self.handle, _stream_handle(stream), C.byref(st)))
        return st.value

    def kernel_times(self, stream=None) -> dict:
        n = len(abi.KERNEL_CLASSES)
        ms = (C.c_float * n)()
        cnt = (C.c_uint32 * n)()
        self.lib.strelka_pathtracer_get_kernel_times(self.handle, _stream_handle(stream), ms, cnt, n)
        return {name: (ms[i], cnt[i]) for i, name in enumerate(abi.KERNEL_CLASSES)}

    def counters(self, stream=None) -> dict:
        """Traversal visit counters since the last call (needs count=True)."""
        out = (C.c_uint64 * 6)()
        self.lib.strelka_pathtracer_get_counters(self.handle, _stream_handle(stream), out, 6)
        keys = ["extend_inner", "extend_leaf", "shadow_inner", "shadow_leaf", "extend_rays", "shadow_rays"]
        return {k: int(out[i]) for i, k in enumerate(keys)}

    def set_nrc(self, cache: "RadianceCache | None", train_paths: int = 16384, train_steps: int = 1,
                diffuse_roughness: float = 0.25) -> None:
        """Renders with the radiance cache (wavefront mode), or without it when
        `cache` is None.  The cache object must outlive its use here."""
        cfg = abi.StrelkaNrcRenderConfig(1 if cache is not None else 0, train_paths, train_steps, diffuse_roughness)
        abi.check(self.lib.strelka_pathtracer_set_nrc(self.handle, cache.handle if cache is not None else None,
                                                      C.byref(cfg)))
        self._cache = cache

    def train_nrc(self, desc: abi.PathTracerDesc, frame_index: int = 0, batches: int = 1, stream=None) -> None:
        """Trains the attached cache on `batches` batches of the frame's
        training paths (one Adam step group per batch) without rendering."""
        abi.check(self.lib.strelka_pathtracer_train_nrc(self.handle, C.byref(desc), frame_index, batches,
                                                        _stream_handle(stream)))

    def close(self) -> None:
        if self.handle:
            self.lib.strelka_pathtracer_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class RadianceCache:
    """Online-trained neural radiance cache: a multi-resolution hash grid and
    a fully fused FP16 MLP (strelka_nrc_*).  Records are StrelkaNrcRecord
    rows (16 float32: pos, dir, normal, roughness, target rgb, slot, pad) in
    device memory."""

    def __init__(self, scene_min, scene_max, learning_rate: float = 1e-2, seed: int = 1, log2_table_size: int = 19):
        self.lib = abi.load()
        cfg = abi.StrelkaNrcConfig((C.c_float * 3)(*[float(v) for v in scene_min]),
                                   (C.c_float * 3)(*[float(v) for v in scene_max]), learning_rate, seed,
                                   log2_table_size, (C.c_uint32 * 3)())
        h = C.c_void_p()
        abi.check(self.lib.strelka_nrc_create(C.byref(cfg), C.byref(h)))
        self.handle = h
        nm = C.c_uint32()
        ng = C.c_uint64()
        abi.check(self.lib.strelka_nrc_info(h, C.byref(nm), C.byref(ng), None))
        self.num_mlp_params = nm.value
        self.num_grid_params = ng.value

    def train(self, records, n: int, stream=None) -> float:
        loss = C.c_float()
        abi.check(self.lib.strelka_nrc_train(self.handle, ptr(records), n, C.byref(loss), _stream_handle(stream)))
        return loss.value

    def infer(self, records, n: int, out, stream=None) -> None:
        abi.check(self.lib.strelka_nrc_infer(self.handle, ptr(records), n, ptr(out), _stream_handle(stream)))

    def params(self) -> tuple[np.ndarray, np.ndarray]:
        mlp = np.zeros(self.num_mlp_params, np.float32)
        grid = np.zeros(self.num_grid_params, np.float32)
        abi.check(self.lib.strelka_nrc_get_params(self.handle, mlp.ctypes.data, grid.ctypes.data))
        return mlp, grid

    def set_params(self, mlp: np.ndarray | None, grid: np.ndarray | None) -> None:
        m = None if mlp is None else np.ascontiguousarray(mlp, np.float32)
        g = None if grid is None else np.ascontiguousarray(grid, np.float32)
        abi.check(self.lib.strelka_nrc_set_params(self.handle, None if m is None else m.ctypes.data,
                                                  None if g is None else g.ctypes.data))

    def close(self) -> None:
        if self.handle:
            self.lib.strelka_nrc_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batch_config(mode: int = abi.BATCH_WAVEFRONT, block_size: int = 128, queue_chunk: int = 256,
                 material_sort: bool = False, use_graph: bool = True) -> abi.StrelkaBatchConfig:
    return abi.StrelkaBatchConfig(mode, block_size, queue_chunk, 1 if material_sort else 0, 1 if use_graph else 0)


class Batch:
    """Many scene/camera jobs rendered as one batch (strelka_batch_*).  Each
    job is a PathTracerDesc with its own constants and sample buffer; the
    scenes (DeviceScene objects) must outlive the batch's use of them."""

    def __init__(self):
        self.lib = abi.load()
        h = C.c_void_p()
        abi.check(self.lib.strelka_batch_create(C.byref(h)))
        self.handle = h
        self._descs = None

    def set_jobs(self, descs, stream=None) -> None:
        arr = (abi.PathTracerDesc * max(len(descs), 1))(*descs)
        abi.check(self.lib.strelka_batch_set_jobs(self.handle, arr, len(descs), _stream_handle(stream)))
        self._descs = (descs, arr)

    def set_frame(self, frame_offset: int, stream=None) -> None:
        abi.check(self.lib.strelka_batch_set_frame(self.handle, frame_offset, _stream_handle(stream)))

    def execute(self, config: abi.StrelkaBatchConfig | None = None, stream=None) -> None:
        abi.check(self.lib.strelka_batch_execute(self.handle, C.byref(config) if config is not None else None,
                                                 _stream_handle(stream)))

    def autotune(self, repeats: int = 3, stream=None):
        """Returns (best config, [(config, ms), ...])."""
        cap = 64
        entries = (abi.StrelkaBatchTuneEntry * cap)()
        n = C.c_uint32()
        best = abi.StrelkaBatchConfig()
        abi.check(self.lib.strelka_batch_autotune(self.handle, repeats, entries, cap, C.byref(n), C.byref(best),
                                                  _stream_handle(stream)))
        return best, [(entries[i].config, entries[i].ms) for i in range(min(n.value, cap))]

    def job_latency(self, stream=None) -> list:
        ms = (C.c_float * abi.BATCH_MAX_JOBS)()
        n = self.lib.strelka_batch_job_latency(self.handle, _stream_handle(stream), ms, abi.BATCH_MAX_JOBS)
        if n < 0:
            abi.check(n)
        return [ms[i] for i in range(n)]

    def device_status(self, stream=None) -> int:
        st = C.c_uint32(0)
        abi.check(self.lib.strelka_batch_get_device_status(self.handle, _stream_handle(stream), C.byref(st)))
        return st.value

    def info(self) -> dict:
        total = C.c_uint64()
        jobs = C.c_uint32()
        keys = C.c_uint32()
        abi.check(self.lib.strelka_batch_info(self.handle, C.byref(total), C.byref(jobs), C.byref(keys)))
        return {"total_paths": total.value, "jobs": jobs.value, "sort_keys": keys.value}

    def close(self) -> None:
        if self.handle:
            self.lib.strelka_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ReductionPass:
    """ReductionPass (shaders/reduction.hlsl:9-32)."""

    def execute(self, desc: abi.ReductionDesc, w: int, h: int, frame_index: int = 0, stream=None) -> None:
        abi.check(abi.load().strelka_reduction_execute(C.byref(desc), w, h, frame_index, _stream_handle(stream)))


class Accumulation:
    """Accumulation (shaders/accumulation.hlsl:86-108)."""

    def execute(self, desc: abi.AccumulationDesc, w: int, h: int, frame_index: int = 0, stream=None) -> None:
        abi.check(abi.load().strelka_accumulation_execute(C.byref(desc), w, h, frame_index, _stream_handle(stream)))


class Tonemap:
    """Tonemap (shaders/tonemap.hlsl:66-88)."""

    def execute(self, desc: abi.TonemapDesc, w: int, h: int, frame_index: int = 0, stream=None) -> None:
        abi.check(abi.load().strelka_tonemap_execute(C.byref(desc), w, h, frame_index, _stream_handle(stream)))


class UpscalePass:
    """UpscalePass (shaders/upscalepass.hlsl:9-21): bilinear, clamp to edge."""

    def execute(self, desc: abi.UpscaleDesc, w: int, h: int, frame_index: int = 0, stream=None) -> None:
        abi.check(abi.load().strelka_upscale_execute(C.byref(desc), w, h, frame_index, _stream_handle(stream)))


def upscale_param(width: int, height: int) -> abi.Upscalepassparam:
    """The constants PtRender::drawFrame fills for the upscale pass
    (src/render/ptrender.cpp:871-876): the output size and its inverse."""
    return abi.Upscalepassparam((width, height), (1.0 / width, 1.0 / height))


def tonemap_upscale(tm_param, inp, up_param, out=None, out_rgba8=None, stream=None) -> None:
    """Tonemap + upscale (+ the final 8-bit blit) fused (strelka_tonemap_upscale_execute)."""
    abi.check(abi.load().strelka_tonemap_upscale_execute(C.byref(tm_param), ptr(inp), C.byref(up_param), ptr(out),
                                                         ptr(out_rgba8), _stream_handle(stream)))


def resolve(pt_param, sample_buffer, tm_param, acc_param=None, history=None, acc_out=None, tonemap_out=None,
            rgba8_out=None, stream=None) -> None:
    """Fused reduce + accumulate + tonemap (strelka_resolve_execute)."""
    lib = abi.load()
    acc = acc_param is not None
    abi.check(lib.strelka_resolve_execute(C.byref(pt_param), ptr(sample_buffer), 1 if acc else 0,
                                          C.byref(acc_param) if acc else None, ptr(history), ptr(acc_out),
                                          C.byref(tm_param), ptr(tonemap_out), ptr(rgba8_out), _stream_handle(stream)))


def accumulation_param(width: int, height: int, iteration: int) -> abi.AccumulationParam:
    """The fields PtRender::drawFrame fills (src/render/ptrender.cpp:805-825) that the kernel reads."""
    p = abi.AccumulationParam()
    p.dimension[0] = width
    p.dimension[1] = height
    p.iteration = iteration
    p.alpha = 0.1
    p.isPt = 1.0
    return p


def tonemap_param(width: int, height: int, kind: int) -> abi.Tonemapparam:
    return abi.Tonemapparam((width, height), kind, 0)
