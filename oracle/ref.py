"""Python bindings of oracle/_ref/libstrelka_ref.so: the reference's own
shader code compiled on the host (oracle/build_ref.sh, oracle/hlsl2cpp.py,
oracle/ref/).

TEST INFRASTRUCTURE ONLY: it checks the oracle's restatement (oracle.c)
against the reference's source, function by function and image by image.
Only the tests import this module.

The library is built from the reference tree where it lies, so it exists
only where that tree was present at build time (or where the built file was
carried along).  `available()` says whether it can be loaded.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import OracleScene, SceneView, _ptr
from . import load as _load_oracle

_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_DIR, "_ref", "libstrelka_ref.so")
_lib: C.CDLL | None = None


def build() -> None:
    subprocess.run(["sh", os.path.join(_DIR, "build_ref.sh")], check=True)


def available() -> bool:
    try:
        load()
        return True
    except OSError:
        return False


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        build()
    if not os.path.exists(LIB_PATH):
        raise OSError(f"{LIB_PATH} is not built (the reference tree was not present)")
    _load_oracle()  # the materials it calls live in liboracle.so
    lib = C.CDLL(LIB_PATH)
    vp, u32, f32 = C.c_void_p, C.c_uint32, C.c_float
    sigs = {
        "strelka_ref_pathtrace": (C.c_int, [vp, C.POINTER(OracleScene), vp, C.c_uint64, C.c_uint64, vp, C.c_int]),
        "strelka_ref_trace": (C.c_int, [C.POINTER(OracleScene), vp, u32, vp, vp, C.c_int, C.c_int]),
        "strelka_ref_jenkins_hash": (u32, [u32]),
        "strelka_ref_init_rng": (u32, [u32, u32, u32, u32, u32]),
        "strelka_ref_xorshift": (u32, [C.POINTER(u32)]),
        "strelka_ref_rand": (f32, [C.POINTER(u32)]),
        "strelka_ref_permute": (u32, [u32, u32, u32]),
        "strelka_ref_randfloat": (f32, [u32, u32]),
        "strelka_ref_unpack_normal": (None, [u32, vp]),
        "strelka_ref_unpack_uv": (None, [u32, vp]),
        "strelka_ref_unpack_tangent": (None, [u32, vp]),
        "strelka_ref_offset_ray": (None, [vp, vp, vp]),
        "strelka_ref_intersect_ray_box": (C.c_int, [vp, vp, vp, vp, C.POINTER(f32)]),
        "strelka_ref_ray_triangle": (C.c_int, [vp, vp, vp, vp, vp, C.POINTER(f32), C.POINTER(f32), C.POINTER(f32)]),
        "strelka_ref_sample_light": (None, [vp, vp, vp, f32, f32, vp]),
        "strelka_ref_camera_ray": (None, [vp, u32, u32, C.POINTER(u32), u32, vp]),
        "strelka_ref_reduce": (C.c_int, [vp, vp, vp]),
        "strelka_ref_accumulate": (C.c_int, [vp, vp, vp, vp]),
        "strelka_ref_tonemap": (C.c_int, [vp, vp, vp]),
        "strelka_ref_upscale": (C.c_int, [vp, vp, u32, u32, vp]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    _lib = lib
    return lib


def pathtrace(view: SceneView, param, first: int = 0, count: int | None = None, threads: int = 0):
    """The reference's computeMain over sample indices [first, first+count):
    (samples (count*3,) float32, undefined (count,) bool) where `undefined`
    marks samples that read a buffer out of range (a result the reference
    leaves undefined)."""
    lib = load()
    total = param.dimension[0] * param.dimension[1] * param.spp
    if count is None:
        count = total - first
    out = np.zeros(count * 3, np.float32)
    ub = np.zeros(count, np.uint8)
    lib.strelka_ref_pathtrace(C.byref(param), C.byref(view.scene), _ptr(out), first, count, _ptr(ub), threads)
    return out, ub.astype(bool)


def trace(view: SceneView, rays: np.ndarray, any_hit: bool = False, threads: int = 0):
    """The reference's closestHit / anyHit: (hits (n,5) uint32, found (n,) bool)."""
    lib = load()
    rays = np.ascontiguousarray(rays, np.float32)
    n = rays.shape[0]
    hits = np.zeros((n, 5), np.uint32)
    found = np.zeros(n, np.uint8)
    lib.strelka_ref_trace(C.byref(view.scene), _ptr(rays), n, _ptr(hits), _ptr(found), 1 if any_hit else 0, threads)
    return hits, found.astype(bool)


def _f3(v) -> np.ndarray:
    return np.ascontiguousarray(v, np.float32)


def offset_ray(p, n) -> np.ndarray:
    out = np.zeros(3, np.float32)
    load().strelka_ref_offset_ray(_ptr(_f3(p)), _ptr(_f3(n)), _ptr(out))
    return out


def intersect_ray_box(o, invdir, pmin, pmax):
    t = C.c_float(0.0)
    hit = load().strelka_ref_intersect_ray_box(_ptr(_f3(o)), _ptr(_f3(invdir)), _ptr(_f3(pmin)), _ptr(_f3(pmax)),
                                               C.byref(t))
    return bool(hit), t.value


def ray_triangle(o, d, v0, e0, e1):
    t, u, v = C.c_float(0), C.c_float(0), C.c_float(0)
    hit = load().strelka_ref_ray_triangle(_ptr(_f3(o)), _ptr(_f3(d)), _ptr(_f3(v0)), _ptr(_f3(e0)), _ptr(_f3(e1)),
                                          C.byref(t), C.byref(u), C.byref(v))
    return bool(hit), t.value, u.value, v.value


def sample_light(light_bytes: np.ndarray, hit_point, normal, u0: float, u1: float) -> np.ndarray:
    out = np.zeros(12, np.float32)
    lb = np.ascontiguousarray(light_bytes, np.uint8)
    load().strelka_ref_sample_light(_ptr(lb), _ptr(_f3(hit_point)), _ptr(_f3(normal)), u0, u1, _ptr(out))
    return out


def camera_ray(param, px: int, py: int, rng: int, s: int):
    st = C.c_uint32(rng)
    out = np.zeros(6, np.float32)
    load().strelka_ref_camera_ray(C.byref(param), px, py, C.byref(st), s, _ptr(out))
    return out, st.value


def reduce(param, sample_buffer: np.ndarray) -> np.ndarray:
    out = np.zeros(param.dimension[0] * param.dimension[1] * 4, np.float32)
    load().strelka_ref_reduce(C.byref(param), _ptr(np.ascontiguousarray(sample_buffer, np.float32)), _ptr(out))
    return out


def accumulate(param, inp: np.ndarray, hist: np.ndarray) -> np.ndarray:
    out = np.zeros(param.dimension[0] * param.dimension[1] * 4, np.float32)
    load().strelka_ref_accumulate(C.byref(param), _ptr(np.ascontiguousarray(inp, np.float32)),
                                  _ptr(np.ascontiguousarray(hist, np.float32)), _ptr(out))
    return out


def tonemap(param, inp: np.ndarray) -> np.ndarray:
    out = np.zeros(param.dimension[0] * param.dimension[1] * 4, np.float32)
    load().strelka_ref_tonemap(C.byref(param), _ptr(np.ascontiguousarray(inp, np.float32)), _ptr(out))
    return out


def upscale(param, inp: np.ndarray, in_w: int, in_h: int) -> np.ndarray:
    out = np.zeros(param.dimension[0] * param.dimension[1] * 4, np.float32)
    load().strelka_ref_upscale(C.byref(param), _ptr(np.ascontiguousarray(inp, np.float32)), in_w, in_h, _ptr(out))
    return out
