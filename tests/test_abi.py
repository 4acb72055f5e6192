"""The C ABI library loads, exports every declared entry point, and its
struct layouts match the reference's shader structs."""
import ctypes as C
import os
import re

from strelka_b200 import abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in ("strelka_b200.h", "strelka_b200_scenes.h"):
        text = open(os.path.join(ROOT, "include", h)).read()
        text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
        for m in re.finditer(r"^\s*(?:int|void|size_t|const char\*)\s+(strelka_\w+)\s*\(", text, flags=re.M):
            names.add(m.group(1))
    return names


def test_every_declared_symbol_is_exported(lib):
    names = declared_functions()
    assert len(names) >= 20
    for n in sorted(names):
        assert hasattr(lib, n), n


def test_signatures_cover_declarations():
    assert declared_functions() <= set(abi.SIGNATURES)


def test_reference_struct_sizes(lib):
    # shaders/pathtracerparam.h, accumulationparam.h, tonemapparam.h, raytracing.h,
    # instanceconstants.h, lights.h, materials.h, ray.h
    expected = {"PathTracerParam": 336, "AccumulationParam": 416, "Tonemapparam": 16, "BVHNode": 32, "Vertex": 32,
                "InstanceConstants": 208, "UniformLight": 112, "MdlMaterial": 16, "Mdl_resource_info": 16,
                "Ray": 32, "Hit": 20, "BVHInputPosition": 20}
    for name, size in expected.items():
        assert lib.strelka_sizeof(name.encode()) == size, name
        assert C.sizeof(getattr(abi, name)) == size, name


def test_field_offsets():
    assert abi.PathTracerParam.camPos.offset == 256
    assert abi.PathTracerParam.dimension.offset == 272
    assert abi.PathTracerParam.frameNumber.offset == 288
    assert abi.PathTracerParam.spp.offset == 308
    assert abi.PathTracerParam.stratifiedSamplingType.offset == 316
    assert abi.AccumulationParam.iteration.offset == 396
    assert abi.InstanceConstants.lightId.offset == 204
    assert abi.UniformLight.type.offset == 96


def test_error_reporting_without_gpu(lib):
    # argument validation happens before any device call
    rc = lib.strelka_reduction_execute(None, 1, 1, 0, None)
    assert rc == abi.ERR_INVALID_ARGUMENT
    assert "NULL" in abi.last_error()
    out = C.POINTER(abi.BVHNode)()
    cnt = C.c_uint32(7)
    assert lib.strelka_bvh_build(None, 4, C.byref(out), C.byref(cnt)) == abi.ERR_INVALID_ARGUMENT
    assert lib.strelka_bvh_build(None, 0, C.byref(out), C.byref(cnt)) == abi.OK and cnt.value == 0


def header_constants():
    """Enumerators and #define constants of the public header, by name."""
    text = open(os.path.join(ROOT, "include", "strelka_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    out = {}
    for m in re.finditer(r"\b(STRELKA_\w+)\s*=\s*1u\s*<<\s*(\d+)", text):
        out[m.group(1)] = 1 << int(m.group(2))
    for m in re.finditer(r"#define\s+(STRELKA_\w+)\s+\(1u\s*<<\s*(\d+)\)", text):
        out[m.group(1)] = 1 << int(m.group(2))
    return out


def test_pass_flags_match_header():
    c = header_constants()
    assert c["STRELKA_PT_PROFILE"] == abi.PT_PROFILE
    assert c["STRELKA_PT_COUNT"] == abi.PT_COUNT
    assert c["STRELKA_PT_NO_SHADE_SORT"] == abi.PT_NO_SHADE_SORT
    assert c["STRELKA_PT_LARGE_SCENE_KERNELS"] == abi.PT_LARGE_SCENE_KERNELS
    assert c["STRELKA_PT_SMALL_SCENE_KERNELS"] == abi.PT_SMALL_SCENE_KERNELS
    assert c["STRELKA_PT_SERIAL_SHADOW"] == abi.PT_SERIAL_SHADOW
    assert c["STRELKA_PT_FORCE_SHADE_SORT"] == abi.PT_FORCE_SHADE_SORT
    assert c["STRELKA_SHADE_SORT_MIN_PATHS"] == abi.SHADE_SORT_MIN_PATHS
    assert c["STRELKA_LARGE_SCENE_NODES"] == abi.LARGE_SCENE_NODES
