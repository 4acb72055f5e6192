"""The syntax-only HLSL -> C++ rewrite that compiles the reference's shaders
on the host (oracle/hlsl2cpp.py), rule by rule on small snippets."""
import os
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))

import hlsl2cpp  # noqa: E402


def rw(code):
    return hlsl2cpp.rewrite(code, "snippet.hlsl")


def test_parameter_qualifiers():
    out = rw("float f(in float a, out float b, inout uint s, in out float3 c) { b = a; }")
    assert "float a" in out and "float& b" in out and "uint& s" in out and "float3& c" in out
    assert " in " not in out and "out " not in out


def test_float_literals_become_float():
    out = rw("float x = 1.0 / y + 2.5e-3 * 1e9 - .5; float z = 2.f; uint h = 0x02e5be93; int i = 3;")
    assert "1.0f" in out and "2.5e-3f" in out and "1e9f" in out and ".5f" in out
    assert "2.f" in out and "2.ff" not in out
    assert "0x02e5be93" in out and "i = 3;" in out


def test_swizzles_intrinsics_and_zero_casts():
    out = rw("Ray r = (Ray) 0; r.d.xyz = normalize(w.xyz); float3 c = l.color.rgb; float2 p = a.xy; float k = r.d.x;")
    assert "Ray{}" in out
    assert "r.d.xyz() = hl_normalize(w.xyz())" in out
    assert "l.color.rgb()" in out and "a.xy()" in out and "r.d.x;" in out


def test_attributes_semantics_and_host_branch():
    out = rw('[numthreads(256, 1, 1)]\n[shader("compute")]\nvoid computeMain(uint2 i : SV_DispatchThreadID) {}\n'
             "#ifdef __cplusplus\nint host;\n#endif\n")
    assert "numthreads" not in out and "shader(" not in out and "SV_" not in out
    assert "void computeMain(uint2 i)" in out
    assert "__cplusplus" not in out
    assert out.count("\n") == 6  # line numbers are kept


def test_left_to_right_arguments():
    out = rw("float2 u = float2(rand(s), rand(s)); float4 x = float4(rand(s), rand(s), rand(s), rand(s));"
             " float3 c = float3(a, b, 0);")
    assert "float2{rand(s), rand(s)}" in out
    assert "float4{rand(s), rand(s), rand(s), rand(s)}" in out
    assert "float3(a, b, 0)" in out


def test_comments_and_strings_untouched():
    out = rw('// out float in 1.0 dot(a)\nfloat x = dot(a, b); /* min(1.0) */ const char* s = "1.0";')
    assert "// out float in 1.0 dot(a)" in out and "/* min(1.0) */" in out and '"1.0"' in out
    assert "hl_dot(a, b)" in out
