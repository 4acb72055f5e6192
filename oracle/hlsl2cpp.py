"""Mechanical HLSL -> C++ rewrite of the reference's shader sources.

TEST INFRASTRUCTURE: part of the recipe (oracle/build_ref.sh) that compiles
the reference's own shader code, where it lies in the reference tree, into
oracle/_ref/ for checking the oracle's restatement.  The rewritten files are
written only under oracle/_ref/src/ (build output, never committed).

Every rewrite below is a syntax difference between HLSL (as Slang compiles
it) and C++; none changes an expression's operands, operators, evaluation
order or control flow:

* `__cplusplus` -> an undefined name: the shared headers carry a glm branch
  for the reference's C++ host code; the shader branch is the one compiled.
* `in` / `out` / `inout` / `in out` parameter qualifiers: `out T x` and
  `inout T x` become `T& x` (HLSL copy-in/copy-out has the same effect for
  these non-aliasing calls); `in` is dropped.
* unsuffixed floating literals get an `f` suffix: in HLSL they are `float`
  (in C++ they would be `double` and change every mixed expression).
* `.xyz` / `.rgb` / `.xy` swizzles become calls `.xyz()` ... that return a
  view which reads and writes the components; single components (.x, .r)
  stay members.
* HLSL intrinsics (`dot`, `min`, `abs`, `mul`, `sin` ...) are renamed
  `hl_dot` ... so they resolve to the shim's definitions (oracle/ref/shim.h)
  and not to the C library's functions of the same names.
* `(T) 0` zero-casts of structs become `T{}` (value initialisation).
* attributes (`[numthreads(...)]`, `[shader(...)]`) and system-value
  semantics (`: SV_DispatchThreadID`) are removed.
* a vector constructor whose arguments call `rand(` is written with braces
  (`float2{rand(s), rand(s)}`): HLSL evaluates arguments left to right,
  C++ guarantees that order only inside braces.
* lights.h:59 `sampleSphereSolidAngle(..., float2 u)` declares a local `u`
  in its outermost block, which HLSL allows to hide the parameter and C++
  rejects; the parameter is renamed so the local hides nothing and every
  use of `u` in the body still means the local, as in HLSL.

Usage: python oracle/hlsl2cpp.py <reference shaders dir> <output dir>
"""
from __future__ import annotations

import os
import re
import sys

FILES = [
    "pathtracerMdl.hlsl", "raytracing.h", "ray.h", "random.h", "helper.h", "pack.h", "lights.h", "materials.h",
    "instanceconstants.h", "pathtracerparam.h", "mdl_types.hlsl", "tonemap.hlsl", "tonemapparam.h",
    "accumulation.hlsl", "accumulationparam.h", "reduction.hlsl", "upscalepass.hlsl", "upscalepassparam.h",
]

INTRINSICS = [
    "asfloat", "asint", "asuint", "dot", "cross", "normalize", "length", "abs", "saturate", "sqrt", "rsqrt", "min",
    "max", "clamp", "lerp", "all", "any", "isnan", "isinf", "cos", "sin", "acos", "asin", "atan", "atan2", "pow",
    "exp", "exp2", "log", "log2", "frac", "floor", "ceil", "round", "sign", "step", "transpose", "mul", "reflect",
    "NonUniformResourceIndex",
]

FLOAT_LIT = re.compile(r"(?<![\w.])((?:\d+\.\d*|\.\d+)(?:[eE][+-]?\d+)?|\d+[eE][+-]?\d+)(?![\w.])")


def _suffix_floats(code: str) -> str:
    return FLOAT_LIT.sub(lambda m: m.group(1) + "f", code)


def _split_comments(text: str):
    """Yields (is_code, chunk) so that comments and strings are left alone."""
    pat = re.compile(r'//[^\n]*|/\*.*?\*/|"(?:\\.|[^"\\])*"', re.S)
    pos = 0
    for m in pat.finditer(text):
        if m.start() > pos:
            yield True, text[pos:m.start()]
        yield False, m.group(0)
        pos = m.end()
    if pos < len(text):
        yield True, text[pos:]


def _braced_rand_ctors(code: str) -> str:
    out = []
    i = 0
    ctor = re.compile(r"\b(float[234]|uint[234]|int[234])\s*\(")
    while True:
        m = ctor.search(code, i)
        if not m:
            out.append(code[i:])
            break
        start = m.end() - 1  # the '('
        depth = 0
        j = start
        while j < len(code):
            if code[j] == "(":
                depth += 1
            elif code[j] == ")":
                depth -= 1
                if depth == 0:
                    break
            j += 1
        inner = code[start + 1:j]
        if "rand(" in inner:
            out.append(code[i:m.start()] + m.group(1) + "{" + _braced_rand_ctors(inner) + "}")
        else:
            out.append(code[i:start + 1] + _braced_rand_ctors(inner) + ")")
        i = j + 1
    return "".join(out)


def rewrite(text: str, name: str) -> str:
    text = re.sub(r"^[ \t]*\[(numthreads|shader)\([^\]\n]*\)\][ \t]*$", "", text, flags=re.M)
    pieces = []
    for is_code, chunk in _split_comments(text):
        if not is_code:
            pieces.append(chunk)
            continue
        c = chunk
        c = c.replace("__cplusplus", "STRELKA_REF_HOST_GLM_BRANCH")
        c = re.sub(r"\s*:\s*SV_\w+", "", c)
        c = re.sub(r"\bin\s+out\b", "inout", c)
        c = re.sub(r"\b(inout|out)\s+(const\s+)?([A-Za-z_][\w:]*(?:<[^>]*>)?)\s+([A-Za-z_]\w*)", r"\2\3& \4", c)
        c = re.sub(r"(?<![\w.])in\s+(?=[A-Za-z_])", "", c)
        c = _suffix_floats(c)
        c = re.sub(r"\.(xyz|rgb|xy)\b(?!\s*\()", r".\1()", c)
        c = re.sub(r"\(\s*([A-Z][A-Za-z_]\w*)\s*\)\s*0\b", r"\1{}", c)
        c = re.sub(r"(?<![\w.])(" + "|".join(INTRINSICS) + r")\s*\(", r"hl_\1(", c)
        pieces.append(c)
    out = "".join(pieces)
    out = _braced_rand_ctors(out)
    if name == "lights.h":
        old = "float3 sampleSphereSolidAngle(UniformLight l, float3 surfaceNormal, float3 hitPoint, float2 u)"
        if old not in out:
            raise SystemExit("lights.h: sampleSphereSolidAngle signature not found")
        out = out.replace(old, old.replace("float2 u)", "float2 u_hidden_by_local)"))
    return out


def main() -> None:
    src, dst = sys.argv[1], sys.argv[2]
    os.makedirs(dst, exist_ok=True)
    for f in FILES:
        with open(os.path.join(src, f), encoding="utf-8", errors="replace") as fh:
            text = fh.read()
        banner = (f"// Rewritten by oracle/hlsl2cpp.py from the reference's shaders/{f}; build output, "
                  f"not a source file.\n#line 1 \"shaders/{f}\"\n")
        with open(os.path.join(dst, f), "w") as fh:
            fh.write(banner + rewrite(text, f))


if __name__ == "__main__":
    main()
