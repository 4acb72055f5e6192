"""Pins the CPU oracle: known answers from the reference's own tests, hand
computations of the RNG, analytic formulas and FP64 cross-checks."""
import ctypes as C

import numpy as np
import pytest

import oracle
from strelka_b200 import abi, scenes

f32 = np.float32


def py_jenkins(x):
    # shaders/random.h:14-22, computed here independently of the oracle
    m = 0xFFFFFFFF
    x = (x + (x << 10)) & m
    x ^= x >> 6
    x = (x + (x << 3)) & m
    x ^= x >> 11
    x = (x + (x << 15)) & m
    return x


def py_xorshift(s):
    m = 0xFFFFFFFF
    s ^= (s << 13) & m
    s ^= s >> 17
    s ^= (s << 5) & m
    return s


def test_jenkins_known_answers(orc):
    # hand-computed: hash(0) = 0; hash(1) = 0x??? computed by the Python twin
    assert orc.oracle_jenkins_hash(0) == 0
    for x in [1, 2, 12345, 0xDEADBEEF, 0xFFFFFFFF, 7 * 16 + 3]:
        assert orc.oracle_jenkins_hash(x) == py_jenkins(x)
    # first step by hand: x=1 -> 1+1024=1025 -> 1025^16=1041 -> 1041+8328=9369
    x = 1 + (1 << 10)
    x ^= x >> 6
    assert x == 1041
    x = x + (x << 3)
    assert x == 9369


def test_rng_stream(orc):
    # random.h:26-48: pixel (3, 5) of a 64-wide image at frame 7
    seed = (3 + 5 * 64) ^ py_jenkins(7)
    state = py_jenkins(seed)
    assert orc.oracle_init_rng(3, 5, 64, 7) == state
    s = C.c_uint32(state)
    for _ in range(16):
        v = orc.oracle_rand(C.byref(s))
        state = py_xorshift(state)
        expect = np.frombuffer(np.uint32(0x3F800000 | (state >> 9)).tobytes(), np.float32)[0] - f32(1.0)
        assert s.value == state
        assert np.float32(v) == expect
        assert 0.0 <= v < 1.0


def test_uint_to_float_extremes(orc):
    # uintToFloat(0xFFFFFFFF) = 1 - 2^-23; uintToFloat(x < 512) = 0
    s = C.c_uint32(0)
    # xorshift(0) stays 0 forever -> rand = 0
    assert orc.oracle_rand(C.byref(s)) == 0.0 and s.value == 0


def slab(orc, o, d, pmin, pmax):
    o = np.asarray(o, f32)
    d = np.asarray(d, f32)
    inv = (f32(1.0) / d).astype(f32)
    lo = np.asarray(pmin, f32)
    hi = np.asarray(pmax, f32)
    t = C.c_float(0)
    r = orc.oracle_intersect_ray_box(o.ctypes.data, inv.ctypes.data, lo.ctypes.data, hi.ctypes.data, C.byref(t))
    return bool(r), t.value


def test_slab_known_answers(orc):
    # tests/intersection/aabb.cpp:16-106 (the reference's commented known answers)
    off = np.array([1e-5] * 3, f32)
    o1 = np.array([1, 1, -4], f32) + off
    d1 = [-1, -1, 4]
    assert slab(orc, o1, d1, [0, 0, 0], [0, 0, 0])[0] is False      # test 1: zero-volume box
    assert slab(orc, o1, d1, [0, 0, 0], [1, 0, 0])[0] is False
    assert slab(orc, o1, d1, [-1, 0, -1], [1, 0, 1])[0] is True     # test 2: plane box
    assert slab(orc, o1, d1, [-1, 0, -1], [1, 2, 1])[0] is True     # test 3: average box
    assert slab(orc, o1, d1, [-0.003, 0, -0.003], [0.003, 0.003, 0.003])[0] is True  # test 4: tiny box
    assert slab(orc, o1, d1, [0, 0, 0], [1, 0, 1])[0] is True       # test 5: angle intersection
    o6 = np.array([1, -1, -4], f32) + off
    assert slab(orc, o6, d1, [-1, 0, -1], [1, 0, 1])[0] is False    # test 6: parallel ray
    o7 = np.array([2.03, -0.03, -2.03], f32) + off
    assert slab(orc, o7, [-2.03, -0.03, 2.03], [-1, 0, -1], [1, 0, 1])[0] is False  # test 7


def test_slab_entry_distance(orc):
    hit, t = slab(orc, [-2, 0.5, 0.5], [1, 0, 0], [0, 0, 0], [1, 1, 1])
    assert hit and t == 2.0
    hit, t = slab(orc, [0.5, 0.5, 0.5], [0, 0, 1], [0, 0, 0], [1, 1, 1])  # inside: t0 clamps to 0
    assert hit and t == 0.0


@pytest.mark.parametrize("name,ref,lo,hi", [("oracle_sinf", np.sin, -13, 13), ("oracle_cosf", np.cos, -13, 13),
                                            ("oracle_acosf", np.arccos, -1, 1)])
def test_own_transcendentals_within_2ulp(orc, name, ref, lo, hi):
    rng = np.random.default_rng(3)
    xs = rng.uniform(lo, hi, 4000).astype(f32)
    fn = getattr(orc, name)
    worst = 0.0
    for x in xs:
        y = np.float64(np.float32(fn(float(x))))
        r = ref(np.float64(x))
        worst = max(worst, abs(y - r) / np.spacing(np.float32(abs(r)) if r != 0 else np.float32(1e-38)))
    assert worst <= 2.0, worst
    assert np.isnan(orc.oracle_acosf(1.0000001)) and orc.oracle_acosf(1.0) == 0.0


def test_pack_unpack(orc):
    out = np.zeros(3, f32)
    # pack.h:4-14: 0 -> (-1,-1,-1); all ones in each field -> ~ (1, 1, 7)
    orc.oracle_unpack_normal(0, out.ctypes.data)
    assert (out == -1).all()
    v = 511 | (511 << 10) | (511 << 20)
    orc.oracle_unpack_normal(v, out.ctypes.data)
    assert np.allclose(out, [511 / 511.99999 * 2 - 1] * 3, atol=1e-6)
    uv = np.zeros(2, f32)
    packed = (8192 | (12288 << 16))
    orc.oracle_unpack_uv(packed, uv.ctypes.data)
    assert np.allclose(uv, [8192 / 16383.99999 * 20 - 10, 12288 / 16383.99999 * 20 - 10], atol=1e-5)


def test_offset_ray(orc):
    # helper.h:12-28: near the origin the offset is float_scale * n
    p = np.array([0.01, 0.5, -2.0], f32)
    n = np.array([0.0, 1.0, 0.0], f32)
    out = np.zeros(3, f32)
    orc.oracle_offset_ray(p.ctypes.data, n.ctypes.data, out.ctypes.data)
    assert out[0] == p[0] + f32(1 / 65536) * f32(0.0)
    # 0.5 >= 1/32: integer offset of 256 ulps
    assert out[1].view(np.int32) == p[1].view(np.int32) + 256
    assert out[2] == p[2]


def interior_rays(n, seed):
    rng = np.random.default_rng(seed)
    rays = np.zeros((n, 8), f32)
    rays[:, :3] = rng.uniform(0.05, 0.95, (n, 3))
    d = rng.normal(size=(n, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 3] = 1e9
    return rays


def test_ray_triangle_matches_fp64():
    s = scenes.cornell(16, 16, sphere_levels=3)
    v = oracle.SceneView(s)
    rays = interior_rays(20000, 9)
    hits, found, _ = oracle.trace(v, rays)
    idx = np.nonzero(found)[0]
    assert idx.size > 100
    t64, u64, v64 = oracle.intersect_fp64(v, rays[idx], hits[idx, 3], hits[idx, 4])
    t32 = hits[idx, 2].view(f32)
    rel = np.abs(t32 - t64) / np.abs(t64)
    assert np.median(rel) < 1e-6 and rel.max() < 1e-3


def tonemap_ref(c, kind):
    c = np.asarray(c, np.float64)
    if kind == 0:
        lum = c @ [0.299, 0.587, 0.114]
        return c * (lum / (lum + 1) / lum)
    if kind == 1:
        A = np.array([[0.59719, 0.35458, 0.04823], [0.07600, 0.90834, 0.01566], [0.02840, 0.13383, 0.83777]])
        B = np.array([[1.60475, -0.53108, -0.07367], [-0.10208, 1.10813, -0.00605], [-0.00327, -0.07276, 1.07602]])
        v = A @ c
        v = (v * (v + 0.0245786) - 0.000090537) / (v * (0.983729 * v + 0.4329510) + 0.238081)
        return np.clip(B @ v, 0, 1)
    x = c
    return np.clip((x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14), 0, 1)


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_tonemap_formulas(kind):
    pts = np.array([[0.18, 0.18, 0.18], [1.0, 0.5, 0.25], [4.0, 2.0, 1.0], [0.01, 0.2, 0.05]], f32)
    img = np.concatenate([pts, np.ones((4, 1), f32)], 1).ravel()
    p = abi.Tonemapparam((4, 1), kind, 0)
    out = oracle.tonemap(p, img).reshape(4, 4)
    for i in range(4):
        assert np.allclose(out[i, :3], tonemap_ref(pts[i], kind), atol=2e-6)
        assert out[i, 3] == 1.0


def test_reinhard_black_is_nan():
    # tonemap.hlsl:59-64 divides by the luminance: black pixels give 0/0
    p = abi.Tonemapparam((1, 1), 0, 0)
    out = oracle.tonemap(p, np.array([0, 0, 0, 1], f32))
    assert np.isnan(out[:3]).all()


def test_accumulate_weights():
    p = abi.AccumulationParam()
    p.dimension[0], p.dimension[1], p.iteration = 2, 1, 3
    inp = np.array([1, 2, 3, 1, 0, 0, 0, 1], f32)
    hist = np.array([2, 2, 2, 1, 4, 4, 4, 1], f32)
    out = oracle.accumulate(p, inp, hist)
    wh, wn = f32(3) / f32(4), f32(1) / f32(4)
    assert out[0] == hist[0] * wh + inp[0] * wn and out[3] == 1.0


def test_reduce_order():
    p = abi.PathTracerParam()
    p.dimension[0], p.dimension[1], p.spp = 1, 1, 3
    sb = np.array([1, 2, 3, 4, 5, 6, 7, 8, 9], f32)
    out = oracle.reduce(p, sb)
    inv = f32(1) / f32(3)
    r = f32(0)
    for s in range(3):
        r = f32(r + inv * sb[3 * s])
    assert out[0] == r and out[3] == 1.0


def _up(w, h):
    from strelka_b200 import abi
    return abi.Upscalepassparam((w, h), (np.float32(1.0) / np.float32(w), np.float32(1.0) / np.float32(h)))


def test_upscale_known_answers():
    # same size: every output centre lands on an input texel centre, exactly
    # when 1/size is exact in FP32 (powers of two), within rounding otherwise
    rng = np.random.default_rng(4)
    img = rng.uniform(0, 3, (4 * 8 * 4)).astype(np.float32)
    out = oracle.upscale(_up(8, 4), img, 8, 4)
    a, b = img.reshape(-1, 4), out.reshape(-1, 4)
    assert np.array_equal(b[:, :3], a[:, :3]) and (b[:, 3] == 1).all()
    img = rng.uniform(0, 3, (5 * 7 * 4)).astype(np.float32)
    out = oracle.upscale(_up(7, 5), img, 7, 5)
    assert np.allclose(out.reshape(-1, 4)[:, :3], img.reshape(-1, 4)[:, :3], rtol=0, atol=1e-5)
    # a constant image stays constant at any size
    c = np.tile(np.array([0.25, 0.5, 2.0, 7.0], np.float32), 6 * 4)
    out = oracle.upscale(_up(13, 9), c, 6, 4).reshape(-1, 4)
    assert np.allclose(out[:, :3], [0.25, 0.5, 2.0], rtol=1e-6, atol=0)
    # 2x1 ramp [0, 1] upscaled to 4x2: centres at texel positions -0.25, 0.25, 0.75, 1.25
    ramp = np.array([0, 0, 0, 1, 1, 1, 1, 1], np.float32)
    out = oracle.upscale(_up(4, 2), ramp, 2, 1).reshape(2, 4, 4)
    assert np.array_equal(out[0, :, 0], np.array([0, 0.25, 0.75, 1], np.float32))
    assert np.array_equal(out[1, :, 0], out[0, :, 0])


def test_mdl_read_known_answers():
    buf = np.zeros(16, np.uint8)
    buf[0:4] = np.frombuffer(np.float32(1.5).tobytes(), np.uint8)
    buf[4:12] = np.frombuffer(np.float64(-2.25).tobytes(), np.uint8)
    buf[13] = 7  # a bool in byte 1 of the last word
    offs = np.array([0, 2, 4, 12, 13, 14, 16, 1000], np.uint32)
    kinds = np.array([0, 0, 1, 4, 4, 4, 3, 0], np.uint32)
    r = oracle.mdl_read(buf, offs, kinds)
    assert np.uint32(r[0]).view(np.float32) == np.float32(1.5)
    assert r[1] == r[0]  # the two low bits of a word offset are ignored
    assert np.uint64(r[2]).view(np.float64) == -2.25
    assert list(r[3:6]) == [0, 1, 0]  # byte 1 of the word is set, bytes 0 and 2 are not
    assert r[6] == 0 and r[7] == 0  # past the end reads 0
