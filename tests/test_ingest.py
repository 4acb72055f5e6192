"""Scene ingest formats (src/hdStrelka/RenderPass.cpp:50-126, Light.cpp:15-198,
src/scene/scene.cpp:459-511): packing against the shader's unpacking
(shaders/pack.h:4-33, restated by the oracle), hand-derived known answers
for the black-body colour and the light translation."""
import ctypes as C

import numpy as np
import pytest

import oracle
from strelka_b200 import abi

F = np.float32


def lib():
    return abi.load()


def pack_normal(n):
    return lib().strelka_pack_normal((C.c_float * 3)(*n))


def pack_uv(uv):
    return lib().strelka_pack_uv((C.c_float * 2)(*uv))


def test_pack_normal_known_answers():
    # (x + 1) / 2 * 511.99999f truncated, fields at bits 0, 10, 20; the
    # float32 literal 511.99999f is exactly 512, so +1 packs to 512
    assert F(511.99999) == F(512.0)
    assert pack_normal((0.0, 0.0, 1.0)) == 256 | (256 << 10) | (512 << 20)
    assert pack_normal((-1.0, 0.0, 0.0)) == 0 | (256 << 10) | (256 << 20)
    v = np.array([0.3, -0.7, 0.648074], F)
    expect = 0
    for k in range(3):
        expect += int(np.uint32((v[k] + F(1)) / F(2) * F(511.99999))) << (10 * k)
    assert pack_normal(v) == expect


def test_pack_round_trips_through_the_shader_unpack():
    o = oracle.load()
    rng = np.random.default_rng(3)
    n = rng.normal(size=(500, 3)).astype(F)
    n /= np.linalg.norm(n, axis=1, keepdims=True)
    out = (C.c_float * 3)()
    for v in n:
        o.oracle_unpack_normal(pack_normal(v), C.cast(out, C.c_void_p))
        assert np.abs(np.array(out) - v).max() <= 2.0 / 511.0 + 1e-6
    uv = rng.uniform(-10, 10, (500, 2)).astype(F)
    o2 = (C.c_float * 2)()
    for t in uv:
        o.oracle_unpack_uv(pack_uv(t), C.cast(o2, C.c_void_p))
        assert np.abs(np.array(o2) - t).max() <= 20.0 / 16383.0 + 1e-5
    assert pack_uv((0.0, 0.0)) == int(F(0.5) * F(16383.99999)) * (1 + (1 << 16))


def test_bake_vertices():
    pts = np.array([[0, 0, 0], [2, 0, 0], [0, 4, 1]], F)
    nrm = np.array([[0, 0, 1], [0, 1, 0], [1, 0, 0]], F)
    uvs = np.array([[0.25, 0.75], [1.0, 0.0], [0.5, 0.5]], F)
    out = (abi.Vertex * 3)()
    mc = (C.c_float * 3)()
    abi.check(lib().strelka_bake_vertices(pts.ctypes.data, nrm.ctypes.data, uvs.ctypes.data, 3, out, mc))
    for k in range(3):
        assert list(out[k].position) == list(pts[k])
        assert out[k].normal == pack_normal(nrm[k])
        assert out[k].uv == pack_uv((uvs[k, 0], F(1) - uvs[k, 1]))  # v flipped
        assert out[k].tangent == 0
    assert np.allclose(np.array(mc), pts.mean(0), rtol=1e-6)
    abi.check(lib().strelka_bake_vertices(pts.ctypes.data, nrm.ctypes.data, None, 3, out, None))
    assert out[0].uv == 0


# the knots of the black-body table at 1000, 6500 and 10000 K
KNOT_1000 = np.array([1.000000, 0.027490, 0.000000], F)
KNOT_6500 = np.array([1.000000, 0.942771, 0.991642], F)
KNOT_10000 = np.array([0.609681, 0.695588, 1.000000], F)


def blackbody(k):
    out = (C.c_float * 3)()
    abi.check(lib().strelka_blackbody_rgb(k, out))
    return np.array(out, F)


@pytest.mark.parametrize("kelvin,knot", [(6500.0, KNOT_6500), (1000.0, KNOT_1000), (500.0, KNOT_1000),
                                         (10000.0, KNOT_10000), (20000.0, KNOT_10000)])
def test_blackbody_at_knots(kelvin, knot):
    # at a knot the Catmull-Rom spline returns the knot, then the luma normalisation
    luma = (knot[0] * F(0.2126) + knot[1] * F(0.7152)) + knot[2] * F(0.0722)
    assert np.allclose(blackbody(kelvin), np.maximum(knot / luma, 0), rtol=2e-6, atol=1e-7)


def test_blackbody_shape():
    t = np.linspace(1000, 10000, 91)
    rgb = np.array([blackbody(k) for k in t])
    assert (rgb >= 0).all()
    luma = rgb @ np.array([0.2126, 0.7152, 0.0722])
    assert np.allclose(luma, 1.0, atol=5e-4)  # above 1 only where a negative blue is clamped (< 1500 K)
    assert (np.diff(rgb[:, 2]) >= -1e-3).all()  # bluer as it gets hotter (the spline wiggles by < 1e-3)
    assert (np.diff(rgb[:, 0]) <= 1e-3).all()


def light(type_, **kw):
    L = abi.StrelkaUsdLight()
    L.type = type_
    L.color[:] = kw.get("color", (1.0, 0.5, 0.25))
    L.intensity = kw.get("intensity", 8.0)
    L.exposure = kw.get("exposure", 0.0)
    L.enableColorTemperature = kw.get("ct", 0)
    L.colorTemperature = kw.get("kelvin", 6500.0)
    x = np.eye(4, dtype=F) if "xform" not in kw else kw["xform"]
    L.xform[:] = x.T.ravel()  # column-major
    L.width, L.height, L.radius = kw.get("width", 2.0), kw.get("height", 1.0), kw.get("radius", 0.5)
    out = abi.UniformLight()
    abi.check(lib().strelka_light_from_usd(C.byref(L), C.byref(out)))
    return out


def f4(v):
    return np.array([v.x, v.y, v.z, v.w], F)


def test_rect_light():
    out = light(0, exposure=1.0)  # intensity 8 * 2^1 = 16 over area 2
    assert out.type == 0
    corners = [f4(out.points[k]) for k in range(4)]
    assert np.array_equal(np.array(corners), np.array([[1, .5, 0, 1], [-1, .5, 0, 1], [-1, -.5, 0, 1], [1, -.5, 0, 1]], F))
    assert np.allclose(f4(out.color), [8.0, 4.0, 2.0, 8.0])


def test_disk_and_sphere_lights():
    x = np.diag([2.0, 2.0, 2.0, 1.0]).astype(F)
    x[:3, 3] = (1.0, 2.0, 3.0)
    d = light(1, xform=x, radius=0.5)  # radius x xform[0][0] = 1
    assert np.array_equal(f4(d.points[0]), np.array([1, 0, 0, 0], F))
    assert np.array_equal(f4(d.points[1]), np.array([1, 2, 3, 1], F))
    assert np.array_equal(f4(d.points[2]), np.array([2, 0, 0, 0], F))  # x axis scaled by xform and radius
    assert np.array_equal(f4(d.normal), np.array([0, 0, 2, 0], F))
    assert np.allclose(f4(d.color)[3], 8.0 / np.pi)
    s = light(2, xform=x, radius=0.5)
    assert s.type == 2
    assert np.array_equal(f4(s.points[1]), np.array([1, 2, 3, 1], F))
    assert np.allclose(f4(s.color)[:3], np.array([1, 0.5, 0.25]) * 8.0 / (4 * np.pi))


def test_color_temperature_and_exposure_clamp():
    out = light(0, ct=1, kelvin=6500.0, color=(1.0, 1.0, 1.0), exposure=80.0)
    bb = blackbody(6500.0)
    per_area = F(8.0) * F(2.0) ** F(50.0) / F(2.0)
    assert np.allclose(f4(out.color)[:3], bb * per_area, rtol=1e-6)
    with pytest.raises(abi.StrelkaError):
        light(3)
