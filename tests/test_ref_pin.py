"""The oracle's restatement against the reference's own shader code.

oracle/_ref/libstrelka_ref.so is the reference's shaders/pathtracerMdl.hlsl
(with raytracing.h, ray.h, random.h, helper.h, pack.h, lights.h) and its
reduction, accumulation, tonemap and upscale shaders, compiled on the host
from the reference tree by oracle/build_ref.sh (syntax-only rewrite,
oracle/hlsl2cpp.py; HLSL types and intrinsics from oracle/ref/shim.h).  Every
comparison is bit for bit.  The library replaces only what the reference
generates with the MDL SDK at run time (the material dispatch functions) by
the project's native materials, so the materials themselves are not pinned
here; everything else is.

Where the reference reads a buffer out of range (a diffuse bounce that hits
a light's emitter reads mdlMaterials[(uint)-1], pathtracerMdl.hlsl:276 with
src/scene/scene.cpp:451), its result is undefined and the oracle ends the
path instead; those samples are reported and excluded.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from strelka_b200 import abi, scenes

ref = pytest.importorskip("oracle.ref")
if not ref.available():
    pytest.skip("oracle/_ref is not built (the reference tree was not present at build time)",
                allow_module_level=True)

F32 = np.float32


def bits(a):
    return np.ascontiguousarray(a, F32).view(np.uint32)


def same_bits(a, b):
    """Bit equality, with any NaN equal to any NaN."""
    a, b = np.ascontiguousarray(a, F32), np.ascontiguousarray(b, F32)
    both_nan = np.isnan(a) & np.isnan(b)
    return bool(np.all((bits(a) == bits(b)) | both_nan))


# ---- random.h / helper.h / pack.h --------------------------------------------

def test_rng_functions():
    lib, r = oracle.load(), ref.load()
    rng = np.random.default_rng(1)
    xs = rng.integers(0, 2**32, 20000, dtype=np.uint64).astype(np.uint32)
    for x in xs[:5000]:
        x = int(x)
        assert lib.oracle_jenkins_hash(x) == r.strelka_ref_jenkins_hash(x)
        px, py, w, f = x & 4095, (x >> 12) & 4095, 1 + ((x >> 7) & 2047), x * 2654435761 & 0xFFFFFFFF
        assert lib.oracle_init_rng(px, py, w, f) == r.strelka_ref_init_rng(px, py, w, 1080, f)
    for x in xs[:200]:
        a, b = C.c_uint32(int(x) | 1), C.c_uint32(int(x) | 1)
        for _ in range(50):
            assert lib.oracle_rand(C.byref(a)) == r.strelka_ref_rand(C.byref(b))
            assert a.value == b.value
    for x in xs[:3000]:
        i, l, p = int(x) % 4096, 1 + int(x) % 97, int(x) * 0x9E3779B1 & 0xFFFFFFFF
        assert lib.oracle_permute(i % l, l, p) == r.strelka_ref_permute(i % l, l, p)
        assert bits(lib.oracle_randfloat(i, p)) == bits(r.strelka_ref_randfloat(i, p))


def test_unpack_and_offset_ray():
    lib, r = oracle.load(), ref.load()
    rng = np.random.default_rng(2)
    for v in rng.integers(0, 2**32, 3000, dtype=np.uint64).astype(np.uint32):
        a, b = np.zeros(3, F32), np.zeros(3, F32)
        lib.oracle_unpack_normal(int(v), a.ctypes.data)
        r.strelka_ref_unpack_normal(int(v), b.ctypes.data)
        assert same_bits(a, b)
        a, b = np.zeros(2, F32), np.zeros(2, F32)
        lib.oracle_unpack_uv(int(v), a.ctypes.data)
        r.strelka_ref_unpack_uv(int(v), b.ctypes.data)
        assert same_bits(a, b)
    mags = np.array([1e-6, 1e-3, 0.02, 1 / 32, 0.5, 3.0, 1e3, 1e6], F32)
    for k in range(4000):
        p = (rng.normal(size=3) * mags[rng.integers(0, len(mags), 3)]).astype(F32)
        n = rng.normal(size=3)
        n = (n / np.linalg.norm(n)).astype(F32)
        a = np.zeros(3, F32)
        lib.oracle_offset_ray(p.ctypes.data, n.ctypes.data, a.ctypes.data)
        assert same_bits(a, ref.offset_ray(p, n)), (p, n)


# ---- ray.h / raytracing.h -----------------------------------------------------

SPECIAL = np.array([0.0, -0.0, 1.0, -1.0, 0.5, np.inf, -np.inf, 1e-30], F32)


def test_slab_test():
    lib = oracle.load()
    rng = np.random.default_rng(3)
    cases = []
    for _ in range(20000):
        o = rng.uniform(-2, 2, 3).astype(F32)
        lo = rng.uniform(-1, 1, 3).astype(F32)
        hi = (lo + rng.uniform(0, 1, 3)).astype(F32)
        inv = rng.normal(size=3).astype(F32)
        k = rng.integers(0, 3)
        if rng.uniform() < 0.3:
            inv[k] = SPECIAL[rng.integers(0, len(SPECIAL))]
        if rng.uniform() < 0.2:
            o[k] = lo[k]  # on a slab plane: 0 * inf cases
        cases.append((o, inv, lo, hi))
    for o, inv, lo, hi in cases:
        t = C.c_float(0.0)
        h0 = lib.oracle_intersect_ray_box(o.ctypes.data, inv.ctypes.data, lo.ctypes.data, hi.ctypes.data, C.byref(t))
        h1, t1 = ref.intersect_ray_box(o, inv, lo, hi)
        assert bool(h0) == h1
        assert same_bits(np.float32(t.value), np.float32(t1))


def test_moller_trumbore():
    lib = oracle.load()
    rng = np.random.default_rng(4)
    for k in range(20000):
        scale = [1.0, 0.003, 1e-3][k % 3]
        v0 = rng.uniform(-1, 1, 3).astype(F32)
        e0 = (rng.normal(size=3) * scale).astype(F32)
        e1 = (rng.normal(size=3) * scale).astype(F32)
        o = rng.uniform(-2, 2, 3).astype(F32)
        target = v0 + e0 * rng.uniform(-0.2, 1.0) + e1 * rng.uniform(-0.2, 1.0)
        d = (target - o)
        d = (d / np.linalg.norm(d)).astype(F32)
        t, u, v = C.c_float(0), C.c_float(0), C.c_float(0)
        h0 = lib.oracle_ray_triangle(o.ctypes.data, d.ctypes.data, v0.ctypes.data, e0.ctypes.data, e1.ctypes.data,
                                     C.byref(t), C.byref(u), C.byref(v))
        h1, t1, u1, v1 = ref.ray_triangle(o, d, v0, e0, e1)
        assert bool(h0) == h1
        assert same_bits(np.float32(t.value), np.float32(t1))
        if h1:
            assert same_bits(np.array([u.value, v.value], F32), np.array([u1, v1], F32))


@pytest.mark.parametrize("scene", ["cornell", "soup", "instanced"])
def test_closest_and_any_hit(scene):
    from gpu_util import interior_rays, vertex_edge_rays

    if scene == "cornell":
        s = scenes.cornell(16, 16, sphere_levels=4)
        rays = np.concatenate([interior_rays(40_000, 5), vertex_edge_rays()])
    elif scene == "soup":
        s = scenes.soup(100_000, 6)
        rays = scenes.rays_soup(60_000, 7)
    else:
        s = scenes.large(width=32, height=16, instances=6, frequency=10, num_textures=2, tex_size=32, env_width=32,
                         env_height=16, max_depth=8, spp=1, seed=3)
        lo, hi = s.bounds()
        rng = np.random.default_rng(8)
        rays = np.zeros((40_000, 8), F32)
        rays[:, :3] = rng.uniform(lo, hi, (40_000, 3))
        d = rng.normal(size=(40_000, 3))
        rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
        rays[:, 3] = 1e9
    view = oracle.SceneView(s)
    for any_hit in (False, True):
        r = rays.copy()
        if any_hit:
            r[:, 3] = np.random.default_rng(9).uniform(0.05, 2.0, r.shape[0]).astype(F32)
        o, of, _ = oracle.trace(view, r, any_hit=any_hit, prune=0)
        g, gf = ref.trace(view, r, any_hit=any_hit)
        assert gf.sum() > 100
        assert np.array_equal(of, gf)
        assert np.array_equal(o, g)


# ---- lights.h -----------------------------------------------------------------

def _light(kind, rng):
    lb = np.zeros(28, F32)
    li = lb.view(np.int32)
    c = rng.uniform(-1, 1, 3)
    if kind == 0:
        ex = rng.normal(size=3) * rng.uniform(0.1, 1)
        ey = np.cross(ex, rng.normal(size=3))
        ey = ey / np.linalg.norm(ey) * rng.uniform(0.1, 1)
        pts = [c, c + ex, c + ex + ey, c + ey]
        for k, p in enumerate(pts):
            lb[4 * k:4 * k + 3] = p
    elif kind == 1:
        n = rng.normal(size=3)
        n /= np.linalg.norm(n)
        ax = np.cross(n, [0.3, 0.5, 0.8])
        ax /= np.linalg.norm(ax)
        ay = np.cross(n, ax)
        lb[0] = rng.uniform(0.05, 0.6)
        lb[4:7] = c
        lb[8:11] = ax
        lb[12:15] = ay
        lb[20:23] = n
    else:
        lb[0] = rng.uniform(0.05, 0.6)
        lb[4:7] = c
    lb[16:19] = rng.uniform(1, 20, 3)
    li[24] = kind
    return lb.view(np.uint8)


@pytest.mark.parametrize("kind", [0, 1, 2])
def test_light_samplers(kind):
    lib = oracle.load()
    rng = np.random.default_rng(10 + kind)
    for _ in range(400):
        lb = _light(kind, rng)
        for _ in range(10):
            p = rng.uniform(-3, 3, 3).astype(F32)
            n = rng.normal(size=3)
            n = (n / np.linalg.norm(n)).astype(F32)
            u0, u1 = (np.float32(x) for x in rng.uniform(0, 1, 2))
            a = np.zeros(12, F32)
            lib.oracle_sample_light(lb.ctypes.data, p.ctypes.data, u0, u1, a.ctypes.data)
            b = ref.sample_light(lb, p, n, u0, u1)
            assert same_bits(a, b), (kind, a, b)


# ---- pathtracerMdl.hlsl ----------------------------------------------------------

@pytest.mark.parametrize("sampling", [0, 1, 2, 3])
def test_camera_rays(sampling):
    lib = oracle.load()
    s = scenes.cornell(40, 32)
    p = s.param(spp=4, frameNumber=3, stratifiedSamplingType=sampling)
    rng = np.random.default_rng(20 + sampling)
    for _ in range(500):
        px, py, st, sidx = int(rng.integers(0, 40)), int(rng.integers(0, 32)), int(rng.integers(1, 2**32)), \
            int(rng.integers(0, 64))
        a = np.zeros(6, F32)
        sa = C.c_uint32(st)
        lib.oracle_camera_ray(C.byref(p), px, py, C.byref(sa), sidx, a.ctypes.data)
        b, sb = ref.camera_ray(p, px, py, st, sidx)
        assert same_bits(a, b)
        assert sa.value == sb


def _compare_samples(view, p, count=None):
    o = oracle.pathtrace(view, p, count=count)
    g, ub = ref.pathtrace(view, p, count=count)
    o3, g3 = o.reshape(-1, 3), g.reshape(-1, 3)
    ok = (bits(o3) == bits(g3)).all(1)
    assert ok[~ub].all(), np.nonzero(~ok & ~ub)[0][:10]
    return ub.mean()


@pytest.mark.parametrize("sampling", [0, 1, 2, 3])
@pytest.mark.parametrize("depth", [4, 8])
def test_cornell_samples(sampling, depth):
    s = scenes.cornell(48, 40, sphere_levels=4, max_depth=depth)
    view = oracle.SceneView(s)
    p = s.param(spp=2, maxDepth=depth, frameNumber=7, stratifiedSamplingType=sampling)
    undefined = _compare_samples(view, p)
    assert undefined < 0.2


@pytest.mark.parametrize("extra", [1, 2, 3])
def test_disc_sphere_and_several_lights(extra):
    # the light pick over 2-3 lights (pathtracerMdl.hlsl:83-92), the disc and
    # sphere samplers (lights.h:196-219, 59-89, 300-340, the sphere sampler's
    # shadowed `u` kept) and shadow rays that reach another light's emitter
    # first (pathtracerMdl.hlsl:63-74)
    s = scenes.cornell(48, 40, sphere_levels=3, extra_lights=extra)
    view = oracle.SceneView(s)
    for sampling, depth in ((1, 8), (0, 4)):
        p = s.param(spp=4, maxDepth=depth, frameNumber=5 + depth, stratifiedSamplingType=sampling)
        assert p.numLights == 1 + bin(extra).count("1")
        assert _compare_samples(view, p) < 0.2


def test_instanced_textured_scene_without_environment():
    # the large-render generator at toy size: 6 instanced displaced spheres,
    # GGX metal / dielectric / textured Lambert; the environment light is an
    # extension (the reference's miss adds nothing), so it is left out
    s = scenes.large(width=48, height=32, instances=6, frequency=10, num_textures=2, tex_size=64, env_width=32,
                     env_height=16, max_depth=8, spp=2, seed=5)
    s.env = None
    view = oracle.SceneView(s)
    p = s.param(spp=2, frameNumber=11)
    _compare_samples(view, p)


def test_no_lights():
    # numLights == 0 over an empty (zeroed) light buffer, as the reference's
    # host leaves it for a scene without lights: the light pick reads the
    # zeroed lights[0], its pdf becomes 0 * (1/0) = NaN and the path ends
    # after the first hit's emission
    s = scenes.cornell(32, 24, sphere_levels=3)
    s.lights[:] = 0
    view = oracle.SceneView(s)
    p = s.param(spp=1, frameNumber=2, numLights=0)
    _compare_samples(view, p)


# ---- reduction / accumulation / tonemap / upscale --------------------------------

def test_post_passes():
    W, H, S = 37, 23, 5
    rng = np.random.default_rng(30)
    sb = rng.gamma(0.5, 1.0, W * H * S * 3).astype(F32)
    sb[::97] = 0.0
    p = abi.PathTracerParam()
    p.dimension[0], p.dimension[1], p.spp = W, H, S
    red = oracle.reduce(p, sb)
    assert same_bits(red, ref.reduce(p, sb))
    hist = np.concatenate([rng.uniform(0, 3, (W * H, 3)), np.ones((W * H, 1))], 1).astype(F32).ravel()
    from strelka_b200.render import accumulation_param, tonemap_param, upscale_param

    for it in (0, 1, 7, 1000):
        ap = accumulation_param(W, H, it)
        a = oracle.accumulate(ap, red, hist)
        b = ref.accumulate(ap, red, hist)
        assert same_bits(a.reshape(-1, 4)[:, :3], b.reshape(-1, 4)[:, :3])
    img = red.copy()
    img.reshape(-1, 4)[::11, :3] = 0.0  # black pixels: Reinhard gives NaN
    for kind in (0, 1, 2):
        tp = tonemap_param(W, H, kind)
        a = oracle.tonemap(tp, img)
        b = ref.tonemap(tp, img)
        assert same_bits(a, b), kind
    for ow, oh in ((74, 46), (17, 11), (37, 23)):
        up = upscale_param(ow, oh)
        a = oracle.upscale(up, img, W, H)
        b = ref.upscale(up, img, W, H)
        assert same_bits(a.reshape(-1, 4)[:, :3], b.reshape(-1, 4)[:, :3])
