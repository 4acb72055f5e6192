"""The path tracer pass on the GPU against the oracle's restatement of
computeMain / pathTraceCameraRays (shaders/pathtracerMdl.hlsl:165-423) on
the same scene, parameters and RNG seeds.

Bar: relMSE <= 1e-4 of the sample buffer (the image-parity tolerance), and,
since both sides evaluate the same operation sequence and closest-hit ties
resolve as in the reference, every sample bit-identical to the oracle (the
committed golden fixture: 99.9%)."""
import numpy as np
import pytest

import oracle
from gpu_util import bits_equal_fraction, relmse
from strelka_b200 import abi, scenes
from strelka_b200.render import DeviceScene, PathTracer, to_device

pytestmark = pytest.mark.gpu

RELMSE_BAR = 1e-4
EXACT_BAR = 1.0        # every sample bit-identical to the oracle


@pytest.fixture(scope="module")
def cornell(cuda):
    s = scenes.cornell(40, 32, sphere_levels=4)
    return s, oracle.SceneView(s), DeviceScene(s)


def render(torch, s, ds, param, mode, chunk=0):
    total = param.dimension[0] * param.dimension[1] * param.spp
    sb = torch.full((total * 3,), -7.0, dtype=torch.float32, device="cuda")
    pt = PathTracer(mode=mode, chunk_paths=chunk)
    pt.execute(ds.desc(param, sb), total, 1, 0)
    status = pt.device_status()
    torch.cuda.synchronize()
    return sb.cpu().numpy(), status


@pytest.mark.parametrize("mode", [abi.MODE_MEGAKERNEL, abi.MODE_WAVEFRONT])
@pytest.mark.parametrize("sst", [0, 1, 2, 3])
def test_cornell_sampling_types(cuda, cornell, mode, sst):
    s, view, ds = cornell
    p = s.param(spp=2, maxDepth=4, frameNumber=5, stratifiedSamplingType=sst)
    g, status = render(cuda, s, ds, p, mode, chunk=777)
    r = oracle.pathtrace(view, p)
    assert status == 0
    assert np.isfinite(g).all()
    assert relmse(g, r) <= RELMSE_BAR
    assert bits_equal_fraction(g, r) >= EXACT_BAR


@pytest.mark.parametrize("mode", [abi.MODE_MEGAKERNEL, abi.MODE_WAVEFRONT])
def test_cornell_deep_russian_roulette(cuda, cornell, mode):
    # depth 8 exercises Russian roulette (depth > 3, pathtracerMdl.hlsl:374-382)
    s, view, ds = cornell
    p = s.param(spp=4, maxDepth=8, frameNumber=11, stratifiedSamplingType=1)
    g, status = render(cuda, s, ds, p, mode)
    r = oracle.pathtrace(view, p)
    assert status == 0
    assert relmse(g, r) <= RELMSE_BAR
    assert bits_equal_fraction(g, r) >= EXACT_BAR


def test_megakernel_equals_wavefront(cuda, cornell):
    s, view, ds = cornell
    p = s.param(spp=3, maxDepth=6, frameNumber=2, stratifiedSamplingType=1)
    a, _ = render(cuda, s, ds, p, abi.MODE_MEGAKERNEL)
    b, _ = render(cuda, s, ds, p, abi.MODE_WAVEFRONT, chunk=1000)
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


@pytest.mark.parametrize("tail", [1, 3, 7, 100])
def test_tail_kernel_equals_megakernel(cuda, tail):
    # the wavefront finishes bounces >= tail in one persistent kernel; every
    # switch depth gives the megakernel's samples bit for bit
    s = scenes.large(width=48, height=32, instances=6, frequency=6, num_textures=2, tex_size=64, env_width=64,
                     env_height=32, max_depth=8, spp=2, seed=4)
    ds = DeviceScene(s)
    p = s.param(frameNumber=3)
    a, _ = render(cuda, s, ds, p, abi.MODE_MEGAKERNEL)
    total = p.dimension[0] * p.dimension[1] * p.spp
    sb = cuda.full((total * 3,), -7.0, dtype=cuda.float32, device="cuda")
    pt = PathTracer(mode=abi.MODE_WAVEFRONT, chunk_paths=1111, tail_depth=tail)
    pt.execute(ds.desc(p, sb), total, 1, 0)
    assert pt.device_status() == 0
    b = sb.cpu().numpy()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_debug_normals(cuda, cornell):
    # ubo.debug == 1 returns (N + 1) / 2 of the first surface hit
    s, view, ds = cornell
    p = s.param(spp=1, maxDepth=4, debug=1)
    g, _ = render(cuda, s, ds, p, abi.MODE_WAVEFRONT)
    r = oracle.pathtrace(view, p)
    assert bits_equal_fraction(g, r) >= EXACT_BAR


def test_no_lights_terminates(cuda, cornell):
    # numLights == 0 (no environment): the reference breaks after the first
    # hit's emission (lightPdf = 0 * (1/0) = NaN)
    s, view, ds = cornell
    p = s.param(spp=1, maxDepth=4, numLights=0)
    g, _ = render(cuda, s, ds, p, abi.MODE_MEGAKERNEL)
    r = oracle.pathtrace(view, p)
    assert np.array_equal(g.view(np.uint32), r.view(np.uint32))


def test_large_scene_small(cuda):
    # the large-render generator at toy size: instanced GGX / dielectric /
    # textured Lambert spheres under an environment light
    s = scenes.large(width=48, height=32, instances=6, frequency=6, num_textures=2, tex_size=64, env_width=64,
                     env_height=32, max_depth=6, spp=2, seed=3)
    view = oracle.SceneView(s)
    ds = DeviceScene(s)
    p = s.param(frameNumber=1)
    for mode in (abi.MODE_MEGAKERNEL, abi.MODE_WAVEFRONT):
        g, status = render(cuda, s, ds, p, mode)
        r = oracle.pathtrace(view, p)
        assert status == 0
        assert relmse(g, r) <= RELMSE_BAR
        assert bits_equal_fraction(g, r) >= EXACT_BAR


@pytest.mark.parametrize("variant", ["large", "small"])
def test_scene_kernel_variants(cuda, cornell, variant):
    # the wavefront's large-scene traversal variants (shared-memory stacks,
    # leaf tests deferred across the warp from bounce 1 on) and its
    # small-scene ones give the oracle's samples bit for bit; the tail kernel
    # is off so that every bounce runs the wavefront passes
    s, view, ds = cornell
    big = scenes.large(width=48, height=32, instances=6, frequency=6, num_textures=2, tex_size=64, env_width=64,
                       env_height=32, max_depth=8, spp=2, seed=5)
    for sc, v, d, p in ((s, view, ds, s.param(spp=2, maxDepth=8, frameNumber=9, stratifiedSamplingType=1)),
                        (big, oracle.SceneView(big), DeviceScene(big), big.param(frameNumber=2))):
        total = p.dimension[0] * p.dimension[1] * p.spp
        sb = cuda.full((total * 3,), -7.0, dtype=cuda.float32, device="cuda")
        pt = PathTracer(mode=abi.MODE_WAVEFRONT, chunk_paths=1111, tail_depth=100, scene_kernels=variant)
        pt.execute(d.desc(p, sb), total, 1, 0)
        assert pt.device_status() == 0
        g = sb.cpu().numpy()
        r = oracle.pathtrace(v, p)
        assert bits_equal_fraction(g, r) >= EXACT_BAR


@pytest.mark.parametrize("sort", ["auto", True, False])
def test_shade_sort_modes(cuda, sort):
    # the material sort of the shade queue (by default only for chunks of
    # STRELKA_SHADE_SORT_MIN_PATHS paths or more; forced here on a small
    # frame of several materials) changes which lane shades a path, never its
    # samples: every mode gives the oracle's samples bit for bit
    s = scenes.large(width=48, height=32, instances=6, frequency=6, num_textures=2, tex_size=64, env_width=64,
                     env_height=32, max_depth=8, spp=2, seed=7)
    ds = DeviceScene(s)
    p = s.param(frameNumber=4)
    total = p.dimension[0] * p.dimension[1] * p.spp
    sb = cuda.full((total * 3,), -7.0, dtype=cuda.float32, device="cuda")
    pt = PathTracer(mode=abi.MODE_WAVEFRONT, profile=True, shade_sort=sort, tail_depth=100)
    pt.execute(ds.desc(p, sb), total, 1, 0)
    cuda.cuda.synchronize()
    sorts = pt.kernel_times()["sort"][1]
    assert pt.device_status() == 0
    pt.close()
    assert (sorts > 0) == (sort is True)
    assert bits_equal_fraction(sb.cpu().numpy(), oracle.pathtrace(oracle.SceneView(s), p)) >= EXACT_BAR


def test_serial_shadow_equals_overlapped(cuda):
    # STRELKA_PT_SERIAL_SHADOW runs each bounce's shadow queries on the
    # frame's stream instead of beside the next bounce's closest-hit queries:
    # the same samples bit for bit, and the shadow launches are timed
    s = scenes.large(width=48, height=32, instances=6, frequency=6, num_textures=2, tex_size=64, env_width=64,
                     env_height=32, max_depth=8, spp=2, seed=6)
    ds = DeviceScene(s)
    p = s.param(frameNumber=5)
    total = p.dimension[0] * p.dimension[1] * p.spp
    out = []
    for serial in (False, True):
        sb = cuda.full((total * 3,), -7.0, dtype=cuda.float32, device="cuda")
        pt = PathTracer(mode=abi.MODE_WAVEFRONT, chunk_paths=1111, profile=True, serial_shadow=serial)
        pt.execute(ds.desc(p, sb), total, 1, 0)
        cuda.cuda.synchronize()
        times = pt.kernel_times()
        assert pt.device_status() == 0
        assert times["shadow"][1] > 0
        pt.close()
        out.append(sb.cpu().numpy())
    assert np.array_equal(out[0].view(np.uint32), out[1].view(np.uint32))
    assert bits_equal_fraction(out[1], oracle.pathtrace(oracle.SceneView(s), p)) >= EXACT_BAR


def test_frames_captured_in_a_cuda_graph(cuda):
    # once a frame of the scene and size has run, execute and resolve allocate
    # nothing and never synchronise: a sequence of progressive frames
    # (PtRender::drawFrame's path trace, reduce, accumulate, tonemap)
    # captured into a CUDA graph and replayed gives the stream-ordered images
    # bit for bit, the shadow pass's second stream included
    from strelka_b200.render import accumulation_param, resolve, tonemap_param

    W = H = 64
    npx, iters = W * H, 4
    s = scenes.cornell(W, H, sphere_levels=3)
    ds = DeviceScene(s)
    params = [s.param(spp=1, maxDepth=4, frameNumber=it, iteration=it) for it in range(iters)]
    aps = [accumulation_param(W, H, it) for it in range(iters)]
    tp = tonemap_param(W, H, 1)
    pt = PathTracer(mode=abi.MODE_WAVEFRONT)
    sb = cuda.zeros(npx * 3, dtype=cuda.float32, device="cuda")
    acc = [cuda.zeros(npx * 4, dtype=cuda.float32, device="cuda") for _ in range(2)]
    tm = cuda.zeros(npx * 4, dtype=cuda.float32, device="cuda")

    def sequence(stream):
        for it in range(iters):
            pt.execute(ds.desc(params[it], sb), npx, 1, it, stream)
            resolve(params[it], sb, tp, aps[it], acc[it % 2], acc[(it + 1) % 2], tm, None, stream)

    main = cuda.cuda.current_stream()
    sequence(main)
    cuda.cuda.synchronize()
    assert pt.device_status() == 0
    ref_acc, ref_tm = acc[iters % 2].clone(), tm.clone()
    g = cuda.cuda.CUDAGraph()
    side = cuda.cuda.Stream()
    with cuda.cuda.graph(g, stream=side):
        sequence(side)
    for a in acc:
        a.zero_()
    tm.fill_(-1.0)
    g.replay()
    g.replay()
    cuda.cuda.synchronize()
    assert pt.device_status() == 0
    assert cuda.equal(acc[iters % 2].view(cuda.int32), ref_acc.view(cuda.int32))
    assert cuda.equal(tm.view(cuda.int32), ref_tm.view(cuda.int32))
    del g
    pt.close()


def test_golden_fixture(cuda):
    # the fixture is the reference's own shader code compiled on the host
    # (tests/golden/make_golden.py); samples it leaves undefined are skipped
    import os
    path = os.path.join(os.path.dirname(__file__), "golden", "cornell_64x64.npz")
    gold = np.load(path)
    s = scenes.cornell(64, 64, sphere_levels=4)
    ds = DeviceScene(s)
    p = s.param(spp=int(gold["spp"]), maxDepth=int(gold["max_depth"]), frameNumber=int(gold["frame"]),
                stratifiedSamplingType=int(gold["sst"]))
    for mode in (abi.MODE_WAVEFRONT, abi.MODE_MEGAKERNEL):
        g, _ = render(cuda, s, ds, p, mode)
        defined = ~gold["undefined"]
        got, ref = g.reshape(-1, 3)[defined], gold["samples"].reshape(-1, 3)[defined]
        assert relmse(got, ref) <= RELMSE_BAR
        assert bits_equal_fraction(got, ref) == EXACT_BAR


def test_soup_golden_fixture(cuda):
    # closest- and any-hit records of the reference's closestHit / anyHit
    # (compiled on the host, tests/golden/make_golden.py), bit for bit
    import os
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(__file__), "golden"))
    import make_golden
    gold = np.load(os.path.join(os.path.dirname(__file__), "golden", "soup_trace.npz"))
    s, rays = make_golden.soup_inputs()
    ds = DeviceScene(s)
    pt = PathTracer()
    n = rays.shape[0]
    for flags, key in ((abi.TRACE_CLOSEST, "closest"), (abi.TRACE_ANY, "any")):
        hits = cuda.zeros(n * 20, dtype=cuda.uint8, device="cuda")
        pt.trace(ds.trace_desc(to_device(rays), hits, flags))
        cuda.cuda.synchronize()
        assert np.array_equal(hits.cpu().numpy().view(np.uint32).reshape(n, 5), gold[key]), key
    assert pt.device_status() == 0
    pt.close()
