"""The radiance cache inside the wavefront path tracer.

A cache trained online on the frame's own training paths must (a) leave the
renderer's status clean and its output finite; (b) lower the error of a
one-sample-per-pixel image against a converged reference compared with the
plain renderer at the same sample count.  Ending a path at its second vertex
can at best remove the noise of the bounces after it, so the gain is measured
against that floor: the error of plain depth-2 images against a depth-2
reference.  (c) The mean of many cached frames stays closer to the reference
than the plain mean at the same sample count (the cache's bias is below the
noise it removes).  The megakernel mode refuses the cache.
"""
import numpy as np
import pytest

from gpu_util import relmse
from strelka_b200 import abi, scenes
from strelka_b200.render import DeviceScene, PathTracer, RadianceCache

pytestmark = pytest.mark.gpu

W, H, DEPTH = 48, 48, 8


@pytest.fixture(scope="module")
def setup(cuda):
    s = scenes.cornell(W, H, sphere_levels=3)
    ds = DeviceScene(s)
    pt = PathTracer(mode=abi.MODE_MEGAKERNEL)
    # converged references: 8192 samples per pixel, full depth and depth 2
    ref = frame(cuda, s, ds, pt, 900, spp=8192).cpu().numpy()
    ref2 = frame(cuda, s, ds, pt, 901, spp=8192, depth=2).cpu().numpy()
    assert pt.device_status() == 0
    pt.close()
    return s, ds, ref, ref2


def frame(cuda, s, ds, pt, frame_number, spp=1, depth=DEPTH):
    p = s.param(spp=spp, maxDepth=depth, frameNumber=frame_number, stratifiedSamplingType=1)
    sb = cuda.zeros(W * H * spp * 3, dtype=cuda.float32, device="cuda")
    pt.execute(ds.desc(p, sb), W * H * spp, 1, 0)
    return sb.view(W * H, spp, 3).double().mean(1)


def test_cache_lowers_error_at_equal_samples(cuda, setup):
    s, ds, ref, ref2 = setup
    lo, hi = s.bounds()
    plain = PathTracer(mode=abi.MODE_WAVEFRONT)
    plain_err = np.mean([relmse(frame(cuda, s, ds, plain, 5000 + k).cpu().numpy(), ref) for k in range(16)])
    floor = np.mean([relmse(frame(cuda, s, ds, plain, 5000 + k, depth=2).cpu().numpy(), ref2) for k in range(16)])

    cache = RadianceCache(lo, hi, learning_rate=1e-2, seed=3, log2_table_size=16)
    pt = PathTracer(mode=abi.MODE_WAVEFRONT, profile=True)
    pt.set_nrc(cache, train_paths=16384, train_steps=4, diffuse_roughness=0.25)
    for k in range(48):  # warm-up: online training on each frame's training paths
        frame(cuda, s, ds, pt, 100 + k)
    imgs = [frame(cuda, s, ds, pt, 5000 + k) for k in range(16)]
    assert pt.device_status() == 0
    assert all(np.isfinite(i.cpu().numpy()).all() for i in imgs)
    nrc_err = float(np.mean([relmse(i.cpu().numpy(), ref) for i in imgs]))
    times = pt.kernel_times()
    assert times["nrc_train"][1] > 0 and times["nrc_infer"][1] > 0
    # (b) the cache removes most of the noise of the bounces after the second vertex
    assert nrc_err < plain_err, (nrc_err, plain_err, floor)
    assert plain_err - nrc_err >= 0.6 * (plain_err - floor), (nrc_err, plain_err, floor)

    # (c) 64 frames averaged: closer to the reference than the plain mean, same brightness
    many = (sum(frame(cuda, s, ds, pt, 7000 + k) for k in range(64)) / 64).cpu().numpy()
    plain_many = (sum(frame(cuda, s, ds, plain, 7000 + k) for k in range(64)) / 64).cpu().numpy()
    assert relmse(many, ref) < relmse(plain_many, ref), (relmse(many, ref), relmse(plain_many, ref))
    assert abs(many.mean() / ref.mean() - 1.0) < 0.03, (many.mean(), ref.mean())
    pt.close()
    plain.close()
    cache.close()


def test_megakernel_refuses_cache(cuda, setup):
    s, ds, _, _ = setup
    lo, hi = s.bounds()
    cache = RadianceCache(lo, hi, log2_table_size=12)
    pt = PathTracer(mode=abi.MODE_MEGAKERNEL)
    pt.set_nrc(cache)
    with pytest.raises(abi.StrelkaError) as e:
        frame(cuda, s, ds, pt, 1)
    assert e.value.code == abi.ERR_UNSUPPORTED
    pt.set_nrc(None)
    frame(cuda, s, ds, pt, 1)  # detached: renders again
    pt.close()
    cache.close()


def test_cache_disabled_is_bit_identical_to_plain(cuda, setup):
    # a cache object attached with enable = 0 changes nothing
    s, ds, _, _ = setup
    lo, hi = s.bounds()
    cache = RadianceCache(lo, hi, log2_table_size=12)
    a = PathTracer(mode=abi.MODE_WAVEFRONT)
    b = PathTracer(mode=abi.MODE_WAVEFRONT)
    cfg = abi.StrelkaNrcRenderConfig(0, 1024, 1, 0.25)
    abi.check(b.lib.strelka_pathtracer_set_nrc(b.handle, cache.handle, cfg))
    x = frame(cuda, s, ds, a, 3, spp=2).cpu().numpy()
    y = frame(cuda, s, ds, b, 3, spp=2).cpu().numpy()
    assert np.array_equal(x, y)
    a.close()
    b.close()
    cache.close()


def test_chunked_wavefront_with_frozen_cache(cuda, setup):
    # with training off the cache is fixed, and a frame split into several
    # wavefront chunks (each with its own queries and inference) must equal
    # the frame rendered in one chunk, bit for bit
    s, ds, _, _ = setup
    lo, hi = s.bounds()
    cache = RadianceCache(lo, hi, log2_table_size=14, seed=7)
    rng = np.random.default_rng(0)
    mlp, grid = cache.params()
    cache.set_params(None, rng.normal(0, 0.2, grid.size).astype(np.float32))  # a cache that predicts something
    whole = PathTracer(mode=abi.MODE_WAVEFRONT)
    parts = PathTracer(mode=abi.MODE_WAVEFRONT, chunk_paths=1000)
    for pt in (whole, parts):
        pt.set_nrc(cache, train_paths=0, train_steps=1, diffuse_roughness=0.25)
    a = frame(cuda, s, ds, whole, 11, spp=2).cpu().numpy()
    b = frame(cuda, s, ds, parts, 11, spp=2).cpu().numpy()
    assert whole.device_status() == 0 and parts.device_status() == 0
    assert np.isfinite(a).all()
    assert np.array_equal(a, b)
    plain = PathTracer(mode=abi.MODE_WAVEFRONT)
    c = frame(cuda, s, ds, plain, 11, spp=2).cpu().numpy()
    assert not np.array_equal(a, c)  # the cache did take part
    for pt in (whole, parts, plain):
        pt.close()
    cache.close()
