"""Disc, sphere and several lights on the GPU, bit for bit against the oracle
(itself checked against the reference's own shader code in
tests/test_ref_pin.py).

The scenes add to the Cornell box a disc light just under the ceiling light
and/or a sphere light, each with its emitter instance, built the way the
reference builds them (src/scene/scene.cpp:210-361, 418-510).  They cover:
* the light pick over several lights, (uint)(numLights * rand) with pdf
  1/numLights (pathtracerMdl.hlsl:83-92);
* the disc sampler (lights.h:196-219, 303-319) and the sphere sampler with
  its shadowed `u` (lights.h:59-89, 322-340);
* the light-type switch (pathtracerMdl.hlsl:31-50);
* shadow rays whose first hit in depth-first order is another light's
  emitter, which the reference counts as visible (pathtracerMdl.hlsl:63-74).
"""
import numpy as np
import pytest

import oracle
from gpu_util import bits_equal_fraction, relmse
from strelka_b200 import abi, scenes
from strelka_b200.render import DeviceScene, PathTracer, to_device

pytestmark = pytest.mark.gpu

W, H = 64, 48


@pytest.mark.parametrize("extra", [1, 2, 3])
@pytest.mark.parametrize("mode", [abi.MODE_WAVEFRONT, abi.MODE_MEGAKERNEL])
@pytest.mark.parametrize("sampling,depth", [(1, 8), (3, 4)])
def test_light_kinds_bit_exact(cuda, extra, mode, sampling, depth):
    s = scenes.cornell(W, H, sphere_levels=3, extra_lights=extra)
    view, ds = oracle.SceneView(s), DeviceScene(s)
    p = s.param(spp=4, maxDepth=depth, frameNumber=3 + extra, stratifiedSamplingType=sampling)
    assert p.numLights == 1 + bin(extra).count("1")
    n = W * H * 4
    sb = cuda.zeros(n * 3, dtype=cuda.float32, device="cuda")
    pt = PathTracer(mode=mode)
    pt.execute(ds.desc(p, sb), n, 1, 0)
    st = pt.device_status()
    pt.close()
    got = sb.cpu().numpy()
    ref = oracle.pathtrace(view, p)
    assert st == 0
    assert bits_equal_fraction(got, ref) == 1.0
    assert relmse(got, ref) == 0.0
    assert ref.mean() > 0.05


def test_shadow_rays_reach_another_lights_emitter_first(cuda):
    # floor points toward the ceiling light: the disc light hangs in between,
    # so the any-hit query's first hit is often the disc's emitter, which the
    # path tracer counts as the light being visible
    s = scenes.cornell(16, 16, sphere_levels=3, extra_lights=1)
    inst = s.instances.view(np.int32).reshape(-1, 52)
    light_ids = inst[:, 51]
    rng = np.random.default_rng(5)
    n = 20000
    rays = np.zeros((n, 8), np.float32)
    rays[:, 0] = rng.uniform(0.2, 0.8, n)
    rays[:, 1] = 1e-3
    rays[:, 2] = rng.uniform(0.2, 0.8, n)
    target = np.stack([rng.uniform(0.4, 0.6, n), np.full(n, 0.998), rng.uniform(0.4, 0.6, n)], 1)
    d = target - rays[:, :3]
    dist = np.linalg.norm(d, axis=1)
    rays[:, 4:7] = d / dist[:, None]
    rays[:, 3] = dist
    ds = DeviceScene(s)
    pt = PathTracer()
    hits = cuda.zeros(n * 20, dtype=cuda.uint8, device="cuda")
    pt.trace(ds.trace_desc(to_device(rays), hits, abi.TRACE_ANY))
    g = hits.cpu().numpy().view(np.uint32).reshape(n, 5)
    pt.close()
    o, found, _ = oracle.trace(oracle.SceneView(s), rays, any_hit=True)
    assert np.array_equal(g, o)
    first_is_emitter = found & (light_ids[np.minimum(g[:, 3], len(light_ids) - 1)] != -1)
    assert first_is_emitter.mean() > 0.05
