"""The CPU-only generator library (oracle/libworkload.so) builds the same
scenes, bit for bit, as the package's library it is compiled from, so the
benchmark's CPU reference arm renders exactly the workload the GPU arm does
without loading the CUDA library."""
import numpy as np

import oracle
from strelka_b200 import scenes


def _fields(hs):
    return [hs.vb, hs.ib, hs.instances, hs.lights, hs.materials, hs.arg_block, hs.resource_infos, hs.nodes,
            np.frombuffer(bytes(hs.camera), np.uint8)] + list(hs.textures) + (
        [hs.env, hs.env_marginal, hs.env_conditional] if hs.env is not None else [])


def _build_all():
    return [scenes.cornell(64, 48, sphere_levels=3), scenes.cornell(32, 32, sphere_levels=2, extra_lights=3),
            scenes.soup(20_000, 3),
            scenes.large(width=64, height=32, instances=3, frequency=12, num_textures=2, tex_size=64, env_width=64,
                         env_height=32, max_depth=8, spp=2, seed=0)], scenes.rays_soup(1000, 5, shadow=True)


def test_workload_library_matches_package_library():
    scenes.use_generator_library(None)
    want, want_rays = _build_all()
    scenes.use_generator_library(oracle.workload())
    try:
        got, got_rays = _build_all()
    finally:
        scenes.use_generator_library(None)
    assert np.array_equal(got_rays, want_rays)
    for g, w in zip(got, want):
        assert g.num_triangles == w.num_triangles
        for a, b in zip(_fields(g), _fields(w)):
            assert np.array_equal(np.asarray(a).view(np.uint8), np.asarray(b).view(np.uint8))
