"""The GPU's 4-wide traversal rule, replayed by the oracle (prune=2), returns
the reference's closestHit / anyHit records (shaders/raytracing.h:198-286)
bit for bit, ties in t included: skipping the odd-depth boxes of the binary
tree leaves the set of tested triangles unchanged, and closest-hit ties go to
the leaf first in depth-first order, as in the reference's strict t < minHit
loop.  The GPU kernels match this replay exactly (tests/test_gpu_trace.py).
The closest-hit kernels defer leaf tests and run them across the warp; the
oracle's replay of one such warp (oracle.trace_warp) returns the same records
too."""
import numpy as np
import pytest

import oracle
from gpu_util import interior_rays, vertex_edge_rays
from strelka_b200 import scenes


def warp_matches(view, rays, ref):
    """The deferred warp replay's closest hits equal the reference's."""
    got, _, _ = oracle.trace_warp(view, rays)
    return np.array_equal(got, ref)


@pytest.fixture(scope="module")
def cornell():
    s = scenes.cornell(16, 16, sphere_levels=4)
    return oracle.SceneView(s)


@pytest.mark.parametrize("any_hit", [False, True])
def test_ties_at_vertices_and_edges(cornell, any_hit):
    rays = vertex_edge_rays()
    ref, found, _ = oracle.trace(cornell, rays, any_hit=any_hit)
    wide, _, _ = oracle.trace(cornell, rays, any_hit=any_hit, prune=2)
    assert found.mean() > 0.8
    assert np.array_equal(wide, ref)
    if not any_hit:
        assert warp_matches(cornell, rays, ref)


@pytest.mark.parametrize("tmax", [1e9, 0.4])
def test_random_interior_rays(cornell, tmax):
    rays = interior_rays(20_000, 11, tmax=tmax)
    for any_hit in (False, True):
        ref, _, _ = oracle.trace(cornell, rays, any_hit=any_hit)
        wide, _, _ = oracle.trace(cornell, rays, any_hit=any_hit, prune=2)
        assert np.array_equal(wide, ref)
        if not any_hit:
            assert warp_matches(cornell, rays, ref)


def test_soup():
    s = scenes.soup(20_000, 3)
    v = oracle.SceneView(s)
    for shadow in (False, True):
        rays = scenes.rays_soup(20_000, 4, shadow=shadow)
        for any_hit in (False, True):
            ref, _, _ = oracle.trace(v, rays, any_hit=any_hit)
            wide, _, _ = oracle.trace(v, rays, any_hit=any_hit, prune=2)
            assert np.array_equal(wide, ref)
            if not any_hit:
                assert warp_matches(v, rays, ref)


@pytest.mark.parametrize("num_tris", [1, 2, 3, 5])
def test_tiny_trees(num_tris):
    # a leaf root, a root with two leaves, and odd shapes of the first levels
    s = scenes.soup(num_tris, 7)
    v = oracle.SceneView(s)
    rays = scenes.rays_soup(4000, 8)
    for any_hit in (False, True):
        ref, _, _ = oracle.trace(v, rays, any_hit=any_hit)
        wide, _, _ = oracle.trace(v, rays, any_hit=any_hit, prune=2)
        assert np.array_equal(wide, ref)
        if not any_hit:
            assert warp_matches(v, rays, ref)


def test_chain_tree():
    # a BVH of depth n - 1 (much deeper than any builder makes)
    from gpu_util import chain_bvh
    s = chain_bvh(scenes.soup(600, 12))
    v = oracle.SceneView(s)
    rays = scenes.rays_soup(3000, 13)
    for any_hit in (False, True):
        ref, found, _ = oracle.trace(v, rays, any_hit=any_hit)
        wide, _, _ = oracle.trace(v, rays, any_hit=any_hit, prune=2)
        assert np.array_equal(wide, ref)
        if not any_hit:
            assert warp_matches(v, rays, ref)
    # the chain is a valid tree: the reference finds the same hits over it as
    # over the builder's tree
    base, _, _ = oracle.trace(oracle.SceneView(scenes.soup(600, 12)), rays)
    ref, _, _ = oracle.trace(v, rays)
    assert np.array_equal(ref[:, 3:], base[:, 3:]) and found.sum() > 0


def test_instanced_scene():
    # the large-render generator at toy size: several instances, leaves of
    # different instance ids, an environment-lit open scene
    s = scenes.large(width=16, height=8, instances=5, frequency=8, num_textures=1, tex_size=16, env_width=16,
                     env_height=8, max_depth=4, spp=1, seed=9)
    v = oracle.SceneView(s)
    lo, hi = s.bounds()
    rng = np.random.default_rng(14)
    n = 6000
    rays = np.zeros((n, 8), np.float32)
    rays[:, :3] = rng.uniform(lo, hi, (n, 3))
    d = rng.normal(size=(n, 3))
    rays[:, 4:7] = d / np.linalg.norm(d, axis=1, keepdims=True)
    rays[:, 3] = np.where(np.arange(n) % 2 == 0, 1e9, rng.uniform(0.1, 3.0, n))
    for any_hit in (False, True):
        ref, found, _ = oracle.trace(v, rays, any_hit=any_hit)
        wide, _, _ = oracle.trace(v, rays, any_hit=any_hit, prune=2)
        assert found.sum() > 100
        assert np.array_equal(wide, ref)
        if not any_hit:
            assert warp_matches(v, rays, ref)


def test_warp_replay_constants_match_the_kernels():
    # the oracle's replay of a deferring warp uses the kernels' pending-list
    # size and lane threshold
    import os
    import re
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cuh = open(os.path.join(root, "strelka_b200", "csrc", "traverse.cuh")).read()
    orc = open(os.path.join(root, "oracle", "oracle.c")).read()

    def define(text, name):
        return int(re.search(r"#define\s+" + name + r"\s+(\d+)", text).group(1))

    assert define(cuh, "SB_DEFER_CAP") == define(orc, "DEFER_CAP")
    assert define(cuh, "SB_DEFER_LANES") == define(orc, "DEFER_LANES")
    assert define(cuh, "SB_STACK") == define(orc, "WIDE_STACK")
