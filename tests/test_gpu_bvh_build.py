"""BVH construction on the GPU: the nodes follow the host builder's flattened
depth-first layout (src/render/bvh.cpp:169-235), builds are deterministic,
and rays traced over a GPU-built BVH give the oracle's hits over the same
nodes and the same closest distances as over the host SAH BVH."""
import dataclasses

import numpy as np
import pytest

import oracle
from gpu_util import bits_equal_fraction, compare_closest, interior_rays, relmse
from strelka_b200 import abi, scenes
from strelka_b200.render import BvhBuilder, DeviceScene, PathTracer, to_device
from test_bvh import check_layout, world_triangles

pytestmark = pytest.mark.gpu


def positions_of(s):
    tris, ids = world_triangles(s)
    n = tris.shape[0]
    raw = np.zeros((3 * n, 5), np.uint32)
    raw[:, 0:3] = tris.reshape(-1, 3).view(np.uint32)
    idarr = np.array(ids, np.uint32)
    raw[:, 3] = np.repeat(idarr[:, 0], 3)
    raw[:, 4] = np.repeat(idarr[:, 1], 3)
    return raw, n


def run_trace(torch, pt, ds, rays, flags):
    n = rays.shape[0]
    hits = torch.zeros(n * 20, dtype=torch.uint8, device="cuda")
    pt.trace(ds.trace_desc(to_device(rays), hits, flags))
    torch.cuda.synchronize()
    return hits.cpu().numpy().view(np.uint32).reshape(n, 5)


MODES = [abi.BVH_PLOC, abi.BVH_LBVH]


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("ntris", [1, 2, 3, 17, 3000])
def test_layout_from_positions(cuda, ntris, mode):
    s = scenes.soup(ntris, 7)
    raw, n = positions_of(s)
    b = BvhBuilder(mode)
    nodes = b.build(to_device(raw), 3 * n)
    check_layout(nodes.cpu().numpy(), n)
    again = b.build(to_device(raw), 3 * n)
    assert np.array_equal(nodes.cpu().numpy(), again.cpu().numpy())  # deterministic
    b.close()


def test_bad_mode(cuda):
    b = BvhBuilder()
    with pytest.raises(abi.StrelkaError):
        abi.check(b.lib.strelka_bvh_builder_set_mode(b.handle, 7, 16))
    with pytest.raises(abi.StrelkaError):
        abi.check(b.lib.strelka_bvh_builder_set_mode(b.handle, abi.BVH_PLOC, 0))
    b.close()


def test_empty(cuda):
    b = BvhBuilder()
    nodes = b.build(to_device(np.zeros(5, np.uint32)), 0)
    assert nodes.numel() == 0
    b.close()


@pytest.mark.parametrize("mode", MODES)
def test_scene_build_matches_positions_build(cuda, mode):
    # the on-device world transform equals the host's (same arithmetic), so
    # both routes give the same nodes
    s = scenes.cornell(16, 16, sphere_levels=2)
    ds = DeviceScene(s)
    b = BvhBuilder(mode)
    a = b.build_scene(ds).cpu().numpy()
    raw, n = positions_of(s)
    c = b.build(to_device(raw), 3 * n).cpu().numpy()
    check_layout(a, n)
    assert np.array_equal(a, c)
    b.close()


@pytest.fixture(scope="module", params=MODES)
def gpu_bvh_scenes(cuda, request):
    out = []
    for s in (scenes.cornell(24, 16, sphere_levels=4),
              scenes.large(width=20, height=12, instances=3, frequency=16, num_textures=2, tex_size=64, env_width=64,
                           env_height=32, max_depth=6, spp=2, seed=4)):
        b = BvhBuilder(request.param)
        nodes = b.build_scene(DeviceScene(s)).cpu().numpy()
        b.close()
        g = dataclasses.replace(s, nodes=nodes)
        out.append((s, g, DeviceScene(s), DeviceScene(g), oracle.SceneView(g)))
    return out


def test_trace_matches_oracle_and_host_bvh(cuda, gpu_bvh_scenes):
    pt = PathTracer()
    for s, g, ds_host, ds_gpu, view in gpu_bvh_scenes:
        check_layout(g.nodes, g.num_triangles)
        lo, hi = s.bounds()
        rays = interior_rays(50_000, 9, 0.0, 1.0)
        rays[:, :3] = lo + rays[:, :3] * (hi - lo)
        got = run_trace(cuda, pt, ds_gpu, rays, abi.TRACE_CLOSEST)
        o, found, _ = oracle.trace(view, rays)
        assert found.mean() > 0.1
        compare_closest(got, o)
        # closest distances do not depend on the tree
        host = run_trace(cuda, pt, ds_host, rays, abi.TRACE_CLOSEST)
        compare_closest(got, host)
        # any hit keeps the depth-first order of this tree
        sh = rays.copy()
        sh[:, 3] = 0.5
        ga = run_trace(cuda, pt, ds_gpu, sh, abi.TRACE_ANY)
        oa, _, _ = oracle.trace(view, sh, any_hit=True)
        assert np.array_equal(ga, oa)
    assert pt.device_status() == 0


def test_render_over_gpu_bvh(cuda, gpu_bvh_scenes):
    s, g, _, ds_gpu, view = gpu_bvh_scenes[0]
    p = g.param(spp=2, maxDepth=4, frameNumber=3, stratifiedSamplingType=1)
    n = p.dimension[0] * p.dimension[1] * p.spp
    sb = cuda.zeros(n * 3, dtype=cuda.float32, device="cuda")
    pt = PathTracer()
    pt.execute(ds_gpu.desc(p, sb), n, 1, 0)
    assert pt.device_status() == 0
    got = sb.cpu().numpy()
    ref = oracle.pathtrace(view, p)
    assert relmse(got, ref) <= 1e-4
    assert bits_equal_fraction(got, ref) >= 0.999


@pytest.mark.parametrize("mode", MODES)
def test_identical_centroids_and_degenerate_triangles(cuda, mode):
    # every Morton code equal: the radix tree splits by position alone
    n = 1000
    tri = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0]], np.float32)
    pos = np.tile(tri, (n, 1)).astype(np.float32)
    pos[3 * (n // 2):] *= 0.0  # the second half collapses to points (zero-area triangles)
    raw = np.zeros((3 * n, 5), np.uint32)
    raw[:, 0:3] = pos.view(np.uint32)
    raw[:, 3] = 0
    raw[:, 4] = np.repeat(np.arange(n, dtype=np.uint32), 3)
    b = BvhBuilder(mode)
    nodes = b.build(to_device(raw), 3 * n).cpu().numpy()
    b.close()
    check_layout(nodes, n)
    # the root box covers every corner
    f = nodes.view(np.float32).reshape(-1, 8)
    assert np.allclose(f[0, 0:3], 0) and np.allclose(f[0, 4:6], 1, atol=1e-5)
