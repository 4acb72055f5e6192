"""Ray queries on the GPU against the oracle's restatement of closestHit /
anyHit (shaders/raytracing.h:198-286): closest-hit and any-hit records match
bit for bit, ties in t included (closest-hit ties go to the leaf first in
depth-first order, as in the reference); visit counters match the oracle
replaying the GPU's traversal rule (for closest hit, whose leaf tests are
deferred across the warp, the replay of one warp that takes a whole batch)."""
import numpy as np
import pytest

import oracle
from gpu_util import interior_rays, vertex_edge_rays
from strelka_b200 import abi, scenes
from strelka_b200.render import DeviceScene, PathTracer, to_device

pytestmark = pytest.mark.gpu


def run_trace(torch, pt, ds, rays, flags):
    n = rays.shape[0]
    rays_d = to_device(rays)
    hits_d = torch.zeros(n * 20, dtype=torch.uint8, device="cuda")
    cnt = torch.zeros(2, dtype=torch.int64, device="cuda")
    pt.trace(ds.trace_desc(rays_d, hits_d, flags, cnt))
    torch.cuda.synchronize()
    return hits_d.cpu().numpy().view(np.uint32).reshape(n, 5), cnt.cpu().numpy().astype(np.uint64)


@pytest.fixture(scope="module")
def soup_setup(cuda):
    s = scenes.soup(200_000, 0)
    return s, oracle.SceneView(s), DeviceScene(s), PathTracer()


@pytest.fixture(scope="module")
def cornell_setup(cuda):
    s = scenes.cornell(16, 16, sphere_levels=4)
    return s, oracle.SceneView(s), DeviceScene(s), PathTracer()


# The largest queue chunk: with at most this many rays, one warp takes them
# all in a fixed order, so the closest-hit counts are deterministic.
WARP_CHUNK = 4096


def check_warp_counts(torch, ds, view, rays):
    """Closest-hit visit counts of batches of WARP_CHUNK rays, each taken by
    one warp, against the oracle's replay of that warp; records against the
    reference loop."""
    pt = PathTracer(queue_chunk=WARP_CHUNK)
    total = np.zeros(2, np.uint64)
    for a in range(0, rays.shape[0], WARP_CHUNK):
        r = rays[a:a + WARP_CHUNK]
        g, cg = run_trace(torch, pt, ds, r, abi.TRACE_CLOSEST | abi.TRACE_COUNT)
        o, _, co = oracle.trace_warp(view, r)
        ref, _, _ = oracle.trace(view, r)
        assert np.array_equal(cg, co)
        assert np.array_equal(o, ref)
        assert np.array_equal(g, ref)
        total += co
    assert pt.device_status() == 0
    return total


def test_closest_soup(cuda, soup_setup):
    s, view, ds, pt = soup_setup
    rays = scenes.rays_soup(100_000, 1)
    g, _ = run_trace(cuda, pt, ds, rays, abi.TRACE_CLOSEST)
    o, found, _ = oracle.trace(view, rays)
    assert found.sum() > 1000
    assert np.array_equal(g, o)
    assert pt.device_status() == 0


def test_closest_interior_cornell(cuda, cornell_setup):
    s, view, ds, pt = cornell_setup
    rays = interior_rays(100_000, 3)
    g, _ = run_trace(cuda, pt, ds, rays, abi.TRACE_CLOSEST)
    o, found, _ = oracle.trace(view, rays)
    assert found.mean() > 0.8  # the box's front face is open
    assert np.array_equal(g, o)


@pytest.mark.parametrize("flags", [abi.TRACE_CLOSEST, abi.TRACE_ANY])
def test_ties_at_vertices_and_edges(cuda, cornell_setup, flags):
    # rays aimed at shared vertices and edges of the wall grid: many exact
    # ties in t, resolved as the reference resolves them
    s, view, ds, pt = cornell_setup
    rays = vertex_edge_rays()
    g, _ = run_trace(cuda, pt, ds, rays, flags)
    o, found, _ = oracle.trace(view, rays, any_hit=flags == abi.TRACE_ANY)
    assert found.mean() > 0.8
    assert np.array_equal(g, o)


@pytest.mark.parametrize("shadow", [False, True])
def test_any_hit_exact(cuda, soup_setup, shadow):
    s, view, ds, pt = soup_setup
    rays = scenes.rays_soup(100_000, 2, shadow=shadow)
    g, _ = run_trace(cuda, pt, ds, rays, abi.TRACE_ANY)
    o, found, _ = oracle.trace(view, rays, any_hit=True)
    assert found.sum() > 100
    assert np.array_equal(g, o)


@pytest.mark.parametrize("setup", ["soup_setup", "cornell_setup"])
def test_visit_counters(cuda, setup, request):
    # the kernels count 4-wide nodes and triangle tests; the oracle replays
    # the same traversal rule and must count the same
    s, view, ds, pt = request.getfixturevalue(setup)
    rays = scenes.rays_soup(50_000, 4) if setup == "soup_setup" else interior_rays(50_000, 4)
    total = check_warp_counts(cuda, ds, view, rays)
    # with every warp busy the deferral differs, the records do not; the
    # immediate rule (prune=2) bounds the work from below
    g, cg = run_trace(cuda, pt, ds, rays, abi.TRACE_CLOSEST | abi.TRACE_COUNT)
    o, _, co = oracle.trace(view, rays, prune=2)
    assert np.array_equal(g, o)
    assert np.all(cg >= co) and np.all(total >= co)
    shadow = scenes.rays_soup(50_000, 5, shadow=True) if setup == "soup_setup" else interior_rays(50_000, 5, tmax=0.4)
    g, cg = run_trace(cuda, pt, ds, shadow, abi.TRACE_ANY | abi.TRACE_COUNT)
    o, _, co = oracle.trace(view, shadow, any_hit=True, prune=2)
    assert np.array_equal(cg, co)
    assert np.array_equal(g, o)


def test_refine_within_2ulp_of_fp64(cuda, cornell_setup):
    s, view, ds, pt = cornell_setup
    rays = interior_rays(20_000, 7)
    g, _ = run_trace(cuda, pt, ds, rays, abi.TRACE_CLOSEST | abi.TRACE_REFINE)
    found = g[:, 3] != 0xFFFFFFFF
    t64, u64, v64 = oracle.intersect_fp64(view, rays[found], g[found, 3], g[found, 4])
    for col, ref in ((2, t64), (0, u64), (1, v64)):
        got = g[found, col].view(np.float32).astype(np.float64)
        ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
        err = np.abs(got - ref) / ulp
        assert np.percentile(err, 100) <= 2.0, (col, err.max())


def test_host_buffers_entry(cuda, cornell_setup):
    import ctypes as C
    s, view, ds, pt = cornell_setup
    rays = interior_rays(1000, 11)
    stage_r = cuda.zeros(1000 * 32, dtype=cuda.uint8, device="cuda")
    stage_h = cuda.zeros(1000 * 20, dtype=cuda.uint8, device="cuda")
    hits = np.zeros((1000, 5), np.uint32)
    desc = ds.trace_desc(stage_r, stage_h, abi.TRACE_CLOSEST)
    abi.check(abi.load().strelka_trace_host(pt.handle, C.byref(desc), rays.ctypes.data, hits.ctypes.data, None))
    o, _, _ = oracle.trace(view, rays)
    assert np.array_equal(hits, o)


def test_chain_tree_deeper_than_the_walk_cap(cuda):
    # depth 2999 > the 1024-step walk-up of the 4-wide build: its parities
    # come from the pointer-jumping pass; hits equal the reference's
    from gpu_util import chain_bvh
    s = chain_bvh(scenes.soup(3000, 21))
    view, ds, pt = oracle.SceneView(s), DeviceScene(s), PathTracer()
    rays = scenes.rays_soup(20_000, 22)
    for flags in (abi.TRACE_CLOSEST, abi.TRACE_ANY):
        g, _ = run_trace(cuda, pt, ds, rays, flags)
        o, found, _ = oracle.trace(view, rays, any_hit=flags == abi.TRACE_ANY)
        assert found.sum() > 50
        assert np.array_equal(g, o)
    assert pt.device_status() == 0
