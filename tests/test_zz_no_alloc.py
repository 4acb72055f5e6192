"""strelka_trace_execute_noalloc against strelka_trace_execute and the oracle.

The allocation-free entry point serves callers that cannot let the library
allocate device memory (an engine whose own allocator owns the device heap,
or a real-time loop that cannot pay for cudaMalloc's synchronisation).  Its
results must equal those of the regular ray query and of the oracle's
restatement of closestHit / anyHit (shaders/raytracing.h:198-286), bit for
bit, on two calls in a row with different scenes (the shared scratch table is
rebuilt by each call); a call must leave the device's free memory unchanged;
and scenes beyond its fixed scratch must be refused.

This file is named to be collected last, and passes alone in a fresh
process as well as after the other tests.
"""
import ctypes as C

import numpy as np
import pytest

import oracle
from gpu_util import interior_rays
from strelka_b200 import abi, scenes
from strelka_b200.render import DeviceScene, PathTracer, to_device

pytestmark = pytest.mark.gpu


def regular(torch, pt, ds, rays_d, n, flags):
    hits = torch.zeros(n * 20, dtype=torch.uint8, device="cuda")
    pt.trace(ds.trace_desc(rays_d, hits, flags))
    torch.cuda.synchronize()
    return hits.cpu().numpy().view(np.uint32).reshape(n, 5)


def noalloc_call(torch, desc, status):
    abi.check(abi.load().strelka_trace_execute_noalloc(C.byref(desc), C.c_void_p(status.data_ptr()), None))
    torch.cuda.synchronize()


def noalloc(torch, ds, rays_d, n, flags):
    hits = torch.full((n * 20,), 0xAB, dtype=torch.uint8, device="cuda")
    status = torch.full((1,), 0x7777, dtype=torch.int32, device="cuda")
    noalloc_call(torch, ds.trace_desc(rays_d, hits, flags), status)
    return hits.cpu().numpy().view(np.uint32).reshape(n, 5), int(status.item())


def test_noalloc_matches_regular_and_oracle_on_two_calls(cuda):
    pt = PathTracer()
    # call 1: the Cornell box (instanced spheres, rays from inside)
    s1 = scenes.cornell(16, 16, sphere_levels=4)
    r1 = interior_rays(50_000, 31)
    # call 2: a different, larger scene, so the scratch left by call 1 is stale
    s2 = scenes.soup(60_000, 7)
    r2 = scenes.rays_soup(50_000, 8)
    for s, rays in ((s1, r1), (s2, r2)):
        ds, view = DeviceScene(s), oracle.SceneView(s)
        n = rays.shape[0]
        rd = to_device(rays)
        for flags in (abi.TRACE_CLOSEST, abi.TRACE_ANY):
            want = regular(cuda, pt, ds, rd, n, flags)
            got, status = noalloc(cuda, ds, rd, n, flags)
            ref, found, _ = oracle.trace(view, rays, any_hit=flags == abi.TRACE_ANY)
            assert status == 0
            assert np.array_equal(got, want)
            assert np.array_equal(got, ref)
            assert found.sum() > 100
    pt.close()


def test_noalloc_leaves_free_memory_unchanged(cuda):
    # the set-up call (no scene, no rays) makes the runtime reserve the fixed
    # scratch; after it, calls on two different scenes change nothing in the
    # device's free memory
    s1, s2 = scenes.soup(20_000, 11), scenes.soup(50_000, 12)
    ds1, ds2 = DeviceScene(s1), DeviceScene(s2)
    r1, r2 = to_device(scenes.rays_soup(30_000, 13)), to_device(scenes.rays_soup(30_000, 14))
    h1 = cuda.zeros(30_000 * 20, dtype=cuda.uint8, device="cuda")
    h2 = cuda.zeros(30_000 * 20, dtype=cuda.uint8, device="cuda")
    status = cuda.zeros(1, dtype=cuda.int32, device="cuda")
    empty = abi.TraceDesc()
    noalloc_call(cuda, empty, status)
    # warm-up: one call per query kind, so both kernels are loaded
    noalloc_call(cuda, ds1.trace_desc(r1, h1, abi.TRACE_CLOSEST), status)
    noalloc_call(cuda, ds2.trace_desc(r2, h2, abi.TRACE_ANY), status)
    d1, d2 = ds1.trace_desc(r1, h1, abi.TRACE_ANY), ds2.trace_desc(r2, h2, abi.TRACE_CLOSEST)
    free0, _ = cuda.cuda.mem_get_info()
    for d in (d2, d1, d2):
        noalloc_call(cuda, d, status)
        assert int(status.item()) == 0
    free1, _ = cuda.cuda.mem_get_info()
    assert free1 == free0
    assert (h2.cpu().numpy().view(np.uint32).reshape(-1, 5)[:, 3] != 0xFFFFFFFF).sum() > 100


def test_noalloc_refuses_large_scene(cuda):
    s = scenes.soup(140_000, 3)  # 279,999 nodes > 262,144
    ds = DeviceScene(s)
    rays = to_device(scenes.rays_soup(16, 1))
    hits = cuda.zeros(16 * 20, dtype=cuda.uint8, device="cuda")
    desc = ds.trace_desc(rays, hits, abi.TRACE_CLOSEST)
    rc = abi.load().strelka_trace_execute_noalloc(C.byref(desc), None, None)
    assert rc == abi.ERR_INVALID_ARGUMENT
    assert "at most 262144" in abi.last_error()
