"""Host-injected faults: corrupt BVHs, out-of-range ids, empty scenes and bad
arguments end in error statuses, never in a hang or a device fault.

The reference's traversal loops have no bound (a cycle in nodeOffset spins
forever); here every traversal stops after 2*numNodes+2 visits and raises
STRELKA_DEV_TRAVERSAL_CAP, and every fetch is range-checked first."""
import ctypes as C

import numpy as np
import pytest

from gpu_util import interior_rays
from strelka_b200 import abi, scenes
from strelka_b200.render import DeviceScene, PathTracer, to_device

pytestmark = pytest.mark.gpu


def trace(torch, pt, ds, rays, flags=abi.TRACE_CLOSEST):
    n = rays.shape[0]
    r = to_device(rays)
    h = torch.zeros(n * 20, dtype=torch.uint8, device="cuda")
    pt.trace(ds.trace_desc(r, h, flags))
    status = pt.device_status()
    return h.cpu().numpy().view(np.uint32).reshape(n, 5), status


def corrupt(s, fn):
    import copy
    c = copy.copy(s)
    c.nodes = s.nodes.copy()
    fn(c.nodes.view(np.int32).reshape(-1, 8))
    return c


@pytest.fixture(scope="module")
def base(cuda):
    return scenes.cornell(16, 16, sphere_levels=2)


def first_leaf(i):
    return int(np.nonzero(i[:, 3] != -1)[0][0])


def test_cycle_hits_the_visit_cap(cuda, base):
    def make_cycle(i):
        i[first_leaf(i), 7] = 0  # leaf escape back to the root
    s = corrupt(base, make_cycle)
    pt = PathTracer()
    ds = DeviceScene(s)
    rays = interior_rays(2000, 1)
    _, status = trace(cuda, pt, ds, rays)
    assert status & abi.DEV_TRAVERSAL_CAP
    _, status = trace(cuda, pt, ds, rays, abi.TRACE_ANY)
    assert status & abi.DEV_TRAVERSAL_CAP


def test_escape_out_of_range(cuda, base):
    def bad_escape(i):
        i[first_leaf(i), 7] = i.shape[0] + 5
    s = corrupt(base, bad_escape)
    pt = PathTracer()
    _, status = trace(cuda, pt, DeviceScene(s), interior_rays(2000, 2))
    assert status & abi.DEV_NODE_OOB


def test_instance_out_of_range(cuda, base):
    def bad_inst(i):
        i[first_leaf(i), 3] = 100000
    s = corrupt(base, bad_inst)
    pt = PathTracer()
    hits, status = trace(cuda, pt, DeviceScene(s), interior_rays(2000, 3))
    assert status & abi.DEV_INSTANCE_OOB
    assert not (hits[:, 3] == 100000).any()


def test_light_capacity(cuda, base):
    # numLights beyond the light buffer: the pass reports LIGHT_OOB instead of reading past it
    ds = DeviceScene(base)
    p = base.param(spp=1, maxDepth=3, numLights=5)
    total = 16 * 16
    sb = cuda.zeros(total * 3, dtype=cuda.float32, device="cuda")
    pt = PathTracer(mode=abi.MODE_MEGAKERNEL)
    pt.execute(ds.desc(p, sb), total, 1, 0)
    assert pt.device_status() & abi.DEV_LIGHT_OOB


def test_empty_scene(cuda, base):
    import copy
    s = copy.copy(base)
    s.nodes = np.zeros(0, np.uint8)
    ds = DeviceScene(s)
    pt = PathTracer()
    hits, status = trace(cuda, pt, ds, interior_rays(100, 4))
    assert status == 0 and (hits[:, 3] == 0xFFFFFFFF).all()
    p = base.param(spp=1, maxDepth=4)
    sb = cuda.full((16 * 16 * 3,), 5.0, dtype=cuda.float32, device="cuda")
    pt.execute(ds.desc(p, sb), 16 * 16, 1, 0)
    assert pt.device_status() == 0
    assert (sb.cpu().numpy() == 0).all()


def test_bad_execute_arguments(cuda, base):
    ds = DeviceScene(base)
    p = base.param(spp=2, maxDepth=4)
    sb = cuda.zeros(16 * 16 * 2 * 3, dtype=cuda.float32, device="cuda")
    pt = PathTracer()
    with pytest.raises(abi.StrelkaError) as e:
        pt.execute(ds.desc(p, sb), 16 * 16, 1, 0)  # w must be W*H*spp
    assert e.value.code == abi.ERR_INVALID_ARGUMENT
    d = ds.desc(p, None)
    with pytest.raises(abi.StrelkaError):
        pt.execute(d, 16 * 16 * 2, 1, 0)
    # the two scene-kernel overrides exclude each other
    cfg = abi.StrelkaPathTracerConfig(abi.MODE_WAVEFRONT, 0, 0, abi.PT_LARGE_SCENE_KERNELS | abi.PT_SMALL_SCENE_KERNELS, 0, 0)
    h = C.c_void_p()
    assert pt.lib.strelka_pathtracer_create(C.byref(cfg), C.byref(h)) == abi.ERR_INVALID_ARGUMENT
    # so do the two shade-sort overrides
    cfg = abi.StrelkaPathTracerConfig(abi.MODE_WAVEFRONT, 0, 0, abi.PT_NO_SHADE_SORT | abi.PT_FORCE_SHADE_SORT, 0, 0)
    assert pt.lib.strelka_pathtracer_create(C.byref(cfg), C.byref(h)) == abi.ERR_INVALID_ARGUMENT


@pytest.mark.parametrize("arrive", [0, 1])
def test_bounded_wait_gives_up(cuda, arrive):
    # The wait that guards every tensor-core completion in the radiance-cache
    # kernels, on an mbarrier phase that nothing completes: it gives up after
    # its limit and sets the status bit, and the context stays usable.  With
    # the phase completed first, it passes without a bit.
    import time
    lib = abi.load()
    status = cuda.zeros(1, dtype=cuda.int32, device="cuda")
    t0 = time.perf_counter()
    abi.check(lib.strelka_selftest_wait_timeout(2_000_000, arrive, status.data_ptr(), None))
    cuda.cuda.synchronize()
    elapsed = time.perf_counter() - t0
    if arrive:
        assert int(status.item()) == 0
    else:
        assert int(status.item()) == abi.DEV_MMA_TIMEOUT
        assert elapsed >= 2e-3
    assert int((cuda.ones(4, device="cuda") * 2).sum().item()) == 8
    with pytest.raises(abi.StrelkaError):
        abi.check(lib.strelka_selftest_wait_timeout(2_000_000_000, 0, status.data_ptr(), None))
