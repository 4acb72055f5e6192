"""GPU parity at the sizes the workloads are quoted on.

* Cornell box, 512x512, 1 spp per iteration x 64 iterations, depth 4, seed 0
  (frameNumber = iteration), ACESFitted: the whole per-frame sequence of
  PtRender::drawFrame (src/render/ptrender.cpp:735-862) -- path tracer,
  reduction, accumulation into the running history, tonemap -- against the
  oracle's same chain (pathtracerMdl.hlsl:406-423, reduction.hlsl:9-32,
  accumulation.hlsl:86-97, tonemap.hlsl:66-88).  Every sample of every
  iteration, the accumulated image and the tonemapped image are compared bit
  for bit.
* Ray queries on the 1M-triangle soup with 4M rays: closest-hit records
  (t, barycentrics, instance and primitive ids) bit for bit against the
  reference's stackless loop (raytracing.h:198-247), ties included; any-hit
  records of 4M shadow rays (tmax in [0.1, 2]) bit for bit against the
  reference's depth-first loop (raytracing.h:249-286); visit counts equal to
  the oracle's replay of the kernels' traversal rule (closest hit: of one
  warp that takes a 4096-ray batch); and the float-float
  refinement of t and the barycentrics against an FP64 Moller-Trumbore.
"""
import numpy as np
import pytest

import oracle
from gpu_util import relmse
from strelka_b200 import abi, scenes
from strelka_b200.render import (Accumulation, DeviceScene, PathTracer, ReductionPass, Tonemap, accumulation_param,
                                 ptr, to_device, tonemap_param)

pytestmark = pytest.mark.gpu

W = H = 512
ITERATIONS = 64


def test_cornell_512_64_iterations_aces(cuda):
    torch = cuda
    s = scenes.cornell(W, H, sphere_levels=4)
    assert s.num_triangles == 10_252
    view, ds = oracle.SceneView(s), DeviceScene(s)
    pt = PathTracer(mode=abi.MODE_WAVEFRONT)
    npx = W * H
    sb = torch.empty(npx * 3, dtype=torch.float32, device="cuda")
    cur = torch.empty(npx * 4, dtype=torch.float32, device="cuda")
    acc = [torch.zeros(npx * 4, dtype=torch.float32, device="cuda") for _ in range(2)]
    tm = torch.empty(npx * 4, dtype=torch.float32, device="cuda")
    tp = tonemap_param(W, H, 1)
    red, accu, tone = ReductionPass(), Accumulation(), Tonemap()
    o_hist = np.zeros(npx * 4, np.float32)
    sample_mismatch = 0
    for it in range(ITERATIONS):
        p = s.param(spp=1, maxDepth=4, frameNumber=it, iteration=it, stratifiedSamplingType=0)
        pt.execute(ds.desc(p, sb), npx, 1, it)
        red.execute(abi.ReductionDesc(p, ptr(sb), ptr(cur)), npx, 1, it)
        hist, out = acc[it % 2], acc[(it + 1) % 2]
        ap = accumulation_param(W, H, it)
        accu.execute(abi.AccumulationDesc(ap, ptr(cur), ptr(hist), ptr(out)), W, H, it)
        # the oracle's chain for the same iteration
        o_sb = oracle.pathtrace(view, p)
        o_cur = oracle.reduce(p, o_sb)
        o_acc = oracle.accumulate(ap, o_cur, o_hist)
        g_sb = sb.cpu().numpy()
        sample_mismatch += int((g_sb.view(np.uint32) != o_sb.view(np.uint32)).sum())
        assert np.array_equal(out.cpu().numpy().view(np.uint32), o_acc.view(np.uint32)), f"iteration {it}"
        o_hist = o_acc
    tone.execute(abi.TonemapDesc(tp, ptr(acc[ITERATIONS % 2]), ptr(tm)), W, H, ITERATIONS - 1)
    o_tm = oracle.tonemap(tp, o_hist)
    g_tm = tm.cpu().numpy()
    assert pt.device_status() == 0
    pt.close()
    assert sample_mismatch == 0
    assert np.array_equal(g_tm.view(np.uint32), o_tm.view(np.uint32))
    # the image is a converged-looking Cornell box, not black
    rgb = o_hist.reshape(-1, 4)[:, :3]
    assert rgb.mean() > 0.05 and np.isfinite(rgb).all()
    assert relmse(acc[ITERATIONS % 2].cpu().numpy(), o_hist) == 0.0


@pytest.fixture(scope="module")
def soup_1m(cuda):
    s = scenes.soup(1_000_000, 0)
    return s, oracle.SceneView(s), DeviceScene(s), PathTracer()


def _trace(torch, pt, ds, rays_d, n, flags, counters=None):
    hits = torch.zeros(n * 20, dtype=torch.uint8, device="cuda")
    pt.trace(ds.trace_desc(rays_d, hits, flags, counters))
    torch.cuda.synchronize()
    return hits.cpu().numpy().view(np.uint32).reshape(n, 5)


N_RAYS = 4_000_000
# the largest queue chunk: one warp takes a batch this size, so closest-hit
# counts (deferred leaf tests) are deterministic
WARP_CHUNK = 4096


@pytest.mark.parametrize("query", ["closest", "any"])
def test_soup_1m_tris_4m_rays(cuda, soup_1m, query):
    s, view, ds, pt = soup_1m
    shadow = query == "any"
    rays = scenes.rays_soup(N_RAYS, 2 if shadow else 1, shadow=shadow)
    flags = abi.TRACE_ANY if shadow else abi.TRACE_CLOSEST
    rd = to_device(rays)
    g = _trace(cuda, pt, ds, rd, N_RAYS, flags)
    o, found, _ = oracle.trace(view, rays, any_hit=shadow, prune=0)
    assert found.sum() > N_RAYS // 20
    assert np.array_equal(g, o)
    # visit counts: the kernels count what they process; the oracle replays
    # the same rule (closest hit: its warp replay, on one warp's batch)
    cnt = cuda.zeros(2, dtype=cuda.int64, device="cuda")
    g2 = _trace(cuda, pt, ds, rd, N_RAYS, flags | abi.TRACE_COUNT, cnt)
    assert np.array_equal(g2, o)
    if shadow:
        _, _, co = oracle.trace(view, rays, any_hit=True, prune=2)
        assert np.array_equal(cnt.cpu().numpy().astype(np.uint64), co)
    else:
        sub = rays[:WARP_CHUNK]
        ptw = PathTracer(queue_chunk=WARP_CHUNK)
        cw = cuda.zeros(2, dtype=cuda.int64, device="cuda")
        gw = _trace(cuda, ptw, ds, to_device(sub), WARP_CHUNK, flags | abi.TRACE_COUNT, cw)
        ow, _, cow = oracle.trace_warp(view, sub)
        assert np.array_equal(cw.cpu().numpy().astype(np.uint64), cow)
        assert np.array_equal(gw, o[:WARP_CHUNK]) and np.array_equal(ow, o[:WARP_CHUNK])
        assert ptw.device_status() == 0
    assert pt.device_status() == 0


def test_soup_1m_refine_against_fp64(cuda, soup_1m):
    """Refined t, u, v of every closest hit against the FP64 formula.

    Bar: within 2 ulp of the FP64 value for every hit whose FP64 value is
    itself accurate to a small fraction of a float ulp.  A barycentric within
    about 1e-6 of a triangle edge on a 0.003-sized triangle is the difference
    of terms some 10^5 to 10^6 times larger than itself, so neither FP64 nor
    the float-float refinement resolves it to a float ulp of its own tiny
    value; for those the bar is the forward error bound of the float-float
    evaluation, 2^-44 of the terms' magnitude divided by |det|."""
    s, view, ds, pt = soup_1m
    rays = scenes.rays_soup(N_RAYS, 1)
    g = _trace(cuda, pt, ds, to_device(rays), N_RAYS, abi.TRACE_CLOSEST | abi.TRACE_REFINE)
    found = g[:, 3] != 0xFFFFFFFF
    assert found.sum() > N_RAYS // 20
    r = rays[found]
    t64, u64, v64 = oracle.intersect_fp64(view, r, g[found, 3], g[found, 4])
    scale = oracle.intersect_terms_fp64(view, r, g[found, 3], g[found, 4])
    within = []
    for col, ref, sc in ((2, t64, scale[:, 2]), (0, u64, scale[:, 0]), (1, v64, scale[:, 1])):
        got = g[found, col].view(np.float32).astype(np.float64)
        ulp = np.spacing(np.abs(ref).astype(np.float32)).astype(np.float64)
        err = np.abs(got - ref)
        ok_ulp = err <= 2.0 * ulp
        ill = sc * 2.0 ** -44 > 0.25 * ulp  # FP64 or float-float cannot resolve an ulp here
        assert (ok_ulp | (ill & (err <= sc * 2.0 ** -44))).all(), (col, err[~ok_ulp][:8], ulp[~ok_ulp][:8])
        within.append(ok_ulp.mean())
    # almost every hit meets the plain 2-ulp bar
    assert min(within) > 0.995, within
