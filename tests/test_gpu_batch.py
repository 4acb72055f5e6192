"""The batched launch: every job's samples must be bit-identical to the
single-job pass rendering the same descriptor, in every execution mode,
block size, queue chunk, with and without the shade sort and the CUDA graph;
the autotuner, per-job latencies and per-frame seeds must work."""
import numpy as np
import pytest

from strelka_b200 import abi, scenes
from strelka_b200.render import Batch, DeviceScene, PathTracer, batch_config

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def jobs(cuda):
    corn = scenes.cornell(24, 16, sphere_levels=2)
    big = scenes.large(width=20, height=12, instances=3, frequency=12, num_textures=2, tex_size=64, env_width=64,
                       env_height=32, max_depth=6, spp=2, seed=4)
    dc, dl = DeviceScene(corn), DeviceScene(big)
    params = [
        (corn, dc, corn.param(spp=2, maxDepth=4, frameNumber=3, stratifiedSamplingType=1)),
        (corn, dc, corn.look_at(17, 11, (0.3, 0.6, 2.2), (0.5, 0.4, 0.0), 50.0, spp=3, maxDepth=6, frameNumber=9,
                               stratifiedSamplingType=2)),
        (big, dl, big.param(spp=2, maxDepth=6, frameNumber=1)),
        (big, dl, big.look_at(13, 7, (8.0, 6.0, 12.0), (0.0, 1.0, 0.0), 35.0, spp=1, maxDepth=3, frameNumber=5)),
        (corn, dc, corn.param(spp=1, maxDepth=0, frameNumber=2)),  # no bounce: zero samples
        (big, dl, big.look_at(9, 5, (-6.0, 3.0, 10.0), (0.0, 0.5, 0.0), 60.0, spp=4, maxDepth=8, frameNumber=11)),
    ]
    out = []
    for hs, ds, p in params:
        n = p.dimension[0] * p.dimension[1] * p.spp
        out.append((hs, ds, p, cuda.full((n * 3,), -7.0, dtype=cuda.float32, device="cuda")))
    return out


def render_alone(cuda, ds, p, frame_offset=0):
    q = type(p)()
    import ctypes as C
    C.memmove(C.byref(q), C.byref(p), C.sizeof(q))
    q.frameNumber = p.frameNumber + frame_offset
    n = q.dimension[0] * q.dimension[1] * q.spp
    sb = cuda.full((n * 3,), -7.0, dtype=cuda.float32, device="cuda")
    pt = PathTracer(mode=abi.MODE_MEGAKERNEL)
    pt.execute(ds.desc(q, sb), n, 1, 0)
    assert pt.device_status() == 0
    pt.close()
    return sb.cpu().numpy()


CONFIGS = [
    (abi.BATCH_PERSISTENT, 64, 32, False, True),
    (abi.BATCH_PERSISTENT, 256, 1024, False, True),
    (abi.BATCH_PERSISTENT, 128, 96, False, False),
    (abi.BATCH_WAVEFRONT, 128, 256, False, True),
    (abi.BATCH_WAVEFRONT, 64, 32, True, True),
    (abi.BATCH_WAVEFRONT, 256, 1024, True, False),
]


@pytest.mark.parametrize("cfg", CONFIGS)
def test_batch_matches_single_job(cuda, jobs, cfg):
    expect = [render_alone(cuda, ds, p) for _, ds, p, _ in jobs]
    b = Batch()
    b.set_jobs([ds.desc(p, sb) for _, ds, p, sb in jobs])
    for _, _, _, sb in jobs:
        sb.fill_(-7.0)
    b.execute(batch_config(*cfg))
    b.execute(batch_config(*cfg))  # a replay writes the same samples
    assert b.device_status() == 0
    for k, (_, _, _, sb) in enumerate(jobs):
        got = sb.cpu().numpy()
        assert np.array_equal(got.view(np.uint32), expect[k].view(np.uint32)), f"job {k}"
    lat = b.job_latency()
    assert len(lat) == len(jobs) and all(v > 0 for v in lat), lat
    b.close()


def test_autotune_and_frames(cuda, jobs):
    b = Batch()
    b.set_jobs([ds.desc(p, sb) for _, ds, p, sb in jobs])
    info = b.info()
    assert info["jobs"] == len(jobs)
    assert info["total_paths"] == sum(p.dimension[0] * p.dimension[1] * p.spp for _, _, p, _ in jobs)
    best, entries = b.autotune(repeats=1)
    assert len(entries) >= 8
    assert best.blockSize in (64, 128, 256) and best.queueChunk % 32 == 0
    assert min(ms for _, ms in entries) > 0
    # the tuned configuration is the default; a new frame offset changes the seeds
    b.set_frame(7)
    b.execute()
    for k, (_, ds, p, sb) in enumerate(jobs):
        assert np.array_equal(sb.cpu().numpy().view(np.uint32), render_alone(cuda, ds, p, 7).view(np.uint32)), k
    assert b.device_status() == 0
    b.close()


def test_batch_rejects_bad_config(cuda, jobs):
    b = Batch()
    b.set_jobs([ds.desc(p, sb) for _, ds, p, sb in jobs[:2]])
    for bad in [(5, 128, 256, False, True), (abi.BATCH_WAVEFRONT, 96, 256, False, True),
                (abi.BATCH_WAVEFRONT, 128, 33, False, True), (abi.BATCH_PERSISTENT, 128, 256, True, True)]:
        with pytest.raises(abi.StrelkaError) as e:
            b.execute(batch_config(*bad))
        assert e.value.code == abi.ERR_INVALID_ARGUMENT
    b.close()
