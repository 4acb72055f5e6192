"""The multi-GPU sharding logic, exercised by two gloo ranks on the CPU.

Each rank renders its own frames of the same scene with the oracle (standing
in for the GPU pass on a machine without one), using the per-rank frame
numbers of strelka_b200.multigpu.  The ranks' sample seeds must not overlap,
the combined image must equal the progressive mean of all frames rendered in
one process, and the timing reduction must return the maximum."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

W, H, FRAMES = 24, 16, 2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _render_frames(rank):
    import oracle
    from strelka_b200 import multigpu, scenes

    s = scenes.cornell(W, H, sphere_levels=2)
    view = oracle.SceneView(s)
    acc = None
    frames = []
    for step in range(FRAMES):
        p = s.param(spp=1, maxDepth=4, frameNumber=multigpu.frame_number(rank, step), stratifiedSamplingType=1)
        img = oracle.reduce(p, oracle.pathtrace(view, p, threads=1))
        frames.append(p.frameNumber)
        # accumulation.hlsl:86-97, iteration = step
        acc = img if acc is None else acc * np.float32(step / (step + 1)) + img * np.float32(1 / (step + 1))
    return acc, frames


def _worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    from strelka_b200 import multigpu

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        acc, frames = _render_frames(rank)
        combined = multigpu.combine_accumulated(torch.from_numpy(acc), FRAMES, dist)
        slowest = multigpu.max_over_ranks(10.0 + rank, dist)
        gathered = [None] * world
        dist.all_gather_object(gathered, frames)
        if rank == 0:
            q.put((combined.numpy(), slowest, gathered))
    finally:
        dist.destroy_process_group()


def test_two_rank_sharding():
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    combined, slowest, frames = q.get(timeout=300)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    # distinct sample seeds across ranks
    assert len(set(frames[0]) & set(frames[1])) == 0
    # the timing reduction is the maximum over ranks
    assert slowest == 11.0
    # the combined image is the mean of every rank's frames
    per_rank = [_render_frames(r)[0] for r in range(world)]
    expect = (per_rank[0].astype(np.float64) + per_rank[1]) / 2
    assert np.allclose(combined.reshape(-1, 4)[:, :3], expect.reshape(-1, 4)[:, :3], rtol=1e-6, atol=1e-7)
    assert (combined.reshape(-1, 4)[:, 3] == 1).all()


def test_frame_number_bounds():
    from strelka_b200 import multigpu

    assert multigpu.frame_number(3, 7) == 300007
    with pytest.raises(ValueError):
        multigpu.frame_number(0, multigpu.FRAME_STRIDE)


SPLIT_SPP = 4


def _split_worker(rank, world, port, q):
    import torch
    import torch.distributed as dist

    import oracle
    from strelka_b200 import multigpu, scenes

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = scenes.cornell(W, H, sphere_levels=2)
        view = oracle.SceneView(s)
        full = s.param(spp=SPLIT_SPP, maxDepth=4, frameNumber=5, stratifiedSamplingType=3)
        share = multigpu.split_frame_param(full, rank, world)
        samples = oracle.pathtrace(view, share, threads=1)
        img = torch.from_numpy(oracle.reduce(share, samples))
        combined = multigpu.combine_split_frame(img, dist)
        gathered = [None] * world
        dist.all_gather_object(gathered, samples)
        if rank == 0:
            q.put((combined.numpy(), gathered))
    finally:
        dist.destroy_process_group()


def test_two_rank_split_frame():
    """One frame split over two ranks: each rank's samples are bit for bit
    the frame's samples of its share of every pixel, and the all-reduced
    image equals the single-process frame within rounding."""
    import oracle
    from strelka_b200 import scenes

    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_split_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    combined, shares = q.get(timeout=300)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    s = scenes.cornell(W, H, sphere_levels=2)
    full = s.param(spp=SPLIT_SPP, maxDepth=4, frameNumber=5, stratifiedSamplingType=3)
    ref = oracle.pathtrace(oracle.SceneView(s), full, threads=1).reshape(W * H, SPLIT_SPP, 3)
    per = SPLIT_SPP // world
    for r in range(world):
        got = shares[r].reshape(W * H, per, 3)
        assert np.array_equal(got.view(np.uint32), ref[:, r * per:(r + 1) * per].view(np.uint32))
    expect = oracle.reduce(full, ref.ravel()).reshape(-1, 4)
    assert np.allclose(combined.reshape(-1, 4)[:, :3], expect[:, :3], rtol=1e-6, atol=1e-7)
    assert ref.mean() > 0.01
