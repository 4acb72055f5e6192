"""Sharding of the path tracer across GPUs (one process per GPU).

Paths are independent, so the work shards by sample, in two ways:

* independent frames (weak scaling): rank r renders its own frames of the
  same scene with sample seeds no other rank uses (:func:`frame_number`),
  and per-GPU work stays fixed as ranks are added.  Nothing is exchanged
  while frames render; when an application wants a single image, the ranks'
  accumulated images are combined by a weighted sum
  (:func:`combine_accumulated`), one collective of W*H*4 floats after the
  last frame;
* one frame split across the ranks (strong scaling): rank r renders spp/N
  samples per pixel of the frame (:func:`split_frame_param`), exactly the
  frame's samples r*spp/N ... (r+1)*spp/N - 1 of every pixel, and after its
  reduction pass the ranks' images are averaged by one all-reduce of W*H*4
  floats per frame (:func:`combine_split_frame`).

Timing is the maximum over ranks (:func:`max_over_ranks`).
"""
from __future__ import annotations

FRAME_STRIDE = 100_000


def frame_number(rank: int, step: int, stride: int = FRAME_STRIDE) -> int:
    """The PathTracerParam.frameNumber rank `rank` uses for its `step`-th
    frame; distinct across ranks as long as each renders fewer than `stride`
    frames (the RNG seed is frameNumber*spp + sample, random.h:26-30)."""
    if step >= stride:
        raise ValueError("step exceeds the per-rank frame stride")
    return rank * stride + step


def max_over_ranks(value: float, dist=None, device="cpu") -> float:
    """Maximum of a per-rank scalar (elapsed milliseconds) over all ranks."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return float(value)
    import torch

    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def combine_accumulated(image, iterations: int, dist=None):
    """Merges the ranks' progressive means into one: each rank's RGBA32F
    accumulated image (a torch tensor, mean of `iterations` frames) is
    weighted by its frame count and summed across ranks.  Returns the
    combined mean on every rank (alpha stays 1)."""
    import torch

    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return image.clone()
    w = torch.tensor([float(iterations)], dtype=torch.float64, device=image.device)
    total = w.clone()
    dist.all_reduce(total)
    acc = image.to(torch.float64) * w
    dist.all_reduce(acc)
    out = (acc / total).to(image.dtype)
    out.view(-1, 4)[:, 3] = 1.0
    return out


def split_frame_param(param, rank: int, world: int):
    """Rank `rank`'s share of the frame `param` (spp S, frameNumber F): a copy
    with spp = S / world and frameNumber = F * world + rank.  The shader seeds
    sample s of a pixel with frameNumber * spp + s (pathtracerMdl.hlsl:
    414-417), so the share's sample s is bit for bit the frame's sample
    rank * S / world + s.  S must be a multiple of world."""
    import ctypes as C

    from . import abi

    if world < 1 or param.spp % world != 0:
        raise ValueError(f"spp {param.spp} does not split over {world} ranks")
    p = abi.PathTracerParam()
    C.memmove(C.byref(p), C.byref(param), C.sizeof(p))
    p.spp = param.spp // world
    p.frameNumber = param.frameNumber * world + rank
    return p


def combine_split_frame(image, dist=None):
    """The frame's image from the ranks' reduction-pass outputs (RGBA32F, each
    the mean of its spp/N samples): their average over the ranks, summed by
    one all-reduce in place.  Returns `image`, now the same on every rank
    (alpha stays 1)."""
    if dist is None or not dist.is_initialized() or dist.get_world_size() == 1:
        return image
    world = dist.get_world_size()
    dist.all_reduce(image)
    image.mul_(1.0 / world)
    image.view(-1, 4)[:, 3] = 1.0
    return image
