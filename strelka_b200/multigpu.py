"""Sharding of the path tracer across GPUs (one process per GPU).

Paths are independent, so the work shards by sample: rank r renders its own
frames of the same scene with sample seeds no other rank uses
(:func:`frame_number`), and per-GPU work stays fixed as ranks are added
(weak scaling).  Nothing is exchanged while frames render; the one exchange
step, when an application wants a single image, is a weighted sum of the
ranks' accumulated images (:func:`combine_accumulated`), one collective of
W*H*4 floats after the last frame.  Timing is the maximum over ranks
(:func:`max_over_ranks`).
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
