"""Frame sharding across GPUs (one process per GPU, torch.distributed).

Frames are independent, so the path shards by frame: rank r of W processes
frames r, r+W, r+2W, ... of the requested range, accumulates its own FP64
(hist, nhist), and one all-reduce (sum) combines them.  Only num_bins doubles
per vector cross the interconnect; no grid is exchanged.  For npt runs the
summed histogram equals the single-GPU one (the reference sums per-frame
histograms, saxsKernel.cu:190-196).  For nvt runs the reference bins the
intensity summed over all frames once, with the first frame's box and a factor
1/frames (saxsKernel.cu:17-39).  Binning is linear, so each rank may bin its own
sum (as its plan does, with its own 1/frames_r) and the run's histogram is
sum_r frames_r * hist_r / sum_r frames_r (``combine_histogram``); the counts are
those of the first box's k-points, the same on every rank.  ``reduce_intensity``
reduces raw intensity sums instead, for callers that hold them.
"""
from __future__ import annotations

import numpy as np


def shard(frames, rank: int, world: int):
    """The frames of ``rank`` out of ``world`` (round-robin, order preserved)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("need 0 <= rank < world")
    return list(frames)[rank::world]


def frame_range(begin: int, end: int, stride: int):
    """Frames begin..end inclusive every ``stride`` (RunSaxs.cu:137-138)."""
    return range(begin, end + 1, stride)


def allreduce_histogram(hist, nhist, group=None, device=None):
    """Sum FP64 (hist, nhist) over the process group; returns numpy arrays."""
    import torch
    import torch.distributed as dist

    h = np.asarray(hist, dtype=np.float64)
    n = np.asarray(nhist, dtype=np.float64)
    buf = torch.from_numpy(np.concatenate([h, n]))
    if device is not None:
        buf = buf.to(device)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    out = buf.cpu().numpy()
    return out[: h.size].copy(), out[h.size:].copy()


def reduce_intensity(iacc, frames: int, group=None, device=None):
    """Sum an nvt intensity accumulator and its frame count over the group."""
    import torch
    import torch.distributed as dist

    a = torch.from_numpy(np.ascontiguousarray(iacc, dtype=np.float64).reshape(-1))
    c = torch.tensor([float(frames)], dtype=torch.float64)
    if device is not None:
        a, c = a.to(device), c.to(device)
    dist.all_reduce(a, op=dist.ReduceOp.SUM, group=group)
    dist.all_reduce(c, op=dist.ReduceOp.SUM, group=group)
    return a.cpu().numpy().reshape(np.shape(iacc)), int(c.item())


def combine_histogram(hist, nhist, frames: int, ensemble: str = "npt", group=None, device=None):
    """The run's FP64 (hist, nhist) from every rank's own after ``frames`` frames
    on this rank.  npt: the sums.  nvt: sum_r frames_r * hist_r / sum_r frames_r,
    and this rank's nhist (the same on every rank)."""
    if ensemble == "npt":
        return allreduce_histogram(hist, nhist, group=group, device=device)
    import torch
    import torch.distributed as dist

    h = np.asarray(hist, dtype=np.float64)
    buf = torch.from_numpy(np.concatenate([h * float(frames), [float(frames)]]))
    if device is not None:
        buf = buf.to(device)
    dist.all_reduce(buf, op=dist.ReduceOp.SUM, group=group)
    out = buf.cpu().numpy()
    total = out[-1]
    return (out[:-1] / total if total > 0 else np.zeros_like(h)), np.asarray(nhist, dtype=np.float64).copy()


def sharded_histogram(engine, group=None, device=None):
    """``engine``'s histogram combined over the process group (each rank ran its
    own shard of the frames through its own engine)."""
    h, n = engine.histogram()
    return combine_histogram(h, n, engine.frames, engine.ensemble, group=group, device=device)
