"""Differentiable SAXS profile: I(q) of one frame as a function of the positions.

``saxs_profile(xyz, engine, box)`` returns the frame's FP64 profile over all
histogram bins (0 in bin 0 and in bins with no k-point, which the reference
does not report).  Its backward is the hand-written adjoint of the CUDA path
(``saxs_backward_device``): dL/dI(bin) is spread onto the k-points of each bin
and their mirror partners, carried through the form factors, the complex type
sum and |F|^2, taken back through the three pruned DFT passes with conjugated
twiddles, through the z-border padding mean, and gathered at the atoms with the
B-spline derivative weights.  The per-type grids are recomputed in the backward
pass instead of being stored.

Forward and backward stay on the device: the histogram is read into device
tensors and dL/dhist is handed over as one, so an optimisation loop never waits
for the host.  A kernel error is left in the plan's status word; the next
``engine.histogram()`` or ``engine.counters()`` reports it.  No reference
counterpart: the reference has no derivative.
"""
from __future__ import annotations

import numpy as np
import torch


def _profile_of(h, n):
    prof = torch.where(n > 0, h / torch.where(n > 0, n, torch.ones_like(n)), torch.zeros_like(h))
    prof[0] = 0.0
    return prof


class _SaxsProfile(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xyz, engine, box):
        x = xyz.detach().to(engine.device, torch.float32).contiguous()
        cur = torch.cuda.current_stream(engine.device)
        engine.stream.wait_stream(cur)
        engine.reset()
        engine.forward(x, box)
        h, n = engine.histogram_device()
        engine.reset()
        x.record_stream(engine.stream)
        ctx.engine = engine
        ctx.nhist = n
        ctx.box = np.asarray(box, dtype=np.float32)
        ctx.save_for_backward(xyz)
        return _profile_of(h, n).to(xyz.device)

    @staticmethod
    def backward(ctx, grad_out):
        (xyz,) = ctx.saved_tensors
        eng = ctx.engine
        n = ctx.nhist
        g = grad_out.detach().to(eng.device, torch.float64)
        dl = torch.where(n > 0, g / torch.where(n > 0, n, torch.ones_like(n)), torch.zeros_like(g))
        dl[0] = 0.0
        grad = eng.backward_device(xyz.detach().to(eng.device, torch.float32).contiguous(), ctx.box, dl)
        return grad.to(device=xyz.device, dtype=xyz.dtype), None, None


def saxs_profile(xyz: torch.Tensor, engine, box) -> torch.Tensor:
    """Differentiable FP64 I(q) (num_bins,) of positions ``xyz`` (natoms, 3) in ``box``."""
    return _SaxsProfile.apply(xyz, engine, box)


def reported_bins(engine, box=None) -> np.ndarray:
    """Boolean mask of the bins the profile file reports (o >= 1 with counts)."""
    h, n = engine.histogram()
    m = n > 0
    m[0] = False
    return m
