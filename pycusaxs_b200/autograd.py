"""Differentiable SAXS profile: I(q) of one frame as a function of the positions.

``saxs_profile(xyz, engine, box)`` returns the frame's FP64 profile over all
histogram bins (0 in bin 0 and in bins with no k-point, which the reference
does not report).  Its backward is the hand-written adjoint of the CUDA path
(``saxs_backward``): dL/dI(bin) is spread onto the k-points of each bin and
their mirror partners, carried through the form factors, the complex type sum
and |F|^2, taken back through the three pruned DFT passes with conjugated
twiddles, through the z-border padding mean, and gathered at the atoms with the
B-spline derivative weights.  The per-type grids are recomputed in the backward
pass instead of being stored.  No reference counterpart: the reference has no
derivative.
"""
from __future__ import annotations

import numpy as np
import torch


class _SaxsProfile(torch.autograd.Function):
    @staticmethod
    def forward(ctx, xyz, engine, box):
        x = xyz.detach().to(engine.device, torch.float32).contiguous()
        engine.reset()
        engine.forward(x, box)
        h, n = engine.histogram()
        engine.reset()
        prof = np.where(n > 0, h / np.where(n > 0, n, 1.0), 0.0)
        prof[0] = 0.0
        ctx.engine = engine
        ctx.nhist = n
        ctx.box = np.asarray(box, dtype=np.float32)
        ctx.save_for_backward(xyz)
        return torch.from_numpy(prof).to(xyz.device)

    @staticmethod
    def backward(ctx, grad_out):
        (xyz,) = ctx.saved_tensors
        dprof = grad_out.detach().to(torch.float64).cpu().numpy()
        n = ctx.nhist
        dl = np.where(n > 0, dprof / np.where(n > 0, n, 1.0), 0.0)
        dl[0] = 0.0
        g = ctx.engine.backward(xyz.detach().to(ctx.engine.device, torch.float32).contiguous(),
                                ctx.box, dl)
        return g.to(device=xyz.device, dtype=xyz.dtype), None, None


def saxs_profile(xyz: torch.Tensor, engine, box) -> torch.Tensor:
    """Differentiable FP64 I(q) (num_bins,) of positions ``xyz`` (natoms, 3) in ``box``."""
    return _SaxsProfile.apply(xyz, engine, box)


def reported_bins(engine, box=None) -> np.ndarray:
    """Boolean mask of the bins the profile file reports (o >= 1 with counts)."""
    h, n = engine.histogram()
    m = n > 0
    m[0] = False
    return m
