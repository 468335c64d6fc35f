"""FP64 PyTorch restatement of the per-frame SAXS forward, differentiable in the positions.

TEST INFRASTRUCTURE ONLY (gradient checks of the CUDA adjoint).  Same method as
``oracle.saxs_oracle`` (see its header for the reference lines followed), written
with torch ops so that autograd yields dL/dx: cell coordinates and bins are
piecewise constant and taken from the detached geometry (the float32 bin rule of
the oracle's C helper), B-spline weights, spreading, the z-border mean, the
supercell, the R2C transform, the form-factor type sum and |F|^2 are
differentiable.  CPU, float64.
"""
from __future__ import annotations

import math

import numpy as np
import torch

from oracle import saxs_oracle as O


def cubic_weights(u):
    """Order-4 B-spline weights of the four taps at offset u (tap 0 farthest left)."""
    v = 1.0 - u
    return torch.stack([v ** 3 / 6, (3 * u ** 3 - 6 * u ** 2 + 4) / 6,
                        (-3 * u ** 3 + 3 * u ** 2 + 3 * u + 1) / 6, u ** 3 / 6])


def profile(plan: O.OraclePlan, xyz: torch.Tensor, type_of_atom, box):
    """(num_bins,) FP64 profile hist/nhist (0 where nhist == 0 and in bin 0) for one frame."""
    co, oc = O.cell_matrices(box, plan.box_mode)
    ocs = plan.scaled_oc(oc)
    nn = plan.nn
    n = plan.grid
    mw, bins = O.kpoint_bins(nn, ocs, plan.dq, plan.kcut, plan.num_bins, plan.contraction)
    inside = torch.from_numpy(~(mw > plan.kcut))
    P = plan.order
    nt = min(P, 4)
    oc64 = torch.tensor(oc.astype(np.float64))
    x1 = xyz @ oc64.T                                   # (N, 3) fractional
    frac = x1 - torch.round(x1.detach() - 0.5)          # wrap into [0, 1]
    r = frac * torch.tensor([float(v) for v in n], dtype=torch.float64)
    m = torch.floor(r.detach())
    u = r - m
    m = m.long()
    w = [cubic_weights(u[:, d]) for d in range(3)]     # each (4, N)
    toa = torch.as_tensor(np.asarray(type_of_atom), dtype=torch.long)
    border = torch.from_numpy(O.border_planes(n[2]))
    npz = nn[2] // 2 + 1
    acc = torch.zeros((nn[0], nn[1], npz), dtype=torch.complex128)
    mwt = torch.from_numpy(mw.astype(np.float64))
    for t in range(len(plan.types)):
        sel = torch.nonzero(toa == t).flatten()
        g = torch.zeros(n[0] * n[1] * n[2], dtype=torch.float64)
        if sel.numel():
            idx, val = [], []
            for o in range(nt):
                ix = (m[sel, 0] - P + o) % n[0]
                for p in range(nt):
                    iy = (m[sel, 1] - P + p) % n[1]
                    for q in range(nt):
                        iz = (m[sel, 2] - P + q) % n[2]
                        idx.append((ix * n[1] + iy) * n[2] + iz)
                        val.append(w[0][o, sel] * w[1][p, sel] * w[2][q, sel])
            g = g.index_add(0, torch.cat(idx), torch.cat(val))
        g = g.reshape(n[0], n[1], n[2])
        mean = (g[:, :, border].sum() / (n[0] * n[1] * int(border.sum())) if plan.padding is None
                else torch.tensor(float(plan.padding[t]), dtype=torch.float64))
        ex = [min(n[d], nn[d]) for d in range(3)]
        sup = mean * torch.ones(nn, dtype=torch.float64)
        sup = sup.clone()
        sup[: ex[0], : ex[1], : ex[2]] = g[: ex[0], : ex[1], : ex[2]]
        ft = torch.fft.rfftn(sup)
        c = plan.coeffs[t].astype(np.float64)
        s2 = (mwt / (4.0 * math.pi)) ** 2
        f = (c[0] * torch.exp(-c[4] * s2) + c[1] * torch.exp(-c[5] * s2) + c[2] * torch.exp(-c[6] * s2)
             + c[3] * torch.exp(-c[7] * s2) + c[8])
        acc = acc + torch.where(inside, f * ft, torch.zeros_like(ft))
    modx, mody, modz = (torch.from_numpy(v) for v in plan.mod)
    m3 = modx[:, None, None] * mody[None, :, None] * modz[None, None, :npz]
    iv = (acc.real ** 2 + acc.imag ** 2) * m3
    mirror = torch.roll(torch.flip(iv, dims=(0, 1)), shifts=(1, 1), dims=(0, 1))
    pair = iv + mirror
    pair = pair.clone()
    pair[0, 0, 0] = iv[0, 0, 0]
    b = torch.from_numpy(bins.astype(np.int64))
    sel = b >= 0
    hist = torch.zeros(plan.num_bins, dtype=torch.float64).index_add(0, b[sel], pair[sel])
    cnt = np.full(bins.shape, 2.0)
    cnt[0, 0, 0] = 1.0
    nhist = np.bincount(bins[bins >= 0], weights=cnt[bins >= 0], minlength=plan.num_bins)
    nh = torch.from_numpy(nhist[: plan.num_bins])
    out = torch.where(nh > 0, hist / torch.where(nh > 0, nh, torch.ones_like(nh)),
                      torch.zeros_like(hist))
    out = out.clone()
    out[0] = 0.0
    return out, nh
