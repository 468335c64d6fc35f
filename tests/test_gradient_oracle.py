"""The FP64 torch oracle of the forward and its gradient (CPU).

The oracle's autograd gradient is the reference gradient for the CUDA adjoint,
so it is checked here against FP64 central finite differences (h = 1e-3 A =
1e-4 nm) on 32 random atoms x 3 axes, for the log-profile loss of the
refinement workload.
"""
import numpy as np
import pytest
import torch

from oracle import saxs_oracle as O
from oracle import torch_oracle as TO
from pycusaxs_b200.synthetic import cubic_system


def setup(seed=3, n=800, grid=16):
    s = cubic_system(n, 30.0, seed=seed)
    names = sorted({str(e) for e in s.elements})
    ff = O.load_form_factors()
    plan = O.OraclePlan(grid=(grid,) * 3, types=names, coeffs=np.stack([ff[k] for k in names]),
                        box0=s.box, sigma=2.0, qcut=0.8)
    return s, plan, s.type_of_atom(names)


def log_loss(prof, target, sel):
    return ((torch.log(prof[sel]) - torch.log(target[sel])) ** 2).sum()


def test_torch_oracle_profile_equals_numpy_oracle():
    s, plan, toa = setup()
    x = torch.tensor(s.positions.astype(np.float64))
    prof, _ = TO.profile(plan, x, toa, s.box)
    h, n = O.run_frames(plan, [(s.positions, s.box)], toa)
    ref = np.where(n > 0, h / np.where(n > 0, n, 1), 0.0)
    ref[0] = 0.0
    sel = ref > 0
    np.testing.assert_allclose(prof.numpy()[sel], ref[sel], rtol=1e-6)


def test_torch_oracle_gradient_matches_central_differences():
    s, plan, toa = setup()
    x = torch.tensor(s.positions.astype(np.float64), requires_grad=True)
    prof, nh = TO.profile(plan, x, toa, s.box)
    target = prof.detach() * (1 + 0.05 * torch.sin(torch.arange(len(prof), dtype=torch.float64)))
    sel = prof.detach() > 0
    log_loss(prof, target, sel).backward()
    g = x.grad.numpy()
    rng = np.random.default_rng(7)
    h = 1e-3
    worst = 0.0
    for a in rng.choice(s.natoms, 32, replace=False):
        for d in range(3):
            xp = x.detach().clone()
            xp[a, d] += h
            xm = x.detach().clone()
            xm[a, d] -= h
            fd = (log_loss(TO.profile(plan, xp, toa, s.box)[0], target, sel)
                  - log_loss(TO.profile(plan, xm, toa, s.box)[0], target, sel)) / (2 * h)
            fd = float(fd)
            err = abs(g[a, d] - fd) / max(abs(fd), 1e-3 * np.abs(g).max())
            worst = max(worst, err)
    assert worst < 1e-4, worst
