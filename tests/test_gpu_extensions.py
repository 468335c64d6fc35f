"""Opt-in physics extensions on the GPU vs the FP64 oracle: the correct-triclinic
inverse and the given (bulk-solvent) padding, on every DFT path, forward and adjoint."""
import os

import numpy as np
import pytest
import torch

from helpers import assert_profiles_close, engine_hist, oracle_hist
from oracle import saxs_oracle as O
from oracle import torch_oracle as TO
from pycusaxs_b200 import SaxsEngine, pycusaxs_cuda
from pycusaxs_b200.autograd import saxs_profile
from pycusaxs_b200.solvent import given_padding
from pycusaxs_b200.synthetic import SyntheticTopology, cubic_system, triclinic_slab_system
from test_extensions_oracle import SHEARED, sheared_cluster

pytestmark = pytest.mark.gpu


def _run(system, grid, frames, **kw):
    ho, no, _ = oracle_hist(system, grid, frames, **kw)
    h, n, eng = engine_hist(system, grid, frames, **kw)
    eng.close()
    return assert_profiles_close(h, n, ho, no)


@pytest.mark.parametrize("simt", [False, True])
def test_triclinic_mode_slab(cuda, simt):
    s = triclinic_slab_system(5000, 40.0, 40.0, 32.0, 75.0, seed=51)
    old = {k: os.environ.get(k) for k in ("PYCUSAXS_ZDFT", "PYCUSAXS_YDFT", "PYCUSAXS_XDFT")}
    try:
        if simt:
            for k in old:
                os.environ[k] = "simt"
        _run(s, (32, 32, 32), [s.positions], sigma=2.0, qcut=0.7, box_mode=1)
    finally:
        for k, v in old.items():
            if v is None:
                os.environ.pop(k, None)
            else:
                os.environ[k] = v


def test_triclinic_mode_sheared_box(cuda):
    from pycusaxs_b200.synthetic import System

    pos, toa = sheared_cluster()
    el = np.array(["C", "O"], dtype=object)[toa]
    s = System(el, pos, SHEARED)
    _run(s, (48, 48, 48), [s.positions], sigma=2.0, qcut=0.6, box_mode=1)


@pytest.mark.parametrize("simt", [False, True])
def test_given_padding(cuda, simt):
    s = cubic_system(6000, 40.0, seed=52)
    names = sorted({str(e) for e in s.elements}, key=lambda k: k.encode())
    pad = given_padding(names, s.box, (32, 32, 32), "TIP3P", {"Na": 3, "Cl": 3})
    old = os.environ.get("PYCUSAXS_ZDFT")
    try:
        if simt:
            os.environ["PYCUSAXS_ZDFT"] = "simt"
        _run(s, (32, 32, 32), [s.positions], sigma=2.0, qcut=0.7, padding=pad)
    finally:
        if old is None:
            os.environ.pop("PYCUSAXS_ZDFT", None)
        else:
            os.environ["PYCUSAXS_ZDFT"] = old


def test_given_padding_adjoint(cuda):
    s = cubic_system(2000, 30.0, seed=53)
    names = sorted({str(e) for e in s.elements}, key=lambda k: k.encode())
    pad = given_padding(names, s.box, (24, 24, 24), "SPCE")
    ff = O.load_form_factors()
    plan = O.OraclePlan(grid=(24,) * 3, types=names, coeffs=np.stack([ff[k] for k in names]),
                        box0=s.box, sigma=2.0, qcut=0.7, padding=pad.astype(np.float64))
    toa = s.type_of_atom(names)
    x64 = torch.tensor(s.positions.astype(np.float64), requires_grad=True)
    prof_o, _ = TO.profile(plan, x64, toa, s.box)
    sel = prof_o.detach() > 0
    prof_o[sel].log().sum().backward()
    eng = SaxsEngine((24, 24, 24), s.atom_index(), s.natoms, s.box, scale_factor=2.0, qcut=0.7,
                     padding="given", padding_values=pad)
    xg = torch.tensor(s.positions, device=eng.device, requires_grad=True)
    prof = saxs_profile(xg, eng, s.box)
    prof[sel.to(prof.device)].log().sum().backward()
    g, g_ref = xg.grad.double().cpu().numpy(), x64.grad.numpy()
    eng.close()
    assert np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref) < 2e-3


def test_dropin_run_with_extensions(cuda, tmp_path):
    s = triclinic_slab_system(3000, 36.0, 36.0, 30.0, 80.0, seed=54, nframes=2, jitter=0.3)
    out = tmp_path / "x.dat"
    pycusaxs_cuda.run(SyntheticTopology(s), "t", "x", [32], end=1, output=str(out), scale_factor=2.0,
                      qcut=0.7, water_model="TIP4P", sodium=2, chlorine=2, box_mode="triclinic",
                      padding="given")
    names = sorted({str(e) for e in s.elements}, key=lambda k: k.encode())
    pad = given_padding(names, s.box, (32, 32, 32), "TIP4P", {"Na": 2, "Cl": 2})
    h, n, plan = oracle_hist(s, (32, 32, 32), [s.frame(0), s.frame(1)], sigma=2.0, qcut=0.7,
                             box_mode=1, padding=pad)
    want = O.profile_rows(h, n, plan.dq)
    got = [(l[:10], float(l[10:])) for l in out.read_text().splitlines()]
    assert [g[0] for g in got] == [f"{q:10.5f}" for q, _ in want]
    for (_, gi), (_, wi) in zip(got, want):
        assert abs(gi - wi) <= 1e-4 * abs(wi)
    with pytest.raises(RuntimeError):
        pycusaxs_cuda.run(SyntheticTopology(s), "t", "x", [32], end=0, output=str(out),
                          scale_factor=2.0, qcut=0.7, padding="solvent")
