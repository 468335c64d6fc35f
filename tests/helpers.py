"""Shared helpers for the parity tests: run the CUDA engine and the FP64 oracle on the same frames."""
from __future__ import annotations

import numpy as np

from oracle import saxs_oracle as O

# Relative per-bin tolerance of the FP32 CUDA path against the FP64 oracle.
RTOL_PROFILE = 1e-4


def oracle_hist(system, grid, frames, *, scaled_grid=(0, 0, 0), order=4, sigma=2.0, bin_size=0.0,
                qcut=0.5, ensemble="npt", boxes=None, box_mode=0, padding=None):
    names = sorted({str(e) for e in system.elements}, key=lambda s: s.encode())
    ff = O.load_form_factors()
    box0 = system.box if boxes is None else boxes[0]
    plan = O.OraclePlan(grid=tuple(grid), types=names, coeffs=np.stack([ff[n] for n in names]),
                        box0=box0, scaled_grid=tuple(scaled_grid), order=order, sigma=sigma,
                        bin_size=bin_size, qcut=qcut, ensemble=ensemble, box_mode=box_mode,
                        padding=None if padding is None else np.asarray(padding, np.float64))
    fr = [(frames[k], system.box if boxes is None else boxes[k]) for k in range(len(frames))]
    h, n = O.run_frames(plan, fr, system.type_of_atom(names))
    return h, n, plan


def engine_hist(system, grid, frames, *, scaled_grid=(0, 0, 0), order=4, sigma=2.0, bin_size=0.0,
                qcut=0.5, ensemble="npt", boxes=None, max_frames=1, device_input=True, box_mode=0,
                padding=None):
    import torch

    from pycusaxs_b200 import SaxsEngine

    box0 = system.box if boxes is None else boxes[0]
    bx = np.stack([system.box] * len(frames)) if boxes is None else np.asarray(boxes)
    eng = SaxsEngine(grid, system.atom_index(), system.natoms, box0, scaled_grid=scaled_grid,
                     order=order, scale_factor=sigma, bin_size=bin_size, qcut=qcut,
                     ensemble=ensemble, max_frames=max_frames,
                     box_mode="triclinic" if box_mode else "parity",
                     padding="average" if padding is None else "given", padding_values=padding)
    x = np.ascontiguousarray(np.stack(frames), dtype=np.float32)
    if device_input:
        eng.forward(torch.from_numpy(x).to(eng.device), bx)
    else:
        eng.forward_host(x, bx)
    h, n = eng.histogram()
    return h, n, eng


def assert_profiles_close(h, n, ho, no, rtol=RTOL_PROFILE):
    """Exact bin counts (the float32 bin rule) and per-bin relative intensity error."""
    np.testing.assert_array_equal(n, no)
    sel = no > 0
    sel[0] = False
    got = h[sel] / n[sel]
    want = ho[sel] / no[sel]
    err = np.abs(got - want) / np.abs(want)
    assert err.max() <= rtol, f"max rel err {err.max():.3e} at bins {np.nonzero(sel)[0][err > rtol]}"
    return float(err.max())


_CASE_ORACLE = {}


def oracle_case(name, case, system):
    """FP64 oracle (hist, nhist, plan) of a golden case over all its frames,
    computed once per test session."""
    if name not in _CASE_ORACLE:
        g = case["grid"]
        grid = tuple(g * 3 if len(g) == 1 else g)
        sg = case.get("scaled", [0, 0, 0])
        _CASE_ORACLE[name] = oracle_hist(
            system, grid, [system.frame(k) for k in range(case["frames"])],
            scaled_grid=tuple(sg * 3 if len(sg) == 1 else sg), order=case.get("order", 4),
            sigma=case["sigma"], bin_size=case["bin_size"], qcut=case["qcut"],
            ensemble=case.get("simulation") or "npt")
    return _CASE_ORACLE[name]


def check_against_reference_file(got, oracle_rows, ref_rows, rtol):
    """Rows (q, I) of the CUDA path against the reference's file, where the
    reference's own FP32 error can exceed `rtol`: the q text must be identical,
    and per bin the CUDA path may differ from the reference by no more than the
    FP64 oracle of the same method does, plus rtol.  Returns (max relative
    difference CUDA - reference, max relative difference oracle - reference)."""
    qs = [r[0] for r in ref_rows]
    assert [f"{q:10.5f}" for q, _ in got] == qs
    assert [f"{q:10.5f}" for q, _ in oracle_rows] == qs
    c = np.array([i for _, i in got])
    o = np.array([i for _, i in oracle_rows])
    r = np.array([float(x[1]) for x in ref_rows])
    dc = np.abs(c - r) / np.abs(r)
    do = np.abs(o - r) / np.abs(r)
    bad = np.nonzero(dc > do + rtol)[0]
    assert bad.size == 0, f"bins {bad}: cuda-ref {dc[bad]}, oracle-ref {do[bad]}"
    return float(dc.max()), float(do.max())
