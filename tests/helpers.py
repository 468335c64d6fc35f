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
