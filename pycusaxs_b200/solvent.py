"""Bulk-solvent padding densities (the "given" padding mode).

The reference carries an AtomCounter (cpp-src/System/AtomCounter.cpp:17-104)
that turns a water model's mass density, the cell volume and the added ions
into atoms per grid point, but its padding is always the z-border average
(Options.cpp:13 ``myPadding = padding::avg``).  ``given_padding`` computes those
per-grid-point counts so a run can pad the supercell with the bulk solvent's
density instead (``SaxsEngine(..., padding="given")``); it is an opt-in physics
extension, not reference parity.
"""
from __future__ import annotations

import numpy as np

AVOGADRO = 6.022e23
WATER_MOLAR_MASS = 18.015  # g/mol
# mass densities (g/cm^3) of the water models AtomCounter knows
WATER_MODELS = {"SPCE": 0.998, "SPC": 0.998, "TIP3P": 0.982, "TIP4P": 0.999}


def water_molecules(volume_a3: float, model: str) -> float:
    """Water molecules filling `volume_a3` (A^3) at the model's density (SPC/E for
    an unknown model)."""
    rho = WATER_MODELS.get(model.upper().replace("/", ""), WATER_MODELS["SPCE"])
    return rho * volume_a3 * 1e-24 / WATER_MOLAR_MASS * AVOGADRO


def given_padding(type_names, box, grid, water_model: str = "SPCE", ions: dict | None = None):
    """Atoms per grid point of each type in bulk solvent filling the cell: O = waters,
    H = 2 x waters, each ion = its count, divided by nx*ny*nz; 0 for other types."""
    box = np.asarray(box, dtype=np.float64).reshape(3, 3)
    volume = abs(float(np.linalg.det(box)))
    g = tuple(int(v) for v in (grid if len(grid) == 3 else [grid[0]] * 3))
    points = g[0] * g[1] * g[2]
    wm = water_molecules(volume, water_model)
    counts = {"O": wm, "H": 2.0 * wm}
    for k, v in (ions or {}).items():
        counts[k] = counts.get(k, 0.0) + float(v)
    return np.array([counts.get(t, 0.0) / points for t in type_names], dtype=np.float32)
