"""Atomic form-factor coefficients (International Tables 1992, 4 Gaussians + c).

The table is the reference's ``it1992`` map (cpp-src/Utilities/Scattering.cpp:9-189),
extracted verbatim into ``data/it1992.json`` by ``data/extract_form_factors.py``.
Each row is (a1, a2, a3, a4, b1, b2, b3, b4, c) as float32, the layout
``opsfact`` reads (Saxs/opsfact.cu:30-35).
"""
from __future__ import annotations

import json
from functools import lru_cache
from pathlib import Path

import numpy as np

TABLE = Path(__file__).resolve().parent / "data" / "it1992.json"


@lru_cache(maxsize=1)
def table() -> dict:
    raw = json.loads(TABLE.read_text())
    return {k: np.array([float(v) for v in vals], dtype=np.float32) for k, vals in raw.items()}


def form_factor_rows(names, extra: dict | None = None) -> np.ndarray:
    """(T, 9) float32 rows for element names.

    Unknown elements raise ``KeyError``: the reference silently looks them up
    as an empty coefficient vector (Scattering.h:13-24, std::map::operator[])
    and then reads past it on the device.
    """
    tab = table()
    rows = []
    for n in names:
        if extra and n in extra:
            rows.append(np.asarray(extra[n], dtype=np.float32).reshape(9))
        elif n in tab:
            rows.append(tab[n])
        else:
            raise KeyError(f"no form-factor coefficients for element {n!r}")
    return np.stack(rows) if rows else np.zeros((0, 9), np.float32)
