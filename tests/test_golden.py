"""The oracle against golden profiles written by the reference cudaSAXS itself (CPU).

``tests/golden/ref_profiles.json`` holds the I(q) files the reference's own
pycusaxs_cuda.run (built from its sources by oracle/build_ref.sh) wrote for
seeded synthetic systems; ``tests/golden/make_golden.py`` regenerates it on a
GPU host.  The oracle must reproduce every q column exactly (same text) and
every intensity within GOLDEN_RTOL: the reference computes in FP32 (its
padding-mean cancellation is worst in the first bin) and prints 6 digits.
"""
import json
from pathlib import Path

import numpy as np
import pytest

from golden.make_golden import CASES, build_system
from helpers import oracle_hist
from oracle import saxs_oracle as O

GOLDEN = Path(__file__).resolve().parent / "golden" / "ref_profiles.json"
GOLDEN_RTOL = 1e-4


def _expand(v):
    return tuple(v * 3 if len(v) == 1 else v)


def oracle_rows(c):
    s = build_system(c)
    h, n, plan = oracle_hist(s, _expand(c["grid"]), [s.frame(k) for k in range(c["frames"])],
                             scaled_grid=_expand(c.get("scaled", [0, 0, 0])),
                             order=c.get("order", 4), sigma=c["sigma"], bin_size=c["bin_size"],
                             qcut=c["qcut"], ensemble=c.get("simulation") or "npt")
    return O.profile_rows(h, n, plan.dq)


def golden():
    return json.loads(GOLDEN.read_text())


@pytest.mark.parametrize("name", sorted(CASES))
def test_oracle_reproduces_reference_profile(name):
    g = golden()[name]
    assert g["params"] == CASES[name]
    rows = oracle_rows(CASES[name])
    assert [f"{q:10.5f}" for q, _ in rows] == [r[0] for r in g["rows"]]
    ref = np.array([float(r[1]) for r in g["rows"]])
    ora = np.array([i for _, i in rows])
    err = np.abs(ora - ref) / np.abs(ref)
    assert err.max() <= GOLDEN_RTOL, err
