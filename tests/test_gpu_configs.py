"""The benchmarked workloads at their own sizes, against the reference and the FP64 oracle (GPU).

Cases (tests/golden/make_golden.py ``LARGE_CASES``, profiles written by the
reference cudaSAXS itself into tests/golden/ref_profiles_large.json):

* the bench workload: 100k atoms in a 12 nm box, grid 128 -> 256^3, 100 frames
  with 0.05 nm jitter (and its first 4 frames);
* the refinement workload: 50k atoms in a 10 nm box, grid 128 -> 256^3;
* the large triclinic slab: 1M atoms, 25 x 25 x 20 nm with gamma = 80 deg, a
  1.5x dense slab, grid 256 -> 512^3 (1 and 20 frames).

Every case runs through the default batched path (wide-tile tensor-core
spreading, tensor-core y and x passes, up to 20 frames per launch, frames from
host memory) and must reproduce the reference's file: identical q text and
intensities within GOLDEN_RTOL.  The cases the FP64 oracle can replay on the
host in seconds are also compared with it: identical bin counts and
RTOL_PROFILE per bin.  Setting PYCUSAXS_ERROR_LOG to a file path appends each
measured error as a JSON line (the per-config error table is built from it).
"""
import json
import os

import numpy as np
import pytest

from golden.make_golden import LARGE_CASES, LARGE_OUT, build_system
from helpers import RTOL_PROFILE, assert_profiles_close, oracle_hist
from test_golden import GOLDEN_RTOL
from pycusaxs_b200 import SaxsEngine

pytestmark = pytest.mark.gpu

ORACLE_CASES = ["c2_100k_grid128_4f", "c5_50k_grid128", "c3_1m_grid256_1f"]


def _golden():
    return json.loads(LARGE_OUT.read_text())


def _log(**kw):
    path = os.environ.get("PYCUSAXS_ERROR_LOG")
    if path:
        with open(path, "a") as fh:
            fh.write(json.dumps(kw) + "\n")


def _grid(c):
    g = c["grid"]
    return tuple(g * 3 if len(g) == 1 else g)


def _run_batched(c, s):
    """The case's frames from host memory through the default batched path."""
    nf = c["frames"]
    eng = SaxsEngine(_grid(c), s.atom_index(), s.natoms, s.box, scale_factor=c["sigma"],
                     bin_size=c["bin_size"], qcut=c["qcut"], max_frames=min(nf, 20))
    assert eng.info.path & 15 == 15, f"default path not taken (path bits {eng.info.path})"
    frames = s.frames(0, nf)
    eng.forward_host(frames, np.stack([s.box] * nf))
    h, n = eng.histogram()
    counters = eng.counters()
    rows = eng.profile()
    info = eng.info
    eng.close()
    return h, n, rows, counters, info


def _rows_vs_golden(rows, name):
    ref = _golden()[name]["rows"]
    assert [f"{q:10.5f}" for q, _ in rows] == [r[0] for r in ref]
    got = np.array([i for _, i in rows])
    want = np.array([float(r[1]) for r in ref])
    err = np.abs(got - want) / np.abs(want)
    assert err.max() <= GOLDEN_RTOL, (name, err.max())
    return float(err.max())


@pytest.mark.parametrize("name", sorted(LARGE_CASES))
def test_batched_path_matches_reference_file(cuda, name):
    c = LARGE_CASES[name]
    assert _golden()[name]["params"] == c
    s = build_system(c)
    h, n, rows, counters, info = _run_batched(c, s)
    assert counters["status"] == 0
    if name.startswith("c3_"):
        # the dense slab puts more atoms near one wide tile than its atom table
        # holds: the table-chunking path of the spreading kernel ran
        assert counters["table_chunks"] >= 2, counters
    err = _rows_vs_golden(rows, name)
    _log(case=name, comparison="cuda vs reference file", max_rel_err=err, rows=len(rows),
         kbox=list(info.kbox), table_chunks=counters["table_chunks"])


@pytest.mark.parametrize("name", ORACLE_CASES)
def test_batched_path_matches_fp64_oracle(cuda, name):
    c = LARGE_CASES[name]
    s = build_system(c)
    frames = [s.frame(k) for k in range(c["frames"])]
    ho, no, plan = oracle_hist(s, _grid(c), frames, sigma=c["sigma"], bin_size=c["bin_size"],
                               qcut=c["qcut"])
    h, n, rows, counters, info = _run_batched(c, s)
    assert info.num_bins == plan.num_bins
    err = assert_profiles_close(h, n, ho, no, rtol=RTOL_PROFILE)
    _log(case=name, comparison="cuda vs fp64 oracle", max_rel_err=err)
    # the oracle reproduces the reference's file at this size too
    from oracle import saxs_oracle as O

    orows = O.profile_rows(ho, no, plan.dq)
    ref = _golden()[name]["rows"]
    assert [f"{q:10.5f}" for q, _ in orows] == [r[0] for r in ref]
    oi = np.array([i for _, i in orows])
    ri = np.array([float(r[1]) for r in ref])
    oerr = np.abs(oi - ri) / np.abs(ri)
    assert oerr.max() <= GOLDEN_RTOL, oerr
    _log(case=name, comparison="reference file vs fp64 oracle", max_rel_err=float(oerr.max()))
