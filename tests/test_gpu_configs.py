"""The benchmarked workloads at their own sizes, against the FP64 oracle and the reference (GPU).

Cases (tests/golden/make_golden.py ``LARGE_CASES``, profiles written by the
reference cudaSAXS itself into tests/golden/ref_profiles_large.json):

* the bench workload: 100k atoms in a 12 nm box, grid 128 -> 256^3, 100 frames
  with 0.05 nm jitter (and its first 4 frames);
* the refinement workload: 50k atoms in a 10 nm box, grid 128 -> 256^3;
* the large triclinic slab: 1M atoms, 25 x 25 x 20 nm with gamma = 80 deg, a
  1.5x dense slab, grid 256 -> 512^3 (1 and 20 frames).

Every case runs through the default batched path (tensor-core spreading and
y and x passes, up to 20 frames per launch, frames from host memory) and must
match the FP64 oracle over all its frames: identical bin counts and
RTOL_PROFILE (1e-4) per bin.  Against the reference's own file the q text must
be identical, and per bin the CUDA path may differ from the reference only as
much as the FP64 oracle of the same method does (plus GOLDEN_RTOL): at these
sizes the reference's FP32 transforms are themselves up to ~2e-3 (100k atoms,
256^3) and ~6e-3 (1M atoms, 512^3) off the FP64 result in the lowest q bins,
where the padded supercell's large k = 0 term leaks into its neighbours.
Setting PYCUSAXS_ERROR_LOG to a file path appends each measured error as a JSON
line (the per-config error table is built from it).
"""
import json
import os

import numpy as np
import pytest

from golden.make_golden import LARGE_CASES, LARGE_OUT, build_system
from helpers import RTOL_PROFILE, assert_profiles_close, check_against_reference_file, oracle_case
from test_golden import GOLDEN_RTOL
from oracle import saxs_oracle as O
from pycusaxs_b200 import SaxsEngine

pytestmark = pytest.mark.gpu


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
    assert eng.info.path & 7 == 7, f"tensor-core path not taken (path bits {eng.info.path})"
    frames = s.frames(0, nf)
    eng.forward_host(frames, np.stack([s.box] * nf))
    h, n = eng.histogram()
    counters = eng.counters()
    rows = eng.profile()
    info = eng.info
    eng.close()
    return h, n, rows, counters, info


@pytest.mark.parametrize("name", sorted(LARGE_CASES))
def test_batched_path_matches_oracle_and_reference(cuda, name):
    c = LARGE_CASES[name]
    assert _golden()[name]["params"] == c
    s = build_system(c)
    h, n, rows, counters, info = _run_batched(c, s)
    assert counters["status"] == 0
    if name.startswith("c3_"):
        # the dense slab puts more atoms near one 128-column tile than its atom
        # table holds: the table-chunking path of the spreading kernel ran
        assert counters["table_chunks"] >= 2, counters
    ho, no, plan = oracle_case(name, c, s)
    assert info.num_bins == plan.num_bins
    err = assert_profiles_close(h, n, ho, no, rtol=RTOL_PROFILE)
    orows = O.profile_rows(ho, no, plan.dq)
    dc, do = check_against_reference_file(rows, orows, _golden()[name]["rows"], GOLDEN_RTOL)
    _log(case=name, cuda_vs_oracle=err, cuda_vs_reference=dc, reference_vs_oracle=do, rows=len(rows),
         kbox=list(info.kbox), path=info.path, table_chunks=counters["table_chunks"])
