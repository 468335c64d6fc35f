"""The drop-in run() against the reference's own output files (GPU).

Same seeded inputs as tests/golden/make_golden.py fed to the reference
cudaSAXS (small and large cases); the profile files must agree row by row: identical q text and
intensities within GOLDEN_RTOL (the reference's FP32 noise and 6 printed
significant digits on both sides).
"""
import json

import numpy as np
import pytest

from golden.make_golden import ALL_CASES, CASES, LARGE_OUT, build_system
from helpers import check_against_reference_file, oracle_case
from test_golden import GOLDEN_RTOL, golden
from oracle import saxs_oracle as O
from pycusaxs_b200 import pycusaxs_cuda
from pycusaxs_b200.synthetic import SyntheticTopology

pytestmark = pytest.mark.gpu


def _golden_rows(name):
    if name in CASES:
        return golden()[name]["rows"]
    return json.loads(LARGE_OUT.read_text())[name]["rows"]


@pytest.mark.parametrize("name", sorted(ALL_CASES))
def test_dropin_file_matches_reference_file(cuda, tmp_path, name):
    c = ALL_CASES[name]
    out = tmp_path / f"{name}.dat"
    pycusaxs_cuda.run(SyntheticTopology(build_system(c)), "synthetic.tpr", "synthetic.xtc",
                      c["grid"], scaled_grid=c.get("scaled", []), begin=0, end=c["frames"] - 1,
                      stride=1, output=str(out), order=c.get("order", 4), scale_factor=c["sigma"],
                      bin_size=c["bin_size"], qcut=c["qcut"], simulation=c.get("simulation", ""))
    got = [(line[:10], float(line[10:])) for line in open(out)]
    ref = _golden_rows(name)
    if name not in CASES:
        # the large cases: within the reference's own FP32 error of it (see
        # tests/test_gpu_configs.py), judged by the FP64 oracle
        s = build_system(c)
        ho, no, plan = oracle_case(name, c, s)
        check_against_reference_file([(float(q), i) for q, i in got], O.profile_rows(ho, no, plan.dq), ref,
                                     GOLDEN_RTOL)
        return
    assert [g[0] for g in got] == [r[0] for r in ref]
    gi = np.array([g[1] for g in got])
    ri = np.array([float(r[1]) for r in ref])
    err = np.abs(gi - ri) / np.abs(ri)
    assert err.max() <= GOLDEN_RTOL, err
