"""Golden I(q) profiles from the reference cudaSAXS itself.

Runs the reference's own pybind module, built from its sources by
``oracle/build_ref.sh`` into ``oracle/_ref/``, on seeded synthetic systems
(``pycusaxs_b200.synthetic``) through its public ``pycusaxs_cuda.run`` with a
duck-typed topology, one fresh process per case (the reference keeps run
state in process-wide statics).  Needs a CUDA GPU.  The inputs are not stored:
they are regenerated from the seeds, which numpy's PCG64 keeps stable.

    python tests/golden/make_golden.py [--out tests/golden/ref_profiles.json]
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
from pathlib import Path

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
sys.path.insert(0, str(REPO))

CASES = {
    "cubic32_npt2": dict(kind="cubic", natoms=4000, box=40.0, seed=31, jitter=0.4, frames=2,
                         grid=[32], sigma=2.0, qcut=0.6, bin_size=0.0),
    "c1_20k_grid64": dict(kind="cubic", natoms=20000, box=60.0, seed=0, jitter=0.0, frames=1,
                          grid=[64], sigma=2.0, qcut=0.5, bin_size=0.002),
    "ortho_2p5": dict(kind="ortho", natoms=3000, lengths=[30.0, 40.0, 50.0], seed=2, frames=1,
                      grid=[24, 32, 40], sigma=2.5, qcut=0.9, bin_size=0.0),
    "triclinic_slab": dict(kind="triclinic", natoms=5000, abc=[40.0, 40.0, 32.0], gamma=80.0,
                           seed=4, frames=1, grid=[32], sigma=2.0, qcut=0.7, bin_size=0.0),
    "nvt3": dict(kind="cubic", natoms=3000, box=36.0, seed=8, jitter=0.5, frames=3, grid=[32],
                 sigma=2.0, qcut=0.7, bin_size=0.0, simulation="nvt"),
    "order2": dict(kind="cubic", natoms=2000, box=30.0, seed=6, frames=1, grid=[24], sigma=2.0,
                   qcut=0.8, bin_size=0.0, order=2),
    "scaled_unit_sigma": dict(kind="cubic", natoms=1500, box=24.0, seed=10, frames=1, grid=[16],
                              scaled=[32], sigma=1.0, qcut=5.0, bin_size=0.0),
}


def build_system(c):
    from pycusaxs_b200 import synthetic as S

    if c["kind"] == "cubic":
        return S.cubic_system(c["natoms"], c["box"], seed=c["seed"], jitter=c.get("jitter", 0.0),
                              nframes=c["frames"])
    if c["kind"] == "ortho":
        return S.orthorhombic_system(c["natoms"], c["lengths"], seed=c["seed"],
                                     jitter=c.get("jitter", 0.0), nframes=c["frames"])
    a, b, cc = c["abc"]
    return S.triclinic_slab_system(c["natoms"], a, b, cc, c["gamma"], seed=c["seed"],
                                   jitter=c.get("jitter", 0.0), nframes=c["frames"])


def run_case(name: str, out: str) -> None:
    c = CASES[name]
    sys.path.insert(0, str(REPO / "oracle" / "_ref"))
    import pycusaxs_cuda  # the reference build

    from pycusaxs_b200.synthetic import SyntheticTopology

    s = build_system(c)
    pycusaxs_cuda.run(SyntheticTopology(s), "synthetic.tpr", "synthetic.xtc", c["grid"],
                      scaled_grid=c.get("scaled", []), begin=0, end=c["frames"] - 1, stride=1,
                      output=out, order=c.get("order", 4), scale_factor=c["sigma"],
                      bin_size=c["bin_size"], qcut=c["qcut"], simulation=c.get("simulation", ""))


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(HERE / "ref_profiles.json"))
    ap.add_argument("--case")
    ap.add_argument("--case-out")
    args = ap.parse_args(argv)
    if args.case:
        run_case(args.case, args.case_out)
        return 0
    result = {}
    with tempfile.TemporaryDirectory() as td:
        for name, c in CASES.items():
            path = os.path.join(td, name + ".dat")
            subprocess.run([sys.executable, __file__, "--case", name, "--case-out", path],
                           check=True, stdout=subprocess.DEVNULL)
            rows = [[line[:10], line[10:].strip()] for line in open(path)]
            result[name] = {"params": c, "rows": rows}
            print(f"{name}: {len(rows)} rows")
    Path(args.out).parent.mkdir(parents=True, exist_ok=True)
    Path(args.out).write_text(json.dumps(result, indent=1) + "\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
