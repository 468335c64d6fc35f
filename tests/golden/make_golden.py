"""Golden I(q) profiles from the reference cudaSAXS itself.

Runs the reference's own pybind module, built from its sources by
``oracle/build_ref.sh`` into ``oracle/_ref/``, on seeded synthetic systems
(``pycusaxs_b200.synthetic``) through its public ``pycusaxs_cuda.run`` with a
duck-typed topology, one fresh process per case (the reference keeps run
state in process-wide statics).  Needs a CUDA GPU.  The inputs are not stored:
they are regenerated from the seeds, which numpy's PCG64 keeps stable.

``CASES`` (small; the CPU suite replays them through the FP64 oracle) go to
``ref_profiles.json``; ``LARGE_CASES`` - the benchmarked workloads at their
own sizes: 100k atoms on a 256^3 supercell, 50k atoms on 256^3, and the
1M-atom triclinic slab on 512^3 - go to ``ref_profiles_large.json`` and are
checked by the GPU suite (tests/test_gpu_configs.py).

    python tests/golden/make_golden.py [--large] [--only NAME,...]
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


LARGE_CASES = {
    # the bench workload: 100k atoms, 12 nm box, grid 128 -> 256^3, 100 jittered frames
    "c2_100k_grid128_100f": dict(kind="cubic", natoms=100_000, box=120.0, seed=1000, jitter=0.5,
                                 frames=100, grid=[128], sigma=2.0, qcut=0.5, bin_size=0.002),
    # its first 4 frames (replayed by the FP64 oracle)
    "c2_100k_grid128_4f": dict(kind="cubic", natoms=100_000, box=120.0, seed=1000, jitter=0.5,
                               frames=4, grid=[128], sigma=2.0, qcut=0.5, bin_size=0.002),
    # the refinement workload: 50k atoms, 10 nm box, grid 128 -> 256^3
    "c5_50k_grid128": dict(kind="cubic", natoms=50_000, box=100.0, seed=77, frames=1, grid=[128],
                           sigma=2.0, qcut=0.5, bin_size=0.002),
    # 1M atoms, 25 x 25 x 20 nm cell with gamma = 80 deg, 1.5x dense slab, grid 256 -> 512^3
    "c3_1m_grid256_1f": dict(kind="triclinic", natoms=1_000_000, abc=[250.0, 250.0, 200.0],
                             gamma=80.0, seed=0, jitter=0.5, frames=1, grid=[256], sigma=2.0,
                             qcut=0.4, bin_size=0.001),
    "c3_1m_grid256_20f": dict(kind="triclinic", natoms=1_000_000, abc=[250.0, 250.0, 200.0],
                              gamma=80.0, seed=0, jitter=0.5, frames=20, grid=[256], sigma=2.0,
                              qcut=0.4, bin_size=0.001),
}
ALL_CASES = {**CASES, **LARGE_CASES}
LARGE_OUT = HERE / "ref_profiles_large.json"


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
    c = ALL_CASES[name]
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
    ap.add_argument("--out")
    ap.add_argument("--large", action="store_true", help="the LARGE_CASES (ref_profiles_large.json)")
    ap.add_argument("--only", help="comma-separated case names; the file's other cases are kept")
    ap.add_argument("--case")
    ap.add_argument("--case-out")
    args = ap.parse_args(argv)
    if args.case:
        run_case(args.case, args.case_out)
        return 0
    cases = LARGE_CASES if args.large else CASES
    out = Path(args.out) if args.out else (LARGE_OUT if args.large else HERE / "ref_profiles.json")
    names = args.only.split(",") if args.only else list(cases)
    result = json.loads(out.read_text()) if (args.only and out.exists()) else {}
    with tempfile.TemporaryDirectory() as td:
        for name in names:
            c = cases[name]
            path = os.path.join(td, name + ".dat")
            subprocess.run([sys.executable, __file__, "--case", name, "--case-out", path],
                           check=True, stdout=subprocess.DEVNULL)
            rows = [[line[:10], line[10:].strip()] for line in open(path)]
            result[name] = {"params": c, "rows": rows}
            print(f"{name}: {len(rows)} rows")
    result = {k: result[k] for k in cases if k in result}
    out.parent.mkdir(parents=True, exist_ok=True)
    out.write_text(json.dumps(result, indent=1) + "\n")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
