"""Frame sharding + histogram all-reduce on two CPU ranks (gloo).

Each rank computes its shard's histogram with the oracle (the compute stand-in
on a host without a GPU), the ranks all-reduce, and the result must equal the
single-process histogram of all frames.  A second test makes one rank fail
before the collective and checks that the other ends with an error instead of
hanging (short process-group timeout).
"""
import datetime
import os
import socket
import sys
from pathlib import Path

import numpy as np
import pytest
import torch.multiprocessing as mp

REPO = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _system():
    from pycusaxs_b200.synthetic import cubic_system

    return cubic_system(1500, 30.0, seed=51, jitter=0.4, nframes=5)


def _plan(s):
    from oracle import saxs_oracle as O

    names = sorted({str(e) for e in s.elements})
    ff = O.load_form_factors()
    return O.OraclePlan(grid=(16, 16, 16), types=names, coeffs=np.stack([ff[n] for n in names]),
                        box0=s.box, sigma=2.0, qcut=0.8), names


def _worker(rank, world, port, outdir, fail_rank):
    sys.path.insert(0, str(REPO))
    import torch.distributed as dist

    from oracle import saxs_oracle as O
    from pycusaxs_b200 import distributed as D

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=10))
    try:
        s = _system()
        plan, names = _plan(s)
        mine = D.shard(D.frame_range(0, 4, 1), rank, world)
        if rank == fail_rank:
            raise RuntimeError("injected failure before the collective")
        h, n = O.run_frames(plan, [(s.frame(k), s.box) for k in mine], s.type_of_atom(names))
        h, n = D.allreduce_histogram(h, n)
        np.save(os.path.join(outdir, f"r{rank}.npy"), np.concatenate([h, n]))
    except Exception as exc:  # recorded for the parent, then the rank leaves
        Path(outdir, f"err{rank}.txt").write_text(f"{type(exc).__name__}: {exc}")
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def test_sharded_histogram_equals_single_process(tmp_path):
    from oracle import saxs_oracle as O

    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path), -1), nprocs=2,
                       start_method="spawn", join=True)
    s = _system()
    plan, names = _plan(s)
    h, n = O.run_frames(plan, [(s.frame(k), s.box) for k in range(5)], s.type_of_atom(names))
    for r in range(2):
        got = np.load(tmp_path / f"r{r}.npy")
        np.testing.assert_array_equal(got[len(h):], n)
        np.testing.assert_allclose(got[: len(h)], h, rtol=1e-12)


def test_failed_rank_surfaces_as_error_not_hang(tmp_path):
    mp.start_processes(_worker, args=(2, _free_port(), str(tmp_path), 1), nprocs=2,
                       start_method="spawn", join=True)
    assert "injected failure" in (tmp_path / "err1.txt").read_text()
    # rank 0 reached the all-reduce alone and must have ended with an error
    assert (tmp_path / "err0.txt").exists()
    assert not (tmp_path / "r0.npy").exists()


def _nvt_worker(rank, world, port, outdir):
    sys.path.insert(0, str(REPO))
    import torch.distributed as dist

    from oracle import saxs_oracle as O
    from pycusaxs_b200 import distributed as D

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=10))
    try:
        s = _system()
        plan, names = _plan(s)
        plan.ensemble = "nvt"
        toa = s.type_of_atom(names)
        mine = D.shard(D.frame_range(0, 4, 1), rank, world)   # 3 and 2 frames: uneven shares
        # (1) each rank bins its own intensity sum, as its plan does, and the
        # binned histograms are combined
        h, n = O.run_frames(plan, [(s.frame(k), s.box) for k in mine], toa)
        h, n = D.combine_histogram(h, n, len(mine), "nvt")
        # (2) the raw intensity sums are reduced and binned once
        total = sum(O.frame_intensity(plan, s.frame(k), toa, s.box)[0] for k in mine)
        total, frames = D.reduce_intensity(total, len(mine))
        _, bins0 = O.kpoint_bins(plan.nn, plan.scaled_oc(plan.oc0), plan.dq, plan.kcut,
                                 plan.num_bins, plan.contraction)
        h2, n2 = O.histogram(total, bins0, plan.num_bins, 1.0 / frames)
        np.save(os.path.join(outdir, f"nvt{rank}.npy"), np.stack([h, n, h2, n2]))
    except Exception as exc:
        Path(outdir, f"err{rank}.txt").write_text(f"{type(exc).__name__}: {exc}")
    finally:
        try:
            dist.destroy_process_group()
        except Exception:
            pass


def test_sharded_nvt_equals_single_process(tmp_path):
    from oracle import saxs_oracle as O

    mp.start_processes(_nvt_worker, args=(2, _free_port(), str(tmp_path)), nprocs=2,
                       start_method="spawn", join=True)
    assert not list(tmp_path.glob("err*.txt")), [p.read_text() for p in tmp_path.glob("err*.txt")]
    s = _system()
    plan, names = _plan(s)
    plan.ensemble = "nvt"
    h, n = O.run_frames(plan, [(s.frame(k), s.box) for k in range(5)], s.type_of_atom(names))
    for r in range(2):
        hb, nb, hr, nr = np.load(tmp_path / f"nvt{r}.npy")
        np.testing.assert_array_equal(nb, n)
        np.testing.assert_allclose(hb, h, rtol=1e-12)
        np.testing.assert_array_equal(nr, n)
        np.testing.assert_allclose(hr, h, rtol=1e-12)


def test_shard_is_a_partition():
    from pycusaxs_b200 import distributed as D

    frames = D.frame_range(3, 17, 2)
    parts = [D.shard(frames, r, 3) for r in range(3)]
    assert sorted(sum(parts, [])) == list(frames)
    with pytest.raises(ValueError):
        D.shard(frames, 3, 3)
