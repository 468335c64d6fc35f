"""The drop-in ``pycusaxs_cuda.run`` end to end with a topology object (GPU)."""
import numpy as np
import pytest

from helpers import RTOL_PROFILE, oracle_hist
from oracle import saxs_oracle as O
from pycusaxs_b200 import core, pycusaxs_cuda
from pycusaxs_b200.synthetic import SyntheticTopology, cubic_system

pytestmark = pytest.mark.gpu


def _read_rows(path):
    rows = []
    for line in open(path):
        rows.append((line[:10], float(line[10:])))
    return rows


def test_run_writes_the_oracle_profile(cuda, tmp_path):
    s = cubic_system(6000, 40.0, seed=21, jitter=0.4, nframes=4)
    out = tmp_path / "saxs.dat"
    res = pycusaxs_cuda.run(SyntheticTopology(s), "top.tpr", "traj.xtc", [32], begin=0, end=3,
                            stride=1, output=str(out), order=4, scale_factor=2.0, bin_size=0.01,
                            qcut=0.7)
    assert res["grid"] == [32, 32, 32]
    assert res["scaled_grid"] == [0, 0, 0]
    assert "CuSAXS Configuration" in res["summary"]
    h, n, plan = oracle_hist(s, (32, 32, 32), [s.frame(k) for k in range(4)], sigma=2.0,
                             bin_size=0.01, qcut=0.7)
    want = O.profile_rows(h, n, plan.dq)
    got = _read_rows(out)
    assert [r[0] for r in got] == [f"{q:10.5f}" for q, _ in want]
    for (_, gi), (_, wi) in zip(got, want):
        # the file keeps 6 significant digits
        assert abs(gi - wi) <= max(RTOL_PROFILE, 6e-6) * abs(wi)


def test_stride_and_nvt(cuda, tmp_path):
    s = cubic_system(3000, 36.0, seed=22, jitter=0.4, nframes=7)
    out = tmp_path / "nvt.dat"
    pycusaxs_cuda.run(SyntheticTopology(s), "t", "x", [32, 32, 32], begin=1, end=6, stride=2,
                      output=str(out), scale_factor=2.0, qcut=0.7, simulation="nvt")
    frames = [s.frame(k) for k in (1, 3, 5)]
    h, n, plan = oracle_hist(s, (32, 32, 32), frames, sigma=2.0, qcut=0.7, ensemble="nvt")
    want = O.profile_rows(h, n, plan.dq)
    got = _read_rows(out)
    assert len(got) == len(want)
    for (_, gi), (_, wi) in zip(got, want):
        assert abs(gi - wi) <= max(RTOL_PROFILE, 6e-6) * abs(wi)


def test_python_error_in_iterator_is_swallowed_and_no_file(cuda, tmp_path, capsys):
    s = cubic_system(1000, 30.0, seed=23, nframes=5)
    out = tmp_path / "none.dat"
    res = pycusaxs_cuda.run(SyntheticTopology(s, fail_at_frame=2), "t", "x", [16], end=4,
                            output=str(out), scale_factor=2.0, qcut=0.8)
    assert "summary" in res
    assert not out.exists()
    assert "Python error while iterating frames" in capsys.readouterr().err


def test_malformed_frame_stops_iteration_and_writes_what_was_read(cuda, tmp_path, capsys):
    s = cubic_system(1000, 30.0, seed=24, nframes=4)

    class Broken(SyntheticTopology):
        def iter_frames_stream(self, start, stop, step=1, **kw):
            for k, fr in enumerate(super().iter_frames_stream(start, stop, step)):
                if k == 2:
                    fr = {"frame": 2}  # no positions
                yield fr

    out = tmp_path / "partial.dat"
    pycusaxs_cuda.run(Broken(s), "t", "x", [16], end=3, output=str(out), scale_factor=2.0, qcut=0.8)
    assert "Error loading frame data" in capsys.readouterr().err
    h, n, plan = oracle_hist(s, (16, 16, 16), [s.frame(0), s.frame(1)], sigma=2.0, qcut=0.8)
    assert len(_read_rows(out)) == len(O.profile_rows(h, n, plan.dq))


def test_unknown_element_raises(cuda, tmp_path):
    s = cubic_system(500, 30.0, seed=25)
    s.elements[:10] = "Xx"
    with pytest.raises(RuntimeError, match="Xx"):
        pycusaxs_cuda.run(SyntheticTopology(s), "t", "x", [16], output=str(tmp_path / "u.dat"),
                          scale_factor=2.0, qcut=0.8)


def test_core_invoke_returns_summary(cuda, tmp_path):
    s = cubic_system(2000, 30.0, seed=26, nframes=2)
    req = {"topology": "t.tpr", "trajectory": "x.xtc", "grid_size": [16], "initial_frame": 0,
           "last_frame": 1}
    adv = {"out": str(tmp_path / "c.dat"), "scale_factor": 2.0, "qcut": 0.8, "bin_size": 0.01}
    lines = core.invoke_cuda_backend(req, adv, SyntheticTopology(s))
    assert len(lines) == 1 and "CuSAXS Configuration" in lines[0]
    assert (tmp_path / "c.dat").exists()


def test_default_pybind_arguments_give_an_empty_profile(cuda, tmp_path):
    # qcut=0 (the pybind default) clamps the cut-off to 0: one bin, no rows
    s = cubic_system(500, 30.0, seed=27)
    out = tmp_path / "empty.dat"
    pycusaxs_cuda.run(SyntheticTopology(s), "t", "x", [16], output=str(out))
    assert out.read_text() == ""


def test_frames_beyond_one_batch_with_a_bad_frame_in_between(cuda, tmp_path, capsys):
    # 40 frames of 2000 atoms fill more than one 32-frame pinned batch; frame 5's
    # box is unusable, so it is reported and skipped (RunSaxs.cu:195-199) and
    # the profile is that of the other 39 frames
    s = cubic_system(2000, 30.0, seed=28, jitter=0.3, nframes=40)

    class OneBadBox(SyntheticTopology):
        def iter_frames_stream(self, start, stop, step=1, **kw):
            for fr in super().iter_frames_stream(start, stop, step):
                if fr["frame"] == 5:
                    fr = dict(fr, box=np.zeros((3, 3), np.float32))
                yield fr

    out = tmp_path / "skip.dat"
    pycusaxs_cuda.run(OneBadBox(s), "t", "x", [16], end=39, output=str(out), scale_factor=2.0,
                      qcut=0.8)
    assert "Error processing frame 5" in capsys.readouterr().err
    frames = [s.frame(k) for k in range(40) if k != 5]
    h, n, plan = oracle_hist(s, (16, 16, 16), frames, sigma=2.0, qcut=0.8)
    want = O.profile_rows(h, n, plan.dq)
    got = _read_rows(out)
    assert [r[0] for r in got] == [f"{q:10.5f}" for q, _ in want]
    for (_, gi), (_, wi) in zip(got, want):
        assert abs(gi - wi) <= max(RTOL_PROFILE, 6e-6) * abs(wi)
