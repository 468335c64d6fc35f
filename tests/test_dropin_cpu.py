"""The drop-in's argument validation, summary text and core wrappers (CPU only).

Messages, exception types and their order follow the reference's pybind layer
(cpp-src/pybind/cuda_bindings.cpp:33-122) and run_cuda_saxs
(cpp-src/cudaSAXS.cu:50-65).
"""
import pytest

from pycusaxs_b200 import core, pycusaxs_cuda


def call(**kw):
    args = dict(obj_topology=None, topology="t.tpr", trajectory="x.xtc", grid=[32])
    args.update(kw)
    return pycusaxs_cuda.run(**args)


@pytest.mark.parametrize("kw,msg", [
    (dict(grid=[]), "Grid must have at least one dimension"),
    (dict(grid=[0]), "Grid dimension must be positive"),
    (dict(grid=[16, -1, 16]), "Grid dimensions must be positive"),
    (dict(grid=[16, 16]), "Grid must have either 1 or 3 dimensions (nx, ny, nz)"),
    (dict(scaled_grid=[0]), "Scaled grid dimension must be positive"),
    (dict(scaled_grid=[32, 0, 32]), "Scaled grid dimensions must be positive"),
    (dict(scaled_grid=[32, 32]), "Scaled grid must have either 1 or 3 dimensions"),
    (dict(stride=0), "Stride must be positive"),
    (dict(order=0), "Spline order must be between 1 and 8"),
    (dict(order=9), "Spline order must be between 1 and 8"),
    (dict(bin_size=-0.1), "Bin size must be non-negative"),
    (dict(qcut=-1.0), "Q cutoff must be non-negative"),
    (dict(scale_factor=-1.0), "Scale factor must be non-negative"),
    (dict(scale_factor=0.0), "Scale factor must be positive when scaled grid is not provided"),
    (dict(begin=-1), "Frame indices must be non-negative"),
    (dict(begin=3, end=2), "Begin frame must be less than or equal to end frame"),
    (dict(topology=""), "Topology path must not be empty."),
    (dict(trajectory=""), "Trajectory path must not be empty."),
])
def test_validation_messages(kw, msg):
    with pytest.raises(ValueError) as e:
        call(**kw)
    assert str(e.value) == msg


def test_validation_order_grid_before_stride():
    with pytest.raises(ValueError, match="Grid dimension must be positive"):
        call(grid=[0], stride=0)


def test_scaled_grid_allows_zero_scale_factor_in_validation():
    # with an explicit scaled grid a zero scale factor passes validation; the run then
    # needs a GPU, which the backend reports as an error (no CPU fallback)
    with pytest.raises(Exception) as e:
        call(scaled_grid=[64], scale_factor=0.0, obj_topology=_NoTopology())
    assert not isinstance(e.value, ValueError)


class _NoTopology:
    def get_atom_index(self):
        return {"C": [0]}

    def read_frame(self, i):
        return i

    def get_box(self):
        return [[10.0, 0, 0], [0, 10.0, 0], [0, 0, 10.0]]

    def iter_frames_stream(self, *a, **k):
        return iter(())


def test_summary_banner_layout():
    s = pycusaxs_cuda.build_summary("a.tpr", "b.xtc", [64, 64, 64], [], 0, 9, 2, 4, 2.0, 0.002,
                                    0.5, "", {"Na": 3, "Cl": 0})
    lines = s.split("\n")
    assert lines[1] == "╔" + "═" * 64 + "╗"
    assert lines[2] == "║" + " " * 18 + "CuSAXS Configuration" + " " * 25 + "║"
    assert "  Topology      : a.tpr" in s
    assert "  Total Frames  : 5" in s                 # (9 - 0) // 2 + 1
    assert "  Grid Size     : (64, 64, 64)" in s
    assert "  Scale Factor  : 2.000" in s
    assert "  Bin Size      : 0.0020" in s
    assert "  Q-cutoff      : 0.500" in s
    assert "  Na⁺ atoms     : 3" in s and "Cl⁻" not in s
    assert "  Padding Mode  : average" in s
    assert s.endswith("\n" + "-" * 66 + "\n")
    assert "\x1b[1mInput Files\x1b[0m" in s           # fmt::emphasis::bold


def test_summary_with_scaled_grid_and_water_model():
    s = pycusaxs_cuda.build_summary("a", "b", [32, 32, 32], [64, 64, 64], 0, 0, 1, 4, 1.0, 0.0,
                                    0.0, "tip3p", {"Na": 0, "Cl": 2})
    assert "  Primary Grid  : (32, 32, 32)" in s
    assert "  Scaled Grid   : (64, 64, 64)" in s
    assert "  Water Model   : tip3p" in s
    assert "  Cl⁻ atoms     : 2" in s


def test_core_returns_backend_error_string_instead_of_raising():
    req = {"topology": "t", "trajectory": "x", "grid_size": [16], "initial_frame": 0,
           "last_frame": 0}
    lines = core.invoke_cuda_backend(req, {"order": 9}, topology=None)
    assert lines == ["cuda backend error: Spline order must be between 1 and 8"]


def test_run_saxs_calculation_validates_paths(tmp_path):
    req = {"topology": str(tmp_path / "missing.tpr"), "trajectory": str(tmp_path / "x.xtc"),
           "grid_size": [16], "initial_frame": 0, "last_frame": 0}
    with pytest.raises(FileNotFoundError):
        core.run_saxs_calculation(req, {})
    (tmp_path / "missing.tpr").write_text("")
    (tmp_path / "x.xtc").write_text("")
    req["initial_frame"], req["last_frame"] = 2, 1
    with pytest.raises(ValueError, match="must be >= initial frame"):
        core.run_saxs_calculation(req, {})


def test_run_saxs_calculation_checks_frames_against_topology(tmp_path):
    (tmp_path / "t.tpr").write_text("")
    (tmp_path / "x.xtc").write_text("")

    class Topo:
        n_frames = 3

    req = {"topology": str(tmp_path / "t.tpr"), "trajectory": str(tmp_path / "x.xtc"),
           "grid_size": [16], "initial_frame": 0, "last_frame": 5}
    with pytest.raises(ValueError, match="Last frame 5 exceeds available frames"):
        core.run_saxs_calculation(req, {}, topology_factory=lambda a, b: Topo())


def test_batch_size_of_run():
    # up to 32 frames, at most 64 MB of positions, at most the frames requested
    assert pycusaxs_cuda._batch_frames(100_000, 100) == 32
    assert pycusaxs_cuda._batch_frames(1_000_000, 20) == 5
    assert pycusaxs_cuda._batch_frames(100_000, 3) == 3
    assert pycusaxs_cuda._batch_frames(50_000_000, 10) == 1


def test_frame_checks_before_batching():
    import numpy as np

    pos = np.zeros((10, 3), np.float32)
    box = np.diag([30.0, 30.0, 30.0]).astype(np.float32)
    assert pycusaxs_cuda._frame_problem(pos, box, 10) == ""
    assert "indexes 11" in pycusaxs_cuda._frame_problem(pos, box, 11)
    assert "positive" in pycusaxs_cuda._frame_problem(pos, np.zeros((3, 3), np.float32), 10)
    bad = box.copy()
    bad[0, 1] = np.nan
    assert "non-finite" in pycusaxs_cuda._frame_problem(pos, bad, 10)
