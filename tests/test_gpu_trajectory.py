"""Frames read from files without MDAnalysis, through the SAXS path (GPU).

A TRR trajectory + GRO topology written from a seeded system: the pinned
read-ahead pipeline (SaxsEngine.run_trajectory) must give the same histogram as
the device path on the frames as read back (to 1e-6: the order of the float
atomics of the spreading differs from run to run at the 1e-8 level), and the
drop-in run() fed by a FileTopology the same profile as run() fed by those
frames from memory.
"""
import numpy as np
import pytest
import torch

from pycusaxs_b200 import SaxsEngine, pycusaxs_cuda
from pycusaxs_b200.synthetic import cubic_system
from pycusaxs_b200.trajectory import FileTopology, NativeTrajectory
from trajfiles import write_gro, write_trr

pytestmark = pytest.mark.gpu


def _files(tmp_path, s, nframes):
    frames_nm = np.stack([s.frame(k) for k in range(nframes)]).astype(np.float64) / 10.0
    boxes_nm = np.stack([s.box.astype(np.float64) / 10.0] * nframes)
    names = [str(e) for e in s.elements]
    write_gro(tmp_path / "s.gro", names, ["MOL"] * len(names), frames_nm[:1], boxes_nm[:1])
    write_trr(tmp_path / "s.trr", frames_nm, boxes_nm, [float(k) for k in range(nframes)])
    return tmp_path / "s.gro", tmp_path / "s.trr"


class _Frames:
    """Topology duck type over frames already in memory."""

    def __init__(self, elements, frames, boxes):
        self.elements, self.frames, self.boxes = elements, frames, boxes
        self.n_frames = len(frames)

    def get_atom_index(self):
        out = {}
        for i, e in enumerate(self.elements):
            out.setdefault(e, []).append(i)
        return out

    def read_frame(self, k):
        self.k = k

    def get_box(self):
        return self.boxes[self.k]

    def iter_frames_stream(self, start, stop, step=1, **_):
        for k in range(start, min(stop, self.n_frames), step):
            yield {"frame": k, "time": float(k), "positions": self.frames[k], "box": self.boxes[k]}


def test_run_trajectory_matches_device_path(cuda, tmp_path):
    s = cubic_system(5000, 40.0, seed=41, jitter=0.4, nframes=11)
    gro, trr = _files(tmp_path, s, 11)
    tr = NativeTrajectory(trr)
    back = [tr.read(k) for k in range(11)]
    xs = np.stack([b[0] for b in back])
    boxes = np.stack([b[1] for b in back])
    kw = dict(scale_factor=2.0, qcut=0.6)
    e1 = SaxsEngine((32, 32, 32), s.atom_index(), s.natoms, boxes[0], max_frames=11, **kw)
    e1.forward(torch.from_numpy(xs).cuda(), boxes)
    h1, n1 = e1.histogram()
    e2 = SaxsEngine((32, 32, 32), s.atom_index(), s.natoms, boxes[0], max_frames=4, **kw)
    done = e2.run_trajectory(tr, batch=4)       # batches of 4, 4, 3 through two pinned buffers
    h2, n2 = e2.histogram()
    assert done == 11
    np.testing.assert_array_equal(n1, n2)
    sel = n1 > 0
    np.testing.assert_allclose(h2[sel], h1[sel], rtol=1e-6)
    e3 = SaxsEngine((32, 32, 32), s.atom_index(), s.natoms, boxes[0], max_frames=4, **kw)
    assert e3.run_trajectory(tr, begin=2, end=9, stride=3) == 3  # frames 2, 5, 8
    e4 = SaxsEngine((32, 32, 32), s.atom_index(), s.natoms, boxes[0], max_frames=3, **kw)
    e4.forward(torch.from_numpy(xs[[2, 5, 8]]).cuda(), boxes[[2, 5, 8]])
    h3, n3 = e3.histogram()
    h4, n4 = e4.histogram()
    np.testing.assert_array_equal(n3, n4)
    np.testing.assert_allclose(h3[n3 > 0], h4[n4 > 0], rtol=1e-6)
    for e in (e1, e2, e3, e4):
        e.close()


def test_dropin_run_from_files_equals_run_from_memory(cuda, tmp_path):
    s = cubic_system(4000, 40.0, seed=42, jitter=0.4, nframes=6)
    gro, trr = _files(tmp_path, s, 6)
    top = FileTopology(gro, trr)
    tr = NativeTrajectory(trr)
    back = [tr.read(k) for k in range(6)]
    mem = _Frames(top.elements, [b[0] for b in back], [b[1] for b in back])
    out_f, out_m = tmp_path / "files.dat", tmp_path / "mem.dat"
    args = dict(begin=0, end=5, stride=1, order=4, scale_factor=2.0, bin_size=0.01, qcut=0.7)
    pycusaxs_cuda.run(top, str(gro), str(trr), [32], output=str(out_f), **args)
    pycusaxs_cuda.run(mem, str(gro), str(trr), [32], output=str(out_m), **args)
    rows_f = [(l[:10], float(l[10:])) for l in out_f.read_text().splitlines()]
    rows_m = [(l[:10], float(l[10:])) for l in out_m.read_text().splitlines()]
    assert [r[0] for r in rows_f] == [r[0] for r in rows_m]
    for (_, a), (_, b) in zip(rows_f, rows_m):
        assert abs(a - b) <= 1e-5 * abs(b)  # the file keeps 6 significant digits
