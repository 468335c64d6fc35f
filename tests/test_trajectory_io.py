"""Frame ingestion without MDAnalysis (CPU): native TRR/XTC/DCD readers, GRO/PDB topologies,
the FileTopology callback contract and the read-ahead streams.

The XTC reader is checked by round trips through the test-side compressor
(tests/trajfiles.py): positions must equal the written integer coordinates
times 1/precision, converted to Angstrom, bit for bit.  No file written by
GROMACS exists here, so parity with GROMACS-written files is unpinned."""
import numpy as np
import pytest

from pycusaxs_b200 import _native
from pycusaxs_b200.trajectory import (BatchStream, FileTopology, GroTrajectory, NativeTrajectory,
                                      NpyTrajectory, box_from_lengths, guess_element, read_gro,
                                      read_pdb)
from trajfiles import write_dcd, write_gro, write_pdb, write_trr, write_xtc


def _frames(F=5, N=7, seed=0):
    rng = np.random.default_rng(seed)
    return rng.uniform(0.0, 3.0, (F, N, 3))


@pytest.mark.parametrize("double", [False, True])
@pytest.mark.parametrize("vf", [False, True])
def test_trr_roundtrip_nm_to_angstrom(tmp_path, double, vf):
    x = _frames()
    boxes = np.stack([np.diag([3.0 + 0.01 * k, 3.1, 3.2]) for k in range(5)])
    boxes[:, 1, 0] = 0.4  # a triclinic row
    times = [2.0 * k for k in range(5)]
    p = tmp_path / "t.trr"
    write_trr(p, x, boxes, times, double=double, with_v=vf, with_f=vf)
    tr = NativeTrajectory(p)
    assert (tr.n_atoms, tr.n_frames) == (7, 5)
    for k in (0, 3, 4, 1):
        pos, box, t = tr.read(k)
        tol = 1e-6 if double else 1e-5
        np.testing.assert_allclose(pos, (x[k] * 10.0).astype(np.float32), rtol=tol, atol=tol)
        np.testing.assert_allclose(box, (boxes[k] * 10.0).astype(np.float32), rtol=tol, atol=tol)
        assert t == pytest.approx(times[k])
    tr.close()


def test_trr_errors(tmp_path):
    p = tmp_path / "bad.trr"
    p.write_bytes(b"\x00\x00\x07\xc9" + b"\x00" * 40)  # magic 1993, then garbage header
    with pytest.raises(_native.SaxsError):
        NativeTrajectory(p)
    q = tmp_path / "t.trr"
    write_trr(q, _frames(F=2), np.stack([np.eye(3) * 3] * 2), [0.0, 1.0])
    tr = NativeTrajectory(q)
    with pytest.raises(_native.SaxsError, match="out of range"):
        tr.read(2)
    raw = q.read_bytes()
    (tmp_path / "cut.trr").write_bytes(raw[: len(raw) - 10])
    with pytest.raises(_native.SaxsError):
        NativeTrajectory(tmp_path / "cut.trr").read(1)


@pytest.mark.parametrize("big", [False, True])
@pytest.mark.parametrize("cosines", [False, True])
def test_dcd_with_unit_cell(tmp_path, big, cosines):
    x = _frames(F=4, N=9, seed=1) * 10.0
    cells = [(30.0 + k, 31.0, 32.0, 90.0, 90.0, 80.0 + k) for k in range(4)]
    p = tmp_path / "t.dcd"
    write_dcd(p, x.astype(np.float32), cells=cells, cosines=cosines, big_endian=big, dt=0.5)
    tr = NativeTrajectory(p)
    assert (tr.n_atoms, tr.n_frames) == (9, 4)
    for k in range(4):
        pos, box, t = tr.read(k)
        np.testing.assert_allclose(pos, x[k].astype(np.float32), rtol=0, atol=0)
        np.testing.assert_allclose(box, box_from_lengths(*cells[k]), rtol=1e-5, atol=1e-4)
        assert t == pytest.approx(0.5 * k)


def test_dcd_without_cell_and_short_file(tmp_path):
    x = _frames(F=3, N=4, seed=2).astype(np.float32)
    p = tmp_path / "t.dcd"
    write_dcd(p, x, cells=None, nset=10)  # header claims more frames than the file holds
    tr = NativeTrajectory(p)
    assert tr.n_frames == 3
    pos, box, _ = tr.read(2)
    np.testing.assert_array_equal(pos, x[2])
    assert np.all(box == 0)


def test_unknown_extension_is_refused(tmp_path):
    p = tmp_path / "x.xyz"
    p.write_bytes(b"\x00" * 16)
    with pytest.raises(_native.SaxsError, match="unsupported trajectory format"):
        NativeTrajectory(p)


def test_element_guessing():
    assert guess_element("CA", "ALA") == "C"
    assert guess_element("CA", "CA") == "Ca"
    assert guess_element("NA", "NA") == "Na"
    assert guess_element("CL", "CL-") == "Cl"
    assert guess_element("1HB", "LEU") == "H"
    assert guess_element("OW", "SOL") == "O"
    assert guess_element("MG", "MG") == "Mg"


def test_gro_topology_and_multiframe_trajectory(tmp_path):
    names = ["OW", "HW1", "HW2", "NA", "CL", "CA"]
    res = ["SOL", "SOL", "SOL", "NA", "CL", "ALA"]
    x = _frames(F=3, N=6, seed=3)
    boxes = np.stack([np.array([[3.0, 0, 0], [0.5, 3.0, 0], [0.2, 0.3, 2.5]])] * 3)
    p = tmp_path / "s.gro"
    write_gro(p, names, res, x, boxes, times=[0.0, 10.0, 20.0])
    top = read_gro(p)
    assert top["elements"] == ["O", "H", "H", "Na", "Cl", "C"]
    np.testing.assert_allclose(top["positions"], np.round(x[0], 3) * 10.0, atol=1e-4)
    np.testing.assert_allclose(top["box"], boxes[0] * 10.0, atol=1e-4)
    tr = GroTrajectory(p)
    assert tr.n_frames == 3
    pos, box, t = tr.read(2)
    np.testing.assert_allclose(pos, np.round(x[2], 3) * 10.0, atol=1e-4)
    assert t == pytest.approx(20.0)


def test_pdb_elements_and_cryst1(tmp_path):
    names = ["N", "CA", "C", "O", "CA"]
    res = ["ALA", "ALA", "ALA", "ALA", "CA"]
    els = ["N", "C", "C", "O", "CA"]
    pos = _frames(F=1, N=5, seed=4)[0] * 10.0
    p = tmp_path / "s.pdb"
    write_pdb(p, names, res, els, pos, cell=(40.0, 41.0, 42.0, 90.0, 90.0, 90.0))
    top = read_pdb(p)
    assert top["elements"] == ["N", "C", "C", "O", "Ca"]
    np.testing.assert_allclose(top["positions"], np.round(pos, 3), atol=1e-4)
    np.testing.assert_allclose(np.diag(top["box"]), [40.0, 41.0, 42.0], atol=1e-5)


def test_file_topology_contract(tmp_path):
    names = ["OW", "HW1", "HW2"] * 4
    res = ["SOL"] * 12
    x = _frames(F=9, N=12, seed=5)
    boxes = np.stack([np.eye(3) * (3.0 + 0.01 * k) for k in range(9)])
    write_gro(tmp_path / "s.gro", names, res, x[:1], boxes[:1])
    write_trr(tmp_path / "s.trr", x, boxes, [float(k) for k in range(9)])
    t = FileTopology(tmp_path / "s.gro", tmp_path / "s.trr", prefetch=3)
    assert t.n_frames == 9 and t.n_atoms == 12
    idx = t.get_atom_index()
    assert idx == {"O": [0, 3, 6, 9], "H": [1, 2, 4, 5, 7, 8, 10, 11]}
    t.read_frame(4)
    np.testing.assert_allclose(t.get_box(), boxes[4] * 10.0, rtol=1e-6)
    assert t.get_step() == 4
    got = [(f["frame"], f["positions"].copy(), f["box"].copy(), f["time"])
           for f in t.iter_frames_stream(1, 8, 3)]
    assert [g[0] for g in got] == [1, 4, 7]
    for k, pos, box, tt in got:
        np.testing.assert_allclose(pos, (x[k] * 10.0).astype(np.float32), rtol=1e-5)
        assert tt == pytest.approx(float(k))
    # stop beyond the end is clipped; reading ahead keeps every yielded frame intact
    frames = list(t.iter_frames_stream(0, 100, 1))
    assert len(frames) == 9
    with pytest.raises(IndexError):
        t.read_frame(9)


def test_read_ahead_does_not_overwrite_the_held_frame(tmp_path):
    x = _frames(F=20, N=5, seed=6)
    write_trr(tmp_path / "a.trr", x, np.stack([np.eye(3) * 3] * 20), [0.0] * 20)
    names = ["C"] * 5
    write_gro(tmp_path / "a.gro", names, ["MOL"] * 5, x[:1], [np.eye(3) * 3])
    t = FileTopology(tmp_path / "a.gro", tmp_path / "a.trr", prefetch=3)
    for f in t.iter_frames_stream(0, 20, 1):
        import time
        time.sleep(0.002)  # give the reader time to run ahead
        np.testing.assert_allclose(f["positions"], (x[f["frame"]] * 10).astype(np.float32), rtol=1e-5)


def test_npy_memmap_trajectory(tmp_path):
    x = _frames(F=4, N=6, seed=7).astype(np.float32) * 10
    np.save(tmp_path / "c.npy", x)
    tr = NpyTrajectory(tmp_path / "c.npy", box=np.eye(3) * 30.0, dt_ps=2.0)
    out = np.empty((6, 3), np.float32)
    pos, box, t = tr.read(3, out=out)
    assert pos is out
    np.testing.assert_array_equal(out, x[3])
    assert t == 6.0 and box.shape == (3, 3)


def test_batch_stream_refills_only_released_buffers(tmp_path):
    x = _frames(F=11, N=4, seed=8)
    write_trr(tmp_path / "b.trr", x, np.stack([np.eye(3) * 3] * 11), [0.0] * 11)
    tr = NativeTrajectory(tmp_path / "b.trr")
    bufs = [np.zeros((3, 4, 3), np.float32) for _ in range(2)]

    class Buf:  # numpy stand-in for a pinned tensor (.numpy())
        def __init__(self, a):
            self.a = a

        def numpy(self):
            return self.a

    st = BatchStream(tr, range(0, 11), 3, [Buf(b) for b in bufs])
    seen = []
    for slot, buf, boxes, n in st:
        a = buf.numpy()[:n].copy()
        seen.extend(a)
        st.release(slot, None)
    st.close()
    np.testing.assert_allclose(np.stack(seen), (x * 10).astype(np.float32), rtol=1e-5)


def _waters(nmol, box_nm, seed):
    """Water-like triples (O then two H 0.1 nm away) spread over a box: the
    pairs and runs the compressor takes apart."""
    rng = np.random.default_rng(seed)
    o = rng.uniform(0.0, box_nm, (nmol, 3))
    h1 = o + rng.normal(0, 0.06, (nmol, 3))
    h2 = o + rng.normal(0, 0.06, (nmol, 3))
    return np.stack([o, h1, h2], axis=1).reshape(-1, 3)


def _expected(ints, precision):
    inv = np.float32(1.0 / np.float64(np.float32(precision)))
    return (ints.astype(np.float32) * inv) * np.float32(10.0)


@pytest.mark.parametrize("large", [False, True])
@pytest.mark.parametrize("precision", [1000.0, 100.0])
def test_xtc_roundtrip(tmp_path, large, precision):
    frames = [_waters(700, 4.0, seed=k) for k in range(4)]
    frames[2] = np.random.default_rng(9).uniform(-1.0, 4.0, (2100, 3))   # no neighbours: lone atoms
    boxes = [np.diag([4.0, 4.1, 4.2]) for _ in range(4)]
    boxes[1][1, 0] = 0.7
    p = tmp_path / "w.xtc"
    written = write_xtc(p, frames, boxes, [0.5 * k for k in range(4)], precision=precision,
                        large=large, seed=3)
    tr = NativeTrajectory(p)
    assert (tr.n_atoms, tr.n_frames) == (2100, 4)
    for k in (3, 0, 2, 1):
        pos, box, t = tr.read(k)
        np.testing.assert_array_equal(pos, _expected(written[k], precision))
        np.testing.assert_array_equal(box, np.asarray(boxes[k], np.float32) * np.float32(10.0))
        assert t == pytest.approx(0.5 * k)
        # and the positions are the frame's to the written precision
        np.testing.assert_allclose(pos, frames[k] * 10.0, atol=10.0 * 0.5 / precision * 1.001 + 1e-4)
    tr.close()


def test_xtc_small_frames_are_plain_floats(tmp_path):
    x = [np.random.default_rng(1).uniform(0, 2, (5, 3)) for _ in range(2)]
    p = tmp_path / "s.xtc"
    write_xtc(p, x, [np.eye(3) * 2.0] * 2, [0.0, 1.0])
    tr = NativeTrajectory(p)
    pos, box, _ = tr.read(1)
    np.testing.assert_array_equal(pos, np.asarray(x[1], np.float32) * np.float32(10.0))
    tr.close()


def test_xtc_corrupt_stream_is_an_error_not_a_crash(tmp_path):
    frames = [_waters(400, 3.0, seed=5)]
    p = tmp_path / "c.xtc"
    write_xtc(p, frames, [np.eye(3) * 3.0], [0.0])
    raw = bytearray(p.read_bytes())
    # keep the header's byte count, zero the stream's second half: the decoder
    # must stop at the end of the stream or at a run past the last atom
    nbytes = int.from_bytes(raw[88:92], "big")
    raw[92 + nbytes // 2: 92 + nbytes] = b"\xff" * (nbytes - nbytes // 2)
    p.write_bytes(bytes(raw))
    tr = NativeTrajectory(p)
    with pytest.raises(_native.SaxsError):
        tr.read(0)
    tr.close()
