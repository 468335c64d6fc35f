"""Output consumers (CPU): the SQLite profile store and solvent subtraction."""
import hashlib
import sqlite3

import numpy as np
import pytest

from pycusaxs_b200.profile_store import (ProfileStore, interpolate_profile, main, profile_key,
                                         read_profile_file, resample_profile, store_run, subtract,
                                         subtract_profiles)
from pycusaxs_b200.trajectory import FileTopology
from trajfiles import write_gro, write_trr

REFERENCE_COLUMNS = [
    "id", "profile_hash", "water_model", "n_water_molecules", "ion_counts", "other_molecules",
    "box_x", "box_y", "box_z", "box_volume", "supercell_scale", "supercell_volume",
    "simulation_time_ps", "n_frames_analyzed", "frame_stride", "grid_size", "bin_size", "qcut",
    "spline_order", "density_g_cm3", "n_atoms", "created_timestamp", "notes", "profile_data"]


def _profile(q0=0.05, dq=0.05, n=20, amp=1.0):
    q = q0 + dq * np.arange(n)
    return [(float(a), float(amp * np.exp(-a))) for a in q]


def _save(db, data, water="TIP3P", ions=None, box=30.0, time=100.0):
    return db.save_profile(profile_data=data, water_model=water, n_water_molecules=900,
                           ion_counts=ions or {"Na": 3, "Cl": 3}, box_x=box, box_y=box, box_z=box,
                           box_volume=box ** 3, supercell_scale=2.0, supercell_volume=8 * box ** 3,
                           simulation_time_ps=time, n_frames_analyzed=10, grid_size=(64, 64, 64),
                           bin_size=0.01, qcut=0.5, order=4, density_g_cm3=1.0, n_atoms=2706)


def test_schema_and_key_match_the_reference_layout(tmp_path):
    with ProfileStore(tmp_path / "p.db") as db:
        cols = [r[1] for r in db.conn.execute("PRAGMA table_info(saxs_profiles)")]
    assert cols == REFERENCE_COLUMNS
    text = "TIP3P|[('Cl', 3), ('Na', 3)]|30.000,30.000,30.000|2.0000|64x64x64|100.00"
    assert profile_key("TIP3P", {"Na": 3, "Cl": 3}, 30.0, 30.0, 30.0, 2.0, (64, 64, 64), 100.0) == \
        hashlib.sha256(text.encode()).hexdigest()


def test_save_find_list_export_delete(tmp_path, capsys):
    data = _profile()
    with ProfileStore(tmp_path / "p.db") as db:
        pid = _save(db, data)
        assert _save(db, data) == pid                      # same key: the existing row
        assert "already exists" in capsys.readouterr().out
        pid2 = _save(db, data, water="SPCE")
        got = db.find_profile("TIP3P", {"Cl": 3, "Na": 3}, 30.0, 30.0, 30.0, 2.0, (64, 64, 64), 100.0)
        assert got["id"] == pid and got["grid_size"] == [64, 64, 64]
        assert got["ion_counts"] == {"Na": 3, "Cl": 3}
        np.testing.assert_allclose(np.asarray(got["profile_data"]), np.asarray(data))
        assert db.find_profile("TIP3P", {}, 30.0, 30.0, 30.0, 2.0, (64, 64, 64), 100.0) is None
        assert {p["id"] for p in db.list_profiles()} == {pid, pid2}
        assert [p["id"] for p in db.list_profiles("SPCE")] == [pid2]
        db.export_profile_csv(pid, tmp_path / "p.csv")
        lines = (tmp_path / "p.csv").read_text().splitlines()
        assert lines[0] == "# SAXS Solvent Profile" and lines[-1].startswith("1.000000,")
        assert db.delete_profile(pid2) and db.get_profile(pid2) is None
        with pytest.raises(ValueError):
            db.export_profile_csv(999, tmp_path / "x.csv")
    # the file is a plain SQLite database other tools can query
    assert sqlite3.connect(str(tmp_path / "p.db")).execute(
        "SELECT count(*) FROM saxs_profiles").fetchone()[0] == 1


def test_subtraction_same_grid_overlap_and_interpolation():
    user = {"profile_data": _profile(n=20, amp=2.0)}
    ref = {"profile_data": _profile(n=20, amp=1.0)}
    q, iq = subtract_profiles(user, ref, 0.5)
    np.testing.assert_allclose(iq, 1.5 * np.exp(-q))
    # reference covers only part of the user range: outside the overlap the user is kept
    ref2 = {"profile_data": _profile(q0=0.2, dq=0.05, n=8, amp=1.0)}
    q, iq = subtract_profiles(user, ref2, 1.0, interp_method="linear")
    inside = (q >= 0.2) & (q <= 0.2 + 0.05 * 7 + 1e-12)
    np.testing.assert_allclose(iq[~inside], 2.0 * np.exp(-q[~inside]))
    np.testing.assert_allclose(iq[inside], np.exp(-q[inside]), rtol=1e-12)
    # a finer reference grid is interpolated onto the user's q
    ref3 = {"profile_data": [(float(a), float(np.exp(-a))) for a in np.linspace(0.01, 1.2, 400)]}
    q, iq = subtract_profiles(user, ref3, 1.0)
    np.testing.assert_allclose(iq, np.exp(-q), rtol=1e-6)
    with pytest.raises(ValueError, match="No overlap"):
        subtract_profiles(user, {"profile_data": _profile(q0=5.0)}, 1.0)


def test_resample_uniform_grid():
    q = np.array([0.0, 0.1, 0.3, 0.6, 1.0])
    qn, iqn = resample_profile(q, q ** 2, 0.05)
    assert len(qn) == 21 and qn[0] == 0.0 and qn[-1] == 1.0
    np.testing.assert_allclose(iqn, qn ** 2, atol=1e-12)   # cubic reproduces a parabola
    np.testing.assert_allclose(interpolate_profile(q, q, qn, method="linear"), qn)


def test_subtract_command_writes_annotated_profile(tmp_path):
    with ProfileStore(tmp_path / "u.db") as db:
        uid = _save(db, _profile(amp=3.0))
    with ProfileStore(tmp_path / "r.db") as db:
        rid = _save(db, _profile(amp=1.0), water="SPCE")
    out = tmp_path / "sub.dat"
    assert main(["--user-db", str(tmp_path / "u.db"), "--user-id", str(uid), "--ref-db",
                 str(tmp_path / "r.db"), "--ref-id", str(rid), "--scale", "2", "--output", str(out),
                 "--dq", "0.1"]) == 0
    text = out.read_text()
    assert "# Reference Profile (subtracted):" in text and "Scaling Factor: 2.000000" in text
    rows = read_profile_file(out)
    assert len(rows) == int(np.ceil((1.0 - 0.05) / 0.1)) + 1
    q = np.array([r[0] for r in rows])
    np.testing.assert_allclose([r[1] for r in rows], np.exp(-q), rtol=2e-4)
    with pytest.raises(ValueError, match="not found"):
        subtract(tmp_path / "u.db", 42, tmp_path / "r.db", rid, 1.0, out)


def test_store_run_with_system_info_from_files(tmp_path):
    # 4 waters + 1 Na + 1 Cl + two residues of MOL
    names = ["OW", "HW1", "HW2"] * 4 + ["NA", "CL"] + ["C1", "O1", "C1", "O1"]
    res = ["SOL"] * 12 + ["NA", "CL"] + ["MOL"] * 4
    rng = np.random.default_rng(0)
    x = rng.uniform(0, 2.0, (3, len(names), 3))
    boxes = np.stack([np.eye(3) * 2.0] * 3)
    write_gro(tmp_path / "s.gro", names, res, x[:1], boxes[:1])
    # residue numbers: the writer numbers every 3 atoms, so MOL atoms 14-17 are residues 5 and 6
    write_trr(tmp_path / "s.trr", x, boxes, [0.0, 2.0, 4.0])
    info = FileTopology(tmp_path / "s.gro", tmp_path / "s.trr").get_system_info()
    assert info["n_water_molecules"] == 4 and info["ion_counts"] == {"Na": 1, "Cl": 1}
    assert info["other_molecules"] == {"MOL": 2}
    assert info["detected_water_model"] == "TIP3P/SPC"
    assert info["box_x"] == pytest.approx(20.0) and info["dt"] == pytest.approx(2.0)
    (tmp_path / "saxs.dat").write_text("".join(f"{q:10.5f}{i:12.5e}\n" for q, i in _profile()))
    pid = store_run(tmp_path / "db.sqlite", tmp_path / "saxs.dat", info, (32, 32, 32), 2.0,
                    first_frame=0, last_frame=2, stride=2, qcut=0.5, order=4)
    with ProfileStore(tmp_path / "db.sqlite") as db:
        p = db.get_profile(pid)
    assert p["n_frames_analyzed"] == 2 and p["simulation_time_ps"] == pytest.approx(4.0)
    assert p["supercell_volume"] == pytest.approx(8 * 20.0 ** 3, rel=1e-6)
    assert len(p["profile_data"]) == 20
