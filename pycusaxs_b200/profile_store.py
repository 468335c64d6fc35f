"""Consumers of the I(q) output: an SQLite profile store and solvent subtraction.

Rebuilt for users of the reference's ``pycusaxs.saxs_database.SaxsDatabase``
(saxs_database.py:15-364) and ``pycusaxs.saxs_subtract`` (saxs_subtract.py:
65-335).  The store keeps the reference's table layout and profile key (the
SHA-256 of "water|sorted ions|box x,y,z|scale|grid|time" with the same number
formats), so databases written by either side can be read and queried by the
other.  Subtraction is non-interactive here (function arguments or the
``python -m pycusaxs_b200.profile_store`` command) instead of the reference's
prompts; the arithmetic is the same: the scaled reference is interpolated onto
the user's q values where the grids differ and subtracted only where both
profiles are defined.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import sqlite3
from pathlib import Path
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

_COLUMNS = (
    "id", "profile_hash", "water_model", "n_water_molecules", "ion_counts", "other_molecules",
    "box_x", "box_y", "box_z", "box_volume", "supercell_scale", "supercell_volume",
    "simulation_time_ps", "n_frames_analyzed", "frame_stride", "grid_size", "bin_size", "qcut",
    "spline_order", "density_g_cm3", "n_atoms", "created_timestamp", "notes", "profile_data",
)

_SCHEMA = """
CREATE TABLE IF NOT EXISTS saxs_profiles (
    id INTEGER PRIMARY KEY AUTOINCREMENT,
    profile_hash TEXT UNIQUE NOT NULL,
    water_model TEXT NOT NULL,
    n_water_molecules INTEGER NOT NULL,
    ion_counts TEXT NOT NULL,
    other_molecules TEXT,
    box_x REAL NOT NULL,
    box_y REAL NOT NULL,
    box_z REAL NOT NULL,
    box_volume REAL NOT NULL,
    supercell_scale REAL NOT NULL,
    supercell_volume REAL NOT NULL,
    simulation_time_ps REAL NOT NULL,
    n_frames_analyzed INTEGER NOT NULL,
    frame_stride INTEGER,
    grid_size TEXT NOT NULL,
    bin_size REAL,
    qcut REAL,
    spline_order INTEGER,
    density_g_cm3 REAL,
    n_atoms INTEGER,
    created_timestamp TEXT DEFAULT CURRENT_TIMESTAMP,
    notes TEXT,
    profile_data TEXT NOT NULL
)
"""


def profile_key(water_model: str, ion_counts: Dict[str, int], box_x: float, box_y: float,
                box_z: float, supercell_scale: float, grid_size: Sequence[int],
                simulation_time_ps: float) -> str:
    """The profile's identity: SHA-256 of the canonical parameter string
    (saxs_database.py:103-135 builds the same string)."""
    ions = sorted(ion_counts.items())
    text = (f"{water_model}|{ions}|{box_x:.3f},{box_y:.3f},{box_z:.3f}|{supercell_scale:.4f}|"
            f"{grid_size[0]}x{grid_size[1]}x{grid_size[2]}|{simulation_time_ps:.2f}")
    return hashlib.sha256(text.encode()).hexdigest()


class ProfileStore:
    """SQLite store of I(q) profiles with their system and run parameters
    (same interface as the reference's SaxsDatabase)."""

    def __init__(self, db_path: str = "saxs_profiles.db"):
        self.db_path = Path(db_path)
        self.conn = sqlite3.connect(str(self.db_path))
        self.conn.row_factory = sqlite3.Row
        cur = self.conn.cursor()
        cur.execute(_SCHEMA)
        cur.execute("CREATE INDEX IF NOT EXISTS idx_profile_hash ON saxs_profiles(profile_hash)")
        cur.execute("CREATE INDEX IF NOT EXISTS idx_water_model ON saxs_profiles(water_model)")
        self.conn.commit()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
        return False

    def close(self) -> None:
        if self.conn is not None:
            self.conn.close()
            self.conn = None

    def save_profile(self, profile_data: List[Tuple[float, float]], water_model: str,
                     n_water_molecules: int, ion_counts: Dict[str, int], box_x: float,
                     box_y: float, box_z: float, box_volume: float, supercell_scale: float,
                     supercell_volume: float, simulation_time_ps: float, n_frames_analyzed: int,
                     grid_size: Tuple[int, int, int], frame_stride: int = 1,
                     bin_size: float | None = None, qcut: float | None = None,
                     order: int | None = None, density_g_cm3: float | None = None,
                     n_atoms: int | None = None, other_molecules: Dict[str, int] | None = None,
                     notes: str | None = None) -> int:
        """Insert a profile; an existing profile with the same key keeps its row and
        its id is returned."""
        key = profile_key(water_model, ion_counts, box_x, box_y, box_z, supercell_scale,
                          grid_size, simulation_time_ps)
        cur = self.conn.cursor()
        try:
            cur.execute(
                "INSERT INTO saxs_profiles (profile_hash, water_model, n_water_molecules, ion_counts, "
                "other_molecules, box_x, box_y, box_z, box_volume, supercell_scale, supercell_volume, "
                "simulation_time_ps, n_frames_analyzed, frame_stride, grid_size, bin_size, qcut, "
                "spline_order, density_g_cm3, n_atoms, notes, profile_data) "
                "VALUES (?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?, ?)",
                (key, water_model, n_water_molecules, json.dumps(ion_counts),
                 json.dumps(other_molecules or {}), box_x, box_y, box_z, box_volume,
                 supercell_scale, supercell_volume, simulation_time_ps, n_frames_analyzed,
                 frame_stride, json.dumps(list(grid_size)), bin_size, qcut, order, density_g_cm3,
                 n_atoms, notes, json.dumps([[float(q), float(i)] for q, i in profile_data])))
            self.conn.commit()
            return int(cur.lastrowid)
        except sqlite3.IntegrityError:
            print(f"Warning: Profile with hash {key[:16]}... already exists in database")
            cur.execute("SELECT id FROM saxs_profiles WHERE profile_hash = ?", (key,))
            return int(cur.fetchone()[0])

    def find_profile(self, water_model: str, ion_counts: Dict[str, int], box_x: float,
                     box_y: float, box_z: float, supercell_scale: float,
                     grid_size: Tuple[int, int, int], simulation_time_ps: float,
                     tolerance: float = 0.01) -> Optional[Dict]:
        key = profile_key(water_model, ion_counts, box_x, box_y, box_z, supercell_scale,
                          grid_size, simulation_time_ps)
        row = self.conn.execute("SELECT * FROM saxs_profiles WHERE profile_hash = ?", (key,)).fetchone()
        return self._row(row) if row else None

    def get_profile(self, profile_id: int) -> Optional[Dict]:
        row = self.conn.execute("SELECT * FROM saxs_profiles WHERE id = ?", (profile_id,)).fetchone()
        return self._row(row) if row else None

    def list_profiles(self, water_model: Optional[str] = None) -> List[Dict]:
        if water_model:
            rows = self.conn.execute("SELECT * FROM saxs_profiles WHERE water_model = ? "
                                     "ORDER BY created_timestamp DESC", (water_model,)).fetchall()
        else:
            rows = self.conn.execute("SELECT * FROM saxs_profiles ORDER BY created_timestamp DESC").fetchall()
        return [self._row(r) for r in rows]

    def delete_profile(self, profile_id: int) -> bool:
        cur = self.conn.execute("DELETE FROM saxs_profiles WHERE id = ?", (profile_id,))
        self.conn.commit()
        return cur.rowcount > 0

    @staticmethod
    def _row(row: sqlite3.Row) -> Dict:
        d = dict(row)
        d["ion_counts"] = json.loads(d["ion_counts"])
        d["other_molecules"] = json.loads(d["other_molecules"]) if d.get("other_molecules") else {}
        d["grid_size"] = json.loads(d["grid_size"])
        d["profile_data"] = json.loads(d["profile_data"])
        return d

    def export_profile_csv(self, profile_id: int, output_path: str) -> None:
        p = self.get_profile(profile_id)
        if p is None:
            raise ValueError(f"Profile with ID {profile_id} not found")
        dens = p.get("density_g_cm3")
        lines = [
            "# SAXS Solvent Profile",
            f"# Water Model: {p['water_model']}",
            f"# Water Molecules: {p['n_water_molecules']}",
            f"# Ion Counts: {p['ion_counts']}",
            f"# Box Size: {p['box_x']:.3f} x {p['box_y']:.3f} x {p['box_z']:.3f} Å",
            f"# Supercell Scale: {p['supercell_scale']:.4f}",
            f"# Simulation Time: {p['simulation_time_ps']:.2f} ps",
            f"# Frames Analyzed: {p['n_frames_analyzed']}",
            f"# Density: {dens:.4f} g/cm³" if dens is not None else "# Density: N/A g/cm³",
            "#",
            "# q (1/Å), I(q) (1/Å³)",
        ]
        lines += [f"{q:.6f},{i:.6e}" for q, i in p["profile_data"]]
        Path(output_path).write_text("\n".join(lines) + "\n")


def read_profile_file(path) -> List[Tuple[float, float]]:
    """(q, I) rows of an I(q) file written by the SAXS run (comment lines skipped)."""
    rows = []
    for line in Path(path).read_text().splitlines():
        line = line.strip()
        if line and not line.startswith("#"):
            parts = line.replace(",", " ").split()
            if len(parts) >= 2:
                rows.append((float(parts[0]), float(parts[1])))
    return rows


def store_run(db_path, profile_file, system_info: Dict, grid_size: Sequence[int],
              supercell_scale: float, first_frame: int, last_frame: int, stride: int = 1,
              bin_size=None, qcut=None, order=None, water_model: str = "", notes=None) -> int:
    """Store a finished run's profile with the system information of its topology
    (the reference CLI's --save-db step, cli.py:240-330): frames first..last with
    `stride`, simulation time from the first to the last processed frame."""
    n = last_frame - first_frame + 1
    frames = (n + stride - 1) // stride
    last = first_frame + (frames - 1) * stride
    dt = float(system_info.get("dt", 0.0) or 0.0)
    with ProfileStore(db_path) as db:
        return db.save_profile(
            profile_data=read_profile_file(profile_file),
            water_model=system_info.get("detected_water_model", water_model) or water_model,
            n_water_molecules=int(system_info.get("n_water_molecules", 0)),
            ion_counts=system_info.get("ion_counts", {}),
            box_x=float(system_info.get("box_x", 0.0)), box_y=float(system_info.get("box_y", 0.0)),
            box_z=float(system_info.get("box_z", 0.0)),
            box_volume=float(system_info.get("box_volume", 0.0)),
            supercell_scale=float(supercell_scale),
            supercell_volume=float(system_info.get("box_volume", 0.0)) * float(supercell_scale) ** 3,
            simulation_time_ps=(last - first_frame) * dt, n_frames_analyzed=frames,
            grid_size=tuple(int(g) for g in grid_size), frame_stride=stride, bin_size=bin_size,
            qcut=qcut, order=order, density_g_cm3=system_info.get("density_g_cm3"),
            n_atoms=system_info.get("n_atoms"), other_molecules=system_info.get("other_molecules", {}),
            notes=notes)


# -- solvent subtraction ----------------------------------------------------------


def interpolate_profile(q_ref: np.ndarray, iq_ref: np.ndarray, q_target: np.ndarray,
                        method: str = "cubic") -> np.ndarray:
    """Reference I(q) on `q_target` (cubic or linear, extrapolated at the ends)."""
    from scipy.interpolate import interp1d

    f = interp1d(q_ref, iq_ref, kind="cubic" if method == "cubic" else "linear",
                 bounds_error=False, fill_value="extrapolate")
    return f(q_target)


def subtract_profiles(user_profile: Dict, ref_profile: Dict, scale: float,
                      interp_method: str = "cubic") -> Tuple[np.ndarray, np.ndarray]:
    """I_user - scale * I_ref on the user's q values inside the overlap of the two
    q ranges; outside it the user's values are kept (saxs_subtract.py:126-205)."""
    u = np.asarray(user_profile["profile_data"], dtype=np.float64)
    r = np.asarray(ref_profile["profile_data"], dtype=np.float64)
    qu, iu, qr, ir = u[:, 0], u[:, 1], r[:, 0], r[:, 1]
    lo, hi = max(qu[0], qr[0]), min(qu[-1], qr[-1])
    if hi <= lo:
        raise ValueError("No overlap between user and reference q-ranges!")
    mask = (qu >= lo) & (qu <= hi)
    same = len(qu) == len(qr) and np.allclose(qu, qr, rtol=1e-6)
    ir_on_u = ir if same else interpolate_profile(qr, ir, qu, method=interp_method)
    out = iu.copy()
    out[mask] = iu[mask] - scale * ir_on_u[mask]
    return qu, out


def resample_profile(q: np.ndarray, iq: np.ndarray, dq: float,
                     method: str = "cubic") -> Tuple[np.ndarray, np.ndarray]:
    """The profile on a uniform grid from q[0] to q[-1] with ceil((q1-q0)/dq)+1 points."""
    n = int(np.ceil((q[-1] - q[0]) / dq)) + 1
    qn = np.linspace(q[0], q[-1], n)
    return qn, interpolate_profile(q, iq, qn, method=method)


def _describe(p: Dict, role: str) -> List[str]:
    def counts(d):
        s = ", ".join(f"{k}: {v}" for k, v in d.items() if v > 0) if d else ""
        return s or "none"

    dens = p.get("density_g_cm3")
    return [
        f"# {role}:",
        f"#   ID: {p['id']}",
        f"#   Water Model: {p['water_model']}",
        f"#   Ions: {counts(p.get('ion_counts', {}))}",
        f"#   Other Molecules: {counts(p.get('other_molecules', {}))}",
        f"#   Grid: {p['grid_size']}",
        f"#   Supercell Scale: {p['supercell_scale']:.4f}",
        f"#   Box: {p['box_x']:.3f} x {p['box_y']:.3f} x {p['box_z']:.3f} Å",
        f"#   Volume: {p['box_volume']:.2f} Ų",
        f"#   Density: {dens:.4f} g/cm³" if dens is not None else "#   Density: N/A g/cm³",
        f"#   Simulation Time: {p['simulation_time_ps']:.2f} ps",
        "#",
    ]


def save_subtracted_profile(output_path, q, iq, user_profile: Dict, ref_profile: Dict, scale: float,
                            resampled: bool = False, original_points: int | None = None) -> None:
    lines = ["# SAXS Profile after Solvent Subtraction", "#"]
    lines += _describe(user_profile, "User Profile")
    lines += _describe(ref_profile, "Reference Profile (subtracted)")
    lines += ["# Subtraction Parameters:", f"#   Scaling Factor: {scale:.6f}",
              "#   Note: Subtraction applied only in overlap region between profiles", "#"]
    if resampled and original_points is not None:
        lines += ["# Output Processing:", f"#   Original data points: {original_points}",
                  f"#   Resampled to: {len(q)} points", f"#   Q spacing (dq): {(q[1] - q[0]):.6f} Å⁻¹", "#"]
    lines.append("# q (Å⁻¹)    I(q) [subtracted]")
    lines += [f"{a:.6f}  {b:.6e}" for a, b in zip(q, iq)]
    Path(output_path).write_text("\n".join(lines) + "\n")


def subtract(user_db, user_id: int, ref_db, ref_id: int, scale: float, output,
             dq: float | None = None, method: str = "cubic") -> Tuple[np.ndarray, np.ndarray]:
    """User profile `user_id` of `user_db` minus `scale` x reference `ref_id` of
    `ref_db`, optionally resampled to spacing `dq`, written to `output`."""
    with ProfileStore(user_db) as u, ProfileStore(ref_db) as r:
        up, rp = u.get_profile(user_id), r.get_profile(ref_id)
    if up is None:
        raise ValueError(f"profile {user_id} not found in {user_db}")
    if rp is None:
        raise ValueError(f"profile {ref_id} not found in {ref_db}")
    q, iq = subtract_profiles(up, rp, scale, interp_method=method)
    n0 = len(q)
    if dq:
        q, iq = resample_profile(q, iq, dq, method=method)
    save_subtracted_profile(output, q, iq, up, rp, scale, resampled=bool(dq), original_points=n0)
    return q, iq


def main(argv=None) -> int:
    ap = argparse.ArgumentParser(description="Subtract a scaled reference solvent profile.")
    ap.add_argument("--user-db", required=True)
    ap.add_argument("--user-id", type=int, required=True)
    ap.add_argument("--ref-db", required=True)
    ap.add_argument("--ref-id", type=int, required=True)
    ap.add_argument("--scale", type=float, required=True)
    ap.add_argument("--output", required=True)
    ap.add_argument("--dq", type=float, default=None)
    ap.add_argument("--method", choices=("cubic", "linear"), default="cubic")
    a = ap.parse_args(argv)
    if a.scale <= 0:
        ap.error("scaling factor must be positive")
    subtract(a.user_db, a.user_id, a.ref_db, a.ref_id, a.scale, a.output, dq=a.dq, method=a.method)
    print(f"Subtracted profile written to {a.output}")
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
