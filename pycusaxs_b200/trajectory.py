"""Frame ingestion without MDAnalysis.

The reference reads its topology and frames through MDAnalysis
(pycusaxs/topology.py:52-75 ``Universe(tpr, xtc)``, 273-286 ``get_atom_index``
from ``atom.element``, 536-577 ``read_frame`` / ``get_box``, 621-737
``iter_frames_stream``).  This module replaces that with:

* ``NativeTrajectory``: GROMACS TRR and XTC (compressed coordinates) and
  CHARMM/NAMD DCD read by the library's native readers (``saxs_traj_*``;
  ctypes releases the GIL during reads);
* ``NpyTrajectory``: coordinates memory-mapped from a ``.npy`` file of shape
  (frames, natoms, 3) float32 Angstrom, boxes from a (3, 3) or (frames, 3, 3)
  array;
* ``read_gro`` / ``read_pdb``: atom names, residue names, elements, first-frame
  positions and box from GROMACS GRO and PDB files (GRO files with several
  frames are also a trajectory: ``GroTrajectory``);
* ``FileTopology``: the reference's topology callback contract over any of the
  above, usable as ``obj_topology`` of ``pycusaxs_cuda.run``;
* ``BatchStream``: a reader thread that fills double-buffered pinned host
  batches while the previous batch is copied and processed
  (``SaxsEngine.run_trajectory``).

Units: Angstrom for positions and box rows, picoseconds for time, as the
reference's frame dicts carry them.  GRO, TRR and XTC store nanometres and are
converted.  Not read: TPR (binary run input).
"""
from __future__ import annotations

import ctypes
import math
import threading
from pathlib import Path
from typing import Iterator

import numpy as np

from . import _native

NM = 10.0  # Angstrom per nanometre

# two-letter element symbols that atom names in GRO/PDB files commonly start with
_TWO_LETTER = {"CL", "NA", "MG", "ZN", "FE", "BR", "CA", "CU", "MN", "LI", "SE", "SI", "CO", "NI",
               "CD", "HG", "AL", "RB", "CS", "SR", "BA", "AG", "AU", "PT", "PB", "SN"}


def guess_element(atom_name: str, resname: str = "") -> str:
    """Element symbol from an atom name.

    Two-letter elements are taken only when the residue is the ion itself
    (resname == atom name, e.g. NA/NA, CL/CL, CA/CA); otherwise the first letter
    (CA of an amino acid is a carbon).  Leading digits (1HB) are skipped.
    """
    name = atom_name.strip().upper().lstrip("0123456789")
    res = resname.strip().upper()
    if not name:
        raise ValueError(f"cannot guess an element from atom name {atom_name!r}")
    two = name[:2]
    if two in _TWO_LETTER and (res == name or res == two or res.rstrip("+-0123456789") == two):
        return two[0] + two[1].lower()
    return name[0]


def box_from_lengths(a, b, c, alpha=90.0, beta=90.0, gamma=90.0) -> np.ndarray:
    """3x3 box rows from edge lengths and angles in degrees (a along x, b in xy)."""
    ca, cb, cg = (math.cos(math.radians(v)) for v in (alpha, beta, gamma))
    sg = math.sin(math.radians(gamma))
    cx = c * cb
    cy = c * (ca - cb * cg) / sg
    cz = math.sqrt(max(c * c - cx * cx - cy * cy, 0.0))
    box = np.array([[a, 0, 0], [b * cg, b * sg, 0], [cx, cy, cz]], dtype=np.float64)
    box[np.abs(box) < 1e-9] = 0.0
    return box.astype(np.float32)


# -- GRO ----------------------------------------------------------------------


def _gro_box(line: str) -> np.ndarray:
    v = [float(x) for x in line.split()]
    if len(v) == 3:
        v += [0.0] * 6
    if len(v) != 9:
        raise ValueError(f"GRO box line needs 3 or 9 numbers: {line!r}")
    # v1(x) v2(y) v3(z) v1(y) v1(z) v2(x) v2(z) v3(x) v3(y), nanometres
    rows = np.array([[v[0], v[3], v[4]], [v[5], v[1], v[6]], [v[7], v[8], v[2]]], dtype=np.float64)
    return (rows * NM).astype(np.float32)


def _gro_frames(path):
    with open(path) as fh:
        while True:
            title = fh.readline()
            if not title:
                return
            n_line = fh.readline()
            if not n_line.strip():
                return
            n = int(n_line)
            names, resnames, resids = [], [], []
            pos = np.empty((n, 3), dtype=np.float32)
            for i in range(n):
                ln = fh.readline()
                resids.append(int(ln[0:5]))
                resnames.append(ln[5:10].strip())
                names.append(ln[10:15].strip())
                pos[i] = (float(ln[20:28]) * NM, float(ln[28:36]) * NM, float(ln[36:44]) * NM)
            box = _gro_box(fh.readline())
            t = 0.0
            if "t=" in title:
                try:
                    t = float(title.split("t=")[1].split()[0])
                except (ValueError, IndexError):
                    t = 0.0
            yield names, resnames, pos, box, t, resids


def read_gro(path) -> dict:
    """First frame of a GRO file: names, resnames, residue numbers, elements,
    positions (A), box rows (A)."""
    names, resnames, pos, box, _, resids = next(_gro_frames(path))
    return {"names": names, "resnames": resnames, "resids": resids,
            "elements": [guess_element(a, r) for a, r in zip(names, resnames)],
            "positions": pos, "box": box}


class GroTrajectory:
    """Every frame of a (multi-frame) GRO file, held in memory."""

    def __init__(self, path):
        frames = list(_gro_frames(path))
        if not frames:
            raise ValueError(f"no frames in {path}")
        self._pos = [f[2] for f in frames]
        self._box = [f[3] for f in frames]
        self._time = [f[4] for f in frames]
        self.n_atoms = self._pos[0].shape[0]
        self.n_frames = len(frames)

    def read(self, k: int, out: np.ndarray | None = None):
        pos = self._pos[k]
        if out is not None:
            out[...] = pos
            pos = out
        return pos, self._box[k], self._time[k]


# -- PDB ----------------------------------------------------------------------


def read_pdb(path) -> dict:
    """ATOM/HETATM records of the first model: names, resnames, elements (columns 77-78,
    else guessed from the name), positions (A), box from CRYST1 (A, degrees)."""
    names, resnames, elements, pos, resids = [], [], [], [], []
    box = np.zeros((3, 3), dtype=np.float32)
    with open(path) as fh:
        for ln in fh:
            rec = ln[:6].strip()
            if rec == "CRYST1":
                a, b, c = float(ln[6:15]), float(ln[15:24]), float(ln[24:33])
                al, be, ga = float(ln[33:40]), float(ln[40:47]), float(ln[47:54])
                box = box_from_lengths(a, b, c, al, be, ga)
            elif rec in ("ATOM", "HETATM"):
                name, res = ln[12:16].strip(), ln[17:20].strip()
                el = ln[76:78].strip() if len(ln) >= 78 else ""
                names.append(name)
                resnames.append(res)
                resids.append(int(ln[22:26]))
                elements.append(el[0].upper() + el[1:].lower() if el else guess_element(name, res))
                pos.append((float(ln[30:38]), float(ln[38:46]), float(ln[46:54])))
            elif rec == "ENDMDL":
                break
    return {"names": names, "resnames": resnames, "resids": resids, "elements": elements,
            "positions": np.asarray(pos, dtype=np.float32).reshape(-1, 3), "box": box}


# -- binary trajectories --------------------------------------------------------


class NativeTrajectory:
    """GROMACS TRR or XTC, or CHARMM/NAMD DCD, through the library's native readers."""

    def __init__(self, path, fmt: int = 0):
        self.lib = _native.load()
        self._h = ctypes.c_void_p()
        _native.check(self.lib.saxs_traj_open(str(path).encode(), fmt, ctypes.byref(self._h)))
        n = ctypes.c_int()
        f = ctypes.c_longlong()
        _native.check(self.lib.saxs_traj_info(self._h, ctypes.byref(n), ctypes.byref(f)))
        self.n_atoms = n.value
        self.n_frames = f.value

    def read(self, k: int, out: np.ndarray | None = None):
        """Frame k: (positions (N, 3) A, box (3, 3) A, time ps); `out` receives the positions."""
        if out is None:
            out = np.empty((self.n_atoms, 3), dtype=np.float32)
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.shape != (self.n_atoms, 3):
            raise ValueError("out must be a C-contiguous float32 array of shape (natoms, 3)")
        t = ctypes.c_double()
        box = np.empty(9, dtype=np.float32)
        # pread-based: concurrent reads of other frames on this handle are safe
        _native.check(self.lib.saxs_traj_read(
            self._h, int(k), out.ctypes.data_as(_native.c_float_p),
            box.ctypes.data_as(_native.c_float_p), ctypes.byref(t)))
        return out, box.reshape(3, 3), t.value

    def close(self):
        if self._h:
            self.lib.saxs_traj_close(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class NpyTrajectory:
    """Coordinates memory-mapped from a .npy file (frames, natoms, 3) float32 Angstrom."""

    def __init__(self, path, box, dt_ps: float = 1.0):
        self._x = np.load(path, mmap_mode="r")
        if self._x.ndim != 3 or self._x.shape[2] != 3:
            raise ValueError("coordinates must have shape (frames, natoms, 3)")
        self.n_frames, self.n_atoms = int(self._x.shape[0]), int(self._x.shape[1])
        b = np.asarray(box, dtype=np.float32)
        self._box = np.broadcast_to(b.reshape(-1, 3, 3), (self.n_frames, 3, 3)) if b.size in (9, 9 * self.n_frames) \
            else None
        if self._box is None:
            raise ValueError("box must be (3, 3) or (frames, 3, 3)")
        self.dt = dt_ps

    def read(self, k: int, out: np.ndarray | None = None):
        src = self._x[k]
        if out is None:
            out = np.array(src, dtype=np.float32)
        else:
            np.copyto(out, src, casting="same_kind")
        return out, np.array(self._box[k]), k * self.dt


def open_trajectory(path, box=None):
    """A reader for `path` by extension: .trr/.xtc/.dcd native, .gro text, .npy memory-mapped."""
    ext = Path(path).suffix.lower()
    if ext in (".trr", ".xtc", ".dcd"):
        return NativeTrajectory(path)
    if ext == ".gro":
        return GroTrajectory(path)
    if ext == ".npy":
        if box is None:
            raise ValueError("a .npy trajectory needs a box")
        return NpyTrajectory(path, box)
    raise ValueError(f"unsupported trajectory format {ext!r} (supported: .trr .xtc .dcd .gro .npy)")


def read_topology(path) -> dict:
    ext = Path(path).suffix.lower()
    if ext == ".gro":
        return read_gro(path)
    if ext == ".pdb":
        return read_pdb(path)
    raise ValueError(f"unsupported topology format {ext!r} (supported: .gro .pdb)")


# -- the reference's topology contract --------------------------------------------

# standard atomic masses (g/mol) for the densities of stored profiles
_MASS = {"H": 1.008, "C": 12.011, "N": 14.007, "O": 15.999, "P": 30.974, "S": 32.06, "Na": 22.990,
         "Cl": 35.45, "K": 39.098, "Ca": 40.078, "Mg": 24.305, "Zn": 65.38, "Fe": 55.845,
         "F": 18.998, "Br": 79.904, "I": 126.904, "Li": 6.94, "Cu": 63.546, "Mn": 54.938, "Se": 78.971}
_WATER_RES = {"SOL", "HOH", "WAT", "TIP3", "TIP4", "TIP5", "SPC", "H2O", "T3P", "T4P"}
_ION_RES = {"NA": "Na", "NA+": "Na", "SOD": "Na", "CL": "Cl", "CL-": "Cl", "CLA": "Cl", "K": "K",
            "K+": "K", "POT": "K", "CA": "Ca", "CAL": "Ca", "MG": "Mg", "MG2": "Mg"}


class FileTopology:
    """Topology + trajectory from files, with the callback contract the drop-in
    ``pycusaxs_cuda.run`` uses (get_atom_index, read_frame, get_box, get_time,
    get_step, iter_frames_stream, n_frames, n_atoms)."""

    def __init__(self, topology, trajectory=None, box=None, prefetch: int = 4):
        top = read_topology(topology)
        self.elements = top["elements"]
        self.resnames = top["resnames"]
        self.resids = top["resids"]
        self.traj = open_trajectory(trajectory if trajectory is not None else topology,
                                    box=box if box is not None else top["box"])
        if self.traj.n_atoms != len(self.elements):
            raise ValueError(f"topology has {len(self.elements)} atoms, trajectory {self.traj.n_atoms}")
        self.prefetch = max(3, int(prefetch))
        self._cur = None

    @property
    def n_frames(self) -> int:
        return self.traj.n_frames

    @property
    def n_atoms(self) -> int:
        return self.traj.n_atoms

    def get_system_info(self) -> dict:
        """System description for the profile store (the keys the reference's
        Topology.get_system_info provides, topology.py:288-450): atom count, box
        edge lengths and volume of the first frame (A, A^3), waters (by residue
        name, counted by their oxygens), ions by residue, other residues, density
        (g/cm^3) and the time between frames (ps)."""
        pos, box, t0 = self.traj.read(0)
        lengths = np.linalg.norm(np.asarray(box, np.float64), axis=1)
        volume = abs(float(np.linalg.det(np.asarray(box, np.float64))))
        n_water, ions, other, water_atoms = 0, {}, {}, []
        seen = set()
        for i, (res, el, rid) in enumerate(zip(self.resnames, self.elements, self.resids)):
            r = res.upper()
            if r in _WATER_RES:
                if el == "O":
                    n_water += 1
                water_atoms.append(i)
            elif r in _ION_RES:
                ions[_ION_RES[r]] = ions.get(_ION_RES[r], 0) + 1
            elif (rid, res) not in seen:  # one count per residue
                seen.add((rid, res))
                other[res] = other.get(res, 0) + 1
        per_water = len(water_atoms) / n_water if n_water else 0
        model = {3: "TIP3P/SPC", 4: "TIP4P", 5: "TIP5P"}.get(int(round(per_water)), "") if n_water else ""
        mass = sum(_MASS.get(e, 0.0) for e in self.elements)
        dt = 0.0
        if self.n_frames > 1:
            dt = float(self.traj.read(1)[2] - t0)
        return {"n_atoms": self.n_atoms, "box_x": float(lengths[0]), "box_y": float(lengths[1]),
                "box_z": float(lengths[2]), "box_volume": volume, "n_water_molecules": n_water,
                "ion_counts": ions, "other_molecules": other, "detected_water_model": model,
                "density_g_cm3": mass / (volume * 0.602214076) if volume > 0 else None, "dt": dt}

    def get_atom_index(self) -> dict:
        out: dict[str, list[int]] = {}
        for i, el in enumerate(self.elements):
            out.setdefault(el, []).append(i)
        return out

    def read_frame(self, frame_number: int):
        if not 0 <= frame_number < self.n_frames:
            raise IndexError(f"Frame {frame_number} out of range [0, {self.n_frames})")
        pos, box, t = self.traj.read(frame_number)
        self._cur = (frame_number, pos, box, t)
        return self._cur

    def _need(self):
        if self._cur is None:
            raise RuntimeError("Call read_frame() before get_box()")
        return self._cur

    def get_box(self) -> np.ndarray:
        return self._need()[2]

    def get_time(self) -> float:
        return self._need()[3]

    def get_step(self) -> int:
        return self._need()[0]

    def get_coordinates(self) -> np.ndarray:
        return self._need()[1]

    def iter_frames_stream(self, start: int, stop: int, step: int = 1, **_ignored) -> Iterator[dict]:
        """Frames start, start+step, ... < stop (stop clipped to n_frames), read ahead
        by a background thread into a ring of `prefetch` buffers.  A yielded
        frame's arrays stay valid until the next frame is requested."""
        frames = range(max(0, start), min(stop, self.n_frames), max(1, step))
        ring = [np.empty((self.n_atoms, 3), dtype=np.float32) for _ in range(self.prefetch)]
        for k, (pos, box, t) in _read_ahead(self.traj, frames, ring):
            yield {"frame": k, "time": t, "positions": pos, "box": box}


def _read_ahead(traj, frames, ring):
    """Yield (k, (positions, box, time)) for k in `frames`, reading ahead into `ring`."""
    import queue

    # the reader fills at most len(ring) - 1 frames past the one the consumer
    # holds: len(ring) - 2 queued plus the one being read
    q: "queue.Queue" = queue.Queue(maxsize=len(ring) - 2)
    stop = threading.Event()

    def work():
        try:
            for i, k in enumerate(frames):
                if stop.is_set():
                    return
                q.put((k, traj.read(k, out=ring[i % len(ring)])))
            q.put(None)
        except BaseException as e:  # surfaced in the consumer
            q.put(e)

    th = threading.Thread(target=work, daemon=True)
    th.start()
    try:
        while True:
            item = q.get()
            if item is None:
                return
            if isinstance(item, BaseException):
                raise item
            yield item
    finally:
        stop.set()
        while th.is_alive():
            try:
                q.get_nowait()
            except Exception:
                pass
            th.join(timeout=0.05)


class BatchStream:
    """Consecutive batches of `frames` read by a thread into two pinned host buffers.

    Iterating yields (slot, buffer, boxes (n, 3, 3), n); after the consumer has
    queued its use of `buffer` (e.g. an asynchronous host-to-device copy) it calls
    ``release(slot, event)`` with a CUDA event recorded after that use.  The
    reader refills a buffer only after it was released and its event completed,
    so one batch is read while the previous one is copied and processed.
    """

    def __init__(self, traj, frames, batch: int, pinned_buffers, readers: int = 4):
        import queue
        from concurrent.futures import ThreadPoolExecutor

        self.traj = traj
        # frames of a batch are read in parallel (the native reader uses pread and
        # releases the GIL); other readers are read by one thread
        self._pool = ThreadPoolExecutor(max_workers=max(1, readers)) \
            if isinstance(traj, NativeTrajectory) and readers > 1 else None
        self.frames = list(frames)
        self.batch = int(batch)
        self.buffers = pinned_buffers
        self._ready: "queue.Queue" = queue.Queue()
        self._free: "queue.Queue" = queue.Queue()
        for slot in range(len(pinned_buffers)):
            self._free.put((slot, None))
        self._thread = threading.Thread(target=self._work, daemon=True)
        self._thread.start()

    def _work(self):
        try:
            for i in range(0, len(self.frames), self.batch):
                ks = self.frames[i:i + self.batch]
                slot, event = self._free.get()
                if slot is None:
                    return
                if event is not None:
                    event.synchronize()
                buf = self.buffers[slot].numpy()
                boxes = np.empty((len(ks), 3, 3), dtype=np.float32)
                if self._pool is not None:
                    res = list(self._pool.map(lambda jk: self.traj.read(jk[1], out=buf[jk[0]]),
                                              enumerate(ks)))
                else:
                    res = [self.traj.read(k, out=buf[j]) for j, k in enumerate(ks)]
                for j, (_, b, _) in enumerate(res):
                    boxes[j] = b
                self._ready.put((slot, boxes, len(ks)))
            self._ready.put(None)
        except BaseException as e:
            self._ready.put(e)

    def release(self, slot: int, event=None) -> None:
        self._free.put((slot, event))

    def __iter__(self):
        while True:
            item = self._ready.get()
            if item is None:
                break
            if isinstance(item, BaseException):
                raise item
            slot, boxes, n = item
            yield slot, self.buffers[slot], boxes, n

    def close(self) -> None:
        self._free.put((None, None))
        self._thread.join(timeout=5)
        if self._pool is not None:
            self._pool.shutdown(wait=True)
