"""Seeded synthetic systems and a topology object that serves them.

There is no trajectory data in this project, so workloads are synthetic:
uniform (or slab-modulated) atoms with a fixed element mix, and frames that
are the first frame plus independent Gaussian jitter.  Units are Angstrom.

``SyntheticTopology`` implements the duck type that the reference's C++ side
calls back into (pycusaxs/topology.py:273-286, 536-577, 621-737):
``get_atom_index()``, ``read_frame(i)``, ``get_box()`` and
``iter_frames_stream(start, stop, step)`` yielding dicts with ``frame``,
``time``, ``positions`` (N, 3) float32 and ``box`` (3, 3).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

MIX_STANDARD = (("H", 0.60), ("C", 0.25), ("O", 0.08), ("N", 0.05), ("S", 0.01), ("P", 0.01))
MIX_LARGE = (("H", 0.55), ("C", 0.30), ("O", 0.10), ("N", 0.03), ("P", 0.02))


@dataclass
class System:
    """Atoms, element of each atom, box rows (3, 3) and the frames' jitter."""

    elements: np.ndarray            # (N,) object array of element symbols
    positions: np.ndarray           # (N, 3) float32, frame 0
    box: np.ndarray                 # (3, 3) float32 rows a, b, c
    jitter: float = 0.0             # Angstrom, per atom per frame
    seed: int = 0
    nframes: int = 1
    _cache: dict = field(default_factory=dict, repr=False)

    @property
    def natoms(self) -> int:
        return int(self.positions.shape[0])

    def atom_index(self) -> dict:
        out: dict[str, list[int]] = {}
        for i, e in enumerate(self.elements):
            out.setdefault(str(e), []).append(i)
        return out

    def type_of_atom(self, names) -> np.ndarray:
        lut = {n: i for i, n in enumerate(names)}
        return np.array([lut.get(str(e), -1) for e in self.elements], dtype=np.int32)

    def frame(self, k: int) -> np.ndarray:
        """Positions of frame k: frame 0 plus N(0, jitter) per coordinate (seeded per k)."""
        if k == 0 or self.jitter == 0.0:
            return self.positions
        rng = np.random.default_rng([self.seed, 1, k])
        return (self.positions + rng.normal(0.0, self.jitter, self.positions.shape)).astype(np.float32)

    def frames(self, start: int, stop: int) -> np.ndarray:
        return np.stack([self.frame(k) for k in range(start, stop)])


def _elements(rng, n, mix):
    names = np.array([m[0] for m in mix], dtype=object)
    p = np.array([m[1] for m in mix], dtype=np.float64)
    return names[rng.choice(len(mix), size=n, p=p / p.sum())]


def cubic_system(natoms: int, box: float, *, seed: int = 0, mix=MIX_STANDARD, jitter: float = 0.0,
                 nframes: int = 1) -> System:
    """Atoms uniform in a cubic periodic box of edge ``box`` Angstrom."""
    rng = np.random.default_rng(seed)
    pos = rng.uniform(0.0, box, size=(natoms, 3)).astype(np.float32)
    return System(_elements(rng, natoms, mix), pos, np.diag([box] * 3).astype(np.float32),
                  jitter=jitter, seed=seed, nframes=nframes)


def orthorhombic_system(natoms: int, lengths, *, seed: int = 0, mix=MIX_STANDARD,
                        jitter: float = 0.0, nframes: int = 1) -> System:
    """Atoms uniform in an orthorhombic box with edges ``lengths`` (Angstrom)."""
    rng = np.random.default_rng(seed)
    L = np.asarray(lengths, dtype=np.float64)
    pos = (rng.uniform(0.0, 1.0, size=(natoms, 3)) * L).astype(np.float32)
    return System(_elements(rng, natoms, mix), pos, np.diag(L).astype(np.float32), jitter=jitter,
                  seed=seed, nframes=nframes)


def triclinic_slab_system(natoms: int, a: float, b: float, c: float, gamma_deg: float, *,
                          seed: int = 0, mix=MIX_LARGE, slab=(0.4, 0.6), slab_factor=1.5,
                          jitter: float = 0.0, nframes: int = 1) -> System:
    """Atoms in a triclinic cell (MDAnalysis lower-triangular rows), denser in a z slab.

    Fractional coordinates are sampled with density ``slab_factor`` times the
    background for fractional z inside ``slab``.
    """
    rng = np.random.default_rng(seed)
    g = math.radians(gamma_deg)
    box = np.array([[a, 0, 0], [b * math.cos(g), b * math.sin(g), 0], [0, 0, c]], dtype=np.float64)
    w_in = (slab[1] - slab[0]) * slab_factor
    w_out = 1.0 - (slab[1] - slab[0])
    n_in = int(round(natoms * w_in / (w_in + w_out)))
    fz_in = rng.uniform(slab[0], slab[1], n_in)
    fz_out = rng.uniform(0.0, w_out, natoms - n_in)
    fz_out = np.where(fz_out < slab[0], fz_out, fz_out + (slab[1] - slab[0]))
    fz = np.concatenate([fz_in, fz_out])
    rng.shuffle(fz)
    frac = np.stack([rng.uniform(0, 1, natoms), rng.uniform(0, 1, natoms), fz], axis=1)
    pos = (frac @ box).astype(np.float32)
    return System(_elements(rng, natoms, mix), pos, box.astype(np.float32), jitter=jitter,
                  seed=seed, nframes=nframes)


# The five workloads (sizes in Angstrom and 1/Angstrom; 1 nm = 10 A).
CONFIGS = {
    # 20k atoms, 6 nm box, grid 64, scale 2 (128^3 transform), q 0-5 /nm in 0.02 /nm bins
    "c1": dict(natoms=20_000, box=60.0, grid=64, scale=2.0, qcut=0.5, bin_size=0.002, frames=1,
               jitter=0.0),
    # 100k atoms, 12 nm box, grid 128, scale 2 (256^3), 100 frames with 0.05 nm jitter
    "c2": dict(natoms=100_000, box=120.0, grid=128, scale=2.0, qcut=0.5, bin_size=0.002,
               frames=100, jitter=0.5),
    # 50k atoms, 10 nm box, grid 128, scale 2 (refinement workload)
    "c5": dict(natoms=50_000, box=100.0, grid=128, scale=2.0, qcut=0.5, bin_size=0.002, frames=1,
               jitter=0.0),
}


def make_config(name: str, seed: int = 0) -> tuple[System, dict]:
    c = dict(CONFIGS[name])
    s = cubic_system(c["natoms"], c["box"], seed=seed, jitter=c["jitter"], nframes=c["frames"])
    return s, c


def large_triclinic(seed: int = 0, natoms: int = 1_000_000, frames: int = 20) -> tuple[System, dict]:
    """1M atoms, 25x25x20 nm cell with gamma = 80 deg, slab 1.5x dense at z in 0.4-0.6."""
    s = triclinic_slab_system(natoms, 250.0, 250.0, 200.0, 80.0, seed=seed, jitter=0.5,
                              nframes=frames)
    return s, dict(natoms=natoms, grid=256, scale=2.0, qcut=0.4, bin_size=0.001, frames=frames,
                   jitter=0.5)


def uneven_systems(n_systems: int = 64, frames: int = 8, seed: int = 0, nmin: int = 5_000,
                   nmax: int = 200_000, density: float = 0.1,
                   grids=(48, 64, 96, 128, 160)) -> list[tuple[System, int]]:
    """Independent cubic systems with log-uniform atom counts in [nmin, nmax].

    Box edge L = (N / density)^(1/3) A (density 0.1 /A^3 = 100 atoms/nm^3); the
    grid is the smallest of ``grids`` not below L (about 1 A spacing).
    Returns [(system, grid)].
    """
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n_systems):
        n = int(round(math.exp(rng.uniform(math.log(nmin), math.log(nmax)))))
        L = (n / density) ** (1.0 / 3.0)
        grid = next((g for g in grids if g >= L), grids[-1])
        s = cubic_system(n, L, seed=10_000 * (seed + 1) + i, jitter=0.5, nframes=frames)
        out.append((s, grid))
    return out


class SyntheticTopology:
    """Topology duck type over a ``System`` (the reference's callback contract)."""

    def __init__(self, system: System, dt_ps: float = 1.0, fail_at_frame: int | None = None,
                 frames=None):
        """``frames``: the positions of every frame, precomputed ((F, N, 3)
        float32); default: each frame generated from the seed when it is read."""
        self.system = system
        self.n_frames = system.nframes if frames is None else len(frames)
        self.dt = dt_ps
        self.ts = None
        self.fail_at_frame = fail_at_frame
        self.frames = frames

    def get_atom_index(self):
        return self.system.atom_index()

    def read_frame(self, frame_number: int):
        if not 0 <= frame_number < self.n_frames:
            raise IndexError(f"Frame {frame_number} out of range [0, {self.n_frames})")
        self.ts = frame_number
        return self.ts

    def get_box(self):
        if self.ts is None:
            raise RuntimeError("Call read_frame() before get_box()")
        return self.system.box.astype(np.float32)

    def iter_frames_stream(self, start: int, stop: int, step: int = 1, **_):
        for k in range(start, min(stop, self.n_frames), step):
            if self.fail_at_frame is not None and k == self.fail_at_frame:
                raise RuntimeError(f"synthetic read failure at frame {k}")
            pos = self.system.frame(k) if self.frames is None else self.frames[k]
            yield {"frame": k, "time": k * self.dt, "positions": pos,
                   "box": self.system.box.astype(np.float32)}
