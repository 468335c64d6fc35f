"""FP64 CPU oracle of the reference's per-frame SAXS path.

TEST INFRASTRUCTURE ONLY.  This module restates, in NumPy (plus a small C
helper for the float32 bin rule, ``oracle/csrc/oracle_bins.c``), the algorithm
of the reference cudaSAXS so that tests, ``__graft_entry__.smoke()`` and the
``cpu_baseline`` leg of ``bench.py`` can check and time the CUDA product.  The
product never imports it.

What is restated, and where it comes from (reference paths):

* grid sizing ``find_closest_product``          saxsKernel.cu:377-469
* inverse cell ``cell_matrices`` (3x3 overload) System/Cell.cpp:111-126
* Delta-q / q-cut reset ``histogram_parameters`` saxsKernel.cu:489-526, :247
* B-spline weights ``bspline_weights``           Saxs/Splines.cu:11-73
* B-spline moduli ``bspmod``                     Utilities/BSpmod.cpp:45-129
* spreading ``spread``                           saxsDeviceKernels.cu:338-398
* z-border mean ``border_mean``                  saxsDeviceKernels.cu:446-465,
                                                 saxsKernel.cu:68-70,150-162
* supercell ``supercell``                        saxsDeviceKernels.cu:413-429
* R2C transform                                  saxsKernel.cu:171 (cuFFT R2C ==
                                                 numpy rfftn on (nnx, nny, nnz))
* form factor ``form_factor``                    Saxs/opsfact.cu:30-35
* type sum, qcut mask                            saxsDeviceKernels.cu:177-216
* modulus                                        saxsDeviceKernels.cu:142-162
* histogram with mirror weighting                saxsDeviceKernels.cu:9-125
* npt/nvt accumulation                           saxsKernel.cu:184-196, :17-39
* profile rows and file format                   saxsKernel.cu:210-225,
                                                 Exec/RunSaxs.cu:224-228

Arithmetic: coordinates are mapped to grid units with the reference's float32
steps (so atoms land in the same cells), the bin index of every k-point uses
the reference's float32 rule, and everything else (spline weights, grids,
transform, form factors, intensities, histogram) is FP64.
"""
from __future__ import annotations

import ctypes
import json
import math
import os
import subprocess
from dataclasses import dataclass, field
from pathlib import Path

import numpy as np

_HERE = Path(__file__).resolve().parent
_REPO = _HERE.parent
FORM_FACTOR_JSON = _REPO / "pycusaxs_b200" / "data" / "it1992.json"

# Contraction mode of the float32 bin rule (see oracle/csrc/oracle_bins.c).
# Pinned against the reference's compiled kernel by tests/test_gpu_bins.py.
DEFAULT_CONTRACTION = 1

# Threads of the FP64 R2C transform (scipy's pocketfft; numpy's rfftn, the same
# algorithm single-threaded, when scipy is absent).  None: every host core.
FFT_WORKERS: int | None = None

SHELL = np.float32(0.07)  # include/Parameters.h:8
KCUT = 50                 # Utilities/BSpmod.h:22
TINY = np.float32(1.0e-7)  # Utilities/BSpmod.cpp:21


# --------------------------------------------------------------------------
# C helper
# --------------------------------------------------------------------------
_LIB = None


def _lib():
    """Load (building on first use with gcc) the C restatement of the bin rule."""
    global _LIB
    if _LIB is not None:
        return _LIB
    out_dir = _HERE / "_lib"
    so = out_dir / "liboracle_bins.so"
    src = _HERE / "csrc" / "oracle_bins.c"
    if not so.exists() or so.stat().st_mtime < src.stat().st_mtime:
        build_c_helper()
    lib = ctypes.CDLL(str(so))
    i64, i32p, f32p = ctypes.c_int64, ctypes.POINTER(ctypes.c_int32), ctypes.POINTER(ctypes.c_float)
    lib.oracle_bins.restype = i64
    lib.oracle_bins.argtypes = [i64, i32p, i32p, i32p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                f32p, ctypes.c_float, ctypes.c_float, ctypes.c_int, ctypes.c_int,
                                f32p, i32p]
    lib.oracle_grid_coords.restype = None
    lib.oracle_grid_coords.argtypes = [i64, f32p, f32p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, f32p]
    _LIB = lib
    return lib


def build_c_helper() -> Path:
    out_dir = _HERE / "_lib"
    out_dir.mkdir(exist_ok=True)
    so = out_dir / "liboracle_bins.so"
    src = _HERE / "csrc" / "oracle_bins.c"
    tmp = out_dir / f".liboracle_bins.{os.getpid()}.so"
    subprocess.run(["gcc", "-O2", "-ffp-contract=off", "-fPIC", "-shared", str(src), "-o", str(tmp),
                    "-lm"], check=True)
    os.replace(tmp, so)
    return so


def _ptr(a, ctype):
    return a.ctypes.data_as(ctypes.POINTER(ctype))


# --------------------------------------------------------------------------
# setup numerics
# --------------------------------------------------------------------------
def load_form_factors() -> dict[str, np.ndarray]:
    """Element -> 9 float32 coefficients (a1..a4, b1..b4, c), Scattering.cpp:9-189."""
    raw = json.loads(FORM_FACTOR_JSON.read_text())
    return {k: np.array([float(v) for v in vals], dtype=np.float32) for k, vals in raw.items()}


def generate_multiples(limit: int) -> list[int]:
    """All 2^a 3^b 5^c 7^d <= limit, sorted (saxsKernel.cu:377-436)."""
    out = set()
    p2 = 1
    while p2 <= limit:
        p3 = p2
        while p3 <= limit:
            p5 = p3
            while p5 <= limit:
                p7 = p5
                while p7 <= limit:
                    out.add(p7)
                    p7 *= 7
                p5 *= 5
            p3 *= 3
        p2 *= 2
    return sorted(out)


def find_closest_product(n: int, sigma: float) -> int:
    """Nearest 2^a3^b5^c7^d to round(n*sigma), ties to the smaller (saxsKernel.cu:449-469)."""
    prod = np.float32(n) * np.float32(sigma)
    target = int(math.floor(abs(float(prod)) + 0.5)) * (1 if prod >= 0 else -1)  # std::round
    closest, best = target, None
    for m in generate_multiples(2 * target):
        d = abs(m - target)
        if best is None or d < best:
            best, closest = d, m
    return closest


def cell_matrices(box, box_mode: int = 0) -> tuple[np.ndarray, np.ndarray]:
    """co (the box rows) and oc from the upper triangle only (Cell.cpp:111-126);
    with box_mode 1 (the opt-in triclinic extension, no reference counterpart)
    oc is the full inverse-transpose H^-T computed in double."""
    co = np.asarray(box, dtype=np.float32).reshape(3, 3)
    if box_mode == 1:
        return co, np.linalg.inv(co.astype(np.float64)).T.astype(np.float32)
    f = np.float32
    oc = np.zeros((3, 3), dtype=np.float32)
    oc[0, 0] = f(1.0 / float(co[0, 0]))
    oc[0, 1] = f(-co[0, 1] / (co[0, 0] * co[1, 1]))
    oc[0, 2] = f((co[0, 1] * co[1, 2] - co[0, 2] * co[1, 1]) / (co[0, 0] * co[1, 1] * co[2, 2]))
    oc[1, 1] = f(1.0 / float(co[1, 1]))
    oc[1, 2] = f(-co[1, 2] / (co[1, 1] * co[2, 2]))
    oc[2, 2] = f(1.0 / float(co[2, 2]))
    return co, oc


def nf_of(n: int) -> int:
    return n // 2 if n % 2 == 0 else n // 2 + 1


def histogram_parameters(nn, oc, sigma, dq, qcut):
    """Effective (Delta-q, q-cut, num_bins) after the reset of saxsKernel.cu:489-526, :247."""
    f = np.float32
    two_pi = f(2.0) * f(math.pi)
    args = [f(two_pi * oc[d, d]) / f(sigma) for d in range(3)]
    fx = [f(nf_of(nn[d]) - 1) for d in range(3)]
    dq0 = [args[0], args[1], args[2], f(dq)]
    cut0 = [f(args[0] * fx[0]), f(args[1] * fx[1]), f(args[2] * fx[2]), f(qcut)]
    dq_eff = max(dq0)
    qcut_eff = min(cut0)
    num_bins = int(f(qcut_eff / dq_eff)) + 1
    return f(dq_eff), f(qcut_eff), num_bins


def bspline_weights(w, order: int = 4):
    """Cardinal B-spline weights x[0..order-1] by the recurrence of Splines.cu:11-73.

    ``w`` may be an array.  Returns (x, dx) with x.shape == (order, *w.shape);
    dx are the derivative weights taken before the last pass (Splines.cu:48-56).
    """
    w = np.asarray(w, dtype=np.float64)
    x = np.zeros((order,) + w.shape)
    dx = np.zeros((order,) + w.shape)
    x[0] = 1.0 - w
    if order > 1:
        x[1] = w

    def one_pass(k1):
        k = k1 + 1
        div = 1.0 / (k - 1)
        x[k - 1] = div * w * x[k - 2]
        for j in range(1, k - 1):
            x[k - j - 1] = div * ((w + j) * x[k - j - 2] + (k - j - w) * x[k - j - 1])
        x[0] = div * (1.0 - w) * x[0]

    for o in range(2, order - 1):
        one_pass(o)
    dx[0] = -x[0]
    for o in range(1, order):
        dx[o] = x[o - 1] - x[o]
    if order >= 2:
        one_pass(order - 1)
    return x, dx


def stencil_weights(g, order: int):
    """Per-tap weights the reference spreads with for a given ``order``.

    The device splines are always evaluated at order 4 (Splines.h:16,
    saxsDeviceKernels.cu:343-345) while the spreading loop runs ``order`` taps
    (:373-395).  Taps 0..min(order,4)-1 take the cubic weights; taps 4.. are
    left unwritten by the reference and are defined here as zero.
    Returns (w, dw) of shape (order, *g.shape).
    """
    x4, dx4 = bspline_weights(g, 4)
    w = np.zeros((order,) + np.shape(g))
    dw = np.zeros((order,) + np.shape(g))
    m = min(order, 4)
    w[:m] = x4[:m]
    dw[:m] = dx4[:m]
    return w, dw


def bspmod(n: int, ndim: int | None = None) -> np.ndarray:
    """Inverse B-spline moduli along one axis (BSpmod.cpp:45-129), FP64."""
    order = 4  # BSpline::order is static 4 (BSpline.cpp:12)
    ndim = max(ndim or n, order + 1)
    d, _ = bspline_weights(np.float64(0.0), order)
    a0 = np.zeros(ndim)
    a0[1:order + 1] = d[:order]
    o = np.arange(n)[:, None]
    p = np.arange(order + 1)[None, :]
    arg = 2.0 * math.pi * (o * p) / n
    s1 = (a0[:order + 1][None, :] * np.cos(arg)).sum(axis=1)
    s2 = (a0[:order + 1][None, :] * np.sin(arg)).sum(axis=1)
    bsp = s1 * s1 + s2 * s2
    for k in range(1, n - 1):
        if not bsp[k] > float(TINY):
            bsp[k] = 0.5 * (bsp[k - 1] + bsp[k + 1])
    nf = n // 2

    def gsum(m, p):
        x = math.pi * m / n
        s = 1.0
        for k in range(1, KCUT + 1):
            s += (x / (x + math.pi * k)) ** p + (x / (x - math.pi * k)) ** p
        return s

    for k in range(n):
        m = k if k < nf else k - n
        if m != 0:
            lam = gsum(m, order) / gsum(m, 2 * order)
            bsp[k] /= lam * lam
    return 1.0 / bsp


def border_planes(nz: int) -> np.ndarray:
    """Boolean mask over z of the padding border (saxsKernel.h:107-110, saxsDeviceKernels.cu:453-462)."""
    dz = int(SHELL * np.float32(nz) / np.float32(2))
    z = np.arange(nz)
    return ~((z > dz) & (z < nz - dz))


# --------------------------------------------------------------------------
# per-frame pieces
# --------------------------------------------------------------------------
def grid_coords(xyz, oc, n, mode: int = DEFAULT_CONTRACTION) -> np.ndarray:
    """Float32 grid coordinates r = n * frac(oc . x) per saxsDeviceKernels.cu:355-361."""
    xyz = np.ascontiguousarray(xyz, dtype=np.float32).reshape(-1, 3)
    ocf = np.ascontiguousarray(oc, dtype=np.float32).reshape(9)
    out = np.empty_like(xyz)
    _lib().oracle_grid_coords(xyz.shape[0], _ptr(xyz, ctypes.c_float), _ptr(ocf, ctypes.c_float),
                              int(n[0]), int(n[1]), int(n[2]), mode, _ptr(out, ctypes.c_float))
    return out


def stencil(r, n, order):
    """Per-atom tap indices and weights along each axis (saxsDeviceKernels.cu:362-389)."""
    r = np.asarray(r, dtype=np.float32)
    m = r.astype(np.int64)  # static_cast<int>, r >= 0
    g = (r - m.astype(np.float32)).astype(np.float64)
    idx, wts, dws = [], [], []
    for d in range(3):
        w, dw = stencil_weights(g[:, d], order)
        taps = m[:, d][None, :] - order + np.arange(order)[:, None]
        taps = np.where(taps >= 0, taps, taps + n[d])
        idx.append(taps)
        wts.append(w)
        dws.append(dw)
    return idx, wts, dws


def spread(r, n, order) -> np.ndarray:
    """FP64 density grid (nx, ny, nz) of one type from grid coordinates ``r``."""
    nx, ny, nz = (int(v) for v in n)
    if r.shape[0] == 0:
        return np.zeros((nx, ny, nz))
    (ix, iy, iz), (wx, wy, wz), _ = stencil(r, n, order)
    flat = (ix[:, None, None, :] * ny + iy[None, :, None, :]) * nz + iz[None, None, :, :]
    w = wx[:, None, None, :] * wy[None, :, None, :] * wz[None, None, :, :]
    grid = np.bincount(flat.ravel(), weights=w.ravel(), minlength=nx * ny * nz)
    return grid.reshape(nx, ny, nz)


def border_mean(grid) -> float:
    mask = border_planes(grid.shape[2])
    sel = grid[:, :, mask]
    return float(sel.sum() / sel.size)


def supercell(grid, mean, nn) -> np.ndarray:
    sup = np.full(tuple(int(v) for v in nn), mean, dtype=np.float64)
    ex = [min(grid.shape[d], int(nn[d])) for d in range(3)]
    sup[:ex[0], :ex[1], :ex[2]] = grid[:ex[0], :ex[1], :ex[2]]
    return sup


def fft_workers() -> int:
    return int(FFT_WORKERS) if FFT_WORKERS else (os.cpu_count() or 1)


def rfftn(a) -> np.ndarray:
    """Unnormalised FP64 R2C transform over all axes (the half spectrum along the
    last axis), as cuFFT's R2C at saxsKernel.cu:171."""
    try:
        import scipy.fft as sf
    except ImportError:
        return np.fft.rfftn(a)
    return sf.rfftn(a, workers=fft_workers())


def form_factor(q, coeffs) -> np.ndarray:
    """f(q) = sum_i a_i exp(-b_i (q/4pi)^2) + c  (opsfact.cu:30-35), FP64."""
    c = np.asarray(coeffs, dtype=np.float64)
    s2 = (np.asarray(q, dtype=np.float64) / (4.0 * math.pi)) ** 2
    return (c[0] * np.exp(-c[4] * s2) + c[1] * np.exp(-c[5] * s2) + c[2] * np.exp(-c[6] * s2)
            + c[3] * np.exp(-c[7] * s2) + c[8])


def kpoint_bins(nn, ocs, bin_size, qcut, num_bins, mode: int = DEFAULT_CONTRACTION):
    """Float32 |q| and bin (or -1) of every half-spectrum point, shape (nnx, nny, nnz//2+1)."""
    nnx, nny, nnz = (int(v) for v in nn)
    npz = nnz // 2 + 1
    i, j, k = np.meshgrid(np.arange(nnx, dtype=np.int32), np.arange(nny, dtype=np.int32),
                          np.arange(npz, dtype=np.int32), indexing="ij")
    i, j, k = (np.ascontiguousarray(a.ravel()) for a in (i, j, k))
    mw = np.empty(i.size, dtype=np.float32)
    b = np.empty(i.size, dtype=np.int32)
    ocf = np.ascontiguousarray(ocs, dtype=np.float32).reshape(9)
    _lib().oracle_bins(i.size, _ptr(i, ctypes.c_int32), _ptr(j, ctypes.c_int32),
                       _ptr(k, ctypes.c_int32), nnx, nny, nnz, _ptr(ocf, ctypes.c_float),
                       np.float32(bin_size), np.float32(qcut), int(num_bins), mode,
                       _ptr(mw, ctypes.c_float), _ptr(b, ctypes.c_int32))
    shape = (nnx, nny, npz)
    return mw.reshape(shape), b.reshape(shape)


def mirror_values(field3):
    """field3[(-i) % nnx, (-j) % nny, k] for every (i, j, k) (saxsDeviceKernels.cu:83-84,105)."""
    return np.roll(field3[::-1, ::-1, :], shift=(1, 1), axis=(0, 1))


def histogram(ivals, bins, num_bins, fact: float = 1.0):
    """Mirror-weighted FP64 histogram of saxsDeviceKernels.cu:9-125."""
    pair = ivals + mirror_values(ivals)
    pair[0, 0, 0] = ivals[0, 0, 0]
    cnt = np.full(ivals.shape, 2.0)
    cnt[0, 0, 0] = 1.0
    sel = bins >= 0
    hist = np.bincount(bins[sel], weights=(pair[sel] * fact), minlength=num_bins)[:num_bins]
    nhist = np.bincount(bins[sel], weights=cnt[sel], minlength=num_bins)[:num_bins]
    return hist, nhist


# --------------------------------------------------------------------------
# whole path
# --------------------------------------------------------------------------
@dataclass
class OraclePlan:
    """Setup of one run, as RunSaxs::Run does it (RunSaxs.cu:117-133)."""

    grid: tuple[int, int, int]
    types: list[str]                 # element names, sorted like std::map keys
    coeffs: np.ndarray               # (T, 9) float32 form-factor rows
    box0: np.ndarray                 # frame-0 box (3, 3)
    scaled_grid: tuple[int, int, int] = (0, 0, 0)
    order: int = 4
    sigma: float = 1.0
    bin_size: float = 0.0
    qcut: float = 0.0
    ensemble: str = "npt"
    contraction: int = DEFAULT_CONTRACTION
    box_mode: int = 0                # 1: triclinic extension (oc = H^-T, q from its transpose)
    padding: np.ndarray | None = None  # given padding per type (atoms per grid point)
    nn: tuple[int, int, int] = field(init=False)
    dq: np.float32 = field(init=False)
    kcut: np.float32 = field(init=False)
    num_bins: int = field(init=False)
    mod: tuple[np.ndarray, np.ndarray, np.ndarray] = field(init=False)

    def __post_init__(self):
        if any(self.scaled_grid):
            self.nn = tuple(int(v) for v in self.scaled_grid)
        else:
            self.nn = tuple(find_closest_product(int(n), self.sigma) for n in self.grid)
        _, oc0 = cell_matrices(self.box0, self.box_mode)
        self.dq, self.kcut, self.num_bins = histogram_parameters(self.nn, oc0, self.sigma,
                                                                 self.bin_size, self.qcut)
        ndim = max(self.nn)
        self.mod = tuple(bspmod(n, ndim) for n in self.nn)
        self.oc0 = oc0

    def scaled_oc(self, oc) -> np.ndarray:
        """sigma' * oc with sigma' = nx/nnx in float (saxsKernel.cu:71-79), as the
        map from k indices to q / 2 pi (rows); transposed in the triclinic mode."""
        s = np.float32(self.grid[0]) / np.float32(self.nn[0])
        m = (s * np.asarray(oc, dtype=np.float32)).astype(np.float32)
        return np.ascontiguousarray(m.T) if self.box_mode == 1 else m


def frame_intensity(plan: OraclePlan, xyz, type_of_atom, box, *, return_parts=False):
    """Modulus grid |sum_t f_t F_t|^2 * M over the half spectrum for one frame (FP64).

    ``type_of_atom[a]`` is the index into ``plan.types`` of atom a (or -1 to skip).
    """
    _, oc = cell_matrices(box, plan.box_mode)
    ocs = plan.scaled_oc(oc)
    nn = plan.nn
    mw, bins = kpoint_bins(nn, ocs, plan.dq, plan.kcut, plan.num_bins, plan.contraction)
    inside = ~(mw > plan.kcut)
    r = grid_coords(xyz, oc, plan.grid, plan.contraction)
    acc = np.zeros(mw.shape, dtype=np.complex128)
    means = []
    for t, _name in enumerate(plan.types):
        sel = np.nonzero(np.asarray(type_of_atom) == t)[0]
        g = spread(r[sel], plan.grid, plan.order)
        mean = border_mean(g) if plan.padding is None else float(plan.padding[t])
        means.append(mean)
        sup = supercell(g, mean, nn)
        ft = rfftn(sup)
        del sup
        f = form_factor(mw[inside], plan.coeffs[t])
        acc[inside] += f * ft[inside]
    modx, mody, modz = plan.mod
    npz = nn[2] // 2 + 1
    m3 = modx[:, None, None] * mody[None, :, None] * modz[None, None, :npz]
    ivals = (acc.real ** 2 + acc.imag ** 2) * m3
    if return_parts:
        return ivals, bins, {"means": means, "ocs": ocs, "mw": mw}
    return ivals, bins


def run_frames(plan: OraclePlan, frames, type_of_atom):
    """FP64 (hist, nhist) over frames [(xyz, box), ...] per the npt/nvt rules."""
    nb = plan.num_bins
    if plan.ensemble == "nvt":
        total = None
        for xyz, box in frames:
            iv, _ = frame_intensity(plan, xyz, type_of_atom, box)
            total = iv if total is None else total + iv
        ocs0 = plan.scaled_oc(plan.oc0)
        _, bins0 = kpoint_bins(plan.nn, ocs0, plan.dq, plan.kcut, nb, plan.contraction)
        fact = 1.0 / len(frames)
        return histogram(total, bins0, nb, fact)
    hist = np.zeros(nb)
    nhist = np.zeros(nb)
    for xyz, box in frames:
        iv, bins = frame_intensity(plan, xyz, type_of_atom, box)
        h, n = histogram(iv, bins, nb)
        hist += h
        nhist += n
    return hist, nhist


def profile_rows(hist, nhist, bin_size):
    """(q, I) rows o >= 1 with nhist != 0 (saxsKernel.cu:210-225)."""
    rows = []
    for o in range(1, len(hist)):
        if nhist[o] != 0.0:
            q = float(np.float32(o) * np.float32(bin_size))
            rows.append((q, hist[o] / nhist[o]))
    return rows


def format_rows(rows) -> str:
    """Text of the I(q) file: setw(10) fixed 5 then setw(12) scientific 5 (RunSaxs.cu:226-227)."""
    return "".join(f"{q:10.5f}{i:12.5e}\n" for q, i in rows)
