"""The float32 k-point bin rule, pinned exactly (GPU).

The reference bins every half-spectrum point with float32 arithmetic compiled
by nvcc (saxsDeviceKernels.cu:67-125).  Points whose |q| is a multiple of the
bin width sit on bin edges, so the result depends on the exact float steps
and on nvcc's fused multiply-adds.  Bin counts are integers, so they are
compared exactly: the CUDA path against the oracle's C restatement, and both
against the reference's own kernel (oracle/_ref/libref_kernels.so) when built.
"""
import ctypes

import numpy as np
import pytest

from helpers import engine_hist
from oracle import saxs_oracle as O
from pycusaxs_b200.synthetic import System

pytestmark = pytest.mark.gpu

GEOMS = [
    # (grid, box rows, sigma, qcut, bin)
    ((128, 128, 128), np.diag([120.0] * 3), 2.0, 0.5, 0.002),   # the 100k-atom workload
    ((64, 64, 64), np.diag([60.0] * 3), 2.0, 0.5, 0.002),
    ((48, 40, 56), np.diag([47.0, 41.5, 60.0]), 2.5, 0.9, 0.0),
    ((32, 32, 32), np.array([[36.0, 4.0, -3.0], [0.0, 40.0, 5.0], [0.0, 0.0, 44.0]]), 2.0, 0.8, 0.0),
    ((64, 64, 64), np.array([[250.0, 0, 0], [43.41204, 246.20193, 0], [0, 0, 200.0]]) / 4, 2.0, 0.4,
     0.001),
]


def _system(box, n=64, seed=0):
    rng = np.random.default_rng(seed)
    pos = (rng.uniform(0, 1, (n, 3)) @ np.asarray(box, np.float64)).astype(np.float32)
    return System(np.array(["C"] * n, dtype=object), pos, np.asarray(box, np.float32))


def _oracle_counts(grid, box, sigma, qcut, dq, mode):
    nn = tuple(O.find_closest_product(g, sigma) for g in grid)
    oc = O.cell_matrices(box)[1]
    dq_e, qc_e, nb = O.histogram_parameters(nn, oc, sigma, dq, qcut)
    ocs = (np.float32(grid[0]) / np.float32(nn[0]) * oc).astype(np.float32)
    _, bins = O.kpoint_bins(nn, ocs, dq_e, qc_e, nb, mode)
    _, n = O.histogram(np.zeros(bins.shape), bins, nb)
    return n, (nn, ocs, dq_e, qc_e, nb)


def _ref_counts(ref_dir, nn, ocs, dq, qc, nb):
    lib = ctypes.CDLL(str(ref_dir / "libref_kernels.so"))
    fp = ctypes.POINTER(ctypes.c_float)
    dp = ctypes.POINTER(ctypes.c_double)
    lib.ref_histogram.argtypes = [fp, fp, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_float,
                                  ctypes.c_float, ctypes.c_int, dp, dp]
    h = np.zeros(nb)
    n = np.zeros(nb)
    ireal = np.zeros(nn[0] * nn[1] * (nn[2] // 2 + 1), np.float32)
    o = np.ascontiguousarray(ocs.reshape(9), np.float32)
    rc = lib.ref_histogram(ireal.ctypes.data_as(fp), o.ctypes.data_as(fp), nn[0], nn[1], nn[2],
                           np.float32(dq), np.float32(qc), nb, h.ctypes.data_as(dp),
                           n.ctypes.data_as(dp))
    assert rc == 0
    return n


@pytest.mark.parametrize("geom", GEOMS, ids=range(len(GEOMS)))
def test_bin_counts_exact(cuda, geom):
    grid, box, sigma, qcut, dq = geom
    s = _system(box)
    _, n_gpu, eng = engine_hist(s, grid, [s.positions], sigma=sigma, qcut=qcut, bin_size=dq)
    eng.close()
    n_or, _ = _oracle_counts(grid, box, sigma, qcut, dq, O.DEFAULT_CONTRACTION)
    np.testing.assert_array_equal(n_gpu, n_or)


@pytest.mark.parametrize("geom", GEOMS, ids=range(len(GEOMS)))
def test_bin_counts_match_reference_kernel(cuda, ref_dir, geom):
    grid, box, sigma, qcut, dq = geom
    s = _system(box)
    _, n_gpu, eng = engine_hist(s, grid, [s.positions], sigma=sigma, qcut=qcut, bin_size=dq)
    eng.close()
    n_or, (nn, ocs, dqe, qce, nb) = _oracle_counts(grid, box, sigma, qcut, dq, O.DEFAULT_CONTRACTION)
    n_ref = _ref_counts(ref_dir, nn, ocs, dqe, qce, nb)
    modes = [m for m in (0, 1, 2)
             if np.array_equal(_oracle_counts(grid, box, sigma, qcut, dq, m)[0], n_ref)]
    print(f"oracle contraction modes matching the reference kernel: {modes}")
    np.testing.assert_array_equal(n_gpu, n_ref)
    assert O.DEFAULT_CONTRACTION in modes
