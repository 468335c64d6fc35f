"""Setup numerics of the native library (host C++) against the oracle and known values.

No GPU needed: grid sizing, the inverse cell, the Delta-q / q-cut reset and the
B-spline moduli are host functions of the shared library.
"""
import ctypes

import numpy as np
import pytest

from oracle import saxs_oracle as O
from pycusaxs_b200 import _native


@pytest.fixture(scope="module")
def lib():
    return _native.load()


def _oc(lib, box):
    b = np.ascontiguousarray(np.asarray(box, np.float32).reshape(9))
    out = np.zeros(9, np.float32)
    _native.check(lib.saxs_cell_oc(b.ctypes.data_as(_native.c_float_p),
                                   out.ctypes.data_as(_native.c_float_p)))
    return out.reshape(3, 3)


def test_closest_product_matches_oracle(lib):
    for sigma in (0.5, 1.0, 1.5, 2.0, 2.5, 3.0, 3.5, 7.0, 12.0):
        for n in list(range(1, 130)) + [160, 200, 256, 300, 333]:
            assert lib.saxs_closest_product(n, sigma) == O.find_closest_product(n, sigma), (n, sigma)


def test_closest_product_known_values(lib):
    # nn for the workloads: 64 -> 128, 128 -> 256, 256 -> 512 at sigma 2
    assert lib.saxs_closest_product(64, 2.0) == 128
    assert lib.saxs_closest_product(128, 2.0) == 256
    assert lib.saxs_closest_product(256, 2.0) == 512
    # ties go to the smaller candidate: 2.5*100 = 250 = 2*5^3 exactly
    assert lib.saxs_closest_product(100, 2.5) == 250
    # 128*2.5 = 320 = 2^6*5
    assert lib.saxs_closest_product(128, 2.5) == 320
    # round(11*1.0) = 11 is prime: 10 and 12 tie, the smaller wins
    assert lib.saxs_closest_product(11, 1.0) == 10


@pytest.mark.parametrize("box", [
    np.diag([120.0, 120.0, 120.0]),
    np.diag([60.0, 75.5, 90.25]),
    # MDAnalysis lower-triangular triclinic rows: only the diagonal survives
    [[250.0, 0, 0], [43.41204, 246.20193, 0], [0, 0, 200.0]],
    # a box with upper-triangular entries (the only ones the reference reads)
    [[50.0, 3.0, -2.0], [0.0, 55.0, 4.0], [0.0, 0.0, 60.0]],
])
def test_cell_oc_matches_oracle(lib, box):
    got = _oc(lib, box)
    _, want = O.cell_matrices(box)
    np.testing.assert_array_equal(got, want)
    assert np.all(np.tril(got, -1) == 0)


@pytest.mark.parametrize("nn,box,sigma,dq,qcut", [
    ((256, 256, 256), np.diag([120.0] * 3), 2.0, 0.002, 0.5),
    ((128, 128, 128), np.diag([60.0] * 3), 2.0, 0.002, 0.5),
    ((512, 512, 512), [[250.0, 0, 0], [43.41204, 246.20193, 0], [0, 0, 200.0]], 2.0, 0.001, 0.4),
    ((320, 320, 320), np.diag([90.0] * 3), 2.5, 0.01, 2.0),
    ((160, 180, 200), np.diag([50.0, 60.0, 70.0]), 1.0, 0.0, 0.0),
])
def test_histogram_parameters_match_oracle(lib, nn, box, sigma, dq, qcut):
    oc = np.ascontiguousarray(_oc(lib, box).reshape(9))
    nn_a = (ctypes.c_int * 3)(*nn)
    b, q, n = ctypes.c_float(), ctypes.c_float(), ctypes.c_int()
    _native.check(lib.saxs_histogram_parameters(nn_a, oc.ctypes.data_as(_native.c_float_p), sigma, dq,
                                                qcut, ctypes.byref(b), ctypes.byref(q), ctypes.byref(n)))
    _, oc_o = O.cell_matrices(box)
    want = O.histogram_parameters(nn, oc_o, sigma, dq, qcut)
    assert np.float32(b.value) == want[0]
    assert np.float32(q.value) == want[1]
    assert n.value == want[2]


def test_bench_config_bins(lib):
    # 100k atoms in 120 A, grid 128, sigma 2: Delta-q is reset to 2 pi / 240 A and
    # q-cut 0.5 /A gives 20 bins (19 profile rows).
    _, oc = O.cell_matrices(np.diag([120.0] * 3))
    dq, qc, nb = O.histogram_parameters((256,) * 3, oc, 2.0, 0.002, 0.5)
    assert abs(float(dq) - 2 * np.pi / 240.0) < 1e-7
    assert float(qc) == pytest.approx(0.5)
    assert nb == 20


@pytest.mark.parametrize("n", [16, 64, 100, 128, 135, 256, 320])
def test_bspline_moduli_match_oracle(lib, n):
    out = np.zeros(n, np.float32)
    _native.check(lib.saxs_bspline_moduli(n, n, out.ctypes.data_as(_native.c_float_p)))
    want = O.bspmod(n)
    np.testing.assert_allclose(out, want, rtol=2e-6)
    assert out[0] == pytest.approx(1.0)
