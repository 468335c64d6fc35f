"""The FP64 oracle: internal consistency and textbook identities (CPU only)."""
import numpy as np
import pytest

from oracle import saxs_oracle as O
from pycusaxs_b200.synthetic import cubic_system


def test_spline_partition_of_unity_and_closed_form():
    u = np.linspace(0.0, 1.0, 101)
    x, dx = O.bspline_weights(u, 4)
    np.testing.assert_allclose(x.sum(axis=0), 1.0, atol=1e-15)
    np.testing.assert_allclose(x[0], (1 - u) ** 3 / 6, atol=1e-15)
    np.testing.assert_allclose(x[3], u ** 3 / 6, atol=1e-15)
    np.testing.assert_allclose(x[1], (3 * u ** 3 - 6 * u ** 2 + 4) / 6, atol=1e-15)
    # derivative weights (before the last pass) are the order-3 differences and sum to zero
    np.testing.assert_allclose(dx.sum(axis=0), 0.0, atol=1e-15)
    # numerical derivative of the cubic weights equals dx
    h = 1e-6
    xp, _ = O.bspline_weights(u[1:-1] + h, 4)
    xm, _ = O.bspline_weights(u[1:-1] - h, 4)
    np.testing.assert_allclose((xp - xm) / (2 * h), dx[:, 1:-1], atol=1e-8)


def test_stencil_weights_for_other_orders():
    g = np.array([0.25])
    w2, _ = O.stencil_weights(g, 2)       # first two cubic taps only
    x4, _ = O.bspline_weights(g, 4)
    np.testing.assert_allclose(w2[:, 0], x4[:2, 0])
    w6, _ = O.stencil_weights(g, 6)       # taps 4, 5 defined as zero
    np.testing.assert_allclose(w6[:4, 0], x4[:, 0])
    assert np.all(w6[4:] == 0)


def test_border_planes():
    assert O.border_planes(128).sum() == 9      # dz = int(0.07*128/2) = 4: z<=4 or z>=124
    assert O.border_planes(64).sum() == 5       # dz = 2
    assert O.border_planes(16).sum() == 1       # dz = 0: only z = 0


def test_spread_conserves_mass():
    s = cubic_system(500, 30.0, seed=3)
    oc = O.cell_matrices(s.box)[1]
    r = O.grid_coords(s.positions, oc, (16, 16, 16))
    g = O.spread(r, (16, 16, 16), 4)
    assert g.sum() == pytest.approx(500.0, rel=1e-12)
    assert g.min() >= 0


def test_grid_coords_in_range():
    rng = np.random.default_rng(0)
    xyz = rng.uniform(-500, 500, (2000, 3)).astype(np.float32)
    xyz[:5] = [[0, 0, 0], [30, 30, 30], [60, 60, 60], [-30, 15, 45], [29.999998, 0, 0]]
    oc = O.cell_matrices(np.diag([60.0] * 3))[1]
    r = O.grid_coords(xyz, oc, (64, 64, 64))
    assert r.min() >= 0 and r.max() <= 64


def test_mirror_values():
    a = np.arange(4 * 5 * 3, dtype=float).reshape(4, 5, 3)
    m = O.mirror_values(a)
    for i in range(4):
        for j in range(5):
            np.testing.assert_array_equal(m[i, j], a[(-i) % 4, (-j) % 5])


def test_histogram_of_constant_intensity_is_constant():
    nn = (32, 32, 32)
    oc = O.cell_matrices(np.diag([40.0] * 3))[1]
    plan_dq, plan_q, nb = O.histogram_parameters(nn, oc, 2.0, 0.0, 0.6)
    ocs = (np.float32(16) / np.float32(32) * oc).astype(np.float32)
    _, bins = O.kpoint_bins(nn, ocs, plan_dq, plan_q, nb)
    iv = np.ones(bins.shape)
    h, n = O.histogram(iv, bins, nb)
    sel = n > 0
    np.testing.assert_allclose(h[sel] / n[sel], 1.0)
    assert n[0] >= 1


def test_format_rows_like_iostream():
    # std::fixed setw(10) setprecision(5), then std::scientific setw(12) setprecision(5)
    text = O.format_rows([(0.02618, 12345.678), (0.5, 1.5e-7)])
    assert text == "   0.02618 1.23457e+04\n   0.50000 1.50000e-07\n"


def test_small_run_is_finite_and_positive():
    s = cubic_system(400, 30.0, seed=1)
    names = sorted({str(e) for e in s.elements})
    ff = O.load_form_factors()
    plan = O.OraclePlan(grid=(16, 16, 16), types=names, coeffs=np.stack([ff[n] for n in names]),
                        box0=s.box, sigma=2.0, bin_size=0.0, qcut=0.8)
    h, n = O.run_frames(plan, [(s.positions, s.box)], s.type_of_atom(names))
    rows = O.profile_rows(h, n, plan.dq)
    assert len(rows) == plan.num_bins - 1
    assert all(np.isfinite(i) and i > 0 for _, i in rows)
