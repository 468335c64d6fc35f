"""Opt-in physics extensions in the FP64 oracle (CPU): the correct-triclinic inverse and
the given (bulk-solvent) padding.  Neither is reference parity, so they are checked
against physics and against the average-padding path instead of reference files."""
import numpy as np
import pytest
import torch

from oracle import saxs_oracle as O
from oracle import torch_oracle as TO
from pycusaxs_b200.solvent import given_padding, water_molecules
from pycusaxs_b200.synthetic import cubic_system
from test_physics import NAMES, direct_intensity, signed

SHEARED = np.array([[60.0, 0.0, 0.0], [15.0, 58.0, 0.0], [10.0, 12.0, 55.0]], np.float32)


def sheared_cluster(seed=7, n=300, radius=10.0):
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1)[:, None]
    r = radius * rng.uniform(0, 1, n) ** (1 / 3)
    centre = 0.5 * SHEARED.sum(axis=0)
    pos = (centre + v * r[:, None]).astype(np.float32)
    return pos, rng.choice(2, n).astype(np.int32)


def _grid_vs_direct(box_mode):
    pos, toa = sheared_cluster()
    ff = O.load_form_factors()
    coeffs = np.stack([ff[k] for k in NAMES])
    plan = O.OraclePlan(grid=(64, 64, 64), types=NAMES, coeffs=coeffs, box0=SHEARED, sigma=2.0,
                        qcut=0.6, box_mode=box_mode)
    iv, bins, parts = O.frame_intensity(plan, pos, toa, SHEARED, return_parts=True)
    idx = np.argwhere(bins >= 0)
    m = np.stack([signed(idx[:, d], plan.nn[d]) for d in range(3)], axis=1).astype(np.float64)
    qvec = 2 * np.pi * (m @ parts["ocs"].astype(np.float64).T)
    i_dir, qa, _ = direct_intensity(qvec, pos, toa, coeffs)
    keep = qa > 0
    i_grid = iv[idx[:, 0], idx[:, 1], idx[:, 2]]
    return np.abs(i_grid[keep] - i_dir[keep]) / i_dir[keep], parts


def test_triclinic_mode_matches_the_direct_sum_in_a_sheared_box():
    rel, parts = _grid_vs_direct(box_mode=1)
    assert parts["means"] == [0.0, 0.0]          # vacuum around the cluster
    assert np.median(rel) < 1e-4 and np.quantile(rel, 0.99) < 2e-3


def test_triclinic_mode_maps_positions_and_k_points_by_the_full_inverse():
    # fractional coordinates s with x = s H, and q(m) = 2 pi sigma' H^-1 m; the
    # reference's upper-triangle inverse gets the fractional part wrong whenever the
    # box rows have a lower-triangle shear (the MDAnalysis convention)
    rng = np.random.default_rng(11)
    x = (rng.uniform(0, 1, (50, 3)) @ SHEARED).astype(np.float32)
    H = SHEARED.astype(np.float64)
    s_true = x.astype(np.float64) @ np.linalg.inv(H)
    _, oc1 = O.cell_matrices(SHEARED, 1)
    np.testing.assert_allclose(x.astype(np.float64) @ oc1.astype(np.float64).T, s_true, atol=1e-5)
    _, oc0 = O.cell_matrices(SHEARED, 0)
    assert np.abs(x.astype(np.float64) @ oc0.astype(np.float64).T - s_true).max() > 0.05
    ff = O.load_form_factors()
    plan = O.OraclePlan(grid=(32, 32, 32), types=NAMES, coeffs=np.stack([ff[k] for k in NAMES]),
                        box0=SHEARED, sigma=2.0, qcut=0.6, box_mode=1)
    m = np.array([[1.0, 2.0, -3.0], [4.0, -1.0, 0.0]])
    sig = 32 / plan.nn[0]
    q_true = 2 * np.pi * sig * (np.linalg.inv(H) @ m.T).T
    q_map = 2 * np.pi * m @ plan.scaled_oc(oc1).astype(np.float64).T
    np.testing.assert_allclose(q_map, q_true, rtol=1e-5)


def test_triclinic_mode_equals_parity_for_orthorhombic_boxes():
    s = cubic_system(2000, 36.0, seed=8)
    names = sorted({str(e) for e in s.elements})
    ff = O.load_form_factors()
    kw = dict(grid=(32, 32, 32), types=names, coeffs=np.stack([ff[k] for k in names]), box0=s.box,
              sigma=2.0, qcut=0.7)
    toa = s.type_of_atom(names)
    h0, n0 = O.run_frames(O.OraclePlan(**kw), [(s.positions, s.box)], toa)
    h1, n1 = O.run_frames(O.OraclePlan(box_mode=1, **kw), [(s.positions, s.box)], toa)
    np.testing.assert_array_equal(n0, n1)
    np.testing.assert_allclose(h1, h0, rtol=1e-6)


def test_given_padding_equal_to_the_border_means_reproduces_the_average_mode():
    s = cubic_system(3000, 36.0, seed=9)
    names = sorted({str(e) for e in s.elements})
    ff = O.load_form_factors()
    kw = dict(grid=(32, 32, 32), types=names, coeffs=np.stack([ff[k] for k in names]), box0=s.box,
              sigma=2.0, qcut=0.7)
    toa = s.type_of_atom(names)
    plan = O.OraclePlan(**kw)
    _, _, parts = O.frame_intensity(plan, s.positions, toa, s.box, return_parts=True)
    means = np.asarray(parts["means"], np.float64)
    h0, n0 = O.run_frames(plan, [(s.positions, s.box)], toa)
    h1, n1 = O.run_frames(O.OraclePlan(padding=means, **kw), [(s.positions, s.box)], toa)
    np.testing.assert_array_equal(n0, n1)
    np.testing.assert_allclose(h1, h0, rtol=1e-10)
    # a different padding changes the profile
    h2, _ = O.run_frames(O.OraclePlan(padding=2 * means, **kw), [(s.positions, s.box)], toa)
    assert np.abs(h2 - h0).max() > 1e-3 * np.abs(h0).max()


def test_given_padding_values_follow_atomcounter():
    box = np.diag([30.0, 31.0, 32.0])
    vals = given_padding(["C", "Cl", "H", "Na", "O"], box, (32, 32, 32), "TIP3P", {"Na": 5, "Cl": 4})
    wm = water_molecules(30 * 31 * 32, "TIP3P")
    pts = 32 ** 3
    np.testing.assert_allclose(vals, [0.0, 4 / pts, 2 * wm / pts, 5 / pts, wm / pts], rtol=1e-6)
    assert wm == pytest.approx(0.982 * 29760 * 1e-24 / 18.015 * 6.022e23)
    # unknown models fall back to SPC/E
    assert water_molecules(1000.0, "OPC") == water_molecules(1000.0, "SPCE")


def test_given_padding_gradient_has_no_mean_term():
    # with a given padding the mean does not move with the atoms: the torch oracle's
    # gradient must match central differences of the same (given-padding) loss
    s = cubic_system(600, 28.0, seed=10)
    names = sorted({str(e) for e in s.elements})
    ff = O.load_form_factors()
    pad = given_padding(names, s.box, (16, 16, 16), "SPCE")
    plan = O.OraclePlan(grid=(16,) * 3, types=names, coeffs=np.stack([ff[k] for k in names]),
                        box0=s.box, sigma=2.0, qcut=0.8, padding=pad)
    toa = s.type_of_atom(names)
    x = torch.tensor(s.positions.astype(np.float64), requires_grad=True)
    prof, _ = TO.profile(plan, x, toa, s.box)
    sel = prof.detach() > 0
    (prof[sel].log().sum()).backward()
    g = x.grad.numpy()
    h = 1e-3
    for a in (3, 77, 301):
        for d in range(3):
            xp = x.detach().clone()
            xp[a, d] += h
            xm = x.detach().clone()
            xm[a, d] -= h
            fd = float((TO.profile(plan, xp, toa, s.box)[0][sel].log().sum()
                        - TO.profile(plan, xm, toa, s.box)[0][sel].log().sum()) / (2 * h))
            assert g[a, d] == pytest.approx(fd, rel=1e-4, abs=1e-6 * np.abs(g).max())
