"""CUDA path vs the FP64 oracle on the same seeded frames (GPU).

Bin counts must be identical (the reference's float32 bin rule, exact), and
each reported bin's intensity within RTOL_PROFILE (1e-4) relative.
"""
import numpy as np
import pytest

from helpers import RTOL_PROFILE, assert_profiles_close, engine_hist, oracle_hist
from pycusaxs_b200.synthetic import cubic_system, triclinic_slab_system, System

pytestmark = pytest.mark.gpu


def _run(system, grid, frames, **kw):
    ho, no, plan = oracle_hist(system, grid, frames, **kw)
    h, n, eng = engine_hist(system, grid, frames, **kw)
    assert eng.info.num_bins == plan.num_bins
    assert np.float32(eng.info.bin_size) == plan.dq
    assert np.float32(eng.info.qcut) == plan.kcut
    err = assert_profiles_close(h, n, ho, no)
    eng.close()
    return err


def test_small_cubic(cuda):
    s = cubic_system(4000, 40.0, seed=1)
    _run(s, (32, 32, 32), [s.positions], sigma=2.0, qcut=0.6)


def test_first_workload_20k_atoms_grid64(cuda):
    # 20k atoms in 6 nm, grid 64, scale 2 (128^3 supercell), q-cut 0.5 /A, bins 0.002 /A (reset)
    s = cubic_system(20_000, 60.0, seed=0)
    _run(s, (64, 64, 64), [s.positions], sigma=2.0, qcut=0.5, bin_size=0.002)


def test_orthorhombic_uneven_grid(cuda):
    s = System(*_ortho(3000, (30.0, 40.0, 50.0), seed=2))
    _run(s, (24, 32, 40), [s.positions], sigma=2.5, qcut=0.9)


def _ortho(n, L, seed):
    rng = np.random.default_rng(seed)
    pos = (rng.uniform(0, 1, (n, 3)) * np.array(L)).astype(np.float32)
    el = np.array(["H", "C", "O", "N"], dtype=object)[rng.choice(4, n, p=[.5, .3, .1, .1])]
    return el, pos, np.diag(L).astype(np.float32)


def test_triclinic_rows_use_upper_triangle_only(cuda):
    s = triclinic_slab_system(5000, 40.0, 40.0, 32.0, 80.0, seed=4)
    _run(s, (32, 32, 32), [s.positions], sigma=2.0, qcut=0.7)


def test_upper_triangular_box(cuda):
    rng = np.random.default_rng(5)
    box = np.array([[36.0, 4.0, -3.0], [0.0, 40.0, 5.0], [0.0, 0.0, 44.0]], np.float32)
    frac = rng.uniform(0, 1, (3000, 3))
    pos = (frac @ box).astype(np.float32)
    el = np.array(["C", "O"], dtype=object)[rng.choice(2, 3000)]
    s = System(el, pos, box)
    _run(s, (32, 32, 32), [s.positions], sigma=2.0, qcut=0.8)


@pytest.mark.parametrize("order", [1, 2, 3, 5, 8])
def test_other_spline_orders(cuda, order):
    s = cubic_system(2000, 30.0, seed=6)
    _run(s, (24, 24, 24), [s.positions], sigma=2.0, qcut=0.8, order=order)


def test_npt_three_jittered_frames(cuda):
    s = cubic_system(3000, 36.0, seed=7, jitter=0.5, nframes=3)
    _run(s, (32, 32, 32), [s.frame(k) for k in range(3)], sigma=2.0, qcut=0.7)


def test_nvt_three_jittered_frames(cuda):
    s = cubic_system(3000, 36.0, seed=8, jitter=0.5, nframes=3)
    _run(s, (32, 32, 32), [s.frame(k) for k in range(3)], sigma=2.0, qcut=0.7, ensemble="nvt")


def test_npt_box_changes_between_frames(cuda):
    s = cubic_system(2500, 36.0, seed=9, jitter=0.3, nframes=3)
    boxes = [np.diag([36.0, 36.0, 36.0]), np.diag([35.5, 36.2, 35.8]), np.diag([36.3, 35.7, 36.1])]
    boxes = [b.astype(np.float32) for b in boxes]
    _run(s, (32, 32, 32), [s.frame(k) for k in range(3)], sigma=2.0, qcut=0.7, boxes=boxes)


def test_explicit_supercell_with_unit_scale_reaches_nyquist(cuda):
    # scale_factor 1 (the pybind default) with an explicit 2x supercell: the q-cut
    # clamp uses sigma=1, so the k-box spans the whole spectrum including Nyquist
    s = cubic_system(1500, 24.0, seed=10)
    _run(s, (16, 16, 16), [s.positions], scaled_grid=(32, 32, 32), sigma=1.0, qcut=5.0)


def test_odd_supercell(cuda):
    s = cubic_system(1500, 27.0, seed=11)
    _run(s, (27, 27, 27), [s.positions], sigma=1.0, qcut=0.8)


def test_supercell_smaller_than_grid(cuda):
    s = cubic_system(1500, 30.0, seed=12)
    _run(s, (32, 32, 32), [s.positions], scaled_grid=(24, 24, 24), sigma=1.0, qcut=0.6)


def test_batched_frames_equal_single_frames(cuda):
    s = cubic_system(3000, 36.0, seed=13, jitter=0.5, nframes=5)
    frames = [s.frame(k) for k in range(5)]
    h1, n1, e1 = engine_hist(s, (32, 32, 32), frames, sigma=2.0, qcut=0.7, max_frames=1)
    h5, n5, e5 = engine_hist(s, (32, 32, 32), frames, sigma=2.0, qcut=0.7, max_frames=5)
    np.testing.assert_array_equal(n1, n5)
    np.testing.assert_allclose(h5, h1, rtol=1e-6)
    e1.close()
    e5.close()


def test_host_input_path_equals_device_input(cuda):
    s = cubic_system(3000, 36.0, seed=14, jitter=0.5, nframes=4)
    frames = [s.frame(k) for k in range(4)]
    hd, nd, e1 = engine_hist(s, (32, 32, 32), frames, sigma=2.0, qcut=0.7, max_frames=2)
    hh, nh, e2 = engine_hist(s, (32, 32, 32), frames, sigma=2.0, qcut=0.7, max_frames=2,
                             device_input=False)
    np.testing.assert_array_equal(nd, nh)
    np.testing.assert_allclose(hh, hd, rtol=1e-6)
    e1.close()
    e2.close()


def test_border_sums_match_oracle_grid(cuda):
    from oracle import saxs_oracle as O

    s = cubic_system(3000, 32.0, seed=15)
    h, n, eng = engine_hist(s, (32, 32, 32), [s.positions], sigma=2.0, qcut=0.6)
    got = eng.border_sums()
    oc = O.cell_matrices(s.box)[1]
    r = O.grid_coords(s.positions, oc, (32, 32, 32))
    mask = O.border_planes(32)
    for t, name in enumerate(eng.type_names):
        sel = np.array([str(e) == name for e in s.elements])
        g = O.spread(r[sel], (32, 32, 32), 4)
        assert got[t] == pytest.approx(g[:, :, mask].sum(), rel=1e-6)
    eng.close()


def _two_element(n, lengths, seed):
    rng = np.random.default_rng(seed)
    L = np.asarray(lengths, np.float64)
    pos = (rng.uniform(0, 1, (n, 3)) * L).astype(np.float32)
    el = np.array(["C", "O"], dtype=object)[rng.choice(2, n)]
    return System(el, pos, np.diag(L).astype(np.float32))


def test_long_z_axis_full_spectrum_chunks_z_twiddles(cuda):
    # 16 x 16 x 256 grid, 512 supercell along z, q-cut above Nyquist: the z
    # twiddle table (256 rows x 258 kz) cannot sit in shared memory at once
    s = _two_element(1500, (20.0, 20.0, 320.0), seed=31)
    _run(s, (16, 16, 256), [s.positions], sigma=2.0, qcut=50.0)


def test_long_x_axis_full_spectrum_chunks_x(cuda):
    # 256 x 16 x 16 grid, full kx range of 512: k_xdft_post walks x in chunks
    s = _two_element(1500, (320.0, 20.0, 20.0), seed=32)
    _run(s, (256, 16, 16), [s.positions], sigma=2.0, qcut=50.0)


def test_cli_default_parameters(cuda):
    # the CLI defaults: scale 2.5, bin 0.01 /A, q-cut 2.0 /A (pycusaxs/saxs_defaults.py)
    s = cubic_system(8000, 60.0, seed=33)
    _run(s, (64, 64, 64), [s.positions], sigma=2.5, bin_size=0.01, qcut=2.0)


def test_kbox_intensity_matches_direct_sum_on_isolated_cluster(cuda):
    """CUDA k-box intensities vs the exact direct sum (the physics check on the GPU)."""
    from test_physics import NAMES, cluster, direct_intensity
    from oracle import saxs_oracle as O

    pos, toa, box = cluster()
    s = System(np.array(NAMES, dtype=object)[toa], pos, box)
    h, n, eng = engine_hist(s, (64, 64, 64), [pos], sigma=2.0, qcut=0.6)
    ib = eng.kbox_intensity()                       # (nkz, nky, nkx)
    nkx, nky, nkz = eng.info.kbox
    kz, ky, kx = np.meshgrid(np.arange(nkz), np.arange(nky), np.arange(nkx), indexing="ij")
    m = np.stack([kx - (nkx // 2), ky - (nky // 2), kz], axis=-1).reshape(-1, 3).astype(np.float64)
    ocs = (np.float32(64) / np.float32(128) * O.cell_matrices(box)[1]).astype(np.float64)
    qvec = 2 * np.pi * (m @ ocs.T)
    ff = O.load_form_factors()
    i_dir, qa, _ = direct_intensity(qvec, pos, toa, np.stack([ff[k] for k in NAMES]))
    i_gpu = ib.reshape(-1).astype(np.float64)
    keep = (i_gpu > 0) & (qa > 0)
    rel = np.abs(i_gpu[keep] - i_dir[keep]) / i_dir[keep]
    assert keep.sum() > 3000
    assert np.median(rel) < 1e-4 and np.quantile(rel, 0.99) < 2e-3 and rel.max() < 1e-2
    eng.close()
