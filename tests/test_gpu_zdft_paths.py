"""Tensor-core (tcgen05, 3xTF32) z-, y- and x-axis DFTs vs the FP32 SIMT kernels and the FP64 oracle (GPU).

Plans take a tensor-core kernel whenever its operands fit shared memory
(``info.path`` bits 0, 1, 2 for the z-, y- and x-axis DFTs; bit 3 when the z
pass runs the 128-column wide-tile kernel);
``PYCUSAXS_ZDFT=simt`` / ``PYCUSAXS_YDFT=simt`` / ``PYCUSAXS_XDFT=simt`` at plan
creation keep the SIMT kernel, ``PYCUSAXS_ZDFT=narrow`` the 64-column
tensor-core z kernel, ``PYCUSAXS_ZDFT=atoms`` the atom-GEMM z kernel (path bit
4).  Every z case runs with each of the three z kernels.  Both must give identical bin counts and profiles within the 1e-4
tolerance of the FP64 oracle; the 3xTF32 products are accurate to ~2^-19, and
TC_VS_SIMT_RTOL (2e-5 per bin) bounds the difference between the two kernels.
"""
import contextlib
import os

import numpy as np
import pytest

from helpers import assert_profiles_close, engine_hist, oracle_hist
from pycusaxs_b200.synthetic import System, cubic_system

pytestmark = pytest.mark.gpu

TC_VS_SIMT_RTOL = 2e-5


@contextlib.contextmanager
def dft_mode(var, mode):
    old = os.environ.get(var)
    if mode is None:
        os.environ.pop(var, None)
    else:
        os.environ[var] = mode
    try:
        yield
    finally:
        if old is None:
            os.environ.pop(var, None)
        else:
            os.environ[var] = old


_AXES = {"z": ("PYCUSAXS_ZDFT", 1), "y": ("PYCUSAXS_YDFT", 2), "x": ("PYCUSAXS_XDFT", 4)}


@pytest.fixture(params=["wide", "narrow", "atoms"])
def zmode(request):
    return request.param


def _both(system, grid, frames, expect_tc=True, axis="z", zmode="wide", expect_wide=None, **kw):
    var, bit = _AXES[axis]
    zenv = {"narrow": "narrow", "atoms": "atoms"}.get(zmode) if axis == "z" else None
    with dft_mode(var, zenv):
        h_tc, n_tc, e_tc = engine_hist(system, grid, frames, **kw)
        path_tc = e_tc.info.path
        e_tc.close()
    with dft_mode(var, "simt"):
        h_s, n_s, e_s = engine_hist(system, grid, frames, **kw)
        path_s = e_s.info.path
        e_s.close()
    assert path_s & bit == 0
    assert (path_tc & bit) == (bit if expect_tc else 0)
    if axis == "z" and zmode == "narrow":
        assert path_tc & 8 == 0
    elif axis == "z" and zmode == "atoms":
        if expect_wide:  # every plan that can run the wide tiles can run the atom GEMM
            assert path_tc & 16 == 16, path_tc
    elif axis == "z" and expect_wide is not None:
        assert (path_tc & 8) == (8 if expect_wide else 0), path_tc
    np.testing.assert_array_equal(n_tc, n_s)
    sel = n_s > 0
    sel[0] = False
    diff = np.abs(h_tc[sel] - h_s[sel]) / np.abs(h_s[sel])
    ho, no, _ = oracle_hist(system, grid, frames, **{k: v for k, v in kw.items() if k != "max_frames"})
    err_tc = assert_profiles_close(h_tc, n_tc, ho, no)
    err_s = assert_profiles_close(h_s, n_s, ho, no)
    print(f"path {path_tc}: vs FP64 oracle: tensor cores {err_tc:.2e}, SIMT {err_s:.2e}; "
          f"between them {diff.max():.2e}")
    assert diff.max() <= TC_VS_SIMT_RTOL, diff.max()
    return err_tc, float(diff.max())


def _line_system(n, lengths, seed, elements=("C", "O")):
    rng = np.random.default_rng(seed)
    L = np.asarray(lengths, np.float64)
    pos = (rng.uniform(0, 1, (n, 3)) * L).astype(np.float32)
    el = np.array(elements, dtype=object)[rng.choice(len(elements), n)]
    return System(el, pos, np.diag(L).astype(np.float32))


def test_tc_small_cubic(cuda, zmode):
    s = cubic_system(4000, 40.0, seed=11)
    _both(s, (32, 32, 32), [s.positions], sigma=2.0, qcut=0.6, zmode=zmode, expect_wide=True)


def test_tc_bench_sized_grid128(cuda, zmode):
    # the trajectory workload's plan: grid 128, 256^3 supercell, q-cut 0.5
    s = cubic_system(30_000, 120.0, seed=12)
    _both(s, (128, 128, 128), [s.positions], sigma=2.0, qcut=0.5, bin_size=0.002, zmode=zmode,
          expect_wide=True)


def test_tc_uneven_grid_z_not_multiple_of_8(cuda, zmode):
    # z extent 44 -> K padded to 48 with zero twiddle rows (a partial last ring
    # slot of the wide kernel); x extent 24 and y extent 32
    s = _line_system(3000, (30.0, 40.0, 44.0), 13, ("H", "C", "O", "N"))
    _both(s, (24, 32, 44), [s.positions], sigma=2.5, qcut=0.9, zmode=zmode, expect_wide=True)


def test_tc_ragged_tiles(cuda, zmode):
    # x extent 20 and y extent 28: the last tiles of both axes are partial
    s = _line_system(3000, (25.0, 35.0, 40.0), 113, ("H", "C", "O"))
    _both(s, (20, 28, 32), [s.positions], sigma=2.0, qcut=0.8, zmode=zmode, expect_wide=True)


def test_tc_order2_two_taps(cuda, zmode):
    s = cubic_system(3000, 36.0, seed=14)
    _both(s, (32, 32, 32), [s.positions], order=2, sigma=2.0, qcut=0.7, zmode=zmode)


def test_tc_supercell_smaller_than_grid(cuda, zmode):
    # scaled grid below the grid: the transform crops, spread rows exceed K
    s = cubic_system(3000, 36.0, seed=15)
    _both(s, (40, 40, 40), [s.positions], scaled_grid=(32, 32, 30), qcut=0.6, zmode=zmode)


def test_tc_single_operand_stage_long_z(cuda, zmode):
    # z extent 256, 17 kz values (N = 48): the 64-column kernel's twiddles 96 KB +
    # one 128 KB operand stage fit shared memory, two stages do not; the wide
    # kernel's f16 twiddles (48 KB) fit beside its 133 KB tile: eight ring chunks
    # per item
    s = _line_system(4000, (80.0, 80.0, 320.0), 16)
    _both(s, (32, 32, 256), [s.positions], sigma=2.0, qcut=0.15, zmode=zmode, expect_wide=True)


def test_tc_many_kz_wide_n(cuda, zmode):
    # long z at the largest q-cut the grid allows (reset to ~1.55 /A): the full kz
    # axis, 97 values, N = 200 with one operand stage
    # (N > 128: no wide tiles)
    s = _line_system(1500, (16.0, 16.0, 192.0), 17)
    _both(s, (16, 16, 96), [s.positions], sigma=2.0, qcut=3.5, zmode=zmode, expect_wide=False)


def test_too_many_kz_keeps_simt(cuda):
    # ~126 kz values over a 256-long z axis: the twiddle operands alone (2 x 256 x 256
    # floats) exceed shared memory, so the plan keeps the SIMT kernel
    s = _line_system(1200, (20.0, 20.0, 320.0), 18)
    _both(s, (16, 16, 256), [s.positions], expect_tc=False, sigma=2.0, qcut=50.0)


def test_tc_batched_frames(cuda, zmode):
    s = cubic_system(5000, 40.0, seed=19, jitter=0.5, nframes=3)
    frames = [s.frame(k) for k in range(3)]
    _both(s, (32, 32, 32), frames, sigma=2.0, qcut=0.6, max_frames=3, zmode=zmode, expect_wide=True)


# -- y-axis DFT -------------------------------------------------------------


def test_ytc_small_cubic_fewer_rows_than_block(cuda):
    # x extent 32 of a 128-row block: the rows beyond it are zero
    s = cubic_system(4000, 40.0, seed=21)
    _both(s, (32, 32, 32), [s.positions], axis="y", sigma=2.0, qcut=0.6)


def test_ytc_bench_sized_grid128(cuda):
    s = cubic_system(30_000, 120.0, seed=22)
    _both(s, (128, 128, 128), [s.positions], axis="y", sigma=2.0, qcut=0.5, bin_size=0.002)


def test_ytc_y_extent_not_multiple_of_chunk(cuda):
    # y extent 40: the last K chunk holds 8 y values and 8 zero rows
    s = _line_system(3000, (30.0, 40.0, 44.0), 23, ("H", "C", "O", "N"))
    _both(s, (24, 40, 44), [s.positions], axis="y", sigma=2.5, qcut=0.9)


def test_ytc_two_x_blocks(cuda):
    # x extent 160: two blocks of 128 rows, the second one partly empty
    s = _line_system(3000, (160.0, 40.0, 40.0), 24, ("C", "N", "O"))
    _both(s, (160, 32, 32), [s.positions], axis="y", sigma=2.0, qcut=0.4)


def test_ytc_full_ky_axis_keeps_simt(cuda):
    # q-cut at the grid's limit on a long y axis: 2*nky > 256 columns, SIMT kernel
    s = _line_system(1500, (16.0, 192.0, 16.0), 25)
    _both(s, (16, 96, 16), [s.positions], axis="y", expect_tc=False, sigma=2.0, qcut=3.5)


def test_ytc_batched_frames(cuda):
    s = cubic_system(5000, 40.0, seed=26, jitter=0.5, nframes=3)
    frames = [s.frame(k) for k in range(3)]
    _both(s, (32, 32, 32), frames, axis="y", sigma=2.0, qcut=0.6, max_frames=3)


@pytest.mark.parametrize("form", ["default", "split"])
@pytest.mark.parametrize("axis", ["y", "x"])
def test_yx_tc_many_items_per_cta(cuda, axis, form):
    # 4 frames at grid 128: several hundred items, so every CTA of the persistent
    # y/x kernels processes more than one item and reuses its accumulator and
    # operand stages (one-frame cases give each CTA at most one item).  The y
    # pass by default reads A's remainder from the swizzled shared-memory tile
    # (two MMAs per k step); "split" (PYCUSAXS_DTC=split) keeps head and
    # remainder in tensor memory (three MMAs per k step), the x pass's form.
    s = cubic_system(20_000, 100.0, seed=28, jitter=0.4, nframes=4)
    frames = [s.frame(k) for k in range(4)]
    var, bit = _AXES[axis]
    kw = dict(sigma=2.0, qcut=0.5, bin_size=0.002, max_frames=4)
    with dft_mode(var, None), dft_mode("PYCUSAXS_DTC", "split" if form == "split" else None):
        h_tc, n_tc, e = engine_hist(s, (128, 128, 128), frames, **kw)
        assert e.info.path & bit
        e.close()
    with dft_mode(var, "simt"):
        h_s, n_s, e = engine_hist(s, (128, 128, 128), frames, **kw)
        e.close()
    np.testing.assert_array_equal(n_tc, n_s)
    sel = n_s > 0
    sel[0] = False
    diff = np.abs(h_tc[sel] - h_s[sel]) / np.abs(h_s[sel])
    assert diff.max() <= TC_VS_SIMT_RTOL, diff.max()


# -- x-axis DFT (with form factors, type sum and moduli) --------------------


def test_xtc_small_cubic(cuda):
    s = cubic_system(4000, 40.0, seed=31)
    _both(s, (32, 32, 32), [s.positions], axis="x", sigma=2.0, qcut=0.6)


def test_xtc_bench_sized_grid128(cuda):
    s = cubic_system(30_000, 120.0, seed=32)
    _both(s, (128, 128, 128), [s.positions], axis="x", sigma=2.0, qcut=0.5, bin_size=0.002)


def test_xtc_x_extent_not_multiple_of_chunk(cuda):
    s = _line_system(3000, (30.0, 40.0, 44.0), 33, ("H", "C", "O", "N"))
    _both(s, (24, 40, 44), [s.positions], axis="x", sigma=2.5, qcut=0.9)


def test_xtc_ten_types_sixteen_rows_per_ky(cuda):
    els = ("H", "C", "N", "O", "P", "S", "Na", "Cl", "K", "Mg")
    s = _line_system(5000, (40.0, 40.0, 40.0), 34, els)
    _both(s, (32, 32, 32), [s.positions], axis="x", sigma=2.0, qcut=0.7)


def test_xtc_seventeen_types_keep_simt(cuda):
    els = ("H", "C", "N", "O", "P", "S", "Na", "Cl", "K", "Mg", "Ca", "F", "Br", "I", "Fe", "Zn", "Cu")
    s = _line_system(5000, (40.0, 40.0, 40.0), 35, els)
    _both(s, (32, 32, 32), [s.positions], axis="x", expect_tc=False, sigma=2.0, qcut=0.7)


def test_xtc_triclinic(cuda):
    from pycusaxs_b200.synthetic import triclinic_slab_system
    s = triclinic_slab_system(5000, 40.0, 40.0, 32.0, 80.0, seed=36)
    _both(s, (32, 32, 32), [s.positions], axis="x", sigma=2.0, qcut=0.7)


def test_xtc_full_kx_axis_keeps_simt(cuda):
    s = _line_system(1500, (192.0, 16.0, 16.0), 37)
    _both(s, (96, 16, 16), [s.positions], axis="x", expect_tc=False, sigma=2.0, qcut=3.5)


def test_xtc_batched_frames(cuda):
    s = cubic_system(5000, 40.0, seed=38, jitter=0.5, nframes=3)
    frames = [s.frame(k) for k in range(3)]
    _both(s, (32, 32, 32), frames, axis="x", sigma=2.0, qcut=0.6, max_frames=3)
