"""The wide z kernel's fixed-point tile cannot overflow (CPU, FP64 oracle).

The kernel accumulates each voxel of a type's spread tile as a 32-bit integer
with a power-of-two scale chosen per item from the item's home-bin counts: it
assumes that a voxel receives taps only from atoms whose home bins (the bins of
the first x and y tap column, 4 columns wide) lie within 3 x 3 bins of it, and
that each tap is a product of three cubic weights of at most 2/3 (at most 1/6
with one tap per axis).  So every voxel sum is at most
tapmax * 9 * (largest home-bin count), the bound behind the scale.  These tests
check that inequality on the oracle's FP64 spreading for uniform, clustered and
coincident atoms, every spline order, and grids that leave a partial bin at the
periodic edge.
"""
import numpy as np
import pytest

from oracle import saxs_oracle as O

BIN_W = 4


def tapmax(order):
    return (2.0 / 3.0) ** 3 if min(order, 4) >= 2 else (1.0 / 6.0) ** 3


def home_bin_counts(r, n, order):
    m = r.astype(np.int64)
    xf = (m[:, 0] - order) % n[0]
    yf = (m[:, 1] - order) % n[1]
    tiles = ((n[0] + BIN_W - 1) // BIN_W, (n[1] + BIN_W - 1) // BIN_W)
    counts = np.zeros(tiles, dtype=np.int64)
    np.add.at(counts, (xf // BIN_W, yf // BIN_W), 1)
    return counts


def check(r, n, order):
    grid = O.spread(r, n, order)
    counts = home_bin_counts(r, n, order)
    bound = tapmax(order) * 9 * counts.max() * (1 + 1e-12)
    assert grid.max() <= bound, (grid.max(), bound)
    # the per-column form: the atoms reaching column (x, y) have their home
    # columns in the four columns ending at it, i.e. in at most 3 x 3 bins
    m = r.astype(np.int64)
    xf = (m[:, 0] - order) % n[0]
    yf = (m[:, 1] - order) % n[1]
    for x, y in [(0, 0), (n[0] - 1, n[1] - 1), (n[0] // 2, 1), (3, n[1] - 2)]:
        dx = (x - xf) % n[0]
        dy = (y - yf) % n[1]
        near = (dx < min(order, 4)) & (dy < min(order, 4))
        bins = {(int(a) // BIN_W, int(b) // BIN_W) for a, b in zip(xf[near], yf[near])}
        assert len({bx for bx, _ in bins}) <= 3 and len({by for _, by in bins}) <= 3
        assert grid[x, y].max() <= tapmax(order) * near.sum() * (1 + 1e-12) + 1e-15


@pytest.mark.parametrize("order", [1, 2, 3, 4, 6])
@pytest.mark.parametrize("n", [(32, 32, 32), (33, 30, 17), (29, 37, 24)])
def test_uniform_atoms(order, n):
    rng = np.random.default_rng(order * 100 + n[0])
    r = (rng.random((4000, 3)) * np.array(n)).astype(np.float32)
    check(r, n, order)


@pytest.mark.parametrize("order", [1, 4])
def test_clustered_and_coincident_atoms(order):
    n = (33, 29, 20)
    rng = np.random.default_rng(7 + order)
    cluster = (np.array([5.0, 27.5, 3.0]) + rng.normal(0.0, 0.6, (3000, 3))) % np.array(n)
    coincident = np.tile(np.array([[32.4, 0.3, 19.9]]), (500, 1))
    r = np.concatenate([cluster, coincident]).astype(np.float32)
    check(r, n, order)
