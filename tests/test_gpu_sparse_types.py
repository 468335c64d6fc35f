"""Sparse element types on the direct z kernel (k_spread_zdft_sparse) vs the FP64 oracle (GPU).

With the wide-tile z kernel, an element type whose 8 x 16 column tiles would
see fewer than r atoms on average (r = PYCUSAXS_SPARSE_REACH at plan creation,
default 24) is spread and z-transformed by the direct kernel instead
(``info.path`` bit 5); the other types stay on the wide kernel.  Both must give
the oracle's bin counts and profiles within RTOL_PROFILE, and the same profile
as a plan that keeps every type on the wide kernel (r = 0).  Sending every type to the
direct kernel (a limit above every type's count) checks it on dense types too,
where many atoms add into the same shared-memory accumulators.
"""
import contextlib
import os

import numpy as np
import pytest

from helpers import RTOL_PROFILE, assert_profiles_close, engine_hist, oracle_hist
from pycusaxs_b200.synthetic import cubic_system

pytestmark = pytest.mark.gpu

SPARSE_BIT = 32
WIDE_BIT = 8


@contextlib.contextmanager
def sparse_reach(value):
    old = os.environ.get("PYCUSAXS_SPARSE_REACH")
    if value is None:
        os.environ.pop("PYCUSAXS_SPARSE_REACH", None)
    else:
        os.environ["PYCUSAXS_SPARSE_REACH"] = value
    try:
        yield
    finally:
        if old is None:
            os.environ.pop("PYCUSAXS_SPARSE_REACH", None)
        else:
            os.environ["PYCUSAXS_SPARSE_REACH"] = old


def _run(system, grid, frames, reach, **kw):
    with sparse_reach(reach):
        h, n, eng = engine_hist(system, grid, frames, max_frames=len(frames), **kw)
        path = eng.info.path
        eng.close()
    return h, n, path


def test_rare_types_on_the_direct_kernel_match_the_oracle_and_the_wide_kernel(cuda):
    # 20k atoms, 6 nm, grid 64: the 1% types (S, P: ~200 atoms, ~10 per tile)
    # are sparse, the others stay on the wide kernel
    s = cubic_system(20_000, 60.0, seed=71, jitter=0.3, nframes=3)
    frames = s.frames(0, 3)
    h, n, path = _run(s, (64, 64, 64), frames, None)
    assert path & WIDE_BIT and path & SPARSE_BIT, path
    ho, no, _ = oracle_hist(s, (64, 64, 64), frames)
    assert_profiles_close(h, n, ho, no)
    hw, nw, pw = _run(s, (64, 64, 64), frames, "0")
    assert pw & WIDE_BIT and not pw & SPARSE_BIT, pw
    assert_profiles_close(h, n, hw, nw, rtol=1e-5)


@pytest.mark.parametrize("ensemble", ["npt", "nvt"])
def test_every_type_on_the_direct_kernel(cuda, ensemble):
    s = cubic_system(12_000, 48.0, seed=72, jitter=0.3, nframes=2)
    frames = s.frames(0, 2)
    h, n, path = _run(s, (48, 48, 48), frames, "1e9", ensemble=ensemble)
    assert path & SPARSE_BIT, path
    ho, no, _ = oracle_hist(s, (48, 48, 48), frames, ensemble=ensemble)
    assert_profiles_close(h, n, ho, no, rtol=RTOL_PROFILE)


def test_triclinic_box_with_sparse_types(cuda):
    s = cubic_system(20_000, 60.0, seed=73, jitter=0.2, nframes=2)
    box = np.array([[60.0, 0.0, 0.0], [12.0, 58.0, 0.0], [6.0, 9.0, 55.0]], dtype=np.float32)
    boxes = np.stack([box, box])
    frames = s.frames(0, 2)
    h, n, path = _run(s, (64, 60, 56), frames, None, boxes=boxes)
    assert path & SPARSE_BIT, path
    ho, no, _ = oracle_hist(s, (64, 60, 56), frames, boxes=boxes)
    assert_profiles_close(h, n, ho, no)
