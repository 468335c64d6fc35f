"""Batched form: several systems of uneven size in graph launches bucketed by grid (GPU).

Each system's histogram after the batched launches must equal the one its own
engine gives for the same frames (exact counts, 1e-6 relative intensities),
across two launches (the two alternating graph copies) and two buckets, and
the FP64 oracle's for those frames (exact counts, RTOL_PROFILE per bin).
"""
import numpy as np
import pytest

from helpers import assert_profiles_close, oracle_hist
from pycusaxs_b200 import SaxsEngine
from pycusaxs_b200.batch import BatchedSaxs
from pycusaxs_b200.synthetic import uneven_systems

pytestmark = pytest.mark.gpu


def _spec(s, grid):
    return dict(atom_index=s.atom_index(), natoms=s.natoms, box0=s.box, grid=(grid,) * 3,
                scale_factor=2.0, bin_size=0.002, qcut=0.5)


def test_batched_graph_equals_per_system_engines(cuda):
    import torch

    systems = uneven_systems(5, frames=3, seed=3, nmin=2000, nmax=30000, grids=(32, 48, 64))
    assert len({g for _, g in systems}) >= 2
    batch = BatchedSaxs([_spec(s, g) for s, g in systems], frames=3)
    assert len(batch.buckets) >= 2
    for launch in range(2):
        pos = [s.frames(3 * launch, 3 * launch + 3) if launch else s.frames(0, 3) for s, _ in systems]
        boxes = [np.stack([s.box] * 3) for s, _ in systems]
        batch.run(pos, boxes)
    got = batch.histograms()
    for (s, g), (h, n) in zip(systems, got):
        eng = SaxsEngine((g,) * 3, s.atom_index(), s.natoms, s.box, scale_factor=2.0,
                         bin_size=0.002, qcut=0.5, max_frames=3)
        for launch in range(2):
            x = s.frames(3 * launch, 3 * launch + 3) if launch else s.frames(0, 3)
            eng.forward(torch.from_numpy(x).to(eng.device), np.stack([s.box] * 3))
        hr, nr = eng.histogram()
        eng.close()
        np.testing.assert_array_equal(n, nr)
        sel = nr > 0
        np.testing.assert_allclose(h[sel], hr[sel], rtol=1e-6)
        frames = [s.frame(k) for k in range(6)]
        ho, no, _ = oracle_hist(s, (g,) * 3, frames, sigma=2.0, bin_size=0.002, qcut=0.5)
        assert_profiles_close(h, n, ho, no)
    batch.close()


def test_boxes_are_read_at_every_launch(cuda):
    # a launch with different boxes must bin with those boxes, not the ones seen at capture
    systems = uneven_systems(2, frames=1, seed=4, nmin=2000, nmax=4000, grids=(32,))
    batch = BatchedSaxs([_spec(s, g) for s, g in systems], frames=1)
    pos = [s.frames(0, 1) for s, _ in systems]
    batch.run(pos, [s.box[None] for s, _ in systems])
    h1 = [n.copy() for _, n in batch.histograms()]
    batch.reset()
    batch.run(pos, [(s.box * np.float32(0.98))[None] for s, _ in systems])
    h2 = [n.copy() for _, n in batch.histograms()]
    assert any(not np.array_equal(a, b) for a, b in zip(h1, h2))
    batch.close()
