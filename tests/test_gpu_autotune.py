"""Kernel configuration and the autotuner (GPU).

A plan holds the resources of every configuration it reports as available:
the tensor-core (tcgen05, 3xTF32) or FP32 SIMT kernel for each of the z, y and
x passes, and one or two producer groups in the tensor-core spreading.  Every
candidate must give the same bin counts and, per bin, the same intensity within
2e-5 relative (the bound between the tensor-core and SIMT kernels; the 3xTF32
products are accurate to ~2^-19), and all of them must agree with the FP64
oracle within the 1e-4 profile tolerance.  The tuner must pick a candidate,
reset the accumulators, and reuse a cached choice without timing.
"""
import json

import numpy as np
import pytest
import torch

from helpers import assert_profiles_close, oracle_hist
from pycusaxs_b200 import SaxsEngine, _native
from pycusaxs_b200.synthetic import cubic_system

pytestmark = pytest.mark.gpu

CANDIDATE_RTOL = 2e-5


def _engine(s, nframes, grid=(32, 32, 32)):
    return SaxsEngine(grid, s.atom_index(), s.natoms, s.box, scale_factor=2.0, qcut=0.6,
                      max_frames=nframes)


def test_every_candidate_gives_the_same_histogram(cuda):
    s = cubic_system(6000, 40.0, seed=71, jitter=0.4, nframes=3)
    frames = np.stack([s.frame(k) for k in range(3)])
    boxes = np.stack([s.box] * 3)
    xyz = torch.from_numpy(frames).cuda()
    e = _engine(s, 3)
    cands = e.config_candidates()
    assert e.config() in cands
    assert len(cands) >= 2, cands
    results = []
    for cfg in cands:
        e.reset()
        e.set_config(cfg)
        assert e.config() == cfg
        e.forward(xyz, boxes)
        results.append(e.histogram())
    e.close()
    h0, n0 = results[0]
    sel = n0 > 0
    sel[0] = False
    ho, no, _ = oracle_hist(s, (32, 32, 32), list(frames), sigma=2.0, qcut=0.6)
    for cfg, (h, n) in zip(cands, results):
        np.testing.assert_array_equal(n, n0)
        rel = np.abs(h[sel] - h0[sel]) / np.abs(h0[sel])
        assert rel.max() <= CANDIDATE_RTOL, (cfg, rel.max())
        assert_profiles_close(h, n, ho, no)


def test_unavailable_configuration_is_refused(cuda):
    s = cubic_system(2000, 30.0, seed=72)
    e = _engine(s, 1)
    with pytest.raises(_native.SaxsError):
        e.set_config({"z_producer_groups": 3})
    with pytest.raises(_native.SaxsError):
        e.set_config({"z_producer_groups": 0})
    assert e.config() in e.config_candidates()  # the refused call changed nothing
    e.close()


def test_autotune_picks_a_candidate_resets_and_caches(cuda, tmp_path):
    s = cubic_system(6000, 40.0, seed=73, jitter=0.4, nframes=2)
    frames = np.stack([s.frame(k) for k in range(2)])
    boxes = np.stack([s.box] * 2)
    xyz = torch.from_numpy(frames).cuda()
    cache = tmp_path / "tune.json"
    e = _engine(s, 2)
    out = e.autotune(xyz, boxes, repeats=2, cache=str(cache))
    assert not out["cached"] and out["config"] in e.config_candidates()
    assert e.config() == out["config"] and e.frames == 0
    assert len(out["ms"]) == len(e.config_candidates())
    assert json.loads(cache.read_text())[e.tuning_key()] == out["config"]
    # the tuned engine still computes the same histogram as a fresh default one
    e.forward(xyz, boxes)
    h, n = e.histogram()
    with pytest.raises(RuntimeError):
        e.autotune(xyz, boxes)  # frames already accumulated
    e.close()
    ref = _engine(s, 2)
    ref.forward(xyz, boxes)
    hr, nr = ref.histogram()
    ref.close()
    np.testing.assert_array_equal(n, nr)
    sel = nr > 0
    sel[0] = False
    assert (np.abs(h[sel] - hr[sel]) / np.abs(hr[sel])).max() <= CANDIDATE_RTOL
    e2 = _engine(s, 2)
    hit = e2.autotune(xyz, boxes, cache=str(cache))
    assert hit["cached"] and e2.config() == out["config"] and hit["ms"] == {}
    e2.close()
