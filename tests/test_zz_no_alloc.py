"""The allocation-free entry point ``saxs_forward_noalloc`` (GPU).

Callers that cannot let the library allocate device memory (a host that owns
all device memory through its own pool, or a per-step loop that must not touch
the allocator) run a frame through ``saxs_forward_noalloc`` with buffers they
already own.  These tests call it through the C ABI twice in a row on two
different frames and compare each result with the regular path
(``saxs_forward`` + ``saxs_histogram`` on a reset plan): bin counts exactly,
intensities within the suite's tolerance.  They also run it first on a fresh
plan against the FP64 oracle, with the free device memory compared across that
first call, and check that NaN positions give a NaN histogram (the call is
asynchronous and has no other way to report a kernel's error).  The file is
named so that pytest collects it last; it also passes on its own in a fresh
process.
"""
import ctypes

import numpy as np
import pytest

from helpers import RTOL_PROFILE
from pycusaxs_b200 import SaxsEngine, _native
from pycusaxs_b200.synthetic import cubic_system

pytestmark = pytest.mark.gpu


def _regular(eng, x_dev, box):
    eng.reset()
    eng.forward(x_dev, box)
    return eng.histogram()


def _noalloc(eng, x_dev, box, hist_dev, nhist_dev):
    import torch

    b = np.ascontiguousarray(np.asarray(box, np.float32).reshape(9))
    rc = eng.lib.saxs_forward_noalloc(
        eng._plan, ctypes.c_void_p(x_dev.data_ptr()), b.ctypes.data_as(_native.c_float_p),
        ctypes.c_void_p(hist_dev.data_ptr()), ctypes.c_void_p(nhist_dev.data_ptr()),
        ctypes.c_void_p(eng.stream.cuda_stream))
    _native.check(rc)
    eng.stream.synchronize()
    torch.cuda.synchronize()
    return hist_dev.cpu().numpy(), nhist_dev.cpu().numpy()


def test_two_calls_match_the_regular_forward(cuda):
    import torch

    s = cubic_system(20_000, 60.0, seed=41, jitter=0.5, nframes=2)
    eng = SaxsEngine((64, 64, 64), s.atom_index(), s.natoms, s.box, scale_factor=2.0,
                     bin_size=0.002, qcut=0.5, max_frames=1)
    nb = eng.info.num_bins
    hist_dev = torch.full((nb,), 7.0, dtype=torch.float64, device=eng.device)   # stale contents
    nhist_dev = torch.full((nb,), 7.0, dtype=torch.float64, device=eng.device)
    frames = [torch.from_numpy(s.frame(k)).to(eng.device) for k in range(2)]
    free_before_second = None
    for k, x in enumerate(frames):
        h_ref, n_ref = _regular(eng, x, s.box)
        if k == 1:
            torch.cuda.synchronize()
            free_before_second = torch.cuda.mem_get_info(eng.device)[0]
        h, n = _noalloc(eng, x, s.box, hist_dev, nhist_dev)
        if k == 1:
            # the second call took no device memory
            assert torch.cuda.mem_get_info(eng.device)[0] == free_before_second
        np.testing.assert_array_equal(n, n_ref)
        sel = n_ref > 0
        err = np.abs(h[sel] - h_ref[sel]) / np.abs(h_ref[sel])
        assert err.max() <= RTOL_PROFILE, (k, err.max())
    # the plan's own accumulators were not touched by the allocation-free calls
    h_acc, n_acc = eng.histogram()
    np.testing.assert_array_equal(n_acc, n_ref)
    eng.close()


def test_oversized_plan_is_refused_with_a_clear_error(cuda):
    import torch

    # grid 256 with a 0.6/A cut needs far more than 32 MiB of per-frame scratch
    s = cubic_system(2000, 250.0, seed=42)
    eng = SaxsEngine((256, 256, 256), s.atom_index(), s.natoms, s.box, scale_factor=2.0,
                     qcut=0.6, max_frames=1)
    hist_dev = torch.zeros(eng.info.num_bins, dtype=torch.float64, device=eng.device)
    x = torch.from_numpy(s.positions).to(eng.device)
    b = np.ascontiguousarray(s.box.reshape(9))
    rc = eng.lib.saxs_forward_noalloc(eng._plan, ctypes.c_void_p(x.data_ptr()),
                                      b.ctypes.data_as(_native.c_float_p),
                                      ctypes.c_void_p(hist_dev.data_ptr()),
                                      ctypes.c_void_p(hist_dev.data_ptr()),
                                      ctypes.c_void_p(eng.stream.cuda_stream))
    assert rc == _native.SAXS_E_RANGE
    msg = eng.lib.saxs_last_error().decode()
    assert "bytes of scratch" in msg and str(_native.SAXS_NOALLOC_SCRATCH_BYTES) in msg
    eng.close()


def test_first_call_on_a_fresh_plan_matches_the_oracle_and_allocates_nothing(cuda):
    import torch

    from helpers import assert_profiles_close, oracle_hist

    s = cubic_system(20_000, 60.0, seed=43)
    eng = SaxsEngine((64, 64, 64), s.atom_index(), s.natoms, s.box, scale_factor=2.0,
                     bin_size=0.002, qcut=0.5, max_frames=1)
    nb = eng.info.num_bins
    hist_dev = torch.full((nb,), -1.0, dtype=torch.float64, device=eng.device)
    nhist_dev = torch.full((nb,), -1.0, dtype=torch.float64, device=eng.device)
    x = torch.from_numpy(s.positions).to(eng.device)
    torch.cuda.synchronize()
    free_before = torch.cuda.mem_get_info(eng.device)[0]
    h, n = _noalloc(eng, x, s.box, hist_dev, nhist_dev)   # the plan's first frame
    assert torch.cuda.mem_get_info(eng.device)[0] == free_before
    ho, no, _ = oracle_hist(s, (64, 64, 64), [s.positions], sigma=2.0, bin_size=0.002, qcut=0.5)
    assert_profiles_close(h, n, ho, no)
    assert eng.frames == 0
    eng.close()


def test_nan_positions_give_a_nan_histogram(cuda):
    import torch

    s = cubic_system(5_000, 40.0, seed=44)
    eng = SaxsEngine((32, 32, 32), s.atom_index(), s.natoms, s.box, scale_factor=2.0, qcut=0.6,
                     max_frames=1)
    nb = eng.info.num_bins
    hist_dev = torch.zeros(nb, dtype=torch.float64, device=eng.device)
    nhist_dev = torch.zeros(nb, dtype=torch.float64, device=eng.device)
    bad = s.positions.copy()
    bad[7, 1] = np.nan
    h, n = _noalloc(eng, torch.from_numpy(bad).to(eng.device), s.box, hist_dev, nhist_dev)
    assert np.isnan(h).all() and np.isnan(n).all()
    # the next call, on good positions, is valid again; the plan's status is untouched
    h, n = _noalloc(eng, torch.from_numpy(s.positions).to(eng.device), s.box, hist_dev, nhist_dev)
    assert np.isfinite(h).all() and n.sum() > 0
    assert eng.counters()["status"] == 0
    eng.close()
