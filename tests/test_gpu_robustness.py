"""Device-side failure reporting and frames whose box outgrows the k-box (GPU).

Failures are made without faulting or hanging the GPU:

* the bounded mbarrier wait the pipelined kernels use is run on a barrier that
  nothing arrives at (saxs_debug_wait_probe) for a millisecond, so it gives up
  and sets the plan's status word - the next histogram reports SAXS_E_DEVICE
  naming the kernel, and after a reset the plan computes correct profiles again;
* a NaN position is caught by the sort kernel, which places the atom at the
  cell origin (all later stencil indices stay inside the cell) and reports it;
* a plan whose frame buffers exceed the free device memory is refused before
  anything is allocated (the reference's pre-check, saxsKernel.cu:284-314).

A frame whose box grows past the planned k-box margin widens the plan instead
of being dropped (the reference bins every frame with its own box,
RunSaxs.cu:176-199): npt and nvt results equal the FP64 oracle's.  Graphs and
the allocation-free call, whose buffers cannot move, refuse such a frame.
"""
import ctypes

import numpy as np
import pytest

from helpers import assert_profiles_close, oracle_hist
from pycusaxs_b200 import SaxsEngine, _native
from pycusaxs_b200.synthetic import System, cubic_system

pytestmark = pytest.mark.gpu


def _engine(s, **kw):
    kw.setdefault("max_frames", 1)
    return SaxsEngine((64, 64, 64), s.atom_index(), s.natoms, s.box, scale_factor=2.0,
                      bin_size=0.002, qcut=0.5, **kw)


def _oracle(s, frames, boxes=None, ensemble="npt"):
    return oracle_hist(s, (64, 64, 64), frames, sigma=2.0, bin_size=0.002, qcut=0.5,
                       boxes=boxes, ensemble=ensemble)


def test_wait_probe_reports_a_device_error_and_reset_recovers(cuda):
    import torch

    s = cubic_system(20_000, 60.0, seed=61)
    eng = _engine(s)
    x = torch.from_numpy(s.positions).to(eng.device)
    eng.forward(x, s.box)
    eng.wait_probe(1e-3)
    with pytest.raises(_native.SaxsError) as exc:
        eng.histogram()
    assert exc.value.code == _native.SAXS_E_DEVICE
    assert "k_wait_probe" in str(exc.value)
    assert eng.counters()["status"] == 8
    eng.reset()
    assert eng.counters()["status"] == 0
    eng.forward(x, s.box)
    h, n = eng.histogram()
    ho, no, _ = _oracle(s, [s.positions])
    assert_profiles_close(h, n, ho, no)
    eng.close()


def test_nan_position_is_reported_and_reset_recovers(cuda):
    import torch

    s = cubic_system(20_000, 60.0, seed=62)
    eng = _engine(s)
    bad = s.positions.copy()
    bad[123, 2] = np.nan
    bad[4567, 0] = np.inf
    eng.forward(torch.from_numpy(bad).to(eng.device), s.box)
    with pytest.raises(_native.SaxsError) as exc:
        eng.histogram()
    assert exc.value.code == _native.SAXS_E_DEVICE
    assert "NaN or infinite" in str(exc.value)
    assert eng.counters()["status"] & 16
    eng.reset()
    eng.forward(torch.from_numpy(s.positions).to(eng.device), s.box)
    h, n = eng.histogram()
    ho, no, _ = _oracle(s, [s.positions])
    assert_profiles_close(h, n, ho, no)
    eng.close()


def test_frame_buffers_beyond_free_memory_are_refused_before_allocating(cuda):
    import torch

    s = cubic_system(20_000, 60.0, seed=63)
    free0 = torch.cuda.mem_get_info()[0]
    with pytest.raises(_native.SaxsError) as exc:
        _engine(s, max_frames=2_000_000)
    assert exc.value.code == _native.SAXS_E_NOMEM
    assert "not enough device memory" in str(exc.value)
    assert torch.cuda.mem_get_info()[0] >= free0 - (64 << 20)
    eng = _engine(s)  # the device is still usable
    eng.close()


def _grown(s, factor, seed):
    """The system's frame with positions and box scaled by `factor` (plus jitter)."""
    rng = np.random.default_rng(seed)
    pos = (s.positions * np.float32(factor) + rng.normal(0, 0.3, s.positions.shape)).astype(np.float32)
    return pos, (s.box * np.float32(factor)).astype(np.float32)


def test_growing_box_widens_the_kbox_npt(cuda):
    import torch

    s = cubic_system(20_000, 60.0, seed=64)
    p1, b1 = _grown(s, 1.2, 1)
    eng = _engine(s, max_frames=2)
    k0 = eng.info.kbox
    x = torch.from_numpy(np.stack([s.positions, p1])).to(eng.device)
    eng.forward(x, np.stack([s.box, b1]))
    assert all(a > b for a, b in zip(eng.info.kbox[:2], k0[:2])), (eng.info.kbox, k0)
    h, n = eng.histogram()
    ho, no, _ = _oracle(s, [s.positions, p1], boxes=[s.box, b1])
    assert_profiles_close(h, n, ho, no)
    eng.close()


def test_growing_box_widens_the_kbox_nvt(cuda):
    import torch

    # the nvt intensity sum accumulated on the first k-box moves into the wider one
    s = cubic_system(20_000, 60.0, seed=65)
    p1, b1 = _grown(s, 1.2, 2)
    p2, b2 = _grown(s, 1.0, 3)
    eng = _engine(s, ensemble="nvt")
    for p, b in ((s.positions, s.box), (p1, b1), (p2, b2)):
        eng.forward(torch.from_numpy(p).to(eng.device), b)
    h, n = eng.histogram()
    ho, no, _ = _oracle(s, [s.positions, p1, p2], boxes=[s.box, b1, b2], ensemble="nvt")
    assert_profiles_close(h, n, ho, no)
    eng.close()


def test_graph_and_allocation_free_call_refuse_a_grown_box(cuda):
    import torch

    from pycusaxs_b200.batch import BatchedSaxs

    s = cubic_system(5_000, 40.0, seed=66)
    p1, b1 = _grown(s, 1.25, 4)
    spec = dict(atom_index=s.atom_index(), natoms=s.natoms, box0=s.box, grid=(32,) * 3,
                scale_factor=2.0, bin_size=0.002, qcut=0.6)
    batch = BatchedSaxs([spec], frames=1)
    with pytest.raises(_native.SaxsError) as exc:
        batch.run([p1[None]], [b1[None]])
    assert exc.value.code == _native.SAXS_E_RANGE and "grew" in str(exc.value)
    batch.close()
    eng = SaxsEngine((32, 32, 32), s.atom_index(), s.natoms, s.box, scale_factor=2.0,
                     bin_size=0.002, qcut=0.6)
    x = torch.from_numpy(p1).to(eng.device)
    hist = torch.zeros(eng.info.num_bins, dtype=torch.float64, device=eng.device)
    b = np.ascontiguousarray(b1.reshape(9))
    rc = eng.lib.saxs_forward_noalloc(eng._plan, ctypes.c_void_p(x.data_ptr()),
                                      b.ctypes.data_as(_native.c_float_p),
                                      ctypes.c_void_p(hist.data_ptr()), ctypes.c_void_p(hist.data_ptr()),
                                      ctypes.c_void_p(eng.stream.cuda_stream))
    assert rc == _native.SAXS_E_RANGE
    eng.close()
