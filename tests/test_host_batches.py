"""forward_host's sub-batch schedule (CPU) and its result on the GPU.

The schedule must cover every frame exactly once, in order, with no sub-batch
above the plan's max_frames; by default its sizes grow 1.6-fold from 6 so that
the first (unoverlapped) copy is small.  On the GPU, frames fed from host memory in
that schedule, in single frames, and from device memory in one batch (more than
the 128 frames the sort kernel takes per launch in its parameters) must give the
same histogram: exact bin counts and intensities within 1e-6 relative (the
batches only change the order of the FP64 accumulation).
"""
import numpy as np
import pytest

from pycusaxs_b200.engine import _host_batches


@pytest.mark.parametrize("nf,cap,chunk", [(100, 100, None), (10, 10, None), (1, 1, None), (5, 100, None),
                                          (1000, 100, None), (250, 64, None), (37, 8, 5), (20, 20, [3, 7]),
                                          (9, 4, [16])])
def test_schedule_covers_every_frame_once(nf, cap, chunk):
    b = _host_batches(nf, cap, chunk)
    assert b[0][0] == 0 and b[-1][1] == nf
    assert all(s1 == e0 for (_, e0), (s1, _) in zip(b, b[1:]))
    assert all(1 <= e - s <= cap for s, e in b)


def test_default_schedule_grows_from_six():
    assert [e - s for s, e in _host_batches(100, 100)] == [6, 10, 15, 25, 44]
    assert [e - s for s, e in _host_batches(10, 10)] == [6, 4]
    assert [e - s for s, e in _host_batches(20, 20)] == [6, 14]
    assert [e - s for s, e in _host_batches(20, 20, [3, 7])] == [3, 7, 7, 3]


@pytest.mark.gpu
def test_host_schedules_and_device_batch_agree(cuda):
    import torch

    from pycusaxs_b200 import SaxsEngine
    from pycusaxs_b200.synthetic import cubic_system

    nf = 100
    s = cubic_system(3000, 40.0, seed=91, jitter=0.4, nframes=nf)
    frames = s.frames(0, nf)
    boxes = np.stack([s.box] * nf)
    out = []
    for how in ("device", "host-default", "host-single"):
        e = SaxsEngine((32, 32, 32), s.atom_index(), s.natoms, s.box, scale_factor=2.0, qcut=0.6,
                       max_frames=nf)
        if how == "device":
            e.forward(torch.from_numpy(frames).cuda(), boxes)
        elif how == "host-default":
            e.forward_host(torch.from_numpy(frames).pin_memory(), boxes)
        else:
            e.forward_host(frames, boxes, chunk=1)
        out.append(e.histogram())
        assert e.frames == nf
        e.close()
    h0, n0 = out[0]
    sel = n0 > 0
    for h, n in out[1:]:
        np.testing.assert_array_equal(n, n0)
        np.testing.assert_allclose(h[sel], h0[sel], rtol=1e-6)


@pytest.mark.gpu
def test_batch_above_the_sort_parameter_frames(cuda):
    # 130 frames in one call: the sort kernel takes 128 frames' geometry per launch
    # in its parameters, so this batch needs two sort launches (128 + 2 frames)
    import torch

    from pycusaxs_b200 import SaxsEngine
    from pycusaxs_b200.synthetic import cubic_system

    nf = 130
    s = cubic_system(1500, 36.0, seed=92, jitter=0.4, nframes=nf)
    frames = s.frames(0, nf)
    boxes = np.stack([s.box] * nf)
    out = []
    for batch in (nf, 1):
        e = SaxsEngine((32, 32, 32), s.atom_index(), s.natoms, s.box, scale_factor=2.0, qcut=0.6,
                       max_frames=batch)
        x = torch.from_numpy(frames).cuda()
        for k in range(0, nf, batch):
            e.forward(x[k:k + batch], boxes[k:k + batch])
        out.append(e.histogram())
        e.close()
    (h0, n0), (h1, n1) = out
    np.testing.assert_array_equal(n0, n1)
    sel = n0 > 0
    np.testing.assert_allclose(h0[sel], h1[sel], rtol=1e-6)
