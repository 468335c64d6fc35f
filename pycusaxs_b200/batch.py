"""Batched form: many systems x many frames per CUDA-graph launch.

``BatchedSaxs`` takes a list of independent systems (any atom counts, boxes,
element sets and grids), builds one native plan per system, groups the plans
into buckets by grid shape, and captures one CUDA graph per bucket in which
every system's whole frame pipeline runs on its own graph branch.  A call to
``run`` copies the frames into the systems' device buffers and launches each
bucket's graph once; each system keeps its own FP64 histogram, so its profile is
exactly what the per-frame path would give for the same frames.

No counterpart in the reference, which handles one frame of one system per
call (RunSaxs.cu:154-203).
"""
from __future__ import annotations

import ctypes
from collections import OrderedDict

import numpy as np

from . import _native
from .engine import SaxsEngine, _torch


class BatchedSaxs:
    def __init__(self, systems: list[dict], frames, *, device=None, bucket_by: str = "grid"):
        """``systems``: dicts with ``atom_index``, ``natoms``, ``box0``, ``grid`` and the
        optional SaxsEngine keywords (scaled_grid, order, scale_factor, bin_size,
        qcut, ensemble, box_margin).  ``frames``: frames per launch, one int for
        all systems or one per system."""
        torch = _torch()
        self._torch = torch
        self.lib = _native.load()
        n = len(systems)
        self.frames = [int(frames)] * n if np.isscalar(frames) else [int(f) for f in frames]
        if len(self.frames) != n:
            raise ValueError("one frame count per system is required")
        self.engines: list[SaxsEngine] = []
        self.buffers = []
        for spec, nf in zip(systems, self.frames):
            kw = {k: v for k, v in spec.items() if k not in ("atom_index", "natoms", "box0", "grid")}
            eng = SaxsEngine(spec["grid"], spec["atom_index"], spec["natoms"], spec["box0"],
                             max_frames=nf, device=device, **kw)
            self.engines.append(eng)
            self.buffers.append(torch.empty((nf, spec["natoms"], 3), dtype=torch.float32,
                                            device=eng.device))
        self.device = self.engines[0].device
        self.stream = torch.cuda.Stream(device=self.device)
        self.buckets: "OrderedDict[tuple, list[int]]" = OrderedDict()
        for i, e in enumerate(self.engines):
            key = tuple(e.info.grid) if bucket_by == "grid" else (i,)
            self.buckets.setdefault(key, []).append(i)
        self._graphs = []
        for key, idx in self.buckets.items():
            plans = (ctypes.c_void_p * len(idx))(*[self.engines[i]._plan.value for i in idx])
            ptrs = (ctypes.c_void_p * len(idx))(*[self.buffers[i].data_ptr() for i in idx])
            strides = (ctypes.c_int64 * len(idx))(*[self.buffers[i].stride(0) for i in idx])
            nfs = (ctypes.c_int * len(idx))(*[self.frames[i] for i in idx])
            g = ctypes.c_void_p()
            torch.cuda.synchronize(self.device)
            _native.check(self.lib.saxs_graph_create(plans, ptrs, strides, nfs, len(idx),
                                                     ctypes.byref(g)))
            self._graphs.append((key, idx, g))

    def run(self, positions, boxes) -> None:
        """One launch per bucket.  ``positions[i]``: (frames_i, natoms_i, 3) host
        array or tensor for system i; ``boxes[i]``: (frames_i, 3, 3)."""
        torch = self._torch
        with torch.cuda.stream(self.stream):
            for i, x in enumerate(positions):
                src = x if isinstance(x, torch.Tensor) else torch.from_numpy(
                    np.ascontiguousarray(x, dtype=np.float32))
                self.buffers[i].copy_(src.reshape(self.buffers[i].shape), non_blocking=True)
        for key, idx, g in self._graphs:
            b = np.ascontiguousarray(np.concatenate(
                [np.asarray(boxes[i], dtype=np.float32).reshape(-1, 9) for i in idx]))
            if b.shape[0] != sum(self.frames[i] for i in idx):
                raise ValueError("one box per frame is required")
            _native.check(self.lib.saxs_graph_launch(g, b.ctypes.data_as(_native.c_float_p),
                                                     ctypes.c_void_p(self.stream.cuda_stream)))

    def run_resident(self, boxes) -> None:
        """Launch every bucket on the frames already in the device buffers."""
        for key, idx, g in self._graphs:
            b = np.ascontiguousarray(np.concatenate(
                [np.asarray(boxes[i], dtype=np.float32).reshape(-1, 9) for i in idx]))
            _native.check(self.lib.saxs_graph_launch(g, b.ctypes.data_as(_native.c_float_p),
                                                     ctypes.c_void_p(self.stream.cuda_stream)))

    def synchronize(self) -> None:
        self.stream.synchronize()

    def histograms(self):
        self.synchronize()
        return [e.histogram() for e in self.engines]

    def profiles(self):
        self.synchronize()
        return [e.profile() for e in self.engines]

    def reset(self) -> None:
        self.synchronize()
        for e in self.engines:
            e.reset()

    def close(self) -> None:
        if getattr(self, "_graphs", None) is not None:
            self.synchronize()
            for _, _, g in self._graphs:
                self.lib.saxs_graph_destroy(g)
            self._graphs = None
            for e in self.engines:
                e.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
