"""Python host layer over the C ABI: one SAXS run on one CUDA device.

``SaxsEngine`` owns a native plan (grid sizing, tables, device buffers) and a
CUDA stream.  Frames are pushed either from device memory (``forward``) or
from host memory (``forward_host``: pinned staging, double-buffered H2D on a
copy stream overlapping the previous frames' kernels).  ``profile()`` returns
the I(q) rows the reference writes (saxsKernel.cu:210-225).

PyTorch is used only as plumbing: device/pinned allocations and streams.
"""
from __future__ import annotations

import ctypes
import itertools
import json
import os
from dataclasses import dataclass

import numpy as np

from . import _native
from .formfactors import form_factor_rows

ENSEMBLES = {"npt": _native.SAXS_NPT, "nvt": _native.SAXS_NVT}


def _torch():
    import torch

    if not torch.cuda.is_available():
        raise RuntimeError("pycusaxs_b200 needs a CUDA device (no CPU fallback)")
    return torch


@dataclass
class PlanInfo:
    grid: tuple
    scaled_grid: tuple
    bin_size: float
    qcut: float
    num_bins: int
    kbox: tuple
    device_bytes: int
    frames: int
    path: int = 0  # bits 1, 2, 4: the z-, y-, x-axis DFT on the tensor cores (tcgen05); 8: wide z tiles


CONFIG_KEYS = ("z_tensor_cores", "y_tensor_cores", "x_tensor_cores", "z_wide_tiles", "z_producer_groups",
               "z_atom_gemm")


def entries_from_index(atom_index: dict, natoms: int | None = None):
    """(type names, entry_atom, entry_type) from an element -> indices mapping.

    Types are ordered like the keys of the reference's std::map (byte-wise
    sorted, RunSaxs.cu:108-115), which fixes the order of the type sum.
    """
    names = sorted(atom_index.keys(), key=lambda s: s.encode())
    atoms, types = [], []
    for t, name in enumerate(names):
        idx = np.asarray(list(atom_index[name]), dtype=np.int64).reshape(-1)
        if idx.size and (idx.min() < 0 or (natoms is not None and idx.max() >= natoms)):
            raise ValueError(f"atom index out of range for element {name!r}")
        atoms.append(idx)
        types.append(np.full(idx.size, t, dtype=np.int32))
    ea = np.concatenate(atoms).astype(np.int32) if atoms else np.zeros(0, np.int32)
    et = np.concatenate(types) if types else np.zeros(0, np.int32)
    return names, ea, et


class SaxsEngine:
    """A SAXS run (npt or nvt) over frames of one topology."""

    def __init__(self, grid, atom_index: dict, natoms: int, box0, *, scaled_grid=(0, 0, 0),
                 order: int = 4, scale_factor: float = 1.0, bin_size: float = 0.0,
                 qcut: float = 0.0, ensemble: str = "npt", max_frames: int = 1,
                 box_margin: float = 0.05, device=None, form_factors: dict | None = None,
                 box_mode: str = "parity", padding: str = "average", padding_values=None):
        """``box_mode``: "parity" (the reference's upper-triangle inverse) or
        "triclinic" (full inverse of the box rows); ``padding``: "average" (the
        z-border mean, as the reference) or "given" with ``padding_values``: a
        mapping element -> atoms per grid point or an array in type order (see
        pycusaxs_b200.solvent.given_padding)."""
        torch = _torch()
        self._torch = torch
        self.lib = _native.load()
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = torch.device(device)
        grid = tuple(int(v) for v in (grid if len(grid) == 3 else [grid[0]] * 3))
        sg = tuple(int(v) for v in scaled_grid) if scaled_grid else (0, 0, 0)
        if len(sg) == 1:
            sg = sg * 3
        self.type_names, ea, et = entries_from_index(atom_index, natoms)
        ff = form_factor_rows(self.type_names, form_factors)
        self._ff = np.ascontiguousarray(ff, dtype=np.float32)
        self._ea = np.ascontiguousarray(ea, dtype=np.int32)
        self._et = np.ascontiguousarray(et, dtype=np.int32)
        self.natoms = int(natoms)
        self.max_frames = int(max_frames)
        p = _native.SaxsParams()
        p.grid[:] = grid
        p.scaled_grid[:] = sg
        p.order = int(order)
        p.scale_factor = float(scale_factor)
        p.bin_size = float(bin_size)
        p.qcut = float(qcut)
        if ensemble not in ENSEMBLES:
            raise ValueError(f"unknown ensemble {ensemble!r}")
        self.ensemble = ensemble
        p.ensemble = ENSEMBLES[ensemble]
        p.ntypes = len(self.type_names)
        p.form_factors = self._ff.ctypes.data_as(_native.c_float_p)
        p.natoms = self.natoms
        p.nentries = int(self._ea.size)
        p.entry_atom = self._ea.ctypes.data_as(_native.c_int32_p)
        p.entry_type = self._et.ctypes.data_as(_native.c_int32_p)
        p.box0[:] = [float(v) for v in np.asarray(box0, dtype=np.float32).reshape(9)]
        p.max_frames = self.max_frames
        p.box_margin = float(box_margin)
        if box_mode not in ("parity", "triclinic"):
            raise ValueError(f"box_mode must be 'parity' or 'triclinic', not {box_mode!r}")
        p.box_mode = 1 if box_mode == "triclinic" else 0
        if padding not in ("average", "given"):
            raise ValueError(f"padding must be 'average' or 'given', not {padding!r}")
        self._pad = None
        if padding == "given":
            if padding_values is None:
                raise ValueError("padding='given' needs padding_values")
            if isinstance(padding_values, dict):
                vals = [float(padding_values.get(t, 0.0)) for t in self.type_names]
            else:
                vals = list(np.asarray(padding_values, dtype=np.float32).reshape(-1))
            if len(vals) != len(self.type_names):
                raise ValueError("one padding value per element type is required")
            self._pad = np.ascontiguousarray(vals, dtype=np.float32)
            p.padding_mode = 1
            p.padding_values = self._pad.ctypes.data_as(_native.c_float_p)
        self._params = p
        plan = ctypes.c_void_p()
        with torch.cuda.device(self.device):
            _native.check(self.lib.saxs_plan_create(ctypes.byref(p), ctypes.byref(plan)))
        self._plan = plan
        self.stream = torch.cuda.Stream(device=self.device)
        self._copy_stream = torch.cuda.Stream(device=self.device)
        self._staging = None

    # -- plan information -------------------------------------------------
    @property
    def info(self) -> PlanInfo:
        """Sizes of the plan.  Read afresh on every access: a frame whose box
        grows beyond the k-box margin makes the plan widen its k-box."""
        return self._info()

    def _info(self) -> PlanInfo:
        i = _native.SaxsPlanInfo()
        _native.check(self.lib.saxs_plan_info(self._plan, ctypes.byref(i)))
        return PlanInfo(tuple(i.grid), tuple(i.scaled_grid), float(i.bin_size), float(i.qcut),
                        int(i.num_bins), tuple(i.kbox), int(i.device_bytes),
                        int(i.frames_accumulated), int(i.path))

    @property
    def frames(self) -> int:
        return self._info().frames

    # -- kernel configuration ----------------------------------------------
    def _config_struct(self):
        c = _native.SaxsPlanConfig()
        _native.check(self.lib.saxs_plan_config(self._plan, ctypes.byref(c)))
        return c

    def config(self) -> dict:
        """The kernel configuration in use: tensor cores (1) or FP32 SIMT (0) for
        the z, y and x passes, 128- (1) or 64-column (0) tiles and the producer
        groups of the tensor-core spreading, and whether the spreading runs as
        one tensor-core GEMM over the atoms (``z_atom_gemm``, 128-column tiles;
        the tile and group fields then do not apply)."""
        c = self._config_struct()
        return {k: int(getattr(c, k)) for k in CONFIG_KEYS}

    def config_candidates(self) -> list:
        """Every configuration the plan can run (its resources cover them all)."""
        c = self._config_struct()
        zk = [(0, 0, 1, 0)]  # (tensor cores, wide tiles, producer groups, atom GEMM)
        if c.z_narrow_tiles_available:
            zk += [(1, 0, g, 0) for g in range(1, c.z_producer_groups_max + 1)]
        if c.z_wide_tiles_available:
            zk += [(1, 1, g, 0) for g in range(1, c.z_wide_producer_groups_max + 1)]
        if c.z_atom_gemm_available:
            zk += [(1, 1, 1, 1)]
        ys = [0, 1] if c.y_tensor_cores_available else [0]
        xs = [0, 1] if c.x_tensor_cores_available else [0]
        return [{"z_tensor_cores": z, "y_tensor_cores": y, "x_tensor_cores": x, "z_wide_tiles": w,
                 "z_producer_groups": g, "z_atom_gemm": ag}
                for (z, w, g, ag), y, x in itertools.product(zk, ys, xs)]

    def set_config(self, cfg: dict) -> None:
        """Select one of ``config_candidates()``; work already queued keeps the
        configuration it was launched with."""
        c = self._config_struct()
        for k in CONFIG_KEYS:
            if k in cfg:
                setattr(c, k, int(cfg[k]))
        _native.check(self.lib.saxs_plan_set_config(self._plan, ctypes.byref(c)))

    def tuning_key(self) -> str:
        """What a tuned configuration depends on: the grids, k-box, atoms, element
        types, frames per launch and the device."""
        torch = self._torch
        i = self.info
        prop = torch.cuda.get_device_properties(self.device)
        return "|".join(str(v) for v in (
            "x".join(map(str, i.grid)), "x".join(map(str, i.scaled_grid)), "x".join(map(str, i.kbox)),
            self.natoms, int(self._ea.size), len(self.type_names), self.max_frames,
            prop.name, prop.multi_processor_count))

    def autotune(self, xyz, boxes, repeats: int = 3, cache: str | None = None) -> dict:
        """Time every candidate configuration on the frames ``xyz`` (device
        tensor, as ``forward``) and keep the fastest.

        Each candidate runs once untimed, then ``repeats`` times between CUDA
        events on the engine stream; the median decides.  Tuning runs the frames
        through the plan, so it must come before any frames are accumulated and
        it resets the accumulators afterwards.  ``cache`` (default: the
        PYCUSAXS_TUNE_CACHE environment variable) names a JSON file of earlier
        choices keyed by ``tuning_key()``: a hit is applied without timing.
        Returns {"config": ..., "ms": {candidate: median ms} , "cached": bool}.
        """
        torch = self._torch
        if self.frames:
            raise RuntimeError("autotune must run before frames are accumulated")
        cache = cache if cache is not None else os.environ.get("PYCUSAXS_TUNE_CACHE")
        key = self.tuning_key()
        cands = self.config_candidates()
        if cache and os.path.exists(cache):
            with open(cache) as fh:
                hit = json.load(fh).get(key)
            if hit is not None and hit in cands:
                self.set_config(hit)
                return {"config": dict(hit), "ms": {}, "cached": True}
        times = {}
        for cfg in cands:
            self.set_config(cfg)
            self.forward(xyz, boxes)
            ms = []
            for _ in range(max(1, int(repeats))):
                t0 = torch.cuda.Event(enable_timing=True)
                t1 = torch.cuda.Event(enable_timing=True)
                t0.record(self.stream)
                self.forward(xyz, boxes)
                t1.record(self.stream)
                t1.synchronize()
                ms.append(t0.elapsed_time(t1))
            times[json.dumps(cfg, sort_keys=True)] = float(np.median(ms))
        best = json.loads(min(times, key=times.get))
        self.set_config(best)
        self.reset()
        if cache:
            data = {}
            if os.path.exists(cache):
                with open(cache) as fh:
                    data = json.load(fh)
            data[key] = best
            tmp = f"{cache}.{os.getpid()}.tmp"
            with open(tmp, "w") as fh:
                json.dump(data, fh, indent=1, sort_keys=True)
            os.replace(tmp, cache)
        return {"config": best, "ms": times, "cached": False}

    # -- frames -----------------------------------------------------------
    def forward(self, xyz, boxes) -> None:
        """Process frames already on the device.

        ``xyz``: CUDA float32 tensor (B, natoms, 3) or (natoms, 3), contiguous
        per frame; ``boxes``: (B, 3, 3) or (3, 3) array on the host.
        """
        torch = self._torch
        if xyz.dim() == 2:
            xyz = xyz.unsqueeze(0)
        if xyz.dtype != torch.float32 or xyz.device != self.device:
            raise ValueError("xyz must be a float32 tensor on the plan's device")
        if xyz.shape[1] < self.natoms or xyz.shape[2] != 3 or xyz.stride(2) != 1 or xyz.stride(1) != 3:
            raise ValueError("xyz must have shape (B, natoms, 3) with contiguous rows")
        b = np.ascontiguousarray(np.asarray(boxes, dtype=np.float32).reshape(-1, 9))
        nf = xyz.shape[0]
        if b.shape[0] != nf:
            raise ValueError("one box per frame is required")
        for s in range(0, nf, self.max_frames):
            e = min(nf, s + self.max_frames)
            _native.check(self.lib.saxs_forward(
                self._plan, ctypes.c_void_p(xyz[s].data_ptr()), ctypes.c_int64(xyz.stride(0)),
                e - s, b[s:e].ctypes.data_as(_native.c_float_p),
                ctypes.c_void_p(self.stream.cuda_stream)))

    def forward_host(self, xyz, boxes, chunk: int | None = None) -> None:
        """Process frames held in host memory, (B, natoms, 3) or (natoms, 3).

        ``xyz`` is a numpy array or a CPU torch tensor.  A pinned tensor is
        copied straight to the device; anything else goes through a pinned
        staging buffer first.  Host-to-device copies run on a copy stream,
        double-buffered against the compute stream, in sub-batches (default:
        6, 10, 15, ... frames, see ``_host_batches``; ``chunk`` frames each if
        given) so that the copy of one sub-batch overlaps the kernels of the
        previous one.  The first sub-batch is small because its copy is not
        overlapped; the later ones grow because every sub-batch pays its
        launches' ramp-up and tail.  On a B200 (52-55 GB/s pinned host-to-device
        once warm) with 100 frames of 100k atoms per call, 6/10/15/25/44
        measured 4.00 ms per call against 4.04 ms for 4/8/16/32/40 and 4.15-4.22
        ms for schedules of eight or nine sub-batches growing 1.3-1.4-fold.
        """
        torch = self._torch
        pinned = isinstance(xyz, torch.Tensor) and xyz.device.type == "cpu" and xyz.is_pinned()
        if isinstance(xyz, torch.Tensor) and not pinned:
            xyz = xyz.detach().cpu().numpy()
        if pinned:
            x = xyz if xyz.dtype == torch.float32 else xyz.float()
            if x.dim() == 2:
                x = x.unsqueeze(0)
            x = x.contiguous()
        else:
            x = np.asarray(xyz, dtype=np.float32)
            if x.ndim == 2:
                x = x[None]
        b = np.asarray(boxes, dtype=np.float32).reshape(-1, 9)
        nf = x.shape[0]
        if b.shape[0] != nf:
            raise ValueError("one box per frame is required")
        if x.shape[1] < self.natoms or x.shape[2] != 3:
            raise ValueError("positions must have shape (B, natoms, 3)")
        st = self._staging_buffers(x.shape[1])
        for s, e in _host_batches(nf, self.max_frames, chunk):
            slot = st["next"]
            st["next"] ^= 1
            dev = st["dev"][slot]
            if pinned:
                src = x[s:e]
            else:
                host = st["host"][slot]
                st["copied"][slot].synchronize()              # staging slot free again
                np.copyto(host.numpy()[: e - s], x[s:e])
                src = host[: e - s]
            with torch.cuda.stream(self._copy_stream):
                self._copy_stream.wait_event(st["used"][slot])  # device slot free again
                dev[: e - s].copy_(src, non_blocking=True)
                st["copied"][slot].record(self._copy_stream)
            self.stream.wait_event(st["copied"][slot])
            _native.check(self.lib.saxs_forward(
                self._plan, ctypes.c_void_p(dev.data_ptr()), ctypes.c_int64(dev.stride(0)),
                e - s, np.ascontiguousarray(b[s:e]).ctypes.data_as(_native.c_float_p),
                ctypes.c_void_p(self.stream.cuda_stream)))
            st["used"][slot].record(self.stream)

    def _staging_buffers(self, rows: int):
        torch = self._torch
        if self._staging is None or self._staging["rows"] != rows:
            if self._staging is not None:  # buffers may still be in use by queued work
                self._copy_stream.synchronize()
                self.stream.synchronize()
            shape = (self.max_frames, rows, 3)
            self._staging = {
                "rows": rows,
                "host": [torch.empty(shape, dtype=torch.float32, pin_memory=True) for _ in range(2)],
                "dev": [torch.empty(shape, dtype=torch.float32, device=self.device) for _ in range(2)],
                "copied": [torch.cuda.Event() for _ in range(2)],
                "used": [torch.cuda.Event() for _ in range(2)],
                "next": 0,
            }
            for ev in self._staging["copied"] + self._staging["used"]:
                ev.record(self.stream)
        return self._staging

    # -- results ----------------------------------------------------------
    def run_trajectory(self, traj, begin: int = 0, end: int | None = None, stride: int = 1,
                       batch: int | None = None, shard: tuple | None = None) -> int:
        """Frames begin, begin+stride, ... < end of `traj` (a reader from
        pycusaxs_b200.trajectory: n_frames, n_atoms, read(k, out)) through the plan.

        A reader thread fills two pinned host batches of up to `batch` frames
        (default max_frames) while the previous batch is copied to the device and
        processed; returns the number of frames processed.  ``shard=(rank,
        world)`` keeps this rank's round-robin share of those frames (one
        process per GPU; combine with pycusaxs_b200.distributed.sharded_histogram).
        """
        from .distributed import shard as shard_frames
        from .trajectory import BatchStream

        torch = self._torch
        end = traj.n_frames if end is None else min(int(end), traj.n_frames)
        frames = range(max(0, int(begin)), end, max(1, int(stride)))
        if shard is not None:
            frames = shard_frames(frames, int(shard[0]), int(shard[1]))
        B = self.max_frames if batch is None else max(1, min(int(batch), self.max_frames))
        bufs = [torch.empty((B, traj.n_atoms, 3), dtype=torch.float32).pin_memory() for _ in range(2)]
        stream = BatchStream(traj, frames, B, bufs)
        done = 0
        try:
            for slot, buf, boxes, n in stream:
                self.forward_host(buf[:n], boxes)
                ev = torch.cuda.Event()
                ev.record(self._copy_stream)  # the batch's copies are queued before this
                stream.release(slot, ev)
                done += n
        finally:
            stream.close()
        return done

    def histogram(self):
        """FP64 (hist, nhist) accumulated so far (waits for the device)."""
        nb = self.info.num_bins
        h = np.zeros(nb, dtype=np.float64)
        n = np.zeros(nb, dtype=np.float64)
        _native.check(self.lib.saxs_histogram(self._plan, h.ctypes.data_as(_native.c_double_p),
                                              n.ctypes.data_as(_native.c_double_p),
                                              ctypes.c_void_p(self.stream.cuda_stream)))
        return h, n

    def histogram_device(self):
        """(hist, nhist) as FP64 CUDA tensors, without waiting for the device:
        ordered after the engine's queued work and before anything the caller's
        current stream does next.  A kernel error stays in the plan's status
        word (the next ``histogram()`` or ``counters()`` reports it)."""
        torch = self._torch
        nb = self.info.num_bins
        cur = torch.cuda.current_stream(self.device)
        h = torch.empty(nb, dtype=torch.float64, device=self.device)
        n = torch.empty(nb, dtype=torch.float64, device=self.device)
        self.stream.wait_stream(cur)
        _native.check(self.lib.saxs_histogram_device(self._plan, ctypes.c_void_p(h.data_ptr()),
                                                     ctypes.c_void_p(n.data_ptr()),
                                                     ctypes.c_void_p(self.stream.cuda_stream)))
        cur.wait_stream(self.stream)
        return h, n

    def profile(self):
        """I(q) rows (q, I) for bins o >= 1 with nhist != 0 (saxsKernel.cu:210-225)."""
        h, n = self.histogram()
        return profile_rows(h, n, self.info.bin_size)

    def kbox_intensity(self) -> np.ndarray:
        """Intensities of the last frame over the k-box, shape (nkz, nky, nkx)."""
        nkx, nky, nkz = self.info.kbox
        out = np.zeros(nkz * nky * nkx, dtype=np.float32)
        _native.check(self.lib.saxs_debug_kbox_intensity(
            self._plan, out.ctypes.data_as(_native.c_float_p),
            ctypes.c_void_p(self.stream.cuda_stream)))
        return out.reshape(nkz, nky, nkx)

    def counters(self) -> dict:
        """Kernel diagnostics since creation or the last reset (waits for the
        device): ``status`` (0, or the bits of the kernels that reported an
        error: 1 spreading/z pass, 2 y pass, 4 x pass, 8 wait probe, 16 a NaN or
        infinite position) and ``table_chunks`` (the most atom-table chunks one
        item of the wide spreading kernel needed; 0 when all fitted at once)."""
        out = np.zeros(4, dtype=np.int32)
        _native.check(self.lib.saxs_debug_counters(self._plan, out.ctypes.data_as(_native.c_int_p),
                                                   ctypes.c_void_p(self.stream.cuda_stream)))
        return {"status": int(out[0]), "table_chunks": int(out[1])}

    def wait_probe(self, limit_s: float = 0.001) -> None:
        """Run the kernels' bounded wait on a barrier nothing arrives at, so
        that it gives up after ``limit_s`` and sets the plan's status word (the
        next ``histogram()`` raises; ``reset()`` clears it)."""
        _native.check(self.lib.saxs_debug_wait_probe(self._plan, float(limit_s),
                                                     ctypes.c_void_p(self.stream.cuda_stream)))

    def border_sums(self) -> np.ndarray:
        out = np.zeros(len(self.type_names), dtype=np.float64)
        _native.check(self.lib.saxs_debug_border_sums(
            self._plan, out.ctypes.data_as(_native.c_double_p),
            ctypes.c_void_p(self.stream.cuda_stream)))
        return out

    def backward(self, xyz, box, dl_dhist):
        """dL/dxyz (natoms, 3) float32 CUDA tensor for one frame.

        ``dl_dhist`` holds dL/dhist for every histogram bin of the frame
        (num_bins values; the profile is hist/nhist, so pass dL/dI / nhist, 0
        for unreported bins).  The frame's transforms are recomputed from
        ``xyz``; the plan's accumulators are not touched.
        """
        torch = self._torch
        x = xyz.detach()
        if x.dim() == 3:
            x = x[0]
        if x.dtype != torch.float32 or x.device != self.device or not x.is_contiguous():
            x = x.to(self.device, torch.float32).contiguous()
        if x.shape[0] < self.natoms:
            raise ValueError("xyz must have natoms rows")
        dl = np.ascontiguousarray(np.asarray(dl_dhist, dtype=np.float64).reshape(-1))
        if dl.size != self.info.num_bins:
            raise ValueError(f"dl_dhist must have {self.info.num_bins} entries")
        b = np.ascontiguousarray(np.asarray(box, dtype=np.float32).reshape(9))
        grad = torch.empty((x.shape[0], 3), dtype=torch.float32, device=self.device)
        if x.shape[0] > self.natoms:
            grad.zero_()
        cur = torch.cuda.current_stream(self.device)
        self.stream.wait_stream(cur)
        _native.check(self.lib.saxs_backward(
            self._plan, ctypes.c_void_p(x.data_ptr()), b.ctypes.data_as(_native.c_float_p),
            dl.ctypes.data_as(_native.c_double_p), ctypes.c_void_p(grad.data_ptr()),
            ctypes.c_void_p(self.stream.cuda_stream)))
        cur.wait_stream(self.stream)
        x.record_stream(self.stream)
        return grad

    def backward_device(self, xyz, box, dl_dhist):
        """``backward`` with dL/dhist an FP64 CUDA tensor (num_bins,): nothing
        waits for the host; the work is ordered after the caller's current
        stream and before what it does next."""
        torch = self._torch
        x = xyz.detach()
        if x.dim() == 3:
            x = x[0]
        if x.dtype != torch.float32 or x.device != self.device or not x.is_contiguous():
            x = x.to(self.device, torch.float32).contiguous()
        if x.shape[0] < self.natoms:
            raise ValueError("xyz must have natoms rows")
        dl = dl_dhist.detach().to(self.device, torch.float64).contiguous().reshape(-1)
        if dl.numel() != self.info.num_bins:
            raise ValueError(f"dl_dhist must have {self.info.num_bins} entries")
        b = np.ascontiguousarray(np.asarray(box, dtype=np.float32).reshape(9))
        grad = torch.empty((x.shape[0], 3), dtype=torch.float32, device=self.device)
        if x.shape[0] > self.natoms:
            grad.zero_()
        cur = torch.cuda.current_stream(self.device)
        self.stream.wait_stream(cur)
        _native.check(self.lib.saxs_backward_device(
            self._plan, ctypes.c_void_p(x.data_ptr()), b.ctypes.data_as(_native.c_float_p),
            ctypes.c_void_p(dl.data_ptr()), ctypes.c_void_p(grad.data_ptr()),
            ctypes.c_void_p(self.stream.cuda_stream)))
        cur.wait_stream(self.stream)
        for t in (x, dl):
            t.record_stream(self.stream)
        return grad

    def profile_enable(self, on: bool = True) -> None:
        """Time every kernel of ``forward`` with CUDA events on the engine stream."""
        _native.check(self.lib.saxs_profile_enable(self._plan, int(bool(on))))

    def profile_read(self) -> dict:
        """{stage: (milliseconds, launches)} since the last read (waits for the device)."""
        n = self.lib.saxs_profile_stages()
        ms = np.zeros(n, dtype=np.float64)
        cnt = np.zeros(n, dtype=np.int32)
        _native.check(self.lib.saxs_profile_read(self._plan, ms.ctypes.data_as(_native.c_double_p),
                                                 cnt.ctypes.data_as(_native.c_int_p)))
        return {self.lib.saxs_profile_stage_name(i).decode(): (float(ms[i]), int(cnt[i]))
                for i in range(n)}

    def reset(self) -> None:
        _native.check(self.lib.saxs_reset(self._plan, ctypes.c_void_p(self.stream.cuda_stream)))

    def synchronize(self) -> None:
        self.stream.synchronize()

    def close(self) -> None:
        if getattr(self, "_plan", None):
            self.stream.synchronize()
            self._copy_stream.synchronize()
            self.lib.saxs_plan_destroy(self._plan)
            self._plan = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def _host_batches(nf: int, cap: int, chunk=None):
    """(start, stop) frame ranges of forward_host's sub-batches of an nf-frame call.

    ``chunk`` None: sizes growing 1.6-fold from 6 (6, 10, 15, 25, ...), the last
    sub-batch taking the rest when the rest is at most 1.5 times the next size
    (each copy, at ~22 us per 1.2 MB frame, then mostly hides behind the previous
    sub-batch's ~34 us per frame of kernels, and each sub-batch's fixed ~60 us of
    launch ramp and tail is paid only five times per 100 frames); an int:
    that many frames per sub-batch; a sequence of ints: those sizes in order,
    the last one repeated.  Every size is clamped to [1, cap].
    """
    if chunk is None:
        sizes, left, g = [], nf, 6.0
        while left > 0:
            n = int(round(g))
            take = left if left <= 1.5 * n else n
            sizes.append(take)
            left -= take
            g *= 1.6
    elif isinstance(chunk, (int, np.integer)):
        sizes = [int(chunk)]
    else:
        sizes = [int(c) for c in chunk] or [nf]
    out, s, i = [], 0, 0
    while s < nf:
        n = max(1, min(cap, sizes[min(i, len(sizes) - 1)]))
        out.append((s, min(nf, s + n)))
        s += n
        i += 1
    return out


def profile_rows(hist, nhist, bin_size):
    """(q, I) rows: q = o*bin_size in float32, I = hist/nhist (saxsKernel.cu:210-225)."""
    rows = []
    b = np.float32(bin_size)
    for o in range(1, len(hist)):
        if nhist[o] != 0.0:
            rows.append((float(np.float32(o) * b), float(hist[o] / nhist[o])))
    return rows


def format_profile(rows) -> str:
    """Text of the profile file (RunSaxs.cu:224-228: setw(10) fixed 5, setw(12) scientific 5)."""
    return "".join(f"{q:10.5f}{i:12.5e}\n" for q, i in rows)
