"""SAXS throughput benchmark: frames/s at 100k atoms on a 256^3 supercell.

Workload (one "step"): one batch of the 100-frame trajectory of the 100k-atom
system (12 nm cubic box, H/C/O/N/S/P mix, frame k = frame 0 + N(0, 0.05 nm)
per atom), grid 128, B-spline order 4, scale 2 (256^3 supercell), q-cut
0.5 /A, bin 0.002 /A (reset to the supercell's reciprocal spacing), npt
histogram in FP64 - all through the batched fused forward.

  value  frames/s with the frames already in HBM (device-timed, CUDA events,
         L2 flushed between steps)
  e2e    frames/s through the public API from pinned host buffers: every step
         copies its frames host->device and reads the histogram back
  dropin frames/s through the drop-in pycusaxs_cuda.run (the reference's own
         entry point, here re-implemented), per-frame slope of two runs, the
         same method as the reference arm

usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Under torchrun each rank processes its own 100 frames (weak scaling); the FP64
histograms are summed with one NCCL all-reduce at the end of every step.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time
from pathlib import Path

import numpy as np

REPO = Path(__file__).resolve().parent
sys.path.insert(0, str(REPO))

NATOMS = 100_000
BOX = 120.0
GRID = 128
SCALE = 2.0
QCUT = 0.5
BIN = 0.002
FRAMES = 100
JITTER = 0.5
METRIC = "SAXS frames/s @100k atoms, 256^3 supercell (batched fused forward)"
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--batch", type=int, default=FRAMES)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-multi", action="store_true")
    ap.add_argument("--no-dropin", action="store_true")
    ap.add_argument("--no-tune", action="store_true", help="keep the plan's default kernels")
    return ap.parse_args()


class ClockSampler:
    """SM clock and clock-event (throttle) reasons of the bench GPU, read through NVML
    every 2 ms from a thread while the timed region runs (reading only; nothing is
    set).  Falls back to `nvidia-smi -lms 200` when NVML cannot be loaded."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake_slowdown", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, index: int):
        self.index = index
        self.samples: list[tuple[float, int]] = []
        self.smax = None
        self._stop = threading.Event()
        self._thread = None
        self._nvml = None
        self._handle = None
        self.proc = None
        self.lines: list[str] = []

    def _open_nvml(self):
        import pynvml
        import torch

        pynvml.nvmlInit()
        try:
            props = torch.cuda.get_device_properties(self.index)
            bus = "%08x:%02x:%02x.0" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
            handle = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
        except Exception:
            handle = pynvml.nvmlDeviceGetHandleByIndex(self.index)
        self._nvml, self._handle = pynvml, handle
        self.smax = float(pynvml.nvmlDeviceGetMaxClockInfo(handle, pynvml.NVML_CLOCK_SM))

    def _poll(self):
        nv, h = self._nvml, self._handle
        while True:
            try:
                self.samples.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                     int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))))
            except Exception:
                pass
            if self._stop.wait(0.002):
                break

    def start(self):
        try:
            self._open_nvml()
            self._thread = threading.Thread(target=self._poll, daemon=True)
            self._thread.start()
            t0 = time.time()
            while not self.samples and time.time() - t0 < 1.0:  # first sample before the timed region
                time.sleep(0.001)
            return
        except Exception:
            self._nvml = None
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=lambda: self.lines.extend(l.strip() for l in self.proc.stdout),
                             daemon=True).start()
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self._nvml is not None:
            self._stop.set()
            self._thread.join(timeout=2)
            nv = self._nvml
            reasons = sorted({name for name, const in self.REASONS
                              for _, bits in self.samples if bits & getattr(nv, const, 0)})
            sm = [c for c, _ in self.samples]
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax,
                    "reasons": reasons, "samples": len(sm), "source": "nvml, 2 ms"}
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 6:
                continue
            try:
                sm.append(float(parts[0]))
                smax.append(float(parts[1]))
            except ValueError:
                continue
            for n, v in zip(names, parts[2:6]):
                if v.lower().startswith("active"):
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": sorted(reasons),
                "samples": len(sm), "source": "nvidia-smi, 200 ms"}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if world <= 1:
        return 0, 1, None
    import datetime

    import torch
    import torch.distributed as dist

    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    return dist.get_rank(), world, dist


def barrier(dist):
    if dist is not None:
        dist.barrier()


def max_over_ranks(v: float, dist) -> float:
    if dist is None:
        return v
    import torch

    t = torch.tensor([v], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


# DRAM bytes (read + write) per frame from one ncu capture of each kernel on the
# 20-frame case of the same workload (`bench.py --batch 20`); a launch's traffic
# grows with its frames, so a full launch is scaled by frames per launch.  These
# are constants of the capture named in NCU_CAPTURE, not live measurements.
NCU_DRAM_BYTES_PER_FRAME = {
    "k_spread_zdft_tcw": (32.623360e6 + 270.978304e6) / 20,
    "k_dft_tc<y>": (330.528256e6 + 83.254272e6) / 20,
    "k_dft_tc<x>": (106.054656e6 + 4.113408e6) / 20,
    "k_sort_atoms": (24.513536e6 + 3.240704e6) / 20,
}


NCU_CAPTURE = "ncu --section MemoryWorkloadAnalysis of bench.py --batch 20 (one kernel per capture)"


def traffic_per_launch(kernel: str, frames_per_launch: float):
    """DRAM bytes per launch of `kernel` (None when no capture exists)."""
    per_frame = NCU_DRAM_BYTES_PER_FRAME.get(kernel)
    return None if per_frame is None else round(per_frame * frames_per_launch)


def bench_ours(args):
    import torch

    from pycusaxs_b200 import SaxsEngine
    from pycusaxs_b200.synthetic import cubic_system

    rank, world, dist = dist_setup(args)
    dev = torch.device("cuda", torch.cuda.current_device())
    system = cubic_system(NATOMS, BOX, seed=1000 + rank, jitter=JITTER, nframes=FRAMES)
    frames = system.frames(0, FRAMES)                       # (100, N, 3) float32 host
    boxes = np.stack([system.box] * FRAMES)
    B = min(args.batch, FRAMES)
    eng = SaxsEngine((GRID,) * 3, system.atom_index(), system.natoms, system.box,
                     scale_factor=SCALE, bin_size=BIN, qcut=QCUT, max_frames=B)
    st = eng.stream
    x_dev = torch.from_numpy(frames).to(dev)
    default_cfg = eng.config()
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)
    hist_buf = torch.zeros(2 * eng.info.num_bins, dtype=torch.float64, device=dev)

    # the plan's kernel configuration, tuned on this step's frames before any timing
    tuned = None
    if not args.no_tune:
        t = eng.autotune(x_dev, boxes, repeats=3)
        tuned = {"config": t["config"], "default": default_cfg,
                 "candidates_ms": {k: round(v, 3) for k, v in t["ms"].items()}}

    def step_device():
        eng.forward(x_dev, boxes)

    def reduce_hist():
        if dist is not None:
            h, n = eng.histogram()
            hist_buf.copy_(torch.from_numpy(np.concatenate([h, n])))
            dist.all_reduce(hist_buf)

    # warm-up
    for _ in range(args.warmup):
        step_device()
    st.synchronize()
    eng.reset()
    # timed device-resident steps: L2 flush on the engine stream, then events around the step
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
          for _ in range(args.steps)]
    eng.profile_enable(True)
    clocks = ClockSampler(dev.index)
    clocks.start()
    barrier(dist)
    torch.cuda.synchronize()
    for k in range(args.steps):
        with torch.cuda.stream(st):
            flush.zero_()
        ev[k][0].record(st)
        step_device()
        ev[k][1].record(st)
    torch.cuda.synchronize()
    barrier(dist)
    ck = clocks.stop()
    eng.profile_enable(False)
    stages = eng.profile_read()
    step_ms = [a.elapsed_time(b) for a, b in ev]
    total_s = max_over_ranks(sum(step_ms) / 1e3, dist)
    reduce_hist()
    value = world * FRAMES * args.steps / total_s

    # per-kernel roofline for the dominant stage
    prof = {k: v for k, v in stages.items()}
    dom = max(prof, key=lambda k: prof[k][0])
    info = eng.info
    nkx, nky, nkz = info.kbox
    T = len(eng.type_names)
    M = system.natoms
    ex = ey = ez = GRID
    frames_timed = FRAMES * args.steps
    algo_bytes = {
        # sorted atom records in, Z half-plane out
        "k_spread_zdft": 16 * M + 8 * T * nkz * ex * ey,
        "k_ydft": 8 * T * nkz * ex * ey + 8 * T * nkz * nky * ex,
        "k_xdft_post": 8 * T * nkz * nky * ex + 4 * nkz * nky * nkx,
        # positions in, (bin, rank) keys out and back, sorted records out
        "k_sort_atoms": 12 * M + 8 * M + 8 * M + 16 * M,
        "k_hist": 4 * nkz * nky * nkx,
    }
    algo_flops = {
        "k_spread_zdft": 4 * T * ex * ey * ez * nkz,          # real x complex MAC = 2 FMA
        "k_ydft": 8 * T * nkz * ex * ey * nky,                # complex MAC = 4 FMA
        "k_xdft_post": 8 * T * nkz * nky * ex * nkx,
    }
    peaks = json.loads((REPO / "MEASURED_PEAKS.json").read_text()) if (
        REPO / "MEASURED_PEAKS.json").exists() else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    dom_ms, dom_launches = prof[dom]
    per_launch_s = dom_ms / 1e3 / max(dom_launches, 1)
    frames_per_launch = frames_timed / max(dom_launches, 1)
    achieved = algo_bytes.get(dom, 0) * frames_per_launch / per_launch_s / 1e9
    # the kernel that ran for each stage: plan path bits 0/1/2 = z/y/x DFT on tcgen05,
    # bit 3 = wide z tiles, bit 5 = sparse element types on k_spread_zdft_sparse (the
    # same stage, after the wide kernel)
    path = info.path
    kernel_of = {"k_spread_zdft": ("k_spread_zdft_ag" if path & 16 else "k_spread_zdft_tcw" if path & 8
                                   else "k_spread_zdft_tc") if path & 1 else "k_spread_zdft",
                 "k_ydft": "k_dft_tc<y>" if path & 2 else "k_ydft",
                 "k_xdft_post": "k_dft_tc<x>" if path & 4 else "k_xdft_post"}
    tensor = bool({"k_spread_zdft": 1, "k_ydft": 2, "k_xdft_post": 4}.get(dom, 0) & path)
    roofline = {"bound": "hbm", "kernel": kernel_of.get(dom, dom), "achieved": round(achieved, 1),
                "peak": hbm, "unit": "GB/s", "frac": round(achieved / hbm, 4),
                "traffic": traffic_per_launch(kernel_of.get(dom, dom), frames_per_launch),
                "traffic_note": "DRAM bytes per launch, a constant from one capture (" + NCU_CAPTURE +
                                "), scaled by frames per launch",
                "algorithmic_bytes": round(algo_bytes.get(dom, 0) * frames_per_launch),
                "peak_source": "measured" if peaks else "fallback"}
    if dom == "k_spread_zdft" and path & 32:
        roofline["stage_note"] = ("the stage runs k_spread_zdft_tcw for the dense element types and "
                                  "k_spread_zdft_sparse for the sparse ones; achieved is the stage's")
    if dom in algo_flops:
        useful = algo_flops[dom] * frames_per_launch / per_launch_s / 1e12
        if tensor and dom == "k_spread_zdft" and path & 16:
            # atom GEMM: the tensor cores also do the spreading (K = reaching atoms), so
            # the dense z-DFT FLOP count is no measure of their work
            roofline["tensor"] = {"mma_kind": "f16", "note": "spreading and z DFT as one GEMM over atoms"}
        elif tensor and dom == "k_spread_zdft" and path & 8:
            # wide z kernel: f16 head/remainder of both operands, two kind::f16 MMAs per
            # 16 z against [Bh | Bl], so four f16 products issued per useful one; the
            # dense f16 rate equals the bf16 one
            f16_peak = float(peaks.get("bf16_tflops", 1590.0))
            roofline["tensor"] = {"useful_tflops": round(useful, 2), "issued_tflops": round(4 * useful, 2),
                                  "mma_kind": "f16", "peak_tflops": f16_peak,
                                  "issued_frac": round(4 * useful / f16_peak, 4)}
        elif tensor:
            # 3xTF32: three TF32 MMAs per product; dense TF32 peak = half the bf16 one
            tf32_peak = float(peaks.get("bf16_tflops", 1590.0)) / 2
            roofline["tensor"] = {"useful_tflops": round(useful, 2), "issued_tflops": round(3 * useful, 2),
                                  "mma_kind": "tf32", "peak_tflops": tf32_peak,
                                  "issued_frac": round(3 * useful / tf32_peak, 4)}
        else:
            roofline["fp32_tflops"] = round(useful, 2)
    stage_share = {k: round(v[0] / max(sum(x[0] for x in prof.values()), 1e-9), 4)
                   for k, v in prof.items()}
    # every stage with an algorithmic byte count: achieved GB/s and fraction of the HBM peak
    stage_hbm = {}
    for k, (ms, n) in prof.items():
        if k in algo_bytes and ms > 0 and n > 0:
            gbs = algo_bytes[k] * (frames_timed / n) / (ms / 1e3 / n) / 1e9
            stage_hbm[kernel_of.get(k, k)] = {"gb_s": round(gbs, 1), "frac": round(gbs / hbm, 4)}

    # e2e through the public API from pinned host memory
    host = torch.from_numpy(frames).pin_memory()
    eng.reset()
    for _ in range(max(1, args.warmup)):
        eng.forward_host(host, boxes)
        eng.histogram()
    barrier(dist)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng.forward_host(host, boxes)
        h, n = eng.histogram()
    e2e_s = max_over_ranks(time.perf_counter() - t0, dist)
    e2e = {"value": round(world * FRAMES * args.steps / e2e_s, 1), "unit": "frames/s",
           "h2d_bytes_per_step": int(frames.nbytes), "d2h_bytes_per_step": int(h.nbytes + n.nbytes)}

    # the plain per-frame path (one frame per call), same frames, device resident
    plain = None
    if not args.no_plain:
        eng1 = SaxsEngine((GRID,) * 3, system.atom_index(), system.natoms, system.box,
                          scale_factor=SCALE, bin_size=BIN, qcut=QCUT, max_frames=1)
        for k in range(5):
            eng1.forward(x_dev[k], boxes[k])
        eng1.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(eng1.stream)
        for k in range(FRAMES):
            eng1.forward(x_dev[k], boxes[k])
        b.record(eng1.stream)
        b.synchronize()
        plain = FRAMES / (a.elapsed_time(b) / 1e3)
        eng1.close()

    dropin = None
    if rank == 0 and world == 1 and not args.no_dropin:
        dropin = dropin_rate(system, frames, args)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(system)
    adj = None
    if rank == 0 and world == 1 and not args.no_adjoint:
        adj = refinement()
    multi = None
    if rank == 0 and world == 1 and not args.no_multi:
        multi = multi_system()

    launches = sum(v[1] for v in prof.values())
    out = {
        "metric": METRIC, "value": round(value, 1), "unit": "frames/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(total_s * 1e3 / args.steps, 3), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (FP64 histogram)",
        "data": "synthetic (seeded uniform atoms, Gaussian-jittered frames)",
        "config": {"workload": "100k atoms, 12 nm cubic box, grid 128, order 4, scale 2 "
                               "(256^3 supercell), qcut 0.5/A, 100 frames per step, npt",
                   "frames_per_step_per_gpu": FRAMES, "batch": B, "l2": "flushed between steps",
                   "kbox": [nkx, nky, nkz], "plain_path_frames_per_s": round(plain, 1) if plain else None,
                   "stage_share": stage_share,
                   "stage_kernels": {k: kernel_of.get(k, k) for k in stage_share},
                   "stage_hbm": stage_hbm,
                   "kernel_config": eng.config(), "autotune": tuned,
                   "parallelism": f"frames sharded over {world} GPU(s)",
                   "adjoint": adj, "multi_system": multi},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "dropin": dropin, "clocks": ck,
        "gpu_launches": int(launches),
    }
    eng.close()
    if rank == 0:
        print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()


def refinement(steps: int = 100) -> dict:
    """50k atoms, 10 nm box, grid 128 (256^3): forward vs forward+adjoint, and Adam refinement.

    Target: the same system after a seeded 1 A Gaussian displacement of 5% of
    the atoms; loss = sum over reported bins of (log I - log I_target)^2.
    """
    import torch

    from pycusaxs_b200 import SaxsEngine
    from pycusaxs_b200.autograd import saxs_profile
    from pycusaxs_b200.synthetic import cubic_system

    s = cubic_system(50_000, 100.0, seed=77)
    rng = np.random.default_rng(78)
    moved = s.positions.copy()
    idx = rng.choice(s.natoms, s.natoms // 20, replace=False)
    moved[idx] += rng.normal(0.0, 1.0, (idx.size, 3)).astype(np.float32)
    eng = SaxsEngine((128,) * 3, s.atom_index(), s.natoms, s.box, scale_factor=2.0, bin_size=0.002,
                     qcut=0.5, box_margin=0.05)
    dev = eng.device
    with torch.no_grad():
        target = saxs_profile(torch.tensor(moved, device=dev), eng, s.box)
    # reported bins as an index tensor (a boolean mask would make every step
    # wait for the device to count it)
    idx = torch.nonzero(target > 0).squeeze(1)
    log_target = torch.log(target.index_select(0, idx))
    x = torch.tensor(s.positions, device=dev, requires_grad=True)

    def loss_fn():
        prof = saxs_profile(x, eng, s.box)
        return ((torch.log(prof.index_select(0, idx)) - log_target) ** 2).sum()

    def timed(fn, n):
        """ms per call: CUDA events on the current stream around n calls that
        never wait for the host."""
        for _ in range(3):
            fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(n):
            fn()
        b.record()
        b.synchronize()
        return a.elapsed_time(b) / n

    def fwd():
        with torch.no_grad():
            loss_fn()

    def fwd_bwd():
        x.grad = None
        loss_fn().backward()

    fwd_ms = timed(fwd, 20)
    fb_ms = timed(fwd_bwd, 20)
    opt = torch.optim.Adam([x], lr=3e-4)
    l0 = float(loss_fn().detach())
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        opt.zero_grad()
        loss = loss_fn()
        loss.backward()
        opt.step()
    torch.cuda.synchronize()
    adam_s = time.perf_counter() - t0
    l1 = float(loss_fn().detach())
    eng.close()
    return {"workload": "50k atoms, 10 nm box, grid 128, scale 2 (256^3), log-profile loss",
            "timing": "CUDA events on the current stream around 20 steps (no host waits inside)",
            "forward_ms": round(fwd_ms, 3), "forward_adjoint_ms": round(fb_ms, 3),
            "adjoint_over_forward": round(fb_ms / fwd_ms, 2),
            "adam_steps": steps, "adam_s": round(adam_s, 3), "loss_start": l0, "loss_end": l1}


def multi_system(launches: int = 3) -> dict:
    """64 independent systems (5k-200k atoms, grids 48-160), 8 frames each.

    Batched: one CUDA-graph launch per grid bucket with every system on its own
    branch (frames resident on the device).  Plain: the same 512 frames one at a
    time through per-system engines.
    """
    import torch

    from pycusaxs_b200 import SaxsEngine
    from pycusaxs_b200.batch import BatchedSaxs
    from pycusaxs_b200.synthetic import uneven_systems

    systems = uneven_systems(64, frames=8, seed=11)
    specs = [dict(atom_index=s.atom_index(), natoms=s.natoms, box0=s.box, grid=(g,) * 3,
                  scale_factor=2.0, bin_size=0.002, qcut=0.5) for s, g in systems]
    frames = [s.frames(0, 8) for s, _ in systems]
    boxes = [np.stack([s.box] * 8) for s, _ in systems]
    batch = BatchedSaxs(specs, frames=8)
    batch.run(frames, boxes)
    batch.synchronize()
    for _ in range(2):
        batch.run_resident(boxes)
    batch.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(batch.stream)
    for _ in range(launches):
        batch.run_resident(boxes)
    b.record(batch.stream)
    b.synchronize()
    nframes = 8 * len(systems)
    batched = nframes * launches / (a.elapsed_time(b) / 1e3)
    buckets = {str(k[0]): len(v) for k, v in batch.buckets.items()}
    batch.close()
    # plain per-frame path on the same frames
    total = 0.0
    for (s, g), x, bx in zip(systems, frames, boxes):
        eng = SaxsEngine((g,) * 3, s.atom_index(), s.natoms, s.box, scale_factor=2.0,
                         bin_size=0.002, qcut=0.5, max_frames=1)
        xd = torch.from_numpy(x).to(eng.device)
        eng.forward(xd[0], bx[0])
        eng.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(eng.stream)
        for k in range(8):
            eng.forward(xd[k], bx[k])
        e1.record(eng.stream)
        e1.synchronize()
        total += e0.elapsed_time(e1) / 1e3
        eng.close()
    plain = nframes / total
    return {"workload": "64 systems, 5k-200k atoms (log-uniform), 100 atoms/nm^3, grids "
                        "48-160 by box, scale 2, qcut 0.5/A, 8 frames each",
            "atoms_total": int(sum(s.natoms for s, _ in systems)), "buckets": buckets,
            "batched_frames_per_s": round(batched, 1), "plain_frames_per_s": round(plain, 1),
            "speedup": round(batched / plain, 2)}


def _silenced(fn, *args, **kw):
    """fn(*args, **kw) with file descriptor 1 sent to /dev/null (both drop-ins
    print per-frame banners, the reference's from C++)."""
    sys.stdout.flush()
    devnull = os.open(os.devnull, os.O_WRONLY)
    saved = os.dup(1)
    os.dup2(devnull, 1)
    try:
        return fn(*args, **kw)
    finally:
        sys.stdout.flush()
        os.dup2(saved, 1)
        os.close(devnull)
        os.close(saved)


def slope_rate(run_module, topo, sample: int, steps: int, warmup: int, out: str) -> tuple:
    """Frames/s of run_module.run on `topo` by the per-frame slope: (run of
    2 + sample frames - run of 2 frames) / sample, wall clock, median of `steps`;
    the run's set-up (plan creation, tables) cancels."""
    def run(nframes):
        t0 = time.perf_counter()
        _silenced(run_module.run, topo, "synthetic.tpr", "synthetic.xtc", [GRID], begin=0,
                  end=nframes - 1, stride=1, output=out, scale_factor=SCALE, bin_size=BIN,
                  qcut=QCUT)
        return time.perf_counter() - t0

    for _ in range(max(1, warmup)):
        run(2)
    per_frame = []
    for _ in range(max(1, steps)):
        t_small = run(2)
        t_big = run(2 + sample)
        per_frame.append((t_big - t_small) / sample)
    return 1.0 / statistics.median(per_frame), per_frame


def dropin_rate(system, frames, args) -> dict:
    """This repo's pycusaxs_cuda.run (the drop-in) on the same workload, timed
    like the reference arm: the topology serves the 100 precomputed frames."""
    from pycusaxs_b200 import pycusaxs_cuda
    from pycusaxs_b200.synthetic import SyntheticTopology

    topo = SyntheticTopology(system, frames=frames)
    sample = FRAMES - 2
    value, per = slope_rate(pycusaxs_cuda, topo, sample, min(args.steps, 5), 1, "/tmp/dropin_bench.dat")
    return {"value": round(value, 1), "unit": "frames/s",
            "method": f"per-frame slope: (run of {2 + sample} frames - run of 2 frames) / {sample}, "
                      "wall clock, median of steps; frames served from host memory by the topology",
            "h2d_bytes_per_frame": int(frames[0].nbytes)}


def cpu_baseline(system) -> dict:
    """The FP64 oracle on one frame of the same workload, on this host's cores."""
    from oracle import saxs_oracle as O

    cores = os.cpu_count() or 1
    O.FFT_WORKERS = cores
    names = sorted({str(e) for e in system.elements})
    ff = O.load_form_factors()
    plan = O.OraclePlan(grid=(GRID,) * 3, types=names, coeffs=np.stack([ff[n] for n in names]),
                        box0=system.box, sigma=SCALE, bin_size=BIN, qcut=QCUT)
    toa = system.type_of_atom(names)
    t0 = time.perf_counter()
    O.run_frames(plan, [(system.frame(0), system.box)], toa)
    dt = time.perf_counter() - t0
    return {"value": round(1.0 / dt, 4), "unit": "frames/s", "cores": cores, "kind": "port",
            "sample": f"1 frame of the workload through the FP64 NumPy oracle ({dt:.2f} s): "
                      f"R2C transforms on {cores} threads (scipy pocketfft), spreading and "
                      "binning in single-threaded NumPy"}


def bench_reference(args):
    rank, world, dist = (int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")),
                         None)
    if rank != 0:
        return
    refdir = REPO / "oracle" / "_ref"
    if not any(refdir.glob("pycusaxs_cuda*.so")):
        print(json.dumps({"impl": "reference", "unavailable":
                          "reference build oracle/_ref missing (run oracle/build_ref.sh)"}))
        return
    sys.path.insert(0, str(refdir))
    import pycusaxs_cuda  # the reference cudaSAXS, built from its own sources

    from pycusaxs_b200.synthetic import SyntheticTopology, cubic_system

    system = cubic_system(NATOMS, BOX, seed=1000, jitter=JITTER, nframes=FRAMES)
    topo = SyntheticTopology(system, frames=system.frames(0, FRAMES))
    sample = 10
    value, per_frame = slope_rate(pycusaxs_cuda, topo, sample, args.steps, args.warmup,
                                  "/tmp/ref_bench.dat")
    out = {"metric": METRIC, "value": round(value, 2), "unit": "frames/s", "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup,
           "ms_per_step": round(statistics.median(per_frame) * 1e3 * sample, 3),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "synthetic", "impl": "reference",
           "config": {"workload": "100k atoms, 12 nm cubic box, grid 128, order 4, scale 2 "
                                  "(256^3 supercell), qcut 0.5/A, npt",
                      "method": "per-frame slope: (run of 12 frames - run of 2 frames) / 10, "
                                "frames served from host memory by the topology"},
           "cpu_baseline": {"value": round(value, 2), "unit": "frames/s", "cores": 1,
                            "kind": "reference", "device": "the GPU (the reference has no CPU path)",
                            "sample": f"{sample} frames per step through the reference's own "
                                      "pycusaxs_cuda.run: its unmodified CUDA build (oracle/_ref) "
                                      "on this box's GPU, one host thread"},
           "e2e": {"value": round(value, 2), "unit": "frames/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}}
    print(json.dumps(out))


def main():
    args = parse()
    if args.impl == "reference":
        bench_reference(args)
    else:
        bench_ours(args)


if __name__ == "__main__":
    main()
