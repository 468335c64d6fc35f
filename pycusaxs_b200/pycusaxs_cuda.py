"""Drop-in for the reference's ``pycusaxs_cuda`` extension module.

``run(...)`` has the signature, keyword defaults, validation messages, error
types, returned dict and output file of the reference's pybind11 entry point
(cpp-src/pybind/cuda_bindings.cpp:11-196) and of what it drives:
run_cuda_saxs (cpp-src/cudaSAXS.cu:48-232) and RunSaxs::Run
(cpp-src/Exec/RunSaxs.cu:94-271).  The numerics run in the sm_100a library
through ``SaxsEngine``.

Behaviour kept from the reference, on purpose:

* a Python exception raised by the topology callbacks is printed to stderr and
  swallowed, and no output file is written (RunSaxs.cu:267-270);
* a frame whose data cannot be read ends the iteration; the frames read so far
  are written (RunSaxs.cu:48-92, 160-169);
* a frame that fails to process is reported and skipped (RunSaxs.cu:195-199);
* the returned ``scaled_grid`` is the value given, [0, 0, 0] when it was
  derived from the scale factor (cudaSAXS.cu:93-95, 220-225);
* the requested bin size and q-cut are reset to the supercell's reciprocal
  spacing and Nyquist limit (saxsKernel.cu:489-526).

Deliberate differences: run state is per call (the reference keeps
``Options::Simulation`` and the nvt frame counter in process-wide statics,
Options.cpp:16, saxsKernel.cu:15); an element without form-factor
coefficients raises ``RuntimeError`` instead of reading undefined memory
(Scattering.h:13-24).
"""
from __future__ import annotations

import sys
import time
from typing import Any

import numpy as np

BOLD = "\x1b[1m"
RESET = "\x1b[0m"
CYAN = "\x1b[38;2;0;255;255m"
DEFAULT_OUTPUT = "saxs.dat"  # Options.cpp:15


def _bold(s: str) -> str:
    return f"{BOLD}{s}{RESET}"


def _int_list(values, what: str) -> list[int]:
    try:
        return [int(v) for v in values]
    except TypeError as exc:
        raise TypeError(f"{what} must be a sequence of integers") from exc


def _validate(grid, scaled_grid, begin, end, stride, order, scale_factor, bin_size, qcut):
    """cuda_bindings.cpp:33-122 (same order, same messages, ValueError)."""
    if len(grid) == 0:
        raise ValueError("Grid must have at least one dimension")
    if len(grid) == 1:
        if grid[0] <= 0:
            raise ValueError("Grid dimension must be positive")
    elif len(grid) == 3:
        if grid[0] <= 0 or grid[1] <= 0 or grid[2] <= 0:
            raise ValueError("Grid dimensions must be positive")
    else:
        raise ValueError("Grid must have either 1 or 3 dimensions (nx, ny, nz)")
    norm_grid = [grid[0]] * 3 if len(grid) == 1 else list(grid)
    norm_scaled: list[int] = []
    if len(scaled_grid) > 0:
        if len(scaled_grid) == 1:
            if scaled_grid[0] <= 0:
                raise ValueError("Scaled grid dimension must be positive")
            norm_scaled = [scaled_grid[0]] * 3
        elif len(scaled_grid) == 3:
            if scaled_grid[0] <= 0 or scaled_grid[1] <= 0 or scaled_grid[2] <= 0:
                raise ValueError("Scaled grid dimensions must be positive")
            norm_scaled = list(scaled_grid)
        else:
            raise ValueError("Scaled grid must have either 1 or 3 dimensions")
    if stride <= 0:
        raise ValueError("Stride must be positive")
    if order < 1 or order > 8:
        raise ValueError("Spline order must be between 1 and 8")
    if bin_size < 0.0:
        raise ValueError("Bin size must be non-negative")
    if qcut < 0.0:
        raise ValueError("Q cutoff must be non-negative")
    if scale_factor < 0.0:
        raise ValueError("Scale factor must be non-negative")
    if not norm_scaled and scale_factor == 0.0:
        raise ValueError("Scale factor must be positive when scaled grid is not provided")
    if begin < 0 or end < 0:
        raise ValueError("Frame indices must be non-negative")
    if begin > end:
        raise ValueError("Begin frame must be less than or equal to end frame")
    return norm_grid, norm_scaled


def build_summary(topology, trajectory, grid, scaled, begin, end, stride, order, sigma, dq, qcut,
                  water_model, ions: dict) -> str:
    """The configuration banner run_cuda_saxs returns as 'summary' (cudaSAXS.cu:97-214)."""
    f32 = lambda v: float(np.float32(v))  # noqa: E731  (Options fields are float)
    banner = ("\n"
              "╔" + "═" * 64 + "╗\n"
              "║" + " " * 18 + "CuSAXS Configuration" + " " * 25 + "║\n"
              "╚" + "═" * 64 + "╝\n")
    inputs = f"\n{_bold('Input Files')}\n  Topology      : {topology}\n  Trajectory    : {trajectory}\n"
    total = (end - begin) // stride + 1
    frames = (f"\n{_bold('Frame Selection')}\n  Start Frame   : {begin}\n  End Frame     : {end}\n"
              f"  Stride        : {stride}\n  Total Frames  : {total}\n")
    if scaled:
        gridi = (f"\n{_bold('Grid Parameters')}\n  Primary Grid  : ({grid[0]}, {grid[1]}, {grid[2]})\n"
                 f"  Scaled Grid   : ({scaled[0]}, {scaled[1]}, {scaled[2]})\n"
                 f"  Spline Order  : {order}\n")
    else:
        gridi = (f"\n{_bold('Grid Parameters')}\n  Grid Size     : ({grid[0]}, {grid[1]}, {grid[2]})\n"
                 f"  Spline Order  : {order}\n")
    saxs = (f"\n{_bold('SAXS Parameters')}\n  Scale Factor  : {f32(sigma):.3f}\n"
            f"  Bin Size      : {f32(dq):.4f}\n  Q-cutoff      : {f32(qcut):.3f}\n")
    ion_list = ""
    for sym in sorted(ions):
        n = ions[sym]
        if n > 0:
            s = sym
            if sym in ("Na", "K"):
                s += "⁺"
            elif sym == "Cl":
                s += "⁻"
            elif sym in ("Ca", "Mg"):
                s += "²⁺"
            ion_list += f"  {s} atoms     : {n}\n"
    if water_model:
        solvent = (f"\n{_bold('Solvent Model')}\n  Water Model   : {water_model}\n{ion_list}"
                   "  Padding Mode  : average\n")
    else:
        solvent = f"\n{_bold('Solvent Model')}\n{ion_list}  Padding Mode  : average\n"
    return banner + inputs + frames + gridi + saxs + solvent + "\n" + "-" * 66 + "\n"


def run(obj_topology: Any, topology: str, trajectory: str, grid, scaled_grid=(), begin: int = 0,
        end: int = 0, stride: int = 1, output: str = "", order: int = 4, scale_factor: float = 1.0,
        bin_size: float = 0.0, qcut: float = 0.0, water_model: str = "", sodium: int = 0,
        chlorine: int = 0, simulation: str = "", *, box_mode: str = "parity",
        padding: str = "average") -> dict:
    """Compute the SAXS profile of frames begin..end (inclusive, every ``stride``) and write it.

    Same arguments and defaults as ``pycusaxs_cuda.run`` of the reference
    (cuda_bindings.cpp:172-196).  Returns {'summary', 'grid', 'scaled_grid'}.
    Two keyword-only extensions, off by default (reference behaviour):
    ``box_mode="triclinic"`` inverts the full box matrix instead of its upper
    triangle, and ``padding="given"`` pads the supercell with bulk solvent of
    ``water_model`` (SPC/E if empty) plus ``sodium`` / ``chlorine`` ions
    (pycusaxs_b200.solvent.given_padding) instead of the z-border average.
    """
    grid_l = _int_list(grid, "grid")
    scaled_l = _int_list(scaled_grid or (), "scaled_grid")
    begin, end, stride, order = int(begin), int(end), int(stride), int(order)
    sodium, chlorine = int(sodium), int(chlorine)
    scale_factor, bin_size, qcut = float(scale_factor), float(bin_size), float(qcut)
    norm_grid, norm_scaled = _validate(grid_l, scaled_l, begin, end, stride, order, scale_factor,
                                       bin_size, qcut)
    # run_cuda_saxs checks (cudaSAXS.cu:50-65)
    if not topology:
        raise ValueError("Topology path must not be empty.")
    if not trajectory:
        raise ValueError("Trajectory path must not be empty.")
    ensemble = simulation if simulation else "npt"
    if ensemble not in ("npt", "nvt"):
        # the reference treats any other value as "neither": frames are
        # processed but nothing is binned, so the profile is empty
        ensemble = None
    out_path = output if output else DEFAULT_OUTPUT
    summary = build_summary(topology, trajectory, norm_grid, norm_scaled, begin, end, stride,
                            order, scale_factor, bin_size, qcut, water_model,
                            {"Na": sodium, "Cl": chlorine})
    print(f"{CYAN}{summary}{RESET}", end="")
    result = {"summary": summary, "grid": list(norm_grid),
              "scaled_grid": list(norm_scaled) if norm_scaled else [0, 0, 0]}
    _run_frames(obj_topology, norm_grid, norm_scaled, begin, end, stride, order, scale_factor,
                bin_size, qcut, ensemble, out_path, box_mode=box_mode, padding=padding,
                water_model=water_model, sodium=sodium, chlorine=chlorine)
    return result


class _PythonCallbackError(Exception):
    pass


# Host bytes of positions one pinned batch of run() holds at most.
_BATCH_BYTES = 64 << 20
_BATCH_MAX = 32


def _batch_frames(natoms: int, total: int) -> int:
    """Frames per batch of run(): up to 32, at most 64 MB of positions, at
    most the frames requested."""
    per = max(1, 12 * int(natoms))
    return int(max(1, min(_BATCH_MAX, _BATCH_BYTES // per, max(1, total))))


def _frame_problem(pos, box, natoms: int) -> str:
    """Why a frame cannot be processed (the checks saxs_forward would make),
    or "" - so that a batch never fails for one bad frame."""
    if pos.shape[0] < natoms:
        return f"positions hold {pos.shape[0]} atoms, the topology indexes {natoms}"
    if not np.all(np.isfinite(box)):
        return "box contains a non-finite value"
    if not (box[0, 0] > 0 and box[1, 1] > 0 and box[2, 2] > 0):
        return "box diagonal must be positive"
    return ""


class _PinnedBatches:
    """Frames of run() gathered into two alternating pinned host batches: a
    full batch goes to the device in one ``forward_host`` call (its copy runs
    on the engine's copy stream) while the next one fills; a batch is refilled
    only after its copy has completed.  A batch that fails as a whole is
    processed frame by frame, so that only the failing frames are reported and
    skipped (RunSaxs.cu:195-199)."""

    def __init__(self, engine, natoms: int, size: int):
        import torch

        self.engine = engine
        self.natoms = natoms
        self.size = size
        self.host = [torch.empty((size, natoms, 3), dtype=torch.float32).pin_memory() for _ in range(2)]
        self.view = [h.numpy() for h in self.host]
        self.boxes = [np.zeros((size, 3, 3), dtype=np.float32) for _ in range(2)]
        self.nums = [[], []]
        self.copied = [None, None]
        self.cur = 0

    def add(self, fnum, pos, box):
        b = self.cur
        n = len(self.nums[b])
        if n == 0 and self.copied[b] is not None:
            self.copied[b].synchronize()  # the batch's previous copy is complete
            self.copied[b] = None
        self.view[b][n] = pos[: self.natoms]
        self.boxes[b][n] = box
        self.nums[b].append(fnum)
        if n + 1 == self.size:
            self.flush()

    def flush(self):
        import torch

        b = self.cur
        n = len(self.nums[b])
        if n == 0:
            return
        eng = self.engine
        try:
            eng.forward_host(self.host[b][:n], self.boxes[b][:n])
        except Exception:
            eng._copy_stream.synchronize()
            for k, fnum in enumerate(self.nums[b]):
                try:
                    eng.forward_host(self.view[b][k], self.boxes[b][k])
                except Exception as exc:
                    print(f"Error processing frame {fnum}: {exc}", file=sys.stderr)
        ev = torch.cuda.Event()
        ev.record(eng._copy_stream)  # the batch's copies are queued before this
        self.copied[b] = ev
        self.nums[b] = []
        self.cur ^= 1


def _call(fn, *args):
    try:
        return fn(*args)
    except Exception as exc:  # a Python error inside a topology callback
        raise _PythonCallbackError(f"{type(exc).__name__}: {exc}") from exc


def _run_frames(topo, grid, scaled, begin, end, stride, order, sigma, dq, qcut, ensemble, out_path,
                box_mode="parity", padding="average", water_model="", sodium=0, chlorine=0):
    from .engine import SaxsEngine, format_profile

    t0 = time.perf_counter()
    try:
        index = _call(topo.get_atom_index)
        index = {str(k): [int(i) for i in v] for k, v in dict(index).items()}
        _call(topo.read_frame, 0)
        box0 = np.asarray(_call(topo.get_box), dtype=np.float32).reshape(3, 3)
        natoms = 1 + max((max(v) for v in index.values() if len(v)), default=-1)
        try:
            ext = {}
            if box_mode != "parity":
                ext["box_mode"] = box_mode
            if padding == "given":
                from .engine import entries_from_index
                from .solvent import given_padding

                names = entries_from_index(index, natoms)[0]
                ext["padding"] = "given"
                ext["padding_values"] = given_padding(names, box0, grid, water_model or "SPCE",
                                                      {"Na": sodium, "Cl": chlorine})
            elif padding != "average":
                raise ValueError(f"padding must be 'average' or 'given', not {padding!r}")
            total = len(range(begin, end + 1, stride))
            batch = _batch_frames(natoms, total)
            engine = SaxsEngine(grid, index, natoms, box0, scaled_grid=scaled or (0, 0, 0),
                                order=order, scale_factor=sigma, bin_size=dq, qcut=qcut,
                                ensemble=ensemble or "npt", max_frames=batch, **ext)
        except KeyError as exc:
            raise RuntimeError(f"CuSAXS error: {exc.args[0]}") from None
        except ValueError as exc:
            raise RuntimeError(str(exc)) from None
        info = engine.info
        if info.qcut != np.float32(qcut):
            print("\n--------------------------------------------------\n"
                  f"----- Qcut had to be reset to {info.qcut:.2f} from  {qcut:.2f} ----\n"
                  "--------------------------------------------------\n")
        if info.bin_size != np.float32(dq):
            print("\n--------------------------------------------------\n"
                  f"----- Dq had to be reset to {info.bin_size:.3f} from  {dq:.3f} ----\n"
                  "--------------------------------------------------\n")
        nn = info.scaled_grid
        print(f"  Grid sizes: {grid[0]}x{grid[1]}x{grid[2]} (cell), {nn[0]}x{nn[1]}x{nn[2]} "
              f"(supercell); k-box {info.kbox[0]}x{info.kbox[1]}x{info.kbox[2]}; "
              f"device memory {info.device_bytes / 2**30:.2f} GB")
        frames_iter = iter(_call(topo.iter_frames_stream, begin, end + 1, stride))
        batches = _PinnedBatches(engine, natoms, batch)
        while True:
            try:
                fr = next(frames_iter)
            except StopIteration:
                break
            except Exception as exc:
                raise _PythonCallbackError(f"{type(exc).__name__}: {exc}") from exc
            try:
                fnum = int(fr["frame"])
                ftime = float(fr["time"])
                pos = np.asarray(fr["positions"], dtype=np.float32)
                box = np.asarray(fr["box"], dtype=np.float32).reshape(3, 3)
                if pos.ndim != 2 or pos.shape[1] != 3:
                    raise ValueError("positions must have shape (N, 3)")
            except Exception as exc:
                print(f"Error loading frame data: {exc}", file=sys.stderr)
                break
            print(f"--> Frame: {fnum:<7}  Time Step: {ftime:.2f} ps")
            if ensemble is None:
                continue
            problem = _frame_problem(pos, box, natoms)
            if problem:
                print(f"Error processing frame {fnum}: {problem}", file=sys.stderr)
                continue
            batches.add(fnum, pos, box)
        if ensemble is not None:
            batches.flush()
        rows = engine.profile() if ensemble is not None else []
        engine.close()
        try:
            with open(out_path, "w") as fh:
                fh.write(format_profile(rows))
        except OSError as exc:
            raise RuntimeError(f"Failed to open output file: {out_path}") from exc
        total = len(range(begin, end + 1, stride))
        print(f"Done {total} Steps")
        print(f"Results written to {out_path}")
        elapsed = (time.perf_counter() - t0) * 1e3 / max(total, 1)
        print("\n=========================================================\n"
              f"=           Total Time:    {elapsed:<10.2f} ms/per step       =\n"
              "=========================================================\n")
    except _PythonCallbackError as exc:
        print(f"Python error while iterating frames: {exc}", file=sys.stderr)
