"""Python entry points of the reference's ``pycusaxs.core`` (core.py:56-211), on the new backend.

``invoke_cuda_backend`` and ``run_saxs_calculation`` keep the reference's
names, parameter dictionaries, defaults and error behaviour: backend errors are
returned as ``"cuda backend error: ..."`` strings, a missing backend as
``"cuda backend unavailable: ..."``; only input validation raises.
"""
from __future__ import annotations

import logging
from pathlib import Path
from typing import Any, Callable, Dict, Iterable, List

logger = logging.getLogger("pycusaxs_b200.core")


class SaxsDefaults:
    """Parameter defaults of pycusaxs/saxs_defaults.py:17-29."""

    GRID_SIZE = "128"
    INITIAL_FRAME = 0
    LAST_FRAME = 0
    OUTPUT = ""
    DT = 1
    ORDER = 4
    GRID_SCALED = 0
    SCALE_FACTOR = 2.5
    BIN_SIZE = 0.01
    QCUT = 2.0
    WATER_MODEL = ""
    SODIUM = 0.0
    CHLORINE = 0.0


def invoke_cuda_backend(required_params: Dict[str, Any], advanced_params: Dict[str, Any],
                        topology) -> List[str]:
    """core.py:56-131: call the backend's ``run`` and return its summary lines."""
    try:
        from . import pycusaxs_cuda
        from . import _native

        _native.load()
    except ImportError as exc:
        logger.error("CUDA backend unavailable: %s", exc)
        return [f"cuda backend unavailable: {exc}"]

    grid = list(required_params["grid_size"])
    scaled_raw = advanced_params.get("grid_scaled")
    scaled_grid: List[int] = []
    if isinstance(scaled_raw, (list, tuple)):
        scaled_grid = [int(v) for v in scaled_raw]
    elif isinstance(scaled_raw, int) and scaled_raw > 0:
        scaled_grid = [int(scaled_raw)]
    begin = int(required_params["initial_frame"])
    end = int(required_params["last_frame"])
    stride = max(1, int(advanced_params.get("dt", SaxsDefaults.DT)))
    logger.info("Starting SAXS calculation: frames %d-%d (stride=%d), grid=%s", begin, end, stride,
                grid)
    try:
        result = pycusaxs_cuda.run(
            obj_topology=topology,
            topology=required_params["topology"],
            trajectory=required_params["trajectory"],
            grid=grid,
            scaled_grid=scaled_grid,
            begin=begin,
            end=end,
            stride=stride,
            output=advanced_params.get("out", SaxsDefaults.OUTPUT),
            order=int(advanced_params.get("order", SaxsDefaults.ORDER)),
            scale_factor=float(advanced_params.get("scale_factor", SaxsDefaults.SCALE_FACTOR)),
            bin_size=float(advanced_params.get("bin_size", SaxsDefaults.BIN_SIZE)),
            qcut=float(advanced_params.get("qcut", SaxsDefaults.QCUT)),
            water_model=str(advanced_params.get("water_model", SaxsDefaults.WATER_MODEL)),
            sodium=int(advanced_params.get("sodium", SaxsDefaults.SODIUM)),
            chlorine=int(advanced_params.get("chlorine", SaxsDefaults.CHLORINE)),
            simulation=str(advanced_params.get("simulation", "")),
        )
        logger.info("SAXS calculation completed successfully")
    except Exception as exc:
        logger.error("CUDA backend error: %s", exc)
        return [f"cuda backend error: {exc}"]
    return [result.get("summary", "cuda backend returned no summary")]


# topology / trajectory formats read without MDAnalysis (pycusaxs_b200.trajectory)
NATIVE_TOPOLOGY = (".gro", ".pdb")
NATIVE_TRAJECTORY = (".xtc", ".trr", ".dcd", ".gro")


def _default_topology_factory(topology_path: str, trajectory_path: str):
    """GRO/PDB topology with an XTC/TRR/DCD/GRO trajectory: the native readers;
    anything else (a TPR topology, ...): the reference's MDAnalysis-backed Topology."""
    if (Path(topology_path).suffix.lower() in NATIVE_TOPOLOGY
            and Path(trajectory_path).suffix.lower() in NATIVE_TRAJECTORY):
        from .trajectory import FileTopology

        return FileTopology(topology_path, trajectory_path)
    try:
        from pycusaxs.topology import Topology  # the reference's MDAnalysis-backed loader
    except ImportError as exc:
        raise ImportError("an MDAnalysis-backed Topology (pycusaxs.topology) is required to read "
                          f"{Path(topology_path).suffix or 'these'} topology / "
                          f"{Path(trajectory_path).suffix or 'these'} trajectory files "
                          f"(read natively: topology {', '.join(NATIVE_TOPOLOGY)}; trajectory "
                          f"{', '.join(NATIVE_TRAJECTORY)}): {exc}") from exc
    return Topology(topology_path, trajectory_path)


def run_saxs_calculation(required_params: Dict[str, Any], advanced_params: Dict[str, Any],
                         topology_factory: Callable | None = None) -> Iterable[str]:
    """core.py:134-211: validate paths and frames, load the topology, run the backend.

    ``topology_factory(topology_path, trajectory_path)`` builds the topology
    object (default: the native readers for GRO/PDB topologies with TRR, DCD or
    GRO trajectories, else the reference's MDAnalysis ``Topology``).
    """
    try:
        topology_path = Path(required_params["topology"]).expanduser().resolve()
        trajectory_path = Path(required_params["trajectory"]).expanduser().resolve()
    except (OSError, RuntimeError) as e:
        raise ValueError(f"Invalid file path: {e}")
    begin = int(required_params["initial_frame"])
    end = int(required_params["last_frame"])
    if not topology_path.is_file():
        raise FileNotFoundError(f"Topology file not found: {topology_path}")
    if not trajectory_path.is_file():
        raise FileNotFoundError(f"Trajectory file not found: {trajectory_path}")
    if end < begin:
        raise ValueError(f"Last frame ({end}) must be >= initial frame ({begin})")
    factory = topology_factory or _default_topology_factory
    topo = factory(str(topology_path), str(trajectory_path))
    total_frames = int(getattr(topo, "n_frames"))
    if begin >= total_frames:
        raise ValueError(f"Initial frame {begin} exceeds available frames (0-{total_frames - 1})")
    if end >= total_frames:
        raise ValueError(f"Last frame {end} exceeds available frames (0-{total_frames - 1})")
    lines = []
    if hasattr(topo, "count_molecules"):
        counts = topo.count_molecules()
        summary = (f"Molecule counts — total: {counts[0]}, proteins: {counts[1]}, "
                   f"waters: {counts[2]}, ions: {counts[3]}, others: {counts[4]}")
        logger.info(summary)
        lines.append(summary)
    lines.extend(invoke_cuda_backend(required_params, advanced_params, topo))
    return lines
