"""ctypes binding of the C ABI declared in ``include/pycusaxs_b200.h``.

The shared library is built in-tree (``pycusaxs_b200/build.py``).  Loading
fails loudly when it is missing: there is no CPU fallback for the SAXS path.
"""
from __future__ import annotations

import ctypes
import os
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "lib" / "libpycusaxs_b200.so"

SAXS_OK = 0
SAXS_E_INVALID = -1
SAXS_E_CUDA = -2
SAXS_E_NOMEM = -3
SAXS_E_RANGE = -4
SAXS_E_DEVICE = -5
SAXS_NOALLOC_SCRATCH_BYTES = 32 << 20
SAXS_NPT = 0
SAXS_NVT = 1

#: every symbol the header declares, in declaration order
EXPORTED = (
    "saxs_plan_create", "saxs_plan_destroy", "saxs_plan_info", "saxs_plan_config",
    "saxs_plan_set_config", "saxs_forward", "saxs_histogram",
    "saxs_reset", "saxs_debug_kbox_intensity", "saxs_debug_border_sums", "saxs_debug_counters",
    "saxs_debug_wait_probe", "saxs_backward", "saxs_histogram_device", "saxs_backward_device",
    "saxs_graph_create", "saxs_graph_launch", "saxs_graph_destroy",
    "saxs_forward_noalloc", "saxs_profile_stages", "saxs_profile_stage_name", "saxs_profile_enable", "saxs_profile_read",
    "saxs_traj_open", "saxs_traj_info", "saxs_traj_read", "saxs_traj_close",
    "saxs_closest_product", "saxs_cell_oc", "saxs_histogram_parameters", "saxs_bspline_moduli",
    "saxs_last_error", "saxs_version",
)

c_float_p = ctypes.POINTER(ctypes.c_float)
c_double_p = ctypes.POINTER(ctypes.c_double)
c_int32_p = ctypes.POINTER(ctypes.c_int32)
c_int_p = ctypes.POINTER(ctypes.c_int)


class SaxsParams(ctypes.Structure):
    _fields_ = [
        ("grid", ctypes.c_int * 3),
        ("scaled_grid", ctypes.c_int * 3),
        ("order", ctypes.c_int),
        ("scale_factor", ctypes.c_float),
        ("bin_size", ctypes.c_float),
        ("qcut", ctypes.c_float),
        ("ensemble", ctypes.c_int),
        ("ntypes", ctypes.c_int),
        ("form_factors", c_float_p),
        ("natoms", ctypes.c_int),
        ("nentries", ctypes.c_int),
        ("entry_atom", c_int32_p),
        ("entry_type", c_int32_p),
        ("box0", ctypes.c_float * 9),
        ("max_frames", ctypes.c_int),
        ("box_margin", ctypes.c_float),
        ("box_mode", ctypes.c_int),
        ("padding_mode", ctypes.c_int),
        ("padding_values", c_float_p),
    ]


class SaxsPlanConfig(ctypes.Structure):
    _fields_ = [(n, ctypes.c_int) for n in (
        "z_tensor_cores", "y_tensor_cores", "x_tensor_cores", "z_wide_tiles", "z_producer_groups",
        "z_tensor_cores_available", "y_tensor_cores_available", "x_tensor_cores_available",
        "z_narrow_tiles_available", "z_wide_tiles_available", "z_producer_groups_max",
        "z_wide_producer_groups_max", "z_atom_gemm", "z_atom_gemm_available")]


class SaxsPlanInfo(ctypes.Structure):
    _fields_ = [
        ("grid", ctypes.c_int * 3),
        ("scaled_grid", ctypes.c_int * 3),
        ("bin_size", ctypes.c_float),
        ("qcut", ctypes.c_float),
        ("num_bins", ctypes.c_int),
        ("kbox", ctypes.c_int * 3),
        ("kz_count", ctypes.c_int),
        ("path", ctypes.c_int),
        ("device_bytes", ctypes.c_size_t),
        ("frames_accumulated", ctypes.c_int),
    ]


class SaxsError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, code: int, message: str):
        super().__init__(message)
        self.code = code


_lib = None


def load(path: os.PathLike | str | None = None) -> ctypes.CDLL:
    """Load the library (once).  Raises ImportError if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise ImportError(
            f"pycusaxs_b200 native library not found at {p}; build it with "
            "`python -m pycusaxs_b200.build` (requires nvcc)")
    lib = ctypes.CDLL(str(p))
    vp = ctypes.c_void_p
    lib.saxs_plan_create.argtypes = [ctypes.POINTER(SaxsParams), ctypes.POINTER(vp)]
    lib.saxs_plan_create.restype = ctypes.c_int
    lib.saxs_plan_destroy.argtypes = [vp]
    lib.saxs_plan_destroy.restype = None
    lib.saxs_plan_info.argtypes = [vp, ctypes.POINTER(SaxsPlanInfo)]
    lib.saxs_plan_info.restype = ctypes.c_int
    lib.saxs_plan_config.argtypes = [vp, ctypes.POINTER(SaxsPlanConfig)]
    lib.saxs_plan_config.restype = ctypes.c_int
    lib.saxs_plan_set_config.argtypes = [vp, ctypes.POINTER(SaxsPlanConfig)]
    lib.saxs_plan_set_config.restype = ctypes.c_int
    lib.saxs_forward.argtypes = [vp, vp, ctypes.c_int64, ctypes.c_int, c_float_p, vp]
    lib.saxs_forward.restype = ctypes.c_int
    lib.saxs_histogram.argtypes = [vp, c_double_p, c_double_p, vp]
    lib.saxs_histogram.restype = ctypes.c_int
    lib.saxs_reset.argtypes = [vp, vp]
    lib.saxs_reset.restype = ctypes.c_int
    lib.saxs_debug_kbox_intensity.argtypes = [vp, c_float_p, vp]
    lib.saxs_debug_kbox_intensity.restype = ctypes.c_int
    lib.saxs_debug_border_sums.argtypes = [vp, c_double_p, vp]
    lib.saxs_debug_border_sums.restype = ctypes.c_int
    lib.saxs_debug_counters.argtypes = [vp, c_int_p, vp]
    lib.saxs_debug_counters.restype = ctypes.c_int
    lib.saxs_debug_wait_probe.argtypes = [vp, ctypes.c_double, vp]
    lib.saxs_debug_wait_probe.restype = ctypes.c_int
    lib.saxs_backward.argtypes = [vp, vp, c_float_p, c_double_p, vp, vp]
    lib.saxs_backward.restype = ctypes.c_int
    lib.saxs_histogram_device.argtypes = [vp, vp, vp, vp]
    lib.saxs_histogram_device.restype = ctypes.c_int
    lib.saxs_backward_device.argtypes = [vp, vp, c_float_p, vp, vp, vp]
    lib.saxs_backward_device.restype = ctypes.c_int
    lib.saxs_graph_create.argtypes = [ctypes.POINTER(vp), ctypes.POINTER(vp),
                                      ctypes.POINTER(ctypes.c_int64), c_int_p, ctypes.c_int,
                                      ctypes.POINTER(vp)]
    lib.saxs_graph_create.restype = ctypes.c_int
    lib.saxs_graph_launch.argtypes = [vp, c_float_p, vp]
    lib.saxs_graph_launch.restype = ctypes.c_int
    lib.saxs_graph_destroy.argtypes = [vp]
    lib.saxs_graph_destroy.restype = None
    lib.saxs_forward_noalloc.argtypes = [vp, vp, c_float_p, vp, vp, vp]
    lib.saxs_forward_noalloc.restype = ctypes.c_int
    lib.saxs_profile_stages.argtypes = []
    lib.saxs_profile_stages.restype = ctypes.c_int
    lib.saxs_profile_stage_name.argtypes = [ctypes.c_int]
    lib.saxs_profile_stage_name.restype = ctypes.c_char_p
    lib.saxs_profile_enable.argtypes = [vp, ctypes.c_int]
    lib.saxs_profile_enable.restype = ctypes.c_int
    lib.saxs_profile_read.argtypes = [vp, c_double_p, c_int_p]
    lib.saxs_profile_read.restype = ctypes.c_int
    lib.saxs_traj_open.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.POINTER(vp)]
    lib.saxs_traj_open.restype = ctypes.c_int
    lib.saxs_traj_info.argtypes = [vp, c_int_p, ctypes.POINTER(ctypes.c_longlong)]
    lib.saxs_traj_info.restype = ctypes.c_int
    lib.saxs_traj_read.argtypes = [vp, ctypes.c_longlong, c_float_p, c_float_p, c_double_p]
    lib.saxs_traj_read.restype = ctypes.c_int
    lib.saxs_traj_close.argtypes = [vp]
    lib.saxs_traj_close.restype = None
    lib.saxs_closest_product.argtypes = [ctypes.c_int, ctypes.c_float]
    lib.saxs_closest_product.restype = ctypes.c_int64
    lib.saxs_cell_oc.argtypes = [c_float_p, c_float_p]
    lib.saxs_cell_oc.restype = ctypes.c_int
    lib.saxs_histogram_parameters.argtypes = [c_int_p, c_float_p, ctypes.c_float, ctypes.c_float,
                                              ctypes.c_float, c_float_p, c_float_p, c_int_p]
    lib.saxs_histogram_parameters.restype = ctypes.c_int
    lib.saxs_bspline_moduli.argtypes = [ctypes.c_int, ctypes.c_int, c_float_p]
    lib.saxs_bspline_moduli.restype = ctypes.c_int
    lib.saxs_last_error.argtypes = []
    lib.saxs_last_error.restype = ctypes.c_char_p
    lib.saxs_version.argtypes = []
    lib.saxs_version.restype = ctypes.c_char_p
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != SAXS_OK:
        msg = load().saxs_last_error().decode(errors="replace") or f"status {rc}"
        raise SaxsError(rc, msg)
