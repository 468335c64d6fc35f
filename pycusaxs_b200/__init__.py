"""B200-native (sm_100a) per-frame SAXS path, a drop-in behind pyCuSaxs.

* ``pycusaxs_b200.pycusaxs_cuda.run`` — the reference's ``pycusaxs_cuda.run``
* ``pycusaxs_b200.core`` — ``invoke_cuda_backend`` / ``run_saxs_calculation``
* ``pycusaxs_b200.SaxsEngine`` — frames from host or device memory, batched
"""
from .engine import SaxsEngine, format_profile, profile_rows  # noqa: F401

__all__ = ["SaxsEngine", "format_profile", "profile_rows"]
__version__ = "0.1.0"
