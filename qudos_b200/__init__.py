"""qudos_b200: the QUDOS plane-wave (PWEM) solve path on NVIDIA B200 (sm_100a).

Import this package before torch or any other library that loads cuBLAS, so
that the toolkit's cuBLAS 12.9 (needed for FP32 emulation on the tensor
cores) is the one the process uses.
"""

from . import lib  # noqa: F401  (loads libqdgpu.so; raises if it is missing)
from .lib import QD_PREC_FP64, QD_PREC_MIXED, QDError, device_count  # noqa: F401
from .pwem import Problem, eigh_window_dev, solve_batch, write_energies  # noqa: F401

__all__ = ["Problem", "QDError", "QD_PREC_FP64", "QD_PREC_MIXED", "device_count", "solve_batch", "eigh_window_dev",
           "write_energies"]
