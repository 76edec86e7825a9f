"""qudos_b200: the QUDOS plane-wave (PWEM) solve path on NVIDIA B200 (sm_100a).

The deck writer (`qudos_b200.configs`) is plain Python.  Everything that
computes goes through libqdgpu.so, which is loaded the first time one of the
solver names below is used (`qudos_b200.Problem`, `qudos_b200.lib`, ...); the
load raises if the library is missing, there is no fallback.
"""

import importlib

from . import configs  # noqa: F401  (deck writer, no native code)

_SOLVER_NAMES = {
    "Problem": "pwem", "eigh_window_dev": "pwem", "solve_batch": "pwem", "write_energies": "pwem",
    "QD_PREC_FP64": "lib", "QD_PREC_MIXED": "lib", "QDError": "lib", "device_count": "lib",
}

__all__ = ["Problem", "QDError", "QD_PREC_FP64", "QD_PREC_MIXED", "device_count", "solve_batch", "eigh_window_dev",
           "write_energies", "configs"]


def __getattr__(name):
    mod = _SOLVER_NAMES.get(name)
    if mod is None:
        raise AttributeError("module 'qudos_b200' has no attribute %r" % name)
    value = getattr(importlib.import_module("." + mod, __name__), name)
    globals()[name] = value
    return value
