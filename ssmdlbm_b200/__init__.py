"""ssmdlbm_b200 — B200-native (sm_100a) hot path of the ssmdLBM two-phase jet solver.

The product is libssmd.so (C ABI in include/ssmd.h); this package holds its
CUDA sources (csrc/), the in-tree build (build.py), a ctypes binding (_lib),
parameter builders (configs) and the host-side driver mirror (lbm.Simulation,
which needs torch for device memory).
"""
from . import _lib, configs  # noqa: F401
from ._lib import SSMDError, check, lib  # noqa: F401

__all__ = ["_lib", "configs", "lib", "check", "SSMDError", "Simulation"]


def __getattr__(name):
    if name == "Simulation":
        from .lbm import Simulation
        return Simulation
    raise AttributeError(name)
