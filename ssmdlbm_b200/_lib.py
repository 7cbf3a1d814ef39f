"""ctypes binding of the C ABI in include/ssmd.h (libssmd.so, built in-tree).

The structures mirror the C declarations field for field; the reference's
``struct LBMFields`` member order (src/structs/LBMFields.cuh:26-49) is kept.
Loading fails loudly when the shared library has not been built: there is no
other implementation of the step to fall back to.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_float, c_int32, c_size_t, c_uint32, c_uint64, c_void_p

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("SSMD_LIB") or os.path.join(HERE, "libssmd.so")

SSMD_OK = 0
SSMD_ERR_INVALID_ARGUMENT = 1
SSMD_ERR_CUDA = 2
SSMD_ERR_UNSTABLE = 3
SSMD_ERR_UNSUPPORTED = 4

BC_PERIODIC_COPY = 0
BC_PERIODIC = 1
BC_JET = 2

STORAGE_F32 = 0
STORAGE_F16 = 1
STORAGE_BF16 = 2
STORAGE_F16_G32 = 3  # f - w as half, g as float: the reference's ENABLE_FP16=1 layout

STEP_STORE_MACROS = 1
STEP_AVERAGE = 2
DERIVED_AVERAGES = 1
DERIVED_VORTICITY = 2

PATH_AUTO = 0
PATH_GATHER = 1
PATH_TMA = 2
PATH_SLAB = 3


class LBMFields(ctypes.Structure):
    _fields_ = [(n, c_void_p) for n in (
        "rho", "ux", "uy", "uz", "pxx", "pyy", "pzz", "pxy", "pxz", "pyz",
        "phi", "normx", "normy", "normz", "ind", "fsx", "fsy", "fsz", "f", "g")]


class Params(ctypes.Structure):
    _fields_ = [
        ("nx", c_uint32), ("ny", c_uint32), ("nz", c_uint32),
        ("velocity_set", c_int32), ("storage", c_int32),
        ("bc_x", c_int32), ("bc_y", c_int32), ("bc_z", c_int32),
        ("nu_water", c_float), ("nu_oil", c_float),
        ("omco_water", c_float), ("omco_oil", c_float), ("omco_ref", c_float),
        ("sigma", c_float), ("gamma", c_float), ("omega_g", c_float),
        ("u_oil", c_float), ("oil_cx", c_float), ("oil_cy", c_float), ("oil_r2", c_float),
        ("u_water", c_float), ("water_cx", c_float), ("water_cz", c_float), ("water_r2", c_float),
        ("noise_amp", c_float), ("u_limit", c_float), ("seed", c_uint64),
        ("f_alt", c_void_p), ("g_alt", c_void_p), ("workspace", c_void_p), ("workspace_bytes", c_size_t),
        ("tile_z", c_int32), ("bulk_path", c_int32),
        ("derived", c_void_p), ("closure", c_void_p), ("reserved", c_int32 * 2),
    ]

    def copy(self) -> "Params":
        p = Params()
        ctypes.memmove(ctypes.byref(p), ctypes.byref(self), ctypes.sizeof(Params))
        return p


class Stats(ctypes.Structure):
    _fields_ = [
        ("phi_sum", c_double), ("phi_sum_next", c_double), ("mass", c_double),
        ("momentum", c_double * 3), ("kinetic", c_double), ("u_max", c_double),
        ("nonfinite", c_double), ("cells", c_double),
    ]

    def as_dict(self) -> dict:
        return {
            "phi_sum": self.phi_sum, "phi_sum_next": self.phi_sum_next, "mass": self.mass,
            "momentum": list(self.momentum), "kinetic": self.kinetic, "u_max": self.u_max,
            "nonfinite": self.nonfinite, "cells": self.cells,
        }


class Droplet(ctypes.Structure):
    _fields_ = [("root", c_uint32), ("cells", c_uint32), ("volume", c_double), ("touches_inlet", c_uint32),
                ("reserved", c_uint32)]


class Derived(ctypes.Structure):
    _fields_ = [(n, c_void_p) for n in (
        "avg_phi", "avg_ux", "avg_uy", "avg_uz", "avg_uxux", "avg_uyuy", "avg_uzuz", "avg_uxuy", "avg_uxuz",
        "avg_uyuz", "vort_x", "vort_y", "vort_z", "vort_mag")]


class Closure(ctypes.Structure):
    _fields_ = [("nut", c_void_p), ("sigma_scale", c_void_p)]


MLP_IN = 12
MLP_HIDDEN = 64
MLP_OUT = 2
MLP_PARAMS = 5378
MLP_NET_FLOATS = 5406


class SSMDError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"ssmd error {code}: {msg}")
        self.code = code


_lib = None

# (name, restype, argtypes) of every exported entry point declared in include/ssmd.h
SIGNATURES = [
    ("ssmd_abi_version", c_int32, []),
    ("ssmd_last_error", c_char_p, []),
    ("ssmd_scalar_bytes", c_size_t, [POINTER(Params)]),
    ("ssmd_f_bytes", c_size_t, [POINTER(Params)]),
    ("ssmd_g_bytes", c_size_t, [POINTER(Params)]),
    ("ssmd_workspace_bytes", c_size_t, [POINTER(Params)]),
    ("ssmd_validate", c_int32, [POINTER(Params)]),
    ("ssmd_params_reference", c_int32, [POINTER(Params), c_uint32, c_uint32, c_uint32, c_int32,
                                        c_float, c_float, c_int32, c_int32, c_int32, c_int32,
                                        c_double, c_double, c_double, c_float]),
    ("ssmd_init", c_int32, [POINTER(Params), POINTER(LBMFields), c_void_p]),
    ("ssmd_init_from_macros", c_int32, [POINTER(Params), POINTER(LBMFields), c_void_p]),
    ("ssmd_step", c_int32, [POINTER(LBMFields), POINTER(Params), c_uint64, c_uint32, c_void_p]),
    ("ssmd_capture_graph", c_int32, [POINTER(Params), POINTER(LBMFields), c_uint64, c_int32,
                                     c_uint32, c_void_p, POINTER(c_void_p)]),
    ("ssmd_graph_launch", c_int32, [c_void_p, c_void_p]),
    ("ssmd_graph_destroy", c_int32, [c_void_p]),
    ("ssmd_reduce", c_int32, [POINTER(Params), POINTER(LBMFields), c_uint64, POINTER(Stats), c_void_p]),
    ("ssmd_reduce_static", c_int32, [POINTER(Params), POINTER(LBMFields), c_uint64, POINTER(Stats),
                                     c_void_p]),
    ("ssmd_populations_to_push", c_int32, [POINTER(Params), POINTER(LBMFields), c_uint64, c_int32,
                                           c_void_p, c_void_p]),
    ("ssmd_check_status", c_int32, [POINTER(Params), POINTER(c_uint32), c_void_p]),
    ("ssmd_batch_table_bytes", c_size_t, [POINTER(Params), c_int32]),
    ("ssmd_batch_prepare", c_int32, [POINTER(Params), POINTER(LBMFields), c_int32, c_void_p, c_size_t, c_void_p]),
    ("ssmd_batch_step", c_int32, [POINTER(Params), c_int32, c_uint64, c_uint32, c_void_p, c_void_p]),
    ("ssmd_batch_capture_graph", c_int32, [POINTER(Params), c_int32, c_uint64, c_int32, c_uint32, c_void_p,
                                           c_void_p, POINTER(c_void_p)]),
    ("ssmd_checkpoint_save", c_int32, [POINTER(Params), POINTER(LBMFields), c_uint64, c_char_p, c_void_p]),
    ("ssmd_checkpoint_load", c_int32, [POINTER(Params), POINTER(LBMFields), c_char_p, POINTER(c_uint64),
                                       c_void_p]),
    ("ssmd_centreline", c_int32, [POINTER(Params), POINTER(LBMFields), c_void_p, c_void_p, c_void_p]),
    ("ssmd_droplets_scratch_bytes", c_size_t, [POINTER(Params), c_int32]),
    ("ssmd_droplets", c_int32, [POINTER(Params), POINTER(LBMFields), c_float, c_void_p, c_size_t,
                                POINTER(Droplet), c_int32, POINTER(c_int32), c_void_p]),
    ("ssmd_output_bin", c_int32, [c_char_p, c_char_p, c_uint64, c_void_p, c_uint64]),
    ("ssmd_output_vti", c_int32, [c_char_p, c_uint64, c_uint32, c_uint32, c_uint32, POINTER(c_char_p), c_int32]),
    ("ssmd_output_info", c_int32, [c_char_p, c_char_p, c_char_p, c_float, c_float, c_double, c_double,
                                   c_double, c_uint32, c_uint32, c_uint32, c_int32, c_int32,
                                   ctypes.c_int64, ctypes.c_int64]),
    ("ssmd_profile_enable", c_int32, [c_int32]),
    ("ssmd_profile_read", c_int32, [POINTER(c_float), c_int32, POINTER(c_int32)]),
    ("ssmd_profile_disable", c_int32, []),
    ("ssmd_phase_flux", c_int32, [POINTER(Params), POINTER(LBMFields), c_uint64, POINTER(c_double),
                                  POINTER(c_double), c_void_p]),
    ("ssmd_derived_update", c_int32, [POINTER(Params), POINTER(LBMFields), c_uint32, c_void_p]),
    ("ssmd_mlp_forward", c_int32, [c_void_p, c_void_p, ctypes.c_int64, c_void_p, c_void_p]),
    ("ssmd_mlp_grad", c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_int64, c_void_p, c_void_p,
                                c_void_p]),
    ("ssmd_mlp_grad_workspace_bytes", ctypes.c_size_t, []),
    ("ssmd_mlp_grad_ws", c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_int64, c_void_p, c_void_p,
                                   c_void_p, ctypes.c_size_t, c_void_p]),
    ("ssmd_mlp_adam", c_int32, [c_void_p, c_void_p, c_void_p, c_void_p, ctypes.c_int64, c_float, c_float,
                                c_float, c_float, c_void_p]),
    ("ssmd_mlp_average", c_int32, [c_void_p, c_void_p, c_float, c_void_p]),
    ("ssmd_mlp_status", c_int32, [POINTER(c_uint32)]),
    ("ssmd_closure_features", c_int32, [POINTER(Params), POINTER(LBMFields), c_void_p, c_void_p]),
    ("ssmd_closure_filter", c_int32, [POINTER(Params), POINTER(LBMFields), c_void_p, c_void_p, c_void_p,
                                      c_void_p]),
    ("ssmd_closure_targets", c_int32, [POINTER(Params), c_void_p, c_void_p, c_void_p, c_float, c_void_p,
                                       c_void_p, c_void_p]),
    ("ssmd_closure_apply", c_int32, [POINTER(Params), c_void_p, c_void_p, c_void_p, c_void_p, c_void_p,
                                     c_float, c_void_p]),
    ("ssmd_closure_refresh", c_int32, [POINTER(Params), POINTER(LBMFields), c_void_p, c_float, c_void_p, c_void_p,
                                       c_void_p]),
]


def lib():
    """Load libssmd.so once; raise if it is missing (no fallback path exists)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                f"{LIB_PATH} not found: build it with `python -m ssmdlbm_b200.build` "
                "(the step has no non-CUDA implementation)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code: int) -> None:
    if code != SSMD_OK:
        msg = lib().ssmd_last_error()
        raise SSMDError(code, msg.decode() if msg else "")


def reference_params(nx, ny, nz, velocity_set=19, u_water=0.05, u_oil=0.05, diam_water=13,
                     diam_oil=13, radius_water=-1, radius_oil=-1, reynolds_water=1400.0,
                     reynolds_oil=450.0, weber=500.0, interface_width=4.0) -> Params:
    """Parameters derived exactly as the reference's constexpr namespaces do
    (src/constants.cuh:70-101, src/functions/globalFunctions.cuh:68-104, 232-283);
    defaults are the reference's own values."""
    p = Params()
    check(lib().ssmd_params_reference(ctypes.byref(p), nx, ny, nz, velocity_set, u_water, u_oil,
                                      diam_water, diam_oil, radius_water, radius_oil,
                                      reynolds_water, reynolds_oil, weber, interface_width))
    return p
