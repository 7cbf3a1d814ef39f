"""C ABI checks that need no GPU: exports, struct layout, validation, parameters."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

from ssmdlbm_b200 import _lib, configs
from ssmdlbm_b200._lib import LBMFields, Params, Stats, lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "ssmd.h")


def declared_functions():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(ssmd_[a-z_0-9]+)\s*\(", text)))


def test_every_declared_symbol_is_exported():
    names = declared_functions()
    assert len(names) >= 15
    out = subprocess.run(["nm", "-D", "--defined-only", _lib.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = set(re.findall(r"\sT\s(ssmd_\w+)", out))
    missing = [n for n in names if n not in exported]
    assert not missing, missing
    # and the ctypes binding knows all of them
    bound = {s[0] for s in _lib.SIGNATURES}
    assert set(names) <= bound, set(names) - bound
    L = lib()
    for n in names:
        assert hasattr(L, n)


def test_struct_layout_matches_header(tmp_path):
    """sizeof/offsetof of the C structs equal the ctypes mirrors."""
    members = {
        "LBMFields": [f[0] for f in LBMFields._fields_],
        "ssmd_params": [f[0] for f in Params._fields_],
        "ssmd_stats": [f[0] for f in Stats._fields_],
    }
    src = ['#include <stdio.h>', '#include <stddef.h>', f'#include "{HEADER}"', "int main(void){"]
    for s, ms in members.items():
        src.append(f'printf("{s} %zu\\n", sizeof({s}));')
        for m in ms:
            src.append(f'printf("{s}.{m} %zu\\n", offsetof({s}, {m}));')
    src.append("return 0;}")
    c = tmp_path / "layout.c"
    c.write_text("\n".join(src))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c99", "-o", str(exe), str(c)], check=True)
    got = dict(line.split() for line in subprocess.run([str(exe)], capture_output=True, text=True,
                                                        check=True).stdout.splitlines())
    py = {"LBMFields": LBMFields, "ssmd_params": Params, "ssmd_stats": Stats}
    for s, T in py.items():
        assert int(got[s]) == ctypes.sizeof(T), s
        for m in members[s]:
            assert int(got[f"{s}.{m}"]) == getattr(T, m).offset, (s, m)


def test_lbmfields_member_order_is_the_references():
    # src/structs/LBMFields.cuh:26-49
    assert [f[0] for f in LBMFields._fields_] == [
        "rho", "ux", "uy", "uz", "pxx", "pyy", "pzz", "pxy", "pxz", "pyz", "phi", "normx", "normy",
        "normz", "ind", "fsx", "fsy", "fsz", "f", "g"]


def test_reference_parameters_match_reference_constants():
    # the reference's defaults: u = 0.05, D = 13, Re = 1400 / 450, We = 500, W = 4
    p = _lib.reference_params(128, 256, 256, 19)
    f32 = np.float32
    nu_w = f32(0.05 * 13 / 1400.0)  # FP64 then FP32 (globalFunctions.cuh:234-237)
    nu_o = f32(0.05 * 13 / 450.0)
    assert p.nu_water == nu_w and p.nu_oil == nu_o
    assert p.omco_water == f32(1) - f32(1.0 / (0.5 + 3.0 * float(nu_w)))
    assert p.omco_ref == p.omco_water
    assert p.sigma == f32(f32(f32(0.05) * f32(0.05)) * f32(13)) / f32(500)
    assert p.gamma == f32(0.5)  # 4 * (1/4)(1 - 1/2) / 4 / (1/4)
    assert p.oil_cx == f32(127 * 0.5) and p.oil_cy == f32(0.5) * f32(255 * 0.5)
    assert p.water_cz == f32(0.7) * f32(255 * 0.5)
    assert p.oil_r2 == 36.0 and p.water_r2 == 36.0  # radius = 13 / 2 = 6 in integers
    assert (p.bc_x, p.bc_y, p.bc_z) == (_lib.BC_PERIODIC_COPY, _lib.BC_JET, _lib.BC_JET)
    assert lib().ssmd_validate(ctypes.byref(p)) == 0


@pytest.mark.parametrize("mutate,fragment", [
    (lambda p: setattr(p, "velocity_set", 15), "velocity_set"),
    (lambda p: setattr(p, "storage", 7), "storage"),
    (lambda p: setattr(p, "nu_oil", 0.0), "tau > 1/2"),
    (lambda p: setattr(p, "nu_water", -1e-3), "tau > 1/2"),
    (lambda p: setattr(p, "nx", 4), "axis 0"),
    (lambda p: setattr(p, "bc_x", _lib.BC_JET), "bc_x"),
    (lambda p: setattr(p, "bc_z", _lib.BC_PERIODIC_COPY), "bc_z"),
    (lambda p: setattr(p, "omega_g", 2.5), "omega_g"),
    (lambda p: setattr(p, "sigma", float("nan")), "non-finite"),
    (lambda p: (setattr(p, "nx", 65535), setattr(p, "ny", 65535), setattr(p, "nz", 2)), "axis 2"),
    (lambda p: (setattr(p, "nx", 4096), setattr(p, "ny", 4096), setattr(p, "nz", 4096)), "2^32"),
])
def test_validate_rejects(mutate, fragment):
    p = _lib.reference_params(32, 32, 64, 19)
    mutate(p)
    rc = lib().ssmd_validate(ctypes.byref(p))
    assert rc == _lib.SSMD_ERR_INVALID_ARGUMENT
    assert fragment in lib().ssmd_last_error().decode()


def test_step_rejects_null_pointers_before_touching_the_device():
    p = _lib.reference_params(32, 32, 64, 19)
    f = LBMFields()
    rc = lib().ssmd_step(ctypes.byref(f), ctypes.byref(p), 0, 0, None)
    assert rc == _lib.SSMD_ERR_INVALID_ARGUMENT
    assert "null" in lib().ssmd_last_error().decode()
    ex = ctypes.c_void_p()
    rc = lib().ssmd_capture_graph(ctypes.byref(p), ctypes.byref(f), 0, 3, 0, None, ctypes.byref(ex))
    assert rc == _lib.SSMD_ERR_INVALID_ARGUMENT  # odd step count breaks the A/B parity


def test_sizes():
    p = _lib.reference_params(32, 32, 64, 27)
    n = 32 * 32 * 64
    L = lib()
    assert L.ssmd_scalar_bytes(ctypes.byref(p)) == 4 * n
    assert L.ssmd_f_bytes(ctypes.byref(p)) == 4 * 27 * n
    assert L.ssmd_g_bytes(ctypes.byref(p)) == 4 * 7 * n
    p.storage = _lib.STORAGE_BF16
    assert L.ssmd_f_bytes(ctypes.byref(p)) == 2 * 27 * n
    assert L.ssmd_workspace_bytes(ctypes.byref(p)) >= 512


def test_oil_jet_parameters():
    p = configs.oil_jet(64, 64, 128, 19, tau=0.55, sigma=1e-3, width=4, mobility=0.1, diam=8)
    assert abs(p.nu_oil - (0.55 - 0.5) / 3) < 1e-8
    assert abs(p.omega_g - 1.0 / (0.5 + 0.1 / 0.25)) < 1e-7
    assert abs(p.gamma - 4 * 0.1 / (4 * 0.25)) < 1e-7
    assert p.oil_r2 == 16.0 and p.oil_cx == 31.5 and p.oil_cy == 31.5
    assert lib().ssmd_validate(ctypes.byref(p)) == 0
