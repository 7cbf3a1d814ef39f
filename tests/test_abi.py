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


def _fake_fields_and_params(q=19, storage=_lib.STORAGE_F32):
    """Parameters and non-null placeholder pointers that pass the host checks;
    the calls below must refuse before any of them is dereferenced."""
    p = _lib.reference_params(32, 32, 64, q)
    p.storage = storage
    f = LBMFields()
    for name, _ in LBMFields._fields_:
        setattr(f, name, ctypes.c_void_p(0x1000))
    p.f_alt = p.g_alt = p.workspace = ctypes.c_void_p(0x1000)
    p.workspace_bytes = lib().ssmd_workspace_bytes(ctypes.byref(p))
    return p, f


def _checkpoint_header(magic=b"SSMDCKP2", abi=None, cells=32 * 32 * 64, q=19, storage=0):
    import struct
    abi = lib().ssmd_abi_version() if abi is None else abi
    return struct.pack("<8sIIQQQii16s", magic, abi, ctypes.sizeof(Params), 0, 0, cells, q, storage, b"\0" * 16)


@pytest.mark.parametrize("kw,fragment", [
    (dict(magic=b"SSMDCKP1"), "older format"),
    (dict(abi=999), "not a checkpoint"),
    (dict(q=27), "not a checkpoint"),
    (dict(storage=_lib.STORAGE_BF16), "not a checkpoint"),
    (dict(cells=7), "not a checkpoint"),
    (dict(magic=b"NOTACKPT"), "not a checkpoint"),
])
def test_checkpoint_load_refuses_other_formats_without_touching_the_device(tmp_path, kw, fragment):
    """A checkpoint of another format, ABI, velocity set, storage or size is
    refused from its header, before any device memory is read or written."""
    p, f = _fake_fields_and_params()
    path = tmp_path / "c.ckp"
    path.write_bytes(_checkpoint_header(**kw) + bytes(ctypes.sizeof(Params)))
    steps = ctypes.c_uint64(123)
    rc = lib().ssmd_checkpoint_load(ctypes.byref(p), ctypes.byref(f), str(path).encode(), ctypes.byref(steps), None)
    assert rc == _lib.SSMD_ERR_INVALID_ARGUMENT
    assert fragment in lib().ssmd_last_error().decode()
    assert steps.value == 123
