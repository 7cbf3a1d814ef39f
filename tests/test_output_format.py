"""The reference's output files, byte for byte (no GPU).

ssmd_output_vti is compared with the reference's own writer
(host::PostProcess::vti, built from its sources into oracle/_ref/q19_s/vti_ref)
on the same .bin inputs; the .bin and _info.txt layouts are checked directly.
"""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from ssmdlbm_b200 import _lib
from ssmdlbm_b200._lib import lib
from oracle import build as obuild

NX, NY, NZ = 16, 16, 32  # the lattice the reference writer was built for (case q19_s)


def _write_bins(d, step, rng):
    arrays = {}
    for name in ("phi", "rho"):
        a = rng.standard_normal(NX * NY * NZ).astype(np.float32)
        _lib.check(lib().ssmd_output_bin(str(d).encode(), name.encode(), step, a.ctypes.data, a.size))
        arrays[name] = a
    return arrays


def test_bin_layout(tmp_path):
    rng = np.random.default_rng(0)
    arrays = _write_bins(tmp_path, 42, rng)
    for name, a in arrays.items():
        raw = np.fromfile(tmp_path / f"{name}000042.bin", dtype="<f4")
        assert np.array_equal(raw, a)


def test_vti_matches_reference_writer(tmp_path):
    exe = obuild.vti_binary("q19_s")
    if not os.path.exists(exe):
        pytest.fail(f"{exe} missing: python -m oracle.build --ref")
    ours, ref = tmp_path / "ours", tmp_path / "ref"
    ours.mkdir()
    ref.mkdir()
    rng = np.random.default_rng(1)
    _write_bins(ours, 1234, rng)
    for f in os.listdir(ours):
        shutil.copy(ours / f, ref / f)
    names = (ctypes.c_char_p * 2)(b"phi", b"rho")
    _lib.check(lib().ssmd_output_vti(str(ours).encode(), 1234, NX, NY, NZ, names, 2))
    subprocess.run([exe, str(ref) + "/", "1234"], check=True, capture_output=True)
    a = (ours / "step_001234.vti").read_bytes()
    b = (ref / "step_001234.vti").read_bytes()
    assert len(a) == len(b) and a == b


def test_info_file(tmp_path):
    _lib.check(lib().ssmd_output_info(str(tmp_path).encode(), b"000", b"D3Q19", 0.05, 0.05, 1400.0, 450.0,
                                      500.0, 128, 256, 256, 13, 13, 100000, 1000))
    text = (tmp_path / "000_info.txt").read_text()
    assert "ID:                 000\n" in text
    assert "Water Reynolds:     1400\n" in text and "Water velocity:     0.05\n" in text
    assert "Domain size:        NX=128, NY=256, NZ=256\n" in text
    assert "Output interval:    1000\n\n" in text
