"""Python handles on the oracle: the CPU build (libssmd_oracle.so) and its
FP64 GPU instance (libssmd_oracle_gpu.so).  TEST INFRASTRUCTURE.

Only tests, fixture scripts, the smoke check and bench.py's CPU-baseline leg
use this module; the product path (ssmdlbm_b200) never imports it.

Arrays are numpy, scalar fields shaped [z][y][x], populations [q][z][y][x] in
the reference's push layout.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import build as _build

FIELD_IDS = {"rho": 0, "ux": 1, "uy": 2, "uz": 3, "phi": 4, "pxx": 5, "pyy": 6, "pzz": 7,
             "pxy": 8, "pxz": 9, "pyz": 10, "fsx": 11, "fsy": 12, "fsz": 13, "f": 20, "g": 21}

_lib = None


def lib():
    global _lib
    if _lib is None:
        path = _build.ORACLE_SO
        if not os.path.exists(path):
            path = _build.build_oracle()
        L = ctypes.CDLL(path)
        L.oracle_new.restype = ctypes.c_void_p
        L.oracle_new.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_free.argtypes = [ctypes.c_void_p]
        L.oracle_init_jets.argtypes = [ctypes.c_void_p]
        L.oracle_init_macros.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 5
        L.oracle_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_get.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.oracle_set.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.oracle_centreline.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_droplets.argtypes = [ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p, ctypes.c_void_p,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.oracle_centreline_arrays.argtypes = [ctypes.c_void_p] * 5
        L.oracle_droplets_arrays.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_float, ctypes.c_void_p,
                                             ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                             ctypes.c_void_p]
        L.oracle_noise.restype = ctypes.c_double
        L.oracle_noise.argtypes = [ctypes.c_uint64, ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint32]
        _lib = L
    return _lib


class Oracle:
    """One lattice advanced by the CPU restatement of the reference step."""

    def __init__(self, params, precision: int = 64):
        self.p = params
        self.precision = precision
        self.h = lib().oracle_new(ctypes.byref(params), precision)
        if not self.h:
            raise ValueError("oracle_new failed")
        self.Q = int(params.velocity_set)
        self.shape = (int(params.nz), int(params.ny), int(params.nx))
        self.cells = int(np.prod(self.shape))
        self.steps_done = 0

    def __del__(self):
        if getattr(self, "h", None):
            lib().oracle_free(self.h)
            self.h = None

    def init_jets(self) -> None:
        lib().oracle_init_jets(self.h)
        self.steps_done = 0

    def init_macros(self, rho, ux, uy, uz, phi) -> None:
        arrs = [np.ascontiguousarray(a, dtype=np.float32).reshape(-1) for a in (rho, ux, uy, uz, phi)]
        lib().oracle_init_macros(self.h, *[a.ctypes.data for a in arrs])
        self.steps_done = 0

    def step(self, n: int = 1) -> None:
        lib().oracle_step(self.h, n)
        self.steps_done += n

    def get(self, name: str) -> np.ndarray:
        fid = FIELD_IDS[name]
        n = self.cells * (self.Q if name == "f" else 7 if name == "g" else 1)
        out = np.empty(n, dtype=np.float64)
        if lib().oracle_get(self.h, fid, out.ctypes.data) != 0:
            raise KeyError(name)
        if name in ("f", "g"):
            return out.reshape((-1,) + self.shape)
        return out.reshape(self.shape)

    def set(self, name: str, values: np.ndarray) -> None:
        v = np.ascontiguousarray(values, dtype=np.float32).reshape(-1)
        if lib().oracle_set(self.h, FIELD_IDS[name], v.ctypes.data) != 0:
            raise KeyError(name)

    def centreline(self):
        uz = np.zeros(self.shape[0])
        phi = np.zeros(self.shape[0])
        lib().oracle_centreline(self.h, uz.ctypes.data, phi.ctypes.data)
        return uz, phi

    def droplets(self, threshold: float = 0.5, max_droplets: int = 100000):
        """Components as a structured array (root, cells, volume, touches_inlet), sorted by root."""
        return _droplets(lambda *a: lib().oracle_droplets(self.h, threshold, *a), max_droplets)


def _droplets(call, max_droplets: int):
    root = np.zeros(max_droplets, np.uint32)
    cells = np.zeros(max_droplets, np.uint32)
    vol = np.zeros(max_droplets, np.float64)
    touch = np.zeros(max_droplets, np.uint32)
    n = ctypes.c_int()
    call(root.ctypes.data, cells.ctypes.data, vol.ctypes.data, touch.ctypes.data, max_droplets, ctypes.byref(n))
    k = min(n.value, max_droplets)
    out = np.zeros(k, dtype=[("root", "u4"), ("cells", "u4"), ("volume", "f8"), ("touches_inlet", "u4")])
    out["root"], out["cells"], out["volume"], out["touches_inlet"] = root[:k], cells[:k], vol[:k], touch[:k]
    return out


_gpu_lib = None


def gpu_lib():
    global _gpu_lib
    if _gpu_lib is None:
        path = _build.ORACLE_GPU_SO
        if not os.path.exists(path):
            path = _build.build_oracle_gpu()
        L = ctypes.CDLL(path)
        L.oracle_gpu_new.restype = ctypes.c_void_p
        L.oracle_gpu_new.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_gpu_free.argtypes = [ctypes.c_void_p]
        L.oracle_gpu_init_jets.argtypes = [ctypes.c_void_p]
        L.oracle_gpu_init_macros.argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * 5
        L.oracle_gpu_step.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.oracle_gpu_get.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.oracle_gpu_last_error.restype = ctypes.c_char_p
        _gpu_lib = L
    return _gpu_lib


class GpuOracle:
    """The oracle on the current CUDA device (same interface as Oracle):
    precision 64 (FP64 transcription) or 32 (the reference's FP32
    arithmetic), bit-identical to the CPU build of the same precision.  It
    allocates its own device memory: Q + 25 reals per cell (+ 7 with
    omega_g != 1)."""

    def __init__(self, params, precision: int = 64):
        self.p = params
        self.precision = precision
        self.h = gpu_lib().oracle_gpu_new(ctypes.byref(params), precision)
        if not self.h:
            raise RuntimeError("oracle_gpu_new failed: " + gpu_lib().oracle_gpu_last_error().decode())
        self.Q = int(params.velocity_set)
        self.shape = (int(params.nz), int(params.ny), int(params.nx))
        self.cells = int(np.prod(self.shape))
        self.steps_done = 0

    def close(self) -> None:
        if getattr(self, "h", None):
            gpu_lib().oracle_gpu_free(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def _check(self, rc: int) -> None:
        if rc != 0:
            raise RuntimeError(gpu_lib().oracle_gpu_last_error().decode())

    def init_jets(self) -> None:
        self._check(gpu_lib().oracle_gpu_init_jets(self.h))
        self.steps_done = 0

    def init_macros(self, rho, ux, uy, uz, phi) -> None:
        arrs = [np.ascontiguousarray(a, dtype=np.float32).reshape(-1) for a in (rho, ux, uy, uz, phi)]
        self._check(gpu_lib().oracle_gpu_init_macros(self.h, *[a.ctypes.data for a in arrs]))
        self.steps_done = 0

    def step(self, n: int = 1) -> None:
        self._check(gpu_lib().oracle_gpu_step(self.h, n))
        self.steps_done += n

    def get(self, name: str) -> np.ndarray:
        n = self.cells * (self.Q if name == "f" else 7 if name == "g" else 1)
        out = np.empty(n, dtype=np.float64)
        self._check(gpu_lib().oracle_gpu_get(self.h, FIELD_IDS[name], out.ctypes.data))
        if name in ("f", "g"):
            return out.reshape((-1,) + self.shape)
        return out.reshape(self.shape)

    def centreline(self):
        uz = np.zeros(self.shape[0])
        phi = np.zeros(self.shape[0])
        u, ph = self.get("uz"), self.get("phi")
        lib().oracle_centreline_arrays(ctypes.byref(self.p), u.ctypes.data, ph.ctypes.data, uz.ctypes.data,
                                       phi.ctypes.data)
        return uz, phi

    def droplets(self, threshold: float = 0.5, max_droplets: int = 100000):
        ph = self.get("phi")
        return _droplets(lambda *a: lib().oracle_droplets_arrays(ctypes.byref(self.p), ph.ctypes.data, threshold,
                                                                 *a), max_droplets)


def noise(seed: int, step: int, cell: int, stream: int = 0) -> float:
    return lib().oracle_noise(seed, step, cell, stream)


def seeded_macros(shape, seed: int = 0, blobs: int = 3, u_amp: float = 0.02, width: float = 4.0):
    """Deterministic smooth initial state for parity runs: phi = union of tanh
    spheres, u = a few random Fourier modes of amplitude u_amp, rho = 1 plus a
    1e-3 perturbation.  Returns float32 arrays (rho, ux, uy, uz, phi), [z][y][x]."""
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    phi = np.zeros(shape)
    for _ in range(blobs):
        c = rng.uniform([0.25 * nz, 0.25 * ny, 0.25 * nx], [0.75 * nz, 0.75 * ny, 0.75 * nx])
        r = rng.uniform(0.12, 0.22) * min(nx, ny, nz)
        d = np.sqrt((z - c[0]) ** 2 + (y - c[1]) ** 2 + (x - c[2]) ** 2)
        phi = np.maximum(phi, 0.5 * (1.0 - np.tanh(2.0 * (d - r) / width)))
    u = []
    for _ in range(3):
        a = np.zeros(shape)
        for _m in range(3):
            k = rng.integers(1, 3, size=3)
            ph = rng.uniform(0, 2 * np.pi, size=3)
            a += (np.sin(2 * np.pi * k[0] * z / nz + ph[0]) * np.sin(2 * np.pi * k[1] * y / ny + ph[1])
                  * np.sin(2 * np.pi * k[2] * x / nx + ph[2]))
        u.append(u_amp / 3.0 * a)
    rho = 1.0 + 1e-3 * np.sin(2 * np.pi * x / nx) * np.cos(2 * np.pi * z / nz)
    f32 = lambda a: np.ascontiguousarray(a, dtype=np.float32)
    return f32(rho), f32(u[0]), f32(u[1]), f32(u[2]), f32(phi)
