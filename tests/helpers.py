"""Shared helpers for the parity tests (CUDA path vs oracle vs reference harness)."""
from __future__ import annotations

import numpy as np

from ssmdlbm_b200 import _lib, configs

FIELDS = ("rho", "ux", "uy", "uz", "phi")

# Reference-harness cases (oracle/build.py CASES) as product parameters:
# the same (u, diam, radius, Re, We, W) through the reference's derivation.
HARNESS_KNOBS = {
    "q19_s": dict(vs=19, n=(16, 16, 32), u_water=0.05, u_oil=0.05, diam_water=5, diam_oil=5, radius_water=2,
                  radius_oil=2, reynolds_water=10, reynolds_oil=8, weber=5, interface_width=4.0),
    "q27_s": dict(vs=27, n=(16, 16, 32), u_water=0.05, u_oil=0.05, diam_water=5, diam_oil=5, radius_water=2,
                  radius_oil=2, reynolds_water=10, reynolds_oil=8, weber=5, interface_width=4.0),
    "q19_c1": dict(vs=19, n=(64, 64, 128), u_water=0.05, u_oil=0.05, diam_water=8, diam_oil=8, radius_water=0,
                   radius_oil=4, reynolds_water=24, reynolds_oil=24, weber=20, interface_width=4.0),
    "q27_c2": dict(vs=27, n=(128, 128, 512), u_water=0.05, u_oil=0.05, diam_water=16, diam_oil=16,
                   radius_water=0, radius_oil=8, reynolds_water=120, reynolds_oil=120, weber=40,
                   interface_width=4.0),
    "q19_c2": dict(vs=19, n=(128, 128, 512), u_water=0.05, u_oil=0.05, diam_water=16, diam_oil=16,
                   radius_water=0, radius_oil=8, reynolds_water=120, reynolds_oil=120, weber=40,
                   interface_width=4.0),
}


def harness_params(case: str, periodic_y: bool = False, storage: int = _lib.STORAGE_F32):
    k = dict(HARNESS_KNOBS[case])
    vs = k.pop("vs")
    nx, ny, nz = k.pop("n")
    p = configs.reference_like(nx, ny, nz, vs, **k)
    if periodic_y:
        p.bc_y = _lib.BC_PERIODIC_COPY
    p.storage = storage
    return p


def rel_linf(a: np.ndarray, b: np.ndarray) -> float:
    """||a - b||_inf / ||b||_inf."""
    den = float(np.max(np.abs(b)))
    return float(np.max(np.abs(np.asarray(a, np.float64) - np.asarray(b, np.float64)))) / max(den, 1e-30)


def field_errors(got: dict, ref: dict) -> dict:
    """Relative L-infinity errors: rho and phi as scalar fields, u as a vector
    field (max over cells and components of |du| over the max speed |u|), so
    that a velocity component whose own maximum is tiny is judged against the
    flow's velocity scale."""
    u_ref = np.sqrt(sum(np.asarray(ref[k], np.float64) ** 2 for k in ("ux", "uy", "uz")))
    du = max(float(np.max(np.abs(np.asarray(got[k], np.float64) - np.asarray(ref[k], np.float64))))
             for k in ("ux", "uy", "uz"))
    return {"rho": rel_linf(got["rho"], ref["rho"]), "u": du / max(float(np.max(u_ref)), 1e-30),
            "phi": rel_linf(got["phi"], ref["phi"])}


def compare_fields(got: dict, ref: dict, tol: float) -> dict:
    errs = field_errors(got, ref)
    bad = {k: v for k, v in errs.items() if not v <= tol}
    assert not bad, f"rel Linf above {tol}: {bad} (all: {errs})"
    return errs


def sim_fields(sim) -> dict:
    return {k: sim.field(k) for k in FIELDS}


def oracle_fields(o) -> dict:
    return {k: o.get(k) for k in FIELDS}


def interior_mask(p) -> np.ndarray:
    """Fluid (colliding) cells, [z][y][x]."""
    m = np.ones((p.nz, p.ny, p.nx), dtype=bool)
    for axis, (n, bc) in enumerate(((p.nz, p.bc_z), (p.ny, p.bc_y), (p.nx, p.bc_x))):
        if bc != _lib.BC_PERIODIC:
            sl = [slice(None)] * 3
            sl[axis] = 0
            m[tuple(sl)] = False
            sl[axis] = n - 1
            m[tuple(sl)] = False
    return m


def separable_macros(shape, seed: int = 0, u_amp: float = 0.02, width: float = 4.0):
    """A seeded smooth initial state built from 1-D profiles (outer products in
    float32), cheap enough for lattices of 10^8 cells: phi = a tanh slab
    profile along each axis multiplied together (an interface everywhere the
    profiles cross 1/2), u = products of sines with seeded phases, rho = 1 +
    1e-3 of a product of sines.  Returns (rho, ux, uy, uz, phi), [z][y][x]."""
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    f32 = np.float32

    def slab(n):  # inside [0.15 n, 0.85 n]: no interface on a face or the periodic wrap
        c = rng.uniform(0.4 * n, 0.6 * n)
        r = rng.uniform(0.15 * n, 0.25 * n)
        t = np.arange(n, dtype=np.float64)
        return (0.5 * (1.0 - np.tanh(2.0 * (np.abs(t - c) - r) / width))).astype(f32)

    def wave(n):
        k = rng.integers(1, 4)
        return np.sin(2 * np.pi * k * np.arange(n) / n + rng.uniform(0, 2 * np.pi)).astype(f32)

    def outer(a, b, c, scale=1.0):
        out = np.empty(shape, dtype=f32)
        np.multiply(a[:, None, None], b[None, :, None], out=out)
        out *= c[None, None, :]
        if scale != 1.0:
            out *= f32(scale)
        return out

    phi = outer(slab(nz), slab(ny), slab(nx))
    ux = outer(wave(nz), wave(ny), wave(nx), u_amp)
    uy = outer(wave(nz), wave(ny), wave(nx), u_amp)
    uz = outer(wave(nz), wave(ny), wave(nx), u_amp)
    rho = outer(wave(nz), wave(ny), wave(nx), 1e-3)
    rho += f32(1.0)
    return rho, ux, uy, uz, phi


def blob_macros(shape, seed: int = 0, blobs_per_mcell: float = 12.0, u_amp: float = 0.02, width: float = 4.0):
    """A seeded state for large lattices whose phase field has no plateau
    other than exactly 0: small tanh blobs of radius 2-4 cells (peak phi
    below 1) on water, the profile cut to 0 below 1e-6, and a smooth velocity
    field (products of sines).  Plateaus of phi strictly inside (0, 1) are
    avoided on purpose: there the interface normal grad phi / (|grad phi| +
    1e-9) of the scheme turns FP32 rounding noise into unit vectors and the
    anti-diffusion flux amplifies it, so any two FP32 codes drift apart.
    Returns (rho, ux, uy, uz, phi), float32, [z][y][x]."""
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    f32 = np.float32
    phi = np.zeros(shape, dtype=f32)
    count = max(1, int(blobs_per_mcell * nx * ny * nz / 1e6))
    h = 10  # half-size of the box a blob is evaluated in
    k = np.arange(-h, h + 1, dtype=np.float64)
    for _ in range(count):
        c = rng.uniform([h, h, h], [nz - h - 1, ny - h - 1, nx - h - 1])
        ci = np.floor(c).astype(int)
        r = rng.uniform(2.0, 4.0)
        dz, dy, dx = (k + ci[0] - c[0]), (k + ci[1] - c[1]), (k + ci[2] - c[2])
        d = np.sqrt(dz[:, None, None] ** 2 + dy[None, :, None] ** 2 + dx[None, None, :] ** 2)
        b = 0.5 * (1.0 - np.tanh(2.0 * (d - r) / width))
        b[b < 1e-6] = 0.0
        sl = tuple(slice(ci[a] - h, ci[a] + h + 1) for a in range(3))
        np.maximum(phi[sl], b.astype(f32), out=phi[sl])
    _, ux, uy, uz, _ = separable_macros(shape, seed=seed + 1, u_amp=u_amp)
    rho = np.full(shape, f32(1.0), dtype=f32)
    return rho, ux, uy, uz, phi
