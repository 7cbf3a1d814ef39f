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
