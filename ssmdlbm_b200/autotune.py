"""Autotuner for the bulk kernel: kernel path x z-chunk per lattice.

The fused step has two launch knobs in ssmd_params: ``bulk_path`` (per-cell
gathers, TMA boxes for the phi halo, TMA slabs for the populations) and
``tile_z`` (z planes per 32 x 8 work item).  Which combination is fastest
depends on the velocity set, the storage type, the lattice shape and the face
kinds, so it is measured: every candidate runs a few steps on the device
(CUDA events on the simulation's stream, after a warm-up) and the fastest is
cached in a JSON file keyed by device name and problem signature
($SSMD_AUTOTUNE_CACHE, default ~/.cache/ssmd_b200/autotune.json).

The population buffers are scratch for the search (the state is restored by
re-initialising afterwards), so tune before ``init`` or re-initialise after.
"""
from __future__ import annotations

import json
import os

from . import _lib

# 0: the library's own choice (a makespan model of the block scheduling, 8-64 planes)
CANDIDATE_TILE_Z = (0, 12, 16, 20, 24, 28, 32, 48, 56, 64)


def cache_path() -> str:
    return os.environ.get("SSMD_AUTOTUNE_CACHE") or os.path.join(
        os.path.expanduser("~"), ".cache", "ssmd_b200", "autotune.json")


def signature(p) -> str:
    bgk = int(abs(float(p.omega_g) - 1.0) > 0)
    return (f"q{p.velocity_set}-s{p.storage}-{p.nx}x{p.ny}x{p.nz}-bc{p.bc_x}{p.bc_y}{p.bc_z}-bgk{bgk}")


def _load() -> dict:
    try:
        with open(cache_path()) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def _save(d: dict) -> None:
    path = cache_path()
    os.makedirs(os.path.dirname(path), exist_ok=True)
    tmp = path + ".tmp"
    with open(tmp, "w") as fh:
        json.dump(d, fh, indent=1, sort_keys=True)
    os.replace(tmp, path)


def candidates(p):
    paths = [_lib.PATH_GATHER]
    f_size = 4 if p.storage == _lib.STORAGE_F32 else 2
    g_size = 4 if p.storage in (_lib.STORAGE_F32, _lib.STORAGE_F16_G32) else 2
    if (int(p.nx) * g_size) % 16 == 0:
        paths.append(_lib.PATH_TMA)  # TMA boxes of g
    if f_size == g_size and (int(p.nx) * f_size) % 16 == 0:
        paths.append(_lib.PATH_SLAB)  # f and g slabs of one element size
    nzf = int(p.nz) - (0 if p.bc_z == _lib.BC_PERIODIC else 2)
    return [(path, tz) for path in paths for tz in CANDIDATE_TILE_Z if tz == 0 or tz <= nzf]


def tune(sim, steps: int = 10, force: bool = False, verbose: bool = False) -> dict:
    """Measure every candidate on `sim` (an lbm.Simulation) and store the best
    (bulk_path, tile_z) into sim.p; returns the cache entry."""
    import torch

    import ctypes
    dev = torch.cuda.get_device_name(sim.device)
    key = f"{dev}|{signature(sim.p)}"
    cache = _load()
    if not force and key in cache:
        best = cache[key]
        sim.p.bulk_path, sim.p.tile_z = int(best["bulk_path"]), int(best["tile_z"])
        return best
    L = _lib.lib()
    s = sim.torch_stream
    results = []
    base_path, base_tz = sim.p.bulk_path, sim.p.tile_z
    sim.init()
    for path, tz in candidates(sim.p):
        sim.p.bulk_path, sim.p.tile_z = path, tz
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        try:
            for i in range(2):  # warm-up (also sets the kernel's shared-memory limit)
                _lib.check(L.ssmd_step(ctypes.byref(sim.fields), ctypes.byref(sim.p), i, 0, sim.stream))
            torch.cuda.synchronize(sim.device)
            e0.record(s)
            for i in range(steps):
                _lib.check(L.ssmd_step(ctypes.byref(sim.fields), ctypes.byref(sim.p), i, 0, sim.stream))
            e1.record(s)
            e1.synchronize()
        except _lib.SSMDError:
            continue
        ms = e0.elapsed_time(e1) / steps
        results.append((ms, path, tz))
        if verbose:
            print(f"autotune {signature(sim.p)} path={path} tile_z={tz}: {ms:.4f} ms/step")
    sim.p.bulk_path, sim.p.tile_z = base_path, base_tz
    if not results:
        return {"bulk_path": base_path, "tile_z": base_tz, "ms_per_step": None}
    ms, path, tz = min(results)
    best = {"bulk_path": path, "tile_z": tz, "ms_per_step": ms,
            "tried": [{"bulk_path": p_, "tile_z": t_, "ms": round(m_, 5)} for m_, p_, t_ in sorted(results)]}
    cache = _load()
    cache[key] = best
    _save(cache)
    sim.p.bulk_path, sim.p.tile_z = path, tz
    sim.init()
    return best


# z chunks tried for a batched sweep (the work items of all lattices share one
# persistent launch, so the chunk trades items per lattice against prologues)
SWEEP_TILE_Z = (8, 12, 16, 24, 32, 48, 64)


def sweep_signature(sw) -> str:
    import hashlib
    sigs = ",".join(signature(p) for p in sw.params)
    return f"sweep{sw.count}-" + hashlib.sha1(sigs.encode()).hexdigest()[:16]


def tune_sweep(sw, steps: int = 10, force: bool = False, verbose: bool = False) -> dict:
    """Measure the batched step of a sweep (a batch.Sweep) over SWEEP_TILE_Z,
    set the fastest on it and cache it (same file and device key as tune()).
    The populations are scratch for the search: re-initialise the sweep
    afterwards."""
    import torch
    dev = torch.cuda.get_device_name(sw.device)
    key = f"{dev}|{sweep_signature(sw)}"
    cache = _load()
    if not force and key in cache:
        best = cache[key]
        sw.set_tile_z(int(best["tile_z"]))
        return best
    results = []
    for tz in SWEEP_TILE_Z:
        sw.set_tile_z(tz)
        sw.timed(2)  # warm-up and graph capture
        dt = sw.timed(steps)
        results.append((dt / steps * 1e3, tz))
        if verbose:
            print(f"autotune sweep tile_z={tz}: {dt / steps * 1e3:.4f} ms/step")
    ms, tz = min(results)
    sw.set_tile_z(tz)
    best = {"tile_z": tz, "ms_per_step": ms, "tried": [{"tile_z": t, "ms": round(m, 5)} for m, t in sorted(results)]}
    cache = _load()
    cache[key] = best
    _save(cache)
    return best
