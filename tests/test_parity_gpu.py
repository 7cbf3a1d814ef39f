"""Parity of the CUDA path (through the C ABI) with the oracle and the reference.

Error measure (tests/helpers.field_errors): relative L-infinity of rho and
phi, and of the velocity vector field (max |u - u_ref| over max |u_ref|).
Tolerances:
  * initial state vs oracle: exact macros, populations within 1e-6;
  * FP32 storage vs FP32 oracle after 1 step: 5e-6, after 50 steps: 1e-5;
  * FP32 storage vs the reference's own CUDA kernels after 100 steps: 1e-5
    (the bar of the jet configurations), and no further from the FP64 oracle
    than the reference's own FP32 result is (within 1.5x + 1e-7): both paths
    carry FP32 rounding of ~1e-5 on the smallest velocity components.
"""
import os
import subprocess
import tempfile

import numpy as np
import pytest

from ssmdlbm_b200 import _lib, configs
from oracle.oracle import Oracle, seeded_macros
from oracle import build as obuild
from helpers import (FIELDS, compare_fields, field_errors, harness_params, interior_mask, oracle_fields,
                     rel_linf, sim_fields)

pytestmark = pytest.mark.gpu


def _sim(p):
    from ssmdlbm_b200.lbm import Simulation
    return Simulation(p)


def _geometries(vs):
    """(name, params) over the face kinds, including lattice sizes that are
    not multiples of the 32 x 8 tile."""
    out = []
    p = harness_params("q19_s" if vs == 19 else "q27_s")
    out.append(("ref_jets", p))
    p = harness_params("q19_s" if vs == 19 else "q27_s", periodic_y=True)
    out.append(("copy_xy", p))
    p = configs.reference_like(20, 12, 24, vs, diam_water=4, diam_oil=4, reynolds_water=10,
                               reynolds_oil=6, weber=4)
    out.append(("ragged_jets", p))
    p = configs.oil_jet(24, 20, 40, vs, tau=0.56, sigma=5e-3, mobility=0.1, diam=6, noise=0.02, seed=5)
    out.append(("exact_xy_bgk_noise", p))
    p = configs.periodic_box((18, 16, 20), vs, tau=0.62, sigma=1e-2, mobility=0.125)
    out.append(("periodic_box", p))
    return out


CASES = [(vs, name, p) for vs in (19, 27) for name, p in _geometries(vs)]
IDS = [f"q{vs}-{name}" for vs, name, _ in CASES]


def _init_both(p, seeded: bool, seed=3):
    sim = _sim(p)
    o = Oracle(p, 32)
    if seeded:
        m = seeded_macros((p.nz, p.ny, p.nx), seed=seed)
        sim.init_from_macros(*m)
        o.init_macros(*m)
    else:
        sim.init()
        o.init_jets()
    return sim, o


@pytest.mark.parametrize("vs,name,p", CASES, ids=IDS)
@pytest.mark.parametrize("seeded", [False, True], ids=["jets", "seeded"])
def test_init_matches_oracle(vs, name, p, seeded):
    sim, o = _init_both(p, seeded)
    compare_fields(sim_fields(sim), oracle_fields(o), 0.0)  # macros are copied / set exactly
    m = interior_mask(p)
    for which, key in ((0, "f"), (1, "g")):
        got = sim.populations_push(which)[:, m]
        ref = o.get(key)[:, m]
        assert np.max(np.abs(got - ref)) <= 1e-6, key


@pytest.mark.parametrize("vs,name,p", CASES, ids=IDS)
@pytest.mark.parametrize("seeded", [False, True], ids=["jets", "seeded"])
def test_steps_match_oracle(vs, name, p, seeded):
    sim, o = _init_both(p, seeded)
    sim.step(1, store_macros=True)
    o.step(1)
    compare_fields(sim_fields(sim), oracle_fields(o), 5e-6)
    m = interior_mask(p)
    for which, key in ((0, "f"), (1, "g")):
        got = sim.populations_push(which)[:, m]
        ref = o.get(key)[:, m]
        assert np.max(np.abs(got - ref)) <= 2e-6 * max(1.0, float(np.max(np.abs(ref)))), key
    sim.step(49, store_macros=True)
    o.step(49)
    compare_fields(sim_fields(sim), oracle_fields(o), 1e-5)


def _run_harness(case, steps, periodic_y, macros, workdir):
    exe = obuild.ref_binary(case)
    if not os.path.exists(exe):
        pytest.fail(f"reference harness {exe} missing: build it with python -m oracle.build --ref")
    nz, ny, nx = macros[0].shape if macros is not None else (None, None, None)
    cmd = [exe, "--steps", str(steps), "--dump", os.path.join(workdir, "d"), "--at", str(steps)]
    if periodic_y:
        cmd.append("--periodic-y")
    if macros is not None:
        path = os.path.join(workdir, "m.bin")
        np.concatenate([a.reshape(-1) for a in macros]).astype(np.float32).tofile(path)
        cmd += ["--macros", path]
    subprocess.run(cmd, check=True, timeout=300)
    return np.fromfile(os.path.join(workdir, f"d_{steps}.bin"), dtype=np.float32)


REF_CASES = [("q19_s", False, None), ("q27_s", False, None), ("q19_s", True, 11), ("q27_s", True, 12),
             ("q19_c1", True, None)]


@pytest.mark.parametrize("case,periodic_y,seed", REF_CASES,
                         ids=[f"{c}-{'py' if py else 'jets'}-{s}" for c, py, s in REF_CASES])
def test_matches_reference_kernels_after_100_steps(case, periodic_y, seed):
    """The reference's own CUDA kernels (oracle/_ref harness) vs this path."""
    p = harness_params(case, periodic_y=periodic_y)
    shape = (p.nz, p.ny, p.nx)
    n = int(np.prod(shape))
    macros = seeded_macros(shape, seed=seed) if seed is not None else None
    with tempfile.TemporaryDirectory() as td:
        raw = _run_harness(case, 100, periodic_y, macros, td)
    ref = {k: raw[i * n:(i + 1) * n].reshape(shape) for i, k in enumerate(FIELDS)}
    sim = _sim(p)
    o = Oracle(p, 64)
    if macros is not None:
        sim.init_from_macros(*macros)
        o.init_macros(*macros)
    else:
        sim.init()
        o.init_jets()
    sim.step(100, store_macros=True)
    ours = sim_fields(sim)
    errs = compare_fields(ours, ref, 1e-5)
    if p.nx * p.ny * p.nz <= 64 * 64 * 128:
        o.step(100)
        truth = oracle_fields(o)
        e_ours, e_ref = field_errors(ours, truth), field_errors(ref, truth)
        for k in e_ours:
            assert e_ours[k] <= 1.5 * e_ref[k] + 1e-7, (k, e_ours, e_ref)
        print(case, periodic_y, seed, errs, "vs fp64:", e_ours, "ref vs fp64:", e_ref)


def test_graph_replay_equals_eager_steps():
    p = harness_params("q19_s")
    a, b = _sim(p), _sim(p)
    a.init()
    b.init()
    a.step(6)
    b.run_graph(3, steps=2)
    a.step(1, store_macros=True)
    b.step(1, store_macros=True)
    for k in FIELDS:
        assert np.array_equal(a.field(k), b.field(k)), k
    assert np.array_equal(a.populations_push(0), b.populations_push(0))
    b.close()


def test_reduce_matches_host_sums():
    p = configs.periodic_box((18, 16, 20), 19)
    sim = _sim(p)
    sim.init_from_macros(*seeded_macros((20, 16, 18), seed=4))
    sim.step(3, store_macros=True)
    st = sim.reduce()
    m = interior_mask(p)
    phi, rho = sim.field("phi")[m].astype(np.float64), sim.field("rho")[m].astype(np.float64)
    assert abs(st["phi_sum"] - phi.sum()) <= 1e-9 * abs(phi.sum())
    assert abs(st["mass"] - rho.sum()) <= 1e-12 * rho.sum()
    g = sim.populations_push(1)
    assert abs(st["phi_sum_next"] - g[:, m].astype(np.float64).sum()) <= 1e-9 * abs(st["phi_sum_next"])
    assert st["cells"] == m.sum() and st["nonfinite"] == 0 and st["status"] == 0


def test_periodic_box_conserves_phi_and_mass():
    """Closed periodic box: sum phi and mass are invariants (FP64 reductions);
    FP32 storage drift after 400 steps must stay below 1e-6 relative."""
    p = configs.periodic_box((32, 32, 32), 19, tau=0.6, sigma=1e-2, mobility=0.1)
    sim = _sim(p)
    sim.init_from_macros(*seeded_macros((32, 32, 32), seed=9))
    st0 = sim.reduce()
    sim.step(400, store_macros=True)
    st1 = sim.reduce()
    assert abs(st1["phi_sum_next"] - st0["phi_sum_next"]) <= 1e-6 * st0["phi_sum_next"]
    assert abs(st1["mass"] - st0["mass"]) <= 1e-6 * st0["mass"]


def test_inlet_noise_matches_host_generator():
    from oracle.oracle import noise
    p = configs.oil_jet(24, 24, 32, 19, diam=8, w_in=0.05, noise=0.01, seed=123)
    sim = _sim(p)
    sim.init()
    sim.step(3, store_macros=True)  # the oil inflow of step index 2 wrote uz on the disc
    uz = sim.field("uz")[0]
    ys, xs = np.nonzero(uz)
    assert len(xs) > 10
    for y, x in zip(ys, xs):
        cell = int(x + 24 * y)
        want = np.float32(np.float32(0.05) * (np.float32(1.0) + np.float32(0.01) * np.float32(noise(123, 2, cell))))
        assert uz[y, x] == want


def test_nonfinite_state_is_reported():
    """Failure detection without a GPU fault: a NaN planted in the populations
    from the host shows up in the status word and in ssmd_reduce."""
    import torch
    p = configs.periodic_box((16, 16, 16), 19)
    sim = _sim(p)
    sim.init_from_macros(*seeded_macros((16, 16, 16), seed=1))
    sim.sync()
    f = sim.t["f"]
    f[5 * sim.cells + 1000] = float("nan")
    torch.cuda.synchronize()
    sim.step(1, store_macros=True)
    assert sim.check_status() & 1
    st = sim.reduce(raise_unstable=False)
    assert st["status"] == _lib.SSMD_ERR_UNSTABLE and st["nonfinite"] > 0
    with pytest.raises(_lib.SSMDError):
        sim.reduce()


@pytest.mark.parametrize("storage,tol", [(_lib.STORAGE_F16, 5e-3), (_lib.STORAGE_BF16, 5e-2),
                                         (_lib.STORAGE_F16_G32, 5e-3)])
def test_reduced_storage_error_vs_fp64_oracle(storage, tol):
    p = harness_params("q19_s", periodic_y=True, storage=storage)
    macros = seeded_macros((p.nz, p.ny, p.nx), seed=21)
    sim = _sim(p)
    sim.init_from_macros(*macros)
    o = Oracle(p, 64)
    o.init_macros(*macros)
    sim.step(100, store_macros=True)
    o.step(100)
    errs = field_errors(sim_fields(sim), oracle_fields(o))
    print(storage, errs)
    assert max(errs.values()) <= tol, errs


@pytest.mark.parametrize("vs,storage", [(19, _lib.STORAGE_F32), (27, _lib.STORAGE_F16)])
def test_kernel_paths_agree(vs, storage):
    """The TMA-fed phi halo, the TMA population slabs and the per-cell gather
    agree to FP32 rounding on a jet box whose tiles touch the periodic wrap and
    the inflow / outflow planes, and bit for bit after one step.  The paths are
    separate instantiations of the same device code; where the source leaves a
    product and a sum unfused (a*b + c*d), the compiler may fuse them
    differently in each, a difference of one rounding that later steps carry
    on."""
    p = configs.oil_jet(64, 40, 48, vs, tau=0.56, sigma=5e-3, mobility=0.1, diam=8, noise=0.01, seed=3,
                        storage=storage)
    first, out = [], []
    for path in (_lib.PATH_GATHER, _lib.PATH_TMA, _lib.PATH_SLAB):
        q = p.copy()
        q.bulk_path = path
        sim = _sim(q)
        sim.init_from_macros(*seeded_macros((48, 40, 64), seed=6))
        sim.step(1, store_macros=True)
        first.append(sim_fields(sim))
        sim.step(5, store_macros=True)
        assert sim.check_status() == 0
        out.append((sim_fields(sim), sim.populations_push(0), sim.populations_push(1)))
    for f in first[1:]:
        for k in FIELDS:
            assert np.array_equal(first[0][k], f[k]), k
    for o in out[1:]:
        for k in FIELDS:
            ref = out[0][0][k]
            assert np.abs(o[0][k] - ref).max() <= 1e-6 * max(np.abs(ref).max(), 1e-3), k
        for a, b in ((out[0][1], o[1]), (out[0][2], o[2])):
            # shifted populations f - w: an FP32 ulp of the unshifted value (~w) is
            # ~3e-8; with FP16 storage one rounding of the stored value moves it by
            # up to 2^-11 of its size
            tol = 2e-7 if storage == _lib.STORAGE_F32 else 2.0**-10 * np.abs(a).max()
            assert np.abs(a - b).max() <= tol


@pytest.mark.parametrize("vs,storage", [(27, _lib.STORAGE_F32), (19, _lib.STORAGE_F16)])
def test_z_chunks_agree_bit_for_bit(vs, storage):
    """Work items of 8, 56 and 64 planes and the automatic choice give the same
    bits: each chunk rebuilds its phi ring and carried gradient / curvature sums
    from the same per-plane partial sums, so the chunk boundaries leave no trace."""
    p = configs.oil_jet(64, 40, 140, vs, tau=0.56, sigma=5e-3, mobility=0.1, diam=8, noise=0.01, seed=3,
                        storage=storage)
    out = []
    for tz in (8, 56, 64, 0):
        q = p.copy()
        q.bulk_path = _lib.PATH_GATHER
        q.tile_z = tz
        sim = _sim(q)
        sim.init_from_macros(*seeded_macros((140, 40, 64), seed=7))
        sim.step(3, store_macros=True)
        assert sim.check_status() == 0
        out.append((sim_fields(sim), sim.populations_push(0), sim.populations_push(1)))
    for o in out[1:]:
        for k in FIELDS:
            assert np.array_equal(out[0][0][k], o[0][k]), k
        assert np.array_equal(out[0][1], o[1]) and np.array_equal(out[0][2], o[2])


def test_autotuner_picks_a_measured_candidate(tmp_path, monkeypatch):
    from ssmdlbm_b200 import autotune
    monkeypatch.setenv("SSMD_AUTOTUNE_CACHE", str(tmp_path / "cache.json"))
    p = configs.oil_jet(64, 40, 48, 19, tau=0.56, sigma=5e-3, mobility=0.1, diam=8)
    sim = _sim(p)
    best = autotune.tune(sim, steps=2)
    assert best["ms_per_step"] > 0 and len(best["tried"]) >= 3
    assert (sim.p.bulk_path, sim.p.tile_z) == (best["bulk_path"], best["tile_z"])
    again = autotune.tune(_sim(p))  # served from the cache
    assert again["bulk_path"] == best["bulk_path"] and again["tile_z"] == best["tile_z"]
