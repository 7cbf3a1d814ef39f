"""Batched sweep: one persistent launch for many lattices equals stepping each alone."""
import numpy as np
import pytest

from ssmdlbm_b200 import _lib, configs

pytestmark = pytest.mark.gpu

FIELDS = ("rho", "ux", "uy", "uz", "phi")


def _lattices():
    return [
        configs.oil_jet(32, 32, 64, 19, tau=0.55, sigma=1e-3, mobility=0.1, diam=6, w_in=0.05, noise=0.01, seed=1),
        configs.oil_jet(48, 48, 96, 19, tau=0.58, sigma=5e-3, mobility=0.15, diam=10, w_in=0.03, noise=0.01, seed=2),
        configs.reference_like(24, 40, 56, 19, diam_water=6, diam_oil=6, reynolds_water=10, reynolds_oil=8, weber=5),
        configs.periodic_box((20, 24, 28), 19, tau=0.6, sigma=1e-2, mobility=0.1),
        configs.oil_jet(36, 20, 44, 19, tau=0.52, sigma=2e-3, mobility=0.05, diam=8, w_in=0.08, noise=0.0),
    ]


def test_batched_steps_equal_single_lattice_steps():
    from ssmdlbm_b200.batch import Sweep
    from ssmdlbm_b200.lbm import Simulation
    ps = _lattices()
    sw = Sweep(ps)
    sw.init()
    sw.step(5)
    sw.timed_one_by_one(1)  # single-lattice steps interleave with batched ones
    sw.run_graph(2, steps=2)
    sw.step(1, store_macros=True)
    sw.sync()
    assert sw.steps_done == 11
    for p, bs in zip(ps, sw.sims):
        s = Simulation(p)
        s.init()
        s.step(11, store_macros=True)
        for k in FIELDS:
            assert np.array_equal(s.field(k), bs.field(k)), (p.nx, p.ny, p.nz, k)
        assert np.array_equal(s.populations_push(0), bs.populations_push(0))
        assert bs.check_status() == 0
    sw.close()


def test_sweep_parameters():
    from ssmdlbm_b200.batch import sweep_params
    ps = sweep_params(48, seed=2)
    assert len(ps) == 48
    assert {p.nx for p in ps} <= {32, 48, 64, 96}
    assert all(p.nz == 4 * p.nx and p.ny == p.nx for p in ps)
    assert all(0.02 <= p.u_oil <= 0.08 for p in ps)
    assert all(1e-4 <= p.sigma <= 1e-2 for p in ps)
    cells = sum(p.nx * p.ny * p.nz for p in ps)
    assert 30e6 < cells < 120e6


def test_batched_tile_heights_agree():
    from ssmdlbm_b200.batch import Sweep
    ps = _lattices()[:3]
    out = []
    for tz in (8, 32):
        sw = Sweep(ps, tile_z=tz)
        sw.init()
        sw.step(4, store_macros=True)
        sw.sync()
        out.append([s.field("phi") for s in sw.sims])
        sw.close()
    for a, b in zip(*out):
        assert np.array_equal(a, b)


def test_sweep_rejects_mixed_velocity_sets():
    from ssmdlbm_b200.batch import Sweep
    ps = [configs.periodic_box((16, 16, 16), 19), configs.periodic_box((16, 16, 16), 27)]
    with pytest.raises(RuntimeError):
        Sweep(ps)
