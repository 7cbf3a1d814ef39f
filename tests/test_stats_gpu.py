"""Jet statistics and checkpoints on the device, against the oracle."""
import numpy as np
import pytest

from ssmdlbm_b200 import _lib, configs
from oracle.oracle import Oracle, seeded_macros

pytestmark = pytest.mark.gpu


def _sim(p):
    from ssmdlbm_b200.lbm import Simulation
    return Simulation(p)


def _blobs(shape, seed, n=12, rmin=1.5, rmax=4.0):
    """phi = union of sharp spheres, some straddling the periodic wrap."""
    nz, ny, nx = shape
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    phi = np.zeros(shape)
    for _ in range(n):
        c = rng.uniform([0, 0, 0], [nz, ny, nx])
        r = rng.uniform(rmin, rmax)
        dz = np.minimum(np.abs(z - c[0]), nz - np.abs(z - c[0]))
        dy = np.minimum(np.abs(y - c[1]), ny - np.abs(y - c[1]))
        dx = np.minimum(np.abs(x - c[2]), nx - np.abs(x - c[2]))
        phi = np.maximum(phi, 0.5 * (1 - np.tanh(2 * (np.sqrt(dx * dx + dy * dy + dz * dz) - r))))
    rho, ux, uy, uz, _ = seeded_macros(shape, seed=seed)
    return rho, ux, uy, uz, phi.astype(np.float32)


@pytest.mark.parametrize("geometry", ["periodic_box", "jet_box"])
def test_droplets_match_oracle(geometry):
    if geometry == "periodic_box":
        p = configs.periodic_box((40, 36, 44), 19)
    else:
        p = configs.oil_jet(40, 36, 44, 19, diam=8)
    shape = (int(p.nz), int(p.ny), int(p.nx))
    m = _blobs(shape, seed=3)
    sim = _sim(p)
    sim.init_from_macros(*m)
    o = Oracle(p, 32)
    o.init_macros(*m)
    got = sim.droplets(0.5)
    want = o.droplets(0.5)
    assert len(want) >= 5
    assert np.array_equal(got["root"], want["root"])
    assert np.array_equal(got["cells"], want["cells"])
    assert np.array_equal(got["touches_inlet"], want["touches_inlet"])
    assert np.allclose(got["volume"], want["volume"], rtol=1e-12, atol=0)


def test_centreline_matches_oracle_after_jet_steps():
    p = configs.oil_jet(32, 32, 64, 27, tau=0.56, diam=8, noise=0.01, seed=2)
    sim = _sim(p)
    sim.init()
    sim.step(30, store_macros=True)
    o = Oracle(p, 64)
    o.init_jets()
    o.step(30)
    uz, phi = sim.centreline()
    uz_o, phi_o = o.centreline()
    assert np.max(np.abs(uz - uz_o)) <= 1e-6 * 0.05 * 10
    assert np.max(np.abs(phi - phi_o)) <= 1e-5
    assert uz[1] > 0.04  # the jet leaves the nozzle along the axis


def test_centreline_off_axis_is_the_block_mean():
    """centreline(cx, cy) averages the cells nearest (cx, cy); the fine-run
    statistics of the closure experiment use it to filter the fine field onto
    the coarse cells around the axis."""
    from ssmdlbm_b200.closure import _coarse_axis_cells
    p = configs.oil_jet(32, 32, 64, 19, tau=0.56, diam=8, noise=0.01, seed=2)
    sim = _sim(p)
    sim.init()
    sim.step(20, store_macros=True)
    uzf = sim.field("uz").astype(np.float64)
    phif = sim.field("phi").astype(np.float64)
    uz, phi = sim.centreline(12.5, 20.5)
    assert np.allclose(uz, uzf[:, 20:22, 12:14].mean(axis=(1, 2)), rtol=1e-12, atol=1e-15)
    assert np.allclose(phi, phif[:, 20:22, 12:14].mean(axis=(1, 2)), rtol=1e-12, atol=1e-15)
    uz, _ = sim.centreline(7.0, 9.0)  # a single column
    assert np.allclose(uz, uzf[:, 9, 7], rtol=1e-12, atol=1e-15)
    assert _coarse_axis_cells(15.5) == [15, 16] and _coarse_axis_cells(15.0) == [15]


def test_checkpoint_resume_is_bit_exact(tmp_path):
    p = configs.oil_jet(32, 24, 40, 19, tau=0.56, diam=6, noise=0.01, seed=4)
    a = _sim(p)
    a.init()
    a.step(7)
    path = tmp_path / "ck.bin"
    a.save(path)
    a.step(6, store_macros=True)
    b = _sim(p)
    b.load(path)
    assert b.steps_done == 7
    b.step(6, store_macros=True)
    for k in ("rho", "ux", "uy", "uz", "phi"):
        assert np.array_equal(a.field(k), b.field(k)), k
    assert np.array_equal(a.populations_push(0), b.populations_push(0))
    q = configs.oil_jet(32, 24, 48, 19)
    c = _sim(q)
    with pytest.raises(_lib.SSMDError):
        c.load(path)


@pytest.mark.parametrize("which", ["oil_jet", "two_jets"])
def test_jet_phi_budget(which):
    """sum phi^N - sum phi^0 - sum_t (inflow - outflow) vanishes to 1e-6
    relative, FP64 reductions, over 300 steps of a jet."""
    from ssmdlbm_b200.lbm import Simulation
    if which == "oil_jet":
        p = configs.oil_jet(32, 32, 96, 19, tau=0.55, sigma=1e-3, mobility=0.1, diam=8, w_in=0.05, noise=0.01,
                            seed=1)
    else:
        p = configs.reference_like(24, 40, 56, 27, diam_water=6, diam_oil=6, reynolds_water=10, reynolds_oil=8,
                                   weber=5)
    s = Simulation(p)
    s.init()
    s0 = s.reduce(raise_unstable=False)["phi_sum_next"]
    net = 0.0
    inflow_total = 0.0
    for _ in range(300):
        s.step(1)
        i, o = s.phase_flux()
        net += i - o
        inflow_total += i
    s1 = s.reduce(raise_unstable=False)["phi_sum_next"]
    assert inflow_total > 0.01 * s1  # the inlets did add phi
    assert abs(s1 - s0 - net) <= 1e-6 * s1, (s0, s1, net, s1 - s0 - net)
    assert s.check_status() == 0
    s.close()
