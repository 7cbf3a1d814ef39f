"""Storage precision against the FP64 oracle on the 64 x 64 x 128 D3Q19 oil jet
(nozzle 8, tau 0.55, w 0.05 + 1 % noise, seed 0) after 1000 steps: the jet
statistics of FP32, shifted FP16 and shifted BF16 population storage (FP32
arithmetic throughout) against the same run in FP64 on the host.

The bar for FP16 storage is 1 % on the centreline velocity and the phi mass.
Measured on B200 (errors relative to the FP64 run): FP32 8e-5 / 2e-6 / 5e-8,
FP16 2.4e-4 / 2.5e-4 / 4.3e-4, BF16 2.5e-2 / 1.4e-2 / 6.2e-4 (centreline
u_z, centreline phi, phi mass; BF16 runs keep the phase populations in half,
so their phi mass is conserved like FP16's while u_z carries BF16's 8-bit
mantissa)."""
import os

import numpy as np
import pytest

from ssmdlbm_b200 import _lib, configs
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu

STEPS = 1000


def _params(storage):
    return configs.oil_jet(64, 64, 128, 19, tau=0.55, sigma=1e-3, width=4.0, mobility=0.1, diam=8, w_in=0.05,
                           noise=0.01, seed=0, storage=storage)


@pytest.fixture(scope="module")
def fp64_run():
    o = Oracle(_params(_lib.STORAGE_F32), 64)
    o.init_jets()
    o.step(STEPS)
    uz, phi = o.centreline()
    mass = float(np.asarray(o.get("phi"), np.float64)[1:-1].sum())
    return uz, phi, mass


def _rel(a, b):
    z = slice(1, len(b) - 1)  # fluid planes
    return float(np.linalg.norm(a[z] - b[z]) / np.linalg.norm(b[z]))


@pytest.mark.timeout(600)
@pytest.mark.parametrize("storage,tol_uz,tol_phi,tol_mass", [
    (_lib.STORAGE_F32, 1e-3, 1e-4, 1e-6),
    (_lib.STORAGE_F16, 1e-2, 1e-2, 1e-2),   # the 1 % bar
    (_lib.STORAGE_BF16, 6e-2, 4e-2, 5e-3),  # f's 8-bit mantissa: u_z reported, not held to 1 %
])
def test_jet_statistics_vs_fp64_oracle(fp64_run, storage, tol_uz, tol_phi, tol_mass):
    from ssmdlbm_b200.lbm import Simulation
    uz_o, phi_o, mass_o = fp64_run
    sim = Simulation(_params(storage))
    sim.init()
    sim.step(STEPS, store_macros=True)
    assert sim.check_status() == 0
    uz, phi = sim.centreline()
    mass = float(sim.field("phi").astype(np.float64)[1:-1].sum())
    errs = {"centreline_uz": _rel(uz, uz_o), "centreline_phi": _rel(phi, phi_o),
            "phi_mass": abs(mass - mass_o) / mass_o}
    print(storage, errs)
    assert uz_o[2] > 0.03  # the jet is through the first planes
    assert errs["centreline_uz"] <= tol_uz, errs
    assert errs["centreline_phi"] <= tol_phi, errs
    assert errs["phi_mass"] <= tol_mass, errs


# ---------------------------------------------------------------------------
# The 128 x 128 x 512 D3Q27 jet (nozzle 16, tau 0.52, seed 1) after 1000 steps
# against the FP64 oracle's statistics in tests/golden/c2_fp64_1000.npz, made by
# tests/golden/make_c2_fp64.py on the host cores (an hour of FP64 work, so the
# fixture stands in for a live oracle run).  Measured on B200 (u_z, phi, phi
# mass, phi > 1/2 volume): FP32 1.6e-5 / 2.0e-6 / 2.6e-7 / 2.7e-7, FP16
# 1.7e-3 / 1.5e-4 / 2.2e-4 / 9.6e-5, BF16 2.8e-2 / 1.6e-2 / 1.3e-4 / 1.5e-4.
GOLDEN_C2 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c2_fp64_1000.npz")
C2_TOLERANCES = [  # centreline u_z, centreline phi, phi mass, volume of the phi > 1/2 components
    (_lib.STORAGE_F32, 1e-4, 1e-5, 2e-6, 2e-6),
    (_lib.STORAGE_F16, 1e-2, 1e-2, 1e-2, 1e-2),   # the 1 % bar
    (_lib.STORAGE_BF16, 6e-2, 4e-2, 2e-3, 2e-3),  # f's 8-bit mantissa: u_z reported, not held to 1 %
]


def _c2_params(storage):
    return configs.oil_jet(128, 128, 512, 27, tau=0.52, sigma=1e-3, width=4.0, mobility=0.1, diam=16,
                           w_in=0.05, noise=0.01, seed=1, storage=storage)


@pytest.mark.timeout(600)
@pytest.mark.parametrize("storage,tol_uz,tol_phi,tol_mass,tol_vol", C2_TOLERANCES)
def test_c2_jet_statistics_vs_fp64_fixture(storage, tol_uz, tol_phi, tol_mass, tol_vol):
    from ssmdlbm_b200.lbm import Simulation
    g = np.load(GOLDEN_C2)
    sim = Simulation(_c2_params(storage))
    sim.init()
    sim.step(int(g["steps"]), store_macros=True)
    assert sim.check_status() == 0
    uz, phi = sim.centreline()
    mass = float(sim.field("phi").astype(np.float64)[1:-1].sum())
    d = sim.droplets(0.5)
    errs = {"centreline_uz": _rel(uz, g["uz"]), "centreline_phi": _rel(phi, g["phi"]),
            "phi_mass": abs(mass - float(g["mass"])) / float(g["mass"]),
            "phi_gt_half_volume": abs(float(d["volume"].sum()) - float(g["drop_volume"].sum()))
            / float(g["drop_volume"].sum())}
    print(storage, errs)
    # the same components: their number, and which of them touch the inlet plane
    assert len(d) == len(g["drop_volume"])
    assert sorted(d["touches_inlet"].tolist()) == sorted(g["drop_touch"].tolist())
    assert errs["centreline_uz"] <= tol_uz, errs
    assert errs["centreline_phi"] <= tol_phi, errs
    assert errs["phi_mass"] <= tol_mass, errs
    assert errs["phi_gt_half_volume"] <= tol_vol, errs


@pytest.mark.timeout(600)
def test_gpu_oracle_reproduces_the_host_fixture():
    """The oracle's FP64 GPU instance (oracle/ssmd_oracle_gpu.cu) runs the
    128 x 128 x 512 jet for 1000 steps and gives the same centreline, phi
    mass and components as the host-core run that made c2_fp64_1000.npz,
    bit for bit: the 5000-step fixture of the same jet is made with it."""
    from oracle.oracle import GpuOracle
    g = np.load(GOLDEN_C2)
    o = GpuOracle(_c2_params(_lib.STORAGE_F32), 64)
    o.init_jets()
    o.step(int(g["steps"]))
    uz, phi = o.centreline()
    mass = float(np.asarray(o.get("phi"), np.float64)[1:-1].sum())
    d = o.droplets(0.5)
    o.close()
    assert np.array_equal(uz, g["uz"]) and np.array_equal(phi, g["phi"])
    assert mass == float(g["mass"])
    assert np.array_equal(d["volume"], g["drop_volume"]) and np.array_equal(d["cells"], g["drop_cells"])


# The same jet over C2's full 5000 steps against the FP64 oracle's GPU
# instance (tests/golden/c2_fp64_5000.npz, tests/golden/make_c2_fp64.py
# --gpu).  Measured on B200 (u_z, phi, phi mass, phi > 1/2 volume): FP32
# 1.7e-4 / 2.1e-4 / 1.6e-5 / 1.1e-4; FP16 7.2e-3 / 4.8e-3 / 2.1e-3 / 1.9e-3;
# FP16 with FP32 phase populations 6.2e-3 / 5.8e-3 / 1.6e-5 / 7.4e-5; BF16
# 9.9e-2 / 1.4e-2 / 6.5e-3 / 1.3e-2.  One phi > 1/2 component in all five
# runs (the jet has not broken up), so the droplet-size histograms agree.
GOLDEN_C2_5000 = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "c2_fp64_5000.npz")
C2_5000_TOLERANCES = [  # centreline u_z, centreline phi, phi mass, volume of the phi > 1/2 components
    (_lib.STORAGE_F32, 1e-3, 1e-3, 1e-4, 1e-3),
    (_lib.STORAGE_F16, 1e-2, 1e-2, 1e-2, 1e-2),       # the 1 % bar
    (_lib.STORAGE_F16_G32, 1e-2, 1e-2, 1e-2, 1e-2),   # the 1 % bar
    (_lib.STORAGE_BF16, 0.15, 3e-2, 1e-2, 3e-2),      # f's 8-bit mantissa: u_z reported, not held to 1 %
]


@pytest.mark.timeout(600)
@pytest.mark.parametrize("storage,tol_uz,tol_phi,tol_mass,tol_vol", C2_5000_TOLERANCES)
def test_c2_jet_statistics_after_5000_steps_vs_fp64(storage, tol_uz, tol_phi, tol_mass, tol_vol):
    from ssmdlbm_b200.lbm import Simulation
    g = np.load(GOLDEN_C2_5000)
    sim = Simulation(_c2_params(storage))
    sim.init()
    sim.step(int(g["steps"]), store_macros=True)
    assert sim.check_status() == 0
    uz, phi = sim.centreline()
    mass = float(sim.field("phi").astype(np.float64)[1:-1].sum())
    d = sim.droplets(0.5)
    sim.close()
    hist = np.histogram(np.asarray(d["volume"], np.float64), bins=g["hist_edges"])[0]
    errs = {"centreline_uz": _rel(uz, g["uz"]), "centreline_phi": _rel(phi, g["phi"]),
            "phi_mass": abs(mass - float(g["mass"])) / float(g["mass"]),
            "phi_gt_half_volume": abs(float(d["volume"].sum()) - float(g["drop_volume"].sum()))
            / float(g["drop_volume"].sum())}
    print(storage, errs)
    assert np.array_equal(hist, g["drop_hist"]), (hist[hist > 0], g["drop_hist"][g["drop_hist"] > 0])
    assert errs["centreline_uz"] <= tol_uz, errs
    assert errs["centreline_phi"] <= tol_phi, errs
    assert errs["phi_mass"] <= tol_mass, errs
    assert errs["phi_gt_half_volume"] <= tol_vol, errs
