"""The compile -> simulate -> output pipeline with the reference's command line."""
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HOST = os.path.join(ROOT, "ssmdlbm_b200", "host")


def _compile(vs, sim_id):
    env = dict(os.environ, GPU_ARCH="100")
    subprocess.run(["bash", os.path.join(HOST, "compile.sh"), vs, sim_id], check=True, env=env,
                   capture_output=True, timeout=600)
    return os.path.join(ROOT, "bin", vs, f"{sim_id}sim_{vs}_sm100")


def test_driver_builds_and_checks_arguments():
    exe = _compile("D3Q19", "ci")
    assert os.path.exists(exe)
    r = subprocess.run([exe], capture_output=True, text=True)
    assert r.returncode == 1 and "Usage" in r.stderr
    r = subprocess.run([exe, "D3Q15", "000", "1"], capture_output=True, text=True)
    assert r.returncode == 1


@pytest.mark.gpu
def test_pipeline_writes_reference_outputs_and_matches_the_library():
    from ssmdlbm_b200 import configs
    from ssmdlbm_b200.lbm import Simulation
    args = ["--nx", "32", "--ny", "48", "--nz", "64", "--steps", "20", "--save", "10", "--diam-water", "6",
            "--diam-oil", "6", "--re-water", "20", "--re-oil", "15", "--weber", "8"]
    r = subprocess.run(["bash", os.path.join(HOST, "pipeline.sh"), "D3Q27", "gt1"] + args, capture_output=True,
                       text=True, timeout=900, cwd=ROOT)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "MLUPS" in r.stdout
    d = os.path.join(ROOT, "bin", "D3Q27", "gt1")
    for step in (0, 10, 20):
        for name in ("phi", "rho"):
            assert os.path.getsize(os.path.join(d, f"{name}{step:06d}.bin")) == 32 * 48 * 64 * 4
        assert os.path.exists(os.path.join(d, f"step_{step:06d}.vti"))
    assert os.path.exists(os.path.join(d, "gt1_info.txt"))
    p = configs.reference_like(32, 48, 64, 27, diam_water=6, diam_oil=6, reynolds_water=20, reynolds_oil=15,
                               weber=8)
    sim = Simulation(p)
    sim.init()
    sim.step(21, store_macros=True)
    phi = np.fromfile(os.path.join(d, "phi000020.bin"), dtype=np.float32).reshape(64, 48, 32)
    assert np.array_equal(phi, sim.field("phi"))
