"""Generate the FP64 oracle's jet statistics of the 128 x 128 x 512
D3Q27 + D3Q7 oil jet: c2_fp64_1000.npz (1000 steps, host cores) and
c2_fp64_5000.npz (5000 steps, the oracle's GPU instance).

    OMP_NUM_THREADS=<cores> python tests/golden/make_c2_fp64.py [--steps 1000] [--out FILE]
    python tests/golden/make_c2_fp64.py --gpu --steps 5000 [--out FILE]

The jet: nozzle 16 on the z = 0 face, tau 0.52, sigma 1e-3, interface width 4,
mobility 0.1, inlet w 0.05 with 1 % Gaussian noise (seed 1), x and y exactly
periodic, from quiescent water; every step in FP64, on the host cores (about
an hour for 1000 steps on 8 cores) or with --gpu on the current CUDA device
(oracle/ssmd_oracle_gpu.cu: the same functions, the same bits; the GPU run
also checks itself against c2_fp64_1000.npz on the way).  Stored: the
centreline u_z and phi profiles (FP64, one value per z plane), the phi mass
over the planes 1 .. nz - 2, the droplets (phi > 1/2 components: cells,
volume, whether they touch the first fluid plane) and their size histogram
(HIST_EDGES, component volume).  tests/test_precision_gpu.py and bench.py's
precision leg compare the FP32, FP16 and BF16 storage runs of the same jet
on the GPU against them.
"""
from __future__ import annotations

import argparse
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from ssmdlbm_b200 import _lib, configs  # noqa: E402
from oracle.oracle import GpuOracle, Oracle  # noqa: E402

HERE = os.path.dirname(os.path.abspath(__file__))
# droplet-size histogram: component volume (sum of phi) in powers-of-two bins
HIST_EDGES = np.concatenate([[0.0], 2.0 ** np.arange(0, 31)])


def droplet_histogram(volumes) -> np.ndarray:
    return np.histogram(np.asarray(volumes, np.float64), bins=HIST_EDGES)[0].astype(np.int64)


def c2_params():
    return configs.oil_jet(128, 128, 512, 27, tau=0.52, sigma=1e-3, width=4.0, mobility=0.1, diam=16,
                           w_in=0.05, noise=0.01, seed=1, storage=_lib.STORAGE_F32)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--gpu", action="store_true", help="run the oracle's FP64 GPU instance")
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    out = a.out or os.path.join(HERE, f"c2_fp64_{a.steps}.npz")
    o = GpuOracle(c2_params(), 64) if a.gpu else Oracle(c2_params(), 64)
    o.init_jets()
    t0 = time.time()
    done = 0
    check = os.path.join(HERE, "c2_fp64_1000.npz")
    while done < a.steps:
        k = min(250, a.steps - done)
        o.step(k)
        done += k
        print(f"{done} steps, {time.time() - t0:.0f} s", flush=True)
        if a.gpu and done == 1000 and os.path.exists(check):
            g = np.load(check)
            uz, phi = o.centreline()
            same = np.array_equal(uz, g["uz"]) and np.array_equal(phi, g["phi"])
            print("GPU instance vs the host-core fixture after 1000 steps:", "identical" if same else
                  f"differ (u_z {np.abs(uz - g['uz']).max():.3e}, phi {np.abs(phi - g['phi']).max():.3e})",
                  flush=True)
    uz, phi = o.centreline()
    mass = float(np.asarray(o.get("phi"), np.float64)[1:-1].sum())
    d = o.droplets(0.5)
    np.savez_compressed(out, steps=a.steps, uz=uz, phi=phi, mass=mass,
                        drop_cells=np.asarray(d["cells"], np.int64), drop_volume=np.asarray(d["volume"]),
                        drop_touch=np.asarray(d["touches_inlet"], np.int64),
                        drop_hist=droplet_histogram(d["volume"]), hist_edges=HIST_EDGES,
                        device_s=time.time() - t0)
    print("wrote", out, f"({len(d)} components, {time.time() - t0:.1f} s)", flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
