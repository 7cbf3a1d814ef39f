"""Generate c2_fp64_1000.npz: the FP64 oracle's jet statistics of the
128 x 128 x 512 D3Q27 + D3Q7 oil jet after 1000 steps.

    OMP_NUM_THREADS=<cores> python tests/golden/make_c2_fp64.py [--steps 1000] [--out FILE]

The jet: nozzle 16 on the z = 0 face, tau 0.52, sigma 1e-3, interface width 4,
mobility 0.1, inlet w 0.05 with 1 % Gaussian noise (seed 1), x and y exactly
periodic, from quiescent water; every step in FP64 on the host cores (about
an hour on 8 cores).  Stored: the centreline u_z and phi profiles (FP64, one
value per z plane), the phi mass over the planes 1 .. nz - 2, and the
droplets (phi > 1/2 components: cells, volume, whether they touch the first
fluid plane).  tests/test_precision_gpu.py compares the FP32, FP16 and BF16
storage runs of the same jet on the GPU against it.
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
from oracle.oracle import Oracle  # noqa: E402


def c2_params():
    return configs.oil_jet(128, 128, 512, 27, tau=0.52, sigma=1e-3, width=4.0, mobility=0.1, diam=16,
                           w_in=0.05, noise=0.01, seed=1, storage=_lib.STORAGE_F32)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--out", default=os.path.join(os.path.dirname(os.path.abspath(__file__)), "c2_fp64_1000.npz"))
    a = ap.parse_args()
    o = Oracle(c2_params(), 64)
    o.init_jets()
    t0 = time.time()
    done = 0
    while done < a.steps:
        k = min(250, a.steps - done)
        o.step(k)
        done += k
        print(f"{done} steps, {time.time() - t0:.0f} s", flush=True)
    uz, phi = o.centreline()
    mass = float(np.asarray(o.get("phi"), np.float64)[1:-1].sum())
    d = o.droplets(0.5)
    np.savez_compressed(a.out, steps=a.steps, uz=uz, phi=phi, mass=mass,
                        drop_cells=np.asarray(d["cells"], np.int64), drop_volume=np.asarray(d["volume"]),
                        drop_touch=np.asarray(d["touches_inlet"], np.int64))
    print("wrote", a.out, flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
