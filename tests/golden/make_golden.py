"""Generate the golden fixtures in this directory from the reference itself.

    python tests/golden/make_golden.py --out DIR      (on a machine with a GPU)

Runs the reference-harness binaries built by ``python -m oracle.build --ref``
(the reference's own CUDA kernels, oracle/_ref/<case>/harness) and stores
rho, ux, uy, uz, phi after the listed steps as compressed .npz files
(float32, [z][y][x]).  The CPU tests then pin the oracle against these files.

Cases (16 x 16 x 32 lattices, reference parameters listed in oracle/build.py):
  q19_jets, q27_jets   the reference's two-jet crossflow from its own initial
                       state (initialConditions.cu), steps 1 and 100;
  q19_seed, q27_seed   x,y-periodic jet box from the seeded smooth state of
                       oracle.oracle.seeded_macros (seeds 1 and 2), steps 1 and 50.
"""
from __future__ import annotations

import argparse
import os
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from oracle import build as obuild  # noqa: E402
from oracle.oracle import seeded_macros  # noqa: E402

GOLDEN = {
    "q19_jets": dict(case="q19_s", periodic_y=False, seed=None, at=(1, 100)),
    "q27_jets": dict(case="q27_s", periodic_y=False, seed=None, at=(1, 100)),
    "q19_seed": dict(case="q19_s", periodic_y=True, seed=1, at=(1, 50)),
    "q27_seed": dict(case="q27_s", periodic_y=True, seed=2, at=(1, 50)),
}
FIELDS = ("rho", "ux", "uy", "uz", "phi")


def case_shape(case: str):
    c = obuild.CASES[case]
    return (c["nz"], c["ny"], c["nx"])


def run_harness(case: str, steps: int, at, periodic_y: bool, seed, workdir: str, with_pops=False):
    """Run the reference harness; return {step: dict(field -> array)}."""
    exe = obuild.ref_binary(case)
    shape = case_shape(case)
    n = int(np.prod(shape))
    q = 19 if obuild.CASES[case]["vs"] == "D3Q19" else 27
    cmd = [exe, "--steps", str(steps), "--dump", os.path.join(workdir, "d"),
           "--at", ",".join(str(s) for s in at)]
    if periodic_y:
        cmd.append("--periodic-y")
    if seed is not None:
        m = seeded_macros(shape, seed=seed)
        path = os.path.join(workdir, "macros.bin")
        np.concatenate([a.reshape(-1) for a in m]).astype(np.float32).tofile(path)
        cmd += ["--macros", path]
    subprocess.run(cmd, check=True)
    out = {}
    for s in at:
        raw = np.fromfile(os.path.join(workdir, f"d_{s}.bin"), dtype=np.float32)
        d = {k: raw[i * n:(i + 1) * n].reshape(shape) for i, k in enumerate(FIELDS)}
        if with_pops:
            d["f"] = raw[5 * n:(5 + q) * n].reshape((q,) + shape)
            d["g"] = raw[(5 + q) * n:(12 + q) * n].reshape((7,) + shape)
        out[s] = d
    return out


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=os.path.dirname(os.path.abspath(__file__)))
    a = ap.parse_args()
    os.makedirs(a.out, exist_ok=True)
    for name, spec in GOLDEN.items():
        with tempfile.TemporaryDirectory() as td:
            res = run_harness(spec["case"], max(spec["at"]), spec["at"], spec["periodic_y"],
                              spec["seed"], td)
        arrays = {f"{k}_{s}": v[k] for s, v in res.items() for k in FIELDS}
        np.savez_compressed(os.path.join(a.out, f"{name}.npz"), **arrays)
        print(name, "ok")
    return 0


if __name__ == "__main__":
    sys.exit(main())
