"""Build libssmd.so (sm_100a) in-tree.

    python -m ssmdlbm_b200.build [--force]

Each .cu under csrc/ is compiled in parallel with nvcc for
``-gencode arch=compute_100a,code=sm_100a`` and linked into
ssmdlbm_b200/libssmd.so with the CUDA runtime linked statically, so the
library carries no dependency on the caller's CUDA runtime version.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libssmd.so")
ROOT = os.path.dirname(HERE)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
                     "-Xcompiler", "-fPIC", "-Xcompiler", "-O2", "-Xptxas", "-v"]
SOURCES = ["ssmd_api.cu", "kernels_q19.cu", "kernels_q27.cu", "reduce_static.cu", "stats.cu", "checkpoint.cu", "batch.cu", "mlp.cu", "closure.cu", "derived.cu", "output.cpp"]


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and os.path.exists(c):
            return c
    raise RuntimeError("nvcc not found")


def _deps() -> list[str]:
    out = [os.path.join(ROOT, "include", "ssmd.h")]
    for f in os.listdir(CSRC):
        if f.endswith((".cu", ".cuh", ".h", ".cpp")):
            out.append(os.path.join(CSRC, f))
    return out


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def _compile(src: str, log: bool) -> str:
    obj = os.path.join(OBJ, os.path.splitext(src)[0] + ".o")
    cmd = [nvcc()] + NVCC_FLAGS + ["-c", os.path.join(CSRC, src), "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
    if log:
        with open(os.path.join(OBJ, os.path.splitext(src)[0] + ".ptxas.txt"), "w") as fh:
            fh.write(r.stderr)
    return obj


def build(force: bool = False, verbose: bool = False) -> str:
    deps = _deps()
    if not force and not _stale(LIB, deps):
        return LIB
    os.makedirs(OBJ, exist_ok=True)
    with cf.ThreadPoolExecutor(max_workers=len(SOURCES)) as ex:
        objs = list(ex.map(lambda s: _compile(s, True), SOURCES))
    cmd = [nvcc()] + ARCH + ["-shared", "-cudart", "static", "-o", LIB] + objs
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    if verbose:
        print(f"built {LIB}")
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    build(force=a.force, verbose=True)
    sys.exit(0)
