"""Build the checkers: the CPU oracle and the reference-harness binaries.

    python -m oracle.build [--oracle] [--ref] [--force]

* oracle/_build/libssmd_oracle.so — ssmd_oracle.cpp, g++ -O2 -fopenmp
  -ffp-contract=off (no FMA contraction, so the FP32 instantiation follows
  the written operation order).
* oracle/_build/libssmd_oracle_gpu.so — ssmd_oracle_gpu.cu, the same
  per-cell functions (oracle_cells.h) as FP64 CUDA kernels, nvcc for sm_100a
  with --fmad=false (no contraction, so it matches the CPU build bit for bit).
* oracle/_ref/<case>/harness — the reference's own kernels, compiled by nvcc
  for sm_100a from the reference's sources where they lie (REF_SRC), with
  oracle/ref_harness/constants.cuh.in filled in per case and placed first on
  the include path, plus oracle/ref_harness/harness.cu as the driver.  The
  nvcc flags are those of the reference's compile.sh:58-75 (minus the
  lto/-rdc pair, which only matters for multi-file device linking) with the
  case's velocity set and ENABLE_FP16.  The built binaries travel with the
  repository copy; building them needs the reference's checkout.

Where the reference's sources are: the environment variable SSMD_REFERENCE
names the root of a checkout of brenogemelgo/ssmdLBM (the directory that
holds its compile.sh and src/); without it the recipe looks in
/root/reference, the read-only checkout of the machine these builds were
first made on.  When neither holds src/lbm.cu the reference binaries are
skipped (build_ref returns an empty list).
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF_ROOT = os.environ.get("SSMD_REFERENCE", "/root/reference")
REF_SRC = os.path.join(REF_ROOT, "src")
ORACLE_SO = os.path.join(HERE, "_build", "libssmd_oracle.so")
ORACLE_GPU_SO = os.path.join(HERE, "_build", "libssmd_oracle_gpu.so")
REF_DIR = os.path.join(HERE, "_ref")

# Reference-expressible cases.  diam/radius/Re/We are the reference's own
# constants.cuh knobs; radius_water = 0 disables the water disc while keeping
# nu_water = u_water diam_water / Re_water.
CASES = {
    # two-jet crossflow geometry of the reference, small
    "q19_s": dict(vs="D3Q19", fp16=0, nx=16, ny=16, nz=32, u_water=0.05, u_oil=0.05, diam_water=5,
                  diam_oil=5, radius_water=2, radius_oil=2, re_water=10, re_oil=8, weber=5, width=4),
    "q27_s": dict(vs="D3Q27", fp16=0, nx=16, ny=16, nz=32, u_water=0.05, u_oil=0.05, diam_water=5,
                  diam_oil=5, radius_water=2, radius_oil=2, re_water=10, re_oil=8, weber=5, width=4),
    # x,y-periodic oil jet at the lattice size of the 64x64x128 configuration
    # (tau = 0.55: nu = 0.05 * 8 / 24 = 1/60; sigma = 0.05^2 * 8 / 20 = 1e-3)
    "q19_c1": dict(vs="D3Q19", fp16=0, nx=64, ny=64, nz=128, u_water=0.05, u_oil=0.05, diam_water=8,
                   diam_oil=8, radius_water=0, radius_oil=4, re_water=24, re_oil=24, weber=20, width=4),
    # 128x128x512 D3Q27 oil jet (tau = 0.52: nu = 0.05 * 16 / 120; sigma = 0.05^2 * 16 / 40 = 1e-3)
    "q27_c2": dict(vs="D3Q27", fp16=0, nx=128, ny=128, nz=512, u_water=0.05, u_oil=0.05, diam_water=16,
                   diam_oil=16, radius_water=0, radius_oil=8, re_water=120, re_oil=120, weber=40, width=4),
    "q27_c2_h": dict(vs="D3Q27", fp16=1, nx=128, ny=128, nz=512, u_water=0.05, u_oil=0.05, diam_water=16,
                     diam_oil=16, radius_water=0, radius_oil=8, re_water=120, re_oil=120, weber=40, width=4),
    "q19_c2": dict(vs="D3Q19", fp16=0, nx=128, ny=128, nz=512, u_water=0.05, u_oil=0.05, diam_water=16,
                   diam_oil=16, radius_water=0, radius_oil=8, re_water=120, re_oil=120, weber=40, width=4),
}


def _oracle_deps(src: str) -> list[str]:
    return [src, os.path.join(HERE, "oracle_cells.h"), os.path.join(ROOT, "include", "ssmd.h"),
            os.path.join(ROOT, "ssmdlbm_b200", "csrc", "noise.h")]


def build_oracle_gpu(force: bool = False) -> str:
    src = os.path.join(HERE, "ssmd_oracle_gpu.cu")
    deps = _oracle_deps(src)
    if not force and os.path.exists(ORACLE_GPU_SO) and all(
            os.path.getmtime(d) <= os.path.getmtime(ORACLE_GPU_SO) for d in deps):
        return ORACLE_GPU_SO
    os.makedirs(os.path.dirname(ORACLE_GPU_SO), exist_ok=True)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-O3", "--fmad=false", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a",
           "-Xcompiler", "-fPIC", "-shared", "-cudart", "static", src, "-o", ORACLE_GPU_SO]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"GPU oracle build failed:\n{r.stdout}\n{r.stderr}")
    return ORACLE_GPU_SO


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "ssmd_oracle.cpp")
    deps = _oracle_deps(src)
    if not force and os.path.exists(ORACLE_SO) and all(
            os.path.getmtime(d) <= os.path.getmtime(ORACLE_SO) for d in deps):
        return ORACLE_SO
    os.makedirs(os.path.dirname(ORACLE_SO), exist_ok=True)
    cmd = ["g++", "-O2", "-std=c++17", "-fopenmp", "-ffp-contract=off", "-fPIC", "-shared",
           src, "-o", ORACLE_SO]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{r.stdout}\n{r.stderr}")
    return ORACLE_SO


def _constants(case: str, c: dict) -> str:
    t = open(os.path.join(HERE, "ref_harness", "constants.cuh.in")).read()
    rep = {"@CASE@": case, "@NX@": c["nx"], "@NY@": c["ny"], "@NZ@": c["nz"],
           "@DIAM_WATER@": c["diam_water"], "@DIAM_OIL@": c["diam_oil"],
           "@RADIUS_WATER@": c["radius_water"], "@RADIUS_OIL@": c["radius_oil"],
           "@U_WATER@": repr(float(c["u_water"])), "@U_OIL@": repr(float(c["u_oil"])),
           "@RE_WATER@": c["re_water"], "@RE_OIL@": c["re_oil"], "@WEBER@": c["weber"],
           "@WIDTH@": repr(float(c["width"]))}
    for k, v in rep.items():
        t = t.replace(k, str(v))
    return t


def ref_binary(case: str) -> str:
    return os.path.join(REF_DIR, case, "harness")


def build_ref_case(case: str, force: bool = False) -> str:
    c = CASES[case]
    out_dir = os.path.join(REF_DIR, case)
    exe = ref_binary(case)
    harness = os.path.join(HERE, "ref_harness", "harness.cu")
    os.makedirs(out_dir, exist_ok=True)
    cfile = os.path.join(out_dir, "constants.cuh")
    text = _constants(case, c)
    if not os.path.exists(cfile) or open(cfile).read() != text:
        open(cfile, "w").write(text)
    deps = [harness, cfile, os.path.join(HERE, "ref_harness", "constants.cuh.in")]
    if not force and os.path.exists(exe) and all(os.path.getmtime(d) <= os.path.getmtime(exe) for d in deps):
        return exe
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-O3", "--restrict", "-gencode", "arch=compute_100a,code=sm_100a",
           "--extra-device-vectorization", "--fmad=true", "--extended-lambda", "-std=c++20",
           "-I", out_dir, "-I", REF_SRC, harness, f"-DVS_{c['vs']}", f"-DENABLE_FP16={c['fp16']}",
           "-DBENCHMARK=1", "-DTIME_AVERAGE=0", "-DREYNOLDS_MOMENTS=0", "-DVORTICITY_FIELDS=0",
           "-DPASSIVE_SCALAR=0", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference harness build failed for {case}:\n{r.stdout}\n{r.stderr}")
    return exe


def vti_binary(case: str) -> str:
    return os.path.join(REF_DIR, case, "vti_ref")


def build_vti_case(case: str, force: bool = False) -> str:
    """The reference's host-side .vti writer for the lattice of `case`."""
    out_dir = os.path.join(REF_DIR, case)
    build_ref_case(case, force)  # writes the case's constants.cuh
    exe = vti_binary(case)
    src = os.path.join(HERE, "ref_harness", "vti_ref.cu")
    deps = [src, os.path.join(out_dir, "constants.cuh")]
    if not force and os.path.exists(exe) and all(os.path.getmtime(d) <= os.path.getmtime(exe) for d in deps):
        return exe
    c = CASES[case]
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    cmd = [nvcc, "-O2", "-gencode", "arch=compute_100a,code=sm_100a", "--extended-lambda", "-std=c++20",
           "-I", out_dir, "-I", REF_SRC, src, f"-DVS_{c['vs']}", f"-DENABLE_FP16={c['fp16']}",
           "-DBENCHMARK=0", "-DTIME_AVERAGE=0", "-DREYNOLDS_MOMENTS=0", "-DVORTICITY_FIELDS=0",
           "-DPASSIVE_SCALAR=0", "-o", exe]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"reference vti writer build failed for {case}:\n{r.stdout}\n{r.stderr}")
    return exe


def build_ref(force: bool = False) -> list[str]:
    if not os.path.isfile(os.path.join(REF_SRC, "lbm.cu")):
        return []
    with cf.ThreadPoolExecutor(max_workers=min(8, len(CASES))) as ex:
        out = list(ex.map(lambda k: build_ref_case(k, force), CASES))
    out.append(build_vti_case("q19_s", force))
    return out


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--oracle", action="store_true")
    ap.add_argument("--ref", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    both = not (a.oracle or a.ref)
    if a.oracle or both:
        print(build_oracle(a.force))
        print(build_oracle_gpu(a.force))
    if a.ref or both:
        for e in build_ref(a.force):
            print(e)
