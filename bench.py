"""Benchmark of the fused two-phase jet step (one JSON line on rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Workload: the 128 x 128 x 512 D3Q27 + D3Q7 oil jet (nozzle diameter 16,
w = 0.05 with 1 % Gaussian inlet noise, seed 1, tau = 0.52, sigma = 1e-3,
interface width 4, mobility 0.1, exact periodic x and y, inflow at z = 0 and
outflow at z = nz-1), FP32 population storage.  Synthetic input: the jet
starts from quiescent water, the reference's own initial state.  A step is one
time step of the whole lattice (bulk kernel + boundary kernels, as a CUDA graph
of 2 steps replayed).  MLUPS counts all nx*ny*nz cells per step, the
reference's convention (src/main.cu:199-203).

Multi-GPU: the workload does not shard (one lattice per GPU); with --gpus N
every rank runs an independent replica ("weak" scaling, no collective in the
data path) and rank 0 reports the sum of MLUPS over ranks timed as the max
device time over ranks.

--impl reference runs the reference's own CUDA kernels for the same
configuration (its only implementation of the path), built from its sources
by ``python -m oracle.build --ref`` into oracle/_ref/q27_c2/harness, on the
same GPU with the reference's own step loop (graph + boundary launches +
per-step stream synchronisation, src/main.cu:159-172).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NX, NY, NZ = 128, 128, 512
# the reference's only published figures for the path: MLUPS of the full step,
# D3Q19 / D3Q27 + D3Q7, on an RTX 3050 (its README; lattice size not stated)
PUBLISHED_MLUPS = {19: 440.0, 27: 377.0}
Q = 27
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0


def b_alg(q: int, s_f: int, s_g: int | None = None) -> int:
    """Compulsory bytes per cell update: read + write of f (q s_f), g (7 s_g,
    s_g = s_f unless given) and phi (4)."""
    return 2 * (q * s_f + 7 * (s_f if s_g is None else s_g) + 4)


def element_sizes(storage: int) -> tuple:
    """(bytes per f population, bytes per g population) of a storage kind."""
    from ssmdlbm_b200 import _lib
    return {_lib.STORAGE_F32: (4, 4), _lib.STORAGE_F16: (2, 2), _lib.STORAGE_BF16: (2, 2),
            _lib.STORAGE_F16_G32: (2, 4)}[storage]


def hbm_peak():
    try:
        d = json.load(open(PEAKS_FILE))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """SM clocks, board power and clock-event (throttle) reasons sampled while
    active: NVML read every 10 ms from a thread (the timed region of a default
    run lasts a fraction of a second), `nvidia-smi -lms 100` when NVML cannot
    be loaded.  Read-only: no clock or power setting is touched."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
    PERIOD_S = 0.010

    def __init__(self, index: int):
        self.index = index      # CUDA device ordinal of this rank
        self.uuid = None        # the same device for NVML / nvidia-smi
        try:
            import torch
            if torch.cuda.is_available():
                self.uuid = "GPU-" + str(torch.cuda.get_device_properties(index).uuid)
        except Exception:
            self.uuid = None
        self.proc = None
        self.thread = None
        self.rows = []          # (sm_mhz, sm_max_mhz, power_w, set of reason names)

    # ---------------------------------------------------------------- NVML
    def _nvml_start(self) -> bool:
        try:
            import threading
            import pynvml as nv
            nv.nvmlInit()
            try:
                h = nv.nvmlDeviceGetHandleByUUID(self.uuid)
            except Exception:
                self.uuid = None
                h = nv.nvmlDeviceGetHandleByIndex(self.index)
            smax = nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM)
            bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                    "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                    "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                    "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        except Exception:
            return False
        self._nv, self._stop = nv, threading.Event()

        def loop():
            while True:
                try:
                    sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                    pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                    r = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                    self.rows.append((float(sm), float(smax), pw,
                                      {n for n, b in bits.items() if r & b}))
                except Exception:
                    pass
                if self._stop.wait(self.PERIOD_S):
                    return

        self.thread = threading.Thread(target=loop, daemon=True)
        self.thread.start()
        return True

    # ---------------------------------------------------------- nvidia-smi
    def _smi_start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", self.uuid or str(self.index), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def _smi_stop(self):
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        for l in out.splitlines():
            c = [x.strip() for x in l.split(",")]
            try:
                row = (float(c[1]), float(c[2]), float(c[3]))
            except (ValueError, IndexError):
                continue
            self.rows.append(row + ({n for n, v in zip(self.NAMES, c[5:9])
                                     if v.lower().startswith("active")},))

    def __enter__(self):
        self.source = "nvml" if self._nvml_start() else "nvidia-smi"
        if self.source == "nvidia-smi":
            self._smi_start()
        return self

    def __exit__(self, *exc):
        if self.thread is not None:
            self._stop.set()
            self.thread.join(timeout=5)
            try:
                self._nv.nvmlShutdown()
            except Exception:
                pass
        elif self.proc is not None:
            self._smi_stop()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [r[0] for r in self.rows]
        reasons = set().union(*(r[3] for r in self.rows))
        return {"sm_mhz": statistics.median(sm), "sm_min_mhz": min(sm), "sm_max_mhz": self.rows[-1][1],
                "power_w_max": round(max(r[2] for r in self.rows), 1), "samples": len(sm),
                "source": self.source, "reasons": sorted(reasons)}


def dist_setup(n_gpus: int):
    """One process per GPU (torchrun's RANK / LOCAL_RANK / WORLD_SIZE): NCCL
    when CUDA is present, gloo otherwise (the CPU tests of this plumbing)."""
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch
        import torch.distributed as dist
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=120))
    return world, rank, local


def max_over_ranks(v: float, world: int) -> float:
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([v], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_mlups(cells: int, steps: int, seconds: float, world: int) -> tuple:
    """Whole-job MLUPS of `world` replicas of a lattice of `cells` cells, each
    timed on its own device: the slowest replica's time (max over ranks) sets
    the job time, every replica updated cells * steps.  Returns (seconds,
    MLUPS)."""
    t = max_over_ranks(seconds, world)
    return t, cells * steps * world / t / 1e6


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def workload(storage: int, q: int = Q):
    from ssmdlbm_b200 import configs
    return configs.oil_jet(NX, NY, NZ, q, tau=0.52, sigma=1e-3, width=4.0, mobility=0.1, diam=16,
                           w_in=0.05, noise=0.01, seed=1, storage=storage)


STORAGE_NAMES = {"f32": 0, "f16": 1, "bf16": 2, "f16g32": 3}

# run length of the 128 x 128 x 512 jet as configured (the end-to-end leg runs it whole)
JOB_STEPS = 5000

# The closure network is kept as the exponential moving average of its
# weights along training, decay 0.9999 (about the last 10 000 of its 20 000
# Adam steps).  The networks the runs end on fit the held-out targets more
# tightly but their effect on a coarse run changes sign from one training to
# the next; the long average fits them less tightly and lowered the
# centreline errors for four of five training seeds on the production jet
# (where the decay was chosen) and on all eight jets of the closure study
# (which played no part in the choice).
CLOSURE_WEIGHT_AVERAGE = 0.9999

# DRAM bytes per cell of one bulk launch on the 128 x 128 x 512 jet,
# dram__bytes_read.sum + dram__bytes_write.sum from one ncu capture of that
# launch, keyed by (velocity set, storage): (bytes, the profiles/ summary
# that records the capture, the commit of the captured build).  The bulk
# kernel's device code of these instantiations has not changed since the
# commits named; a change to bulk.cuh or lattice.cuh calls for a new capture
# and new entries here.
NCU_BYTES_PER_CELL = {
    (27, "f32"): (279.2, "profiles/bulk_kernel_q27_f32_oil_jet.md", "e00f0c2"),
    (19, "f32"): (215.0, "profiles/bulk_kernel_q19_f32_oil_jet.md", "e00f0c2"),
    (27, "f16"): (134.2, "profiles/bulk_kernel_q27_f16_oil_jet.md", "e00f0c2"),
}


def time_graph(sim, steps: int, warmup: int, world: int):
    """Device time of exactly `steps` steps after exactly `warmup` untimed
    ones, replayed as 2-step graphs (an odd count ends with one plain step),
    bracketed by barriers (replica_mlups takes the max over ranks)."""
    import torch
    sim.graph(2)
    sim.run_graph(warmup // 2, 2)
    if warmup % 2:
        sim.step(1)
    sim.graph(2)  # captured for the parity the timed steps start at, outside the timing
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    s = sim.torch_stream
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(s)
    sim.run_graph(steps // 2, 2)
    if steps % 2:
        sim.step(1)
    e1.record(s)
    e1.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3


def bulk_launch_ms(sim, launches: int) -> float:
    """Mean duration of the fused bulk kernel, CUDA events on its stream."""
    from ssmdlbm_b200 import _lib
    L = _lib.lib()
    _lib.check(L.ssmd_profile_enable(launches))
    sim.step(launches)
    ms = (ctypes.c_float * launches)()
    cnt = ctypes.c_int32()
    _lib.check(L.ssmd_profile_read(ms, launches, ctypes.byref(cnt)))
    _lib.check(L.ssmd_profile_disable())
    vals = list(ms)[:cnt.value]
    return statistics.mean(vals)


def e2e_run(p, steps: int):
    """End to end through the C ABI with host buffers: pinned upload of the
    initial macroscopic state, ssmd_init_from_macros, capture of a 2-step CUDA
    graph (ssmd_capture_graph, as the reference's pipeline captures its step,
    src/main.cu:153) replayed with an async read-back of the status word after
    every replay, the last two steps as ssmd_step calls (the final one storing
    the macroscopic fields), and the download of phi and rho (the fields the
    reference's pipeline saves).  Capture and graph teardown are timed."""
    import numpy as np
    import torch
    from ssmdlbm_b200 import _lib
    from ssmdlbm_b200.lbm import Simulation
    sim = Simulation(p)
    n = sim.cells
    sim.init()  # the reference's initial state, staged in pinned host memory (untimed)
    sim.sync()
    host_in = {k: torch.empty(n, dtype=torch.float32, pin_memory=True) for k in ("rho", "ux", "uy", "uz", "phi")}
    for k, t in host_in.items():
        t.copy_(sim.t[k])
    host_out = {k: torch.empty(n, dtype=torch.float32, pin_memory=True) for k in ("phi", "rho")}
    status_host = torch.empty(4, dtype=torch.uint8, pin_memory=True)
    L = _lib.lib()
    s = sim.torch_stream
    pr, fl = ctypes.byref(sim.p), ctypes.byref(sim.fields)

    def once(k):
        ex = ctypes.c_void_p()
        with torch.cuda.stream(s):
            for name, t in host_in.items():
                sim.t[name].copy_(t, non_blocking=True)
            _lib.check(L.ssmd_init_from_macros(pr, fl, sim.stream))
            _lib.check(L.ssmd_capture_graph(pr, fl, 0, 2, 0, sim.stream, ctypes.byref(ex)))
            replays = max(k - 2, 0) // 2
            for _ in range(replays):
                _lib.check(L.ssmd_graph_launch(ex, sim.stream))
                status_host.copy_(sim.t["workspace"][:4], non_blocking=True)
            for i in range(2 * replays, k):
                flags = _lib.STEP_STORE_MACROS if i == k - 1 else 0
                _lib.check(L.ssmd_step(fl, pr, i, flags, sim.stream))
                status_host.copy_(sim.t["workspace"][:4], non_blocking=True)
            for name, t in host_out.items():
                t.copy_(sim.t[name], non_blocking=True)
        s.synchronize()
        _lib.check(L.ssmd_graph_destroy(ex))

    once(4)  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    once(steps)
    dt = time.perf_counter() - t0
    replays = max(steps - 2, 0) // 2
    reads = replays + (steps - 2 * replays)  # status words read back
    h2d = 5 * n * 4 / steps
    d2h = (2 * n * 4 + 4 * reads) / steps
    sim.close()
    return n * steps / dt / 1e6, h2d, d2h


def cpu_baseline(p, steps: int = 3):
    """FP64 oracle (the CPU restatement of the step) on the host cores."""
    from oracle.oracle import Oracle
    cores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(cores))
    o = Oracle(p, 64)
    o.init_jets()
    o.step(1)
    t0 = time.perf_counter()
    o.step(steps)
    dt = time.perf_counter() - t0
    n = int(p.nx) * int(p.ny) * int(p.nz)
    return {"value": n * steps / dt / 1e6, "unit": "MLUPS", "cores": int(os.environ["OMP_NUM_THREADS"]),
            "kind": "port",
            "sample": f"FP64 oracle, {steps} steps of the full {NX}x{NY}x{NZ} D3Q27+D3Q7 lattice after 1 "
                      f"warm-up step ({dt:.1f} s)"}


def run_sweep(steps: int = 2000):
    """The 48-lattice sweep (N x N x 4N, N in {32, 48, 64, 96}, seed 2; D3Q19
    f32) for its 2000 steps: batched persistent launches replayed as graphs,
    the z-chunk height from the autotuner (autotune.tune_sweep), against the
    same steps issued lattice by lattice."""
    import torch
    from ssmdlbm_b200 import autotune
    from ssmdlbm_b200.batch import Sweep, sweep_params
    sw = Sweep(sweep_params(48, seed=2))
    tuned = autotune.tune_sweep(sw)
    sw.init()
    sw.timed(4)
    dt = sw.timed(steps)
    sw.timed_one_by_one(4)
    dt_single = sw.timed_one_by_one(steps)
    out = {"lattices": sw.count, "cells": sw.cells, "steps": steps, "tile_z": int(sw.tile_z),
           "tile_z_from": "autotune.tune_sweep", "tuning": tuned.get("tried"),
           "all_lattices_ok": all(s.check_status() == 0 for s in sw.sims),
           "batched_mlups": round(sw.cells * steps / dt / 1e6, 1),
           "one_by_one_mlups": round(sw.cells * steps / dt_single / 1e6, 1),
           "launches_per_step": {"batched": 3, "one_by_one": sw.count * 2}}
    sw.close()
    del sw
    torch.cuda.empty_cache()
    return out


def mlp_throughput(net=None, rows: int = 1 << 24, reps: int = 20):
    """Device throughput of the closure network's kernels (CUDA events):
    forward from a feature array, the gradient with atomics and with the
    reproducible per-CTA reduction, and the fused refresh (features from the
    fields, network, bounds) on the 192 x 192 x 768 coarse lattice.  FLOPs
    are the network's multiply-adds, 2 (12 x 64 + 64 x 64 + 64 x 2) per row
    forward and three times that for the gradient."""
    import ctypes as ct
    import torch
    from ssmdlbm_b200 import _lib, closure
    from ssmdlbm_b200.lbm import Simulation
    L = _lib.lib()
    if net is None:
        net = closure.Network(0)
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    feats = torch.randn(rows, _lib.MLP_IN, device="cuda", generator=g)
    tg = torch.rand(rows, 2, device="cuda", generator=g)
    out = torch.empty(rows, 2, device="cuda")
    st = torch.cuda.current_stream().cuda_stream
    n_ptr, g_ptr, l_ptr = net.net.data_ptr(), net.grad.data_ptr(), net.loss.data_ptr()

    def timed(fn, n_reps, stream=None):
        """Mean device seconds of fn(), CUDA events on the stream it launches on."""
        stream = stream or torch.cuda.current_stream()
        for _ in range(3):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(n_reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3 / n_reps

    flop_row = 2 * (12 * 64 + 64 * 64 + 64 * 2)
    res = {}
    calls = {
        "forward": (lambda: _lib.check(L.ssmd_mlp_forward(n_ptr, feats.data_ptr(), rows, out.data_ptr(), st)), 1),
        "grad_atomic": (lambda: _lib.check(L.ssmd_mlp_grad(n_ptr, feats.data_ptr(), tg.data_ptr(), None, rows, g_ptr,
                                                            l_ptr, st)), 3),
        "grad_reproducible": (lambda: _lib.check(L.ssmd_mlp_grad_ws(n_ptr, feats.data_ptr(), tg.data_ptr(), None, rows,
                                                                     g_ptr, l_ptr, net.ws.data_ptr(),
                                                                     net.ws.numel() * 4, st)), 3)}
    for name, (fn, mult) in calls.items():
        s_per = timed(fn, reps)
        res[name] = {"rows": rows, "g_rows_per_s": round(rows / s_per / 1e9, 3), "ms": round(s_per * 1e3, 4),
                     "tflops": round(flop_row * mult * rows / s_per / 1e12, 2)}
    del feats, tg, out
    cp = closure.coarse_params(c5_params())
    cp.storage = _lib.STORAGE_F16
    sim = Simulation(cp)
    sim.init()
    sim.step(2, store_macros=True)
    n = sim.cells
    nut, cs = torch.empty(n, device="cuda"), torch.empty(n, device="cuda")
    pr, fl = ct.byref(sim.p), ct.byref(sim.fields)
    s_per = timed(lambda: _lib.check(L.ssmd_closure_refresh(pr, fl, n_ptr, 0.05, nut.data_ptr(), cs.data_ptr(),
                                                             sim.stream)), 10, sim.torch_stream)
    step_s = timed(lambda: sim.step(1), 10, sim.torch_stream)
    res["refresh_fused"] = {"cells": n, "g_cells_per_s": round(n / s_per / 1e9, 3), "ms": round(s_per * 1e3, 4),
                            "tflops": round(flop_row * n / s_per / 1e12, 2),
                            "coarse_step_ms": round(step_s * 1e3, 4),
                            "bytes_per_cell": 28, "note": "reads rho, u, phi (20 B) and writes nu_t, sigma factor (8 B)"}
    sim.close()
    del sim
    torch.cuda.empty_cache()
    return res


def jet_stats(sim) -> dict:
    """Centreline u_z and phi (fluid planes), phi mass and droplets of the
    fields the last step stored."""
    uz, phi = sim.centreline()
    d = sim.droplets()
    return {"uz": uz[1:-1], "phi": phi[1:-1], "mass": sim.reduce(raise_unstable=False)["phi_sum_next"],
            "droplets": int(len(d)), "droplet_volume": float(d["volume"].sum()) if len(d) else 0.0}


def stat_diffs(s: dict, ref: dict) -> dict:
    import numpy as np
    rel = lambda a, b: float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30))
    return {"centreline_uz": rel(s["uz"], ref["uz"]), "centreline_phi": rel(s["phi"], ref["phi"]),
            "phi_mass": abs(s["mass"] - ref["mass"]) / max(abs(ref["mass"]), 1e-30),
            "droplets": [s["droplets"], ref["droplets"]],
            "droplet_volume": (abs(s["droplet_volume"] - ref["droplet_volume"]) / ref["droplet_volume"]
                               if ref["droplet_volume"] > 0 else None)}


C2_FP64 = os.path.join(ROOT, "tests", "golden", "c2_fp64_5000.npz")


def run_precision(steps: int = 5000):
    """The 128 x 128 x 512 D3Q27 jet for `steps` steps with FP32, shifted
    FP16, shifted BF16 and FP16-with-FP32-phase population storage (FP32
    arithmetic in all four), judged by the FP64 oracle's statistics of the
    same jet (tests/golden/c2_fp64_5000.npz, computed by the oracle's FP64
    GPU instance): centreline u_z and phi, phi mass, the phi > 1/2 volume and
    the droplet-size histogram."""
    import numpy as np
    import torch
    from ssmdlbm_b200 import _lib
    from ssmdlbm_b200.lbm import Simulation
    g = np.load(C2_FP64)
    assert int(g["steps"]) == steps
    rel = lambda a, b: float(np.linalg.norm(a[1:-1] - b[1:-1]) / np.linalg.norm(b[1:-1]))
    out = {}
    for name, stg in (("f32", _lib.STORAGE_F32), ("f16", _lib.STORAGE_F16), ("bf16", _lib.STORAGE_BF16),
                      ("f16_g32", _lib.STORAGE_F16_G32)):
        sim = Simulation(workload(stg, 27))
        sim.init()
        sim.step(steps, store_macros=True)
        uz, phi = sim.centreline()
        mass = float(sim.field("phi").astype(np.float64)[1:-1].sum())
        d = sim.droplets(0.5)
        hist = np.histogram(np.asarray(d["volume"], np.float64), bins=g["hist_edges"])[0]
        out[name + "_vs_fp64"] = {
            "centreline_uz": rel(uz, g["uz"]), "centreline_phi": rel(phi, g["phi"]),
            "phi_mass": abs(mass - float(g["mass"])) / float(g["mass"]),
            "phi_gt_half_volume": abs(float(d["volume"].sum()) - float(g["drop_volume"].sum()))
            / float(g["drop_volume"].sum()),
            "components": [int(len(d)), int(len(g["drop_volume"]))],
            "droplet_hist_l1": int(np.abs(hist - g["drop_hist"]).sum())}
        sim.close()
        del sim
        torch.cuda.empty_cache()
    return {"workload": f"oil jet D3Q27+D3Q7 {NX}x{NY}x{NZ}, {steps} steps, nozzle 16, tau 0.52, seed 1",
            "judge": "FP64 oracle (oracle_cells.h as FP64 CUDA kernels, bit-identical to the host build), "
                     "statistics in tests/golden/c2_fp64_5000.npz", **out}


def c5_params():
    """384 x 384 x 1536 D3Q27 + D3Q7 jet: nozzle 24, w 0.06 + 1 % noise (seed
    3), sigma 1e-3, tau 0.52, interface width 4, mobility 0.1."""
    from ssmdlbm_b200 import configs
    return configs.oil_jet(384, 384, 1536, 27, tau=0.52, sigma=1e-3, width=4.0, mobility=0.1, diam=24,
                           w_in=0.06, noise=0.01, seed=3)


def run_production(steps: int = 10000, sample_every: int = 1000, spinup: int = 5000, train_steps: int = 20000,
                   update_every: int = 10):
    """The production jet: plain FP32 on the fine 384 x 384 x 1536 lattice
    (the judge, and the source of the training data: filtered 2x onto
    192 x 192 x 768 every `sample_every` steps from `spinup` on, the last
    snapshot held out), the closure network trained on them (Adam, lr 1e-3,
    batch 65536), then the coarse lattice with FP16 storage, plain and with
    the closure refreshed every `update_every` coarse steps, for half the
    steps (acoustic scaling).  Statistics are time averages over the same
    snapshots, on the coarse cells."""
    import torch
    from ssmdlbm_b200 import _lib, closure
    from ssmdlbm_b200.lbm import Simulation
    peak, _ = hbm_peak()
    fine_p = c5_params()
    # the eddy viscosity is bounded by the coarse lattice's molecular one (half
    # the fine one): the closure corrects the flow, it does not take it over
    nut_max = 0.5 * float(fine_p.nu_water)
    r = closure.experiment(fine_p, steps=steps, sample_every=sample_every, spinup=spinup, train_steps=train_steps,
                           batch=65536, lr=1e-3, seed=0, update_every=update_every, nut_max=nut_max,
                           coarse_storage=_lib.STORAGE_F16, average=CLOSURE_WEIGHT_AVERAGE)
    f, pl, cl = r["fine"], r["plain"], r["closure"]
    cp = closure.coarse_params(fine_p)
    cp.storage = _lib.STORAGE_F16
    # ablation: the trained network with one of its two outputs held at the
    # plain method's value (output scale 0, offset nu_t = 0 or factor 1)
    ablation = {}
    P, I = _lib.MLP_PARAMS, _lib.MLP_IN
    for name, k, value in (("nut_only", 1, 1.0), ("sigma_only", 0, 0.0)):
        part = closure.Network(0)
        part.net.copy_(r["net"].net)
        part.net[P + 2 * I + k] = 0.0
        part.net[P + 2 * I + 2 + k] = value
        s = closure.coarse_run(cp, steps // 2, max(1, sample_every // 2), spinup // 2, part, update_every, nut_max)
        ablation[name] = {key: closure.stat_errors(s, f)[key] for key in ("centreline_uz", "centreline_phi",
                                                                          "phi_volume")}
        del part
    # bulk-kernel roofline of the two lattices (fresh runs, 10 launches each)
    bulk = {}
    for name, p, s_f in (("fine_f32", fine_p, 4), ("coarse_f16", cp, 2)):
        sim = Simulation(p)
        sim.init()
        sim.step(2)
        bm = bulk_launch_ms(sim, 10)
        bulk[name] = {"bulk_ms": round(bm, 3),
                      "roofline_frac": round(b_alg(27, s_f) * sim.cells / (bm * 1e-3) / 1e9 / peak, 4),
                      "device_gb": round(torch.cuda.max_memory_allocated() / 1e9, 1)}
        sim.close()
        del sim
        torch.cuda.empty_cache()
        torch.cuda.reset_peak_memory_stats()
    net = r["net"]
    mlups = lambda s: round(s.cells * s.steps / s.device_s / 1e6, 1)
    keys = ("centreline_uz", "centreline_phi", "phi_volume", "droplets", "droplet_volume", "droplets_per_snapshot",
            "droplet_hist_l1")
    return {
        "workload": f"oil jet D3Q27+D3Q7 fine 384x384x1536 FP32 plain, {steps} steps, nozzle 24, w 0.06 + 1% noise, "
                    f"seed 3, tau 0.52, sigma 1e-3; coarse 192x192x768 FP16 storage, {steps // 2} steps, "
                    f"closure refreshed every {update_every} coarse steps; statistics averaged over steps "
                    f"{spinup}..{steps} every {sample_every}",
        "steps": steps,
        "fine": {"mlups": mlups(f), "device_s": round(f.device_s, 3), **bulk["fine_f32"]},
        "coarse_plain": {"mlups": mlups(pl), "device_s": round(pl.device_s, 3)},
        "coarse_closure": {"mlups": mlups(cl), "device_s": round(cl.device_s, 3), **bulk["coarse_f16"]},
        "nut_max": nut_max,
        "training": {"device_s": round(r["train_device_s"], 3), "adam_steps": train_steps, "samples": r["samples"],
                     "heldout_loss": r["heldout_loss"], "reproducible_gradient": True,
                     "weight_average_decay": CLOSURE_WEIGHT_AVERAGE},
        "time_ratio": round(cl.device_s / f.device_s, 4),
        "time_ratio_plain_coarse": round(pl.device_s / f.device_s, 4),
        "errors_vs_filtered_fine": {k: {"plain": r["errors_plain"][k], "closure": r["errors_closure"][k]}
                                    for k in keys},
        "closure_ablation": ablation,
        "fine_droplets_per_snapshot": f.droplets_mean,
        "mlp_status": r["mlp_status"],
        "mlp": mlp_throughput(net),
    }


def run_c4(seeds: int = 8, steps: int = 20000, train_steps: int = 20000,
           average: float | None = None):
    """The closure study's data generation and training: fine D3Q19 jets
    256 x 256 x 1024 (nozzle 32, tau 0.55, sigma 1e-3, M 0.1, 1 % noise),
    inlet w ~ U[0.04, 0.08] per seed, `steps` steps each, filtered 2x onto
    128 x 128 x 512 every 1000 steps from step 10000 (the last snapshot of
    each seed held out); one network trained on all seeds (Adam, lr 1e-3,
    batch 65536, `train_steps` steps, reproducible gradient); per seed, the
    held-out loss and the coarse run with and without the closure against
    the filtered fine run.  `average`: decay of the moving average of the
    weights the network is kept as (None: CLOSURE_WEIGHT_AVERAGE; 0: the last
    step's weights)."""
    import numpy as np
    import torch
    from ssmdlbm_b200 import closure, configs
    rng = np.random.default_rng(4)
    ws = rng.uniform(0.04, 0.08, seeds)
    data = closure.Dataset()
    fines, held = [], []
    for i, w in enumerate(ws):
        p = configs.oil_jet(256, 256, 1024, 19, tau=0.55, sigma=1e-3, width=4.0, mobility=0.1, diam=32,
                            w_in=float(w), noise=0.01, seed=100 + i)
        d = closure.Dataset()
        fines.append((p, closure.fine_run(p, steps, 1000, 10000, 0.05, d)))
        f, t, wt = d.cat()
        nc = d.feats[-1].shape[0]
        held.append((f[-nc:], t[-nc:], wt[-nc:]))
        data.feats.append(f[:-nc])
        data.targets.append(t[:-nc])
        data.weights.append(wt[:-nc])
        del d
    feats, tg, wt = data.cat()
    net = closure.Network(0)
    net.normalise(feats, tg)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    curve = net.train(feats, tg, wt, train_steps, 65536, 1e-3, 0, report_every=max(1, train_steps // 10),
                      average=CLOSURE_WEIGHT_AVERAGE if average is None else average)
    e1.record()
    e1.synchronize()
    per_seed = []
    for (p, fine), (hf, ht, hw), w in zip(fines, held, ws):
        base = closure.Network(0)
        base.net.copy_(net.net)
        P, I, O = 5378, 12, 2
        base.net[:P] = 0.0
        base.net[P + 2 * I + O:] = torch.tensor([0.0, 1.0], device=base.device)  # nu_t = 0, factor 1
        cp = closure.coarse_params(p)
        plain = closure.coarse_run(cp, steps // 2, 500, 5000, None, nut_max=0.05)
        closed = closure.coarse_run(cp, steps // 2, 500, 5000, net, 10, 0.05)
        per_seed.append({"w_in": round(float(w), 4),
                         "heldout_loss": {"no_closure": base.loss_on(hf, ht, hw), "trained": net.loss_on(hf, ht, hw)},
                         "errors_plain": closure.stat_errors(plain, fine),
                         "errors_closure": closure.stat_errors(closed, fine),
                         "fine_droplets_per_snapshot": fine.droplets_mean,
                         "time_ratio_closure": round(closed.device_s / fine.device_s, 4)})
    return {"workload": f"C4: {seeds} fine D3Q19 jets 256x256x1024, {steps} steps, w ~ U[0.04, 0.08]; "
                        f"one network, {train_steps} Adam steps at batch 65536", "samples": int(feats.shape[0]),
            "train_device_s": round(e0.elapsed_time(e1) / 1e3, 3), "train_curve": curve, "seeds": per_seed}


def run_ours(a, world, rank, local):
    import torch
    from ssmdlbm_b200 import _lib
    from ssmdlbm_b200.lbm import Simulation

    from ssmdlbm_b200 import autotune
    p = workload(STORAGE_NAMES[a.storage], a.vs)
    p.bulk_path = a.path
    sim = Simulation(p)
    tuned = autotune.tune(sim) if (a.path == 0 and not a.no_tune) else None
    sim.init()
    with ClockSampler(local) as clk:
        dt_local = time_graph(sim, a.steps, a.warmup, world)
    clocks = clk.summary()
    dt, value = replica_mlups(sim.cells, a.steps, dt_local, world)
    st = sim.reduce(raise_unstable=False)

    # live roofline of the dominant kernel
    bulk_ms = bulk_launch_ms(sim, 40)
    s_f0, s_g0 = element_sizes(STORAGE_NAMES[a.storage])
    bytes_per_launch = b_alg(a.vs, s_f0, s_g0) * sim.cells
    peak, peak_kind = hbm_peak()
    achieved = bytes_per_launch / (bulk_ms * 1e-3) / 1e9
    n_bc = 1  # oil inflow + outflow z in one launch (x, y exact periodic: no ghost copies)
    sim_path, sim_tz = int(sim.p.bulk_path), int(sim.p.tile_z)
    sim.close()
    del sim
    torch.cuda.empty_cache()

    # the single-GPU legs below (storage / velocity-set variants, sweep,
    # closure, precision, production) run at N = 1 only: they are one-GPU
    # measurements, and under torchrun they would only hold the other GPUs
    extras = world == 1 and not a.quick
    variants = {}
    if extras:
        for name, q, stg in (("d3q27_f16", 27, _lib.STORAGE_F16), ("d3q27_bf16", 27, _lib.STORAGE_BF16),
                             ("d3q27_f16_g32", 27, _lib.STORAGE_F16_G32),
                             ("d3q19_f32", 19, _lib.STORAGE_F32), ("d3q19_f16", 19, _lib.STORAGE_F16)):
            pv = workload(stg, q)
            sv = Simulation(pv)
            tv = autotune.tune(sv) if (a.path == 0 and not a.no_tune) else None
            sv.init()
            dv = time_graph(sv, a.steps, a.warmup, world)
            bm = bulk_launch_ms(sv, 20)
            s_f, s_g = element_sizes(stg)
            variants[name] = {"mlups": round(sv.cells * a.steps / dv / 1e6, 1),
                              "bulk_path": int(sv.p.bulk_path), "tile_z": int(sv.p.tile_z),
                              "bulk_ms": round(bm, 4), "bytes_per_cell": b_alg(q, s_f, s_g),
                              "roofline_frac": round(b_alg(q, s_f, s_g) * sv.cells / (bm * 1e-3) / 1e9 / peak, 4)}
            sv.close()
            del sv
            torch.cuda.empty_cache()

    sweep = run_sweep() if extras else None
    precision = run_precision() if extras else None
    production = run_production() if (extras and not a.no_production) else None

    p.bulk_path, p.tile_z = sim_path, sim_tz
    # End to end: the jet's configured job (JOB_STEPS steps from the host's
    # initial state to the download of the final fields), and the same path
    # over the K timed steps alone, where the one-time upload and download
    # weigh K / JOB_STEPS times more
    e2e_steps = max(JOB_STEPS, a.steps)
    barrier(world)
    with ClockSampler(local) as clk_e2e:
        e2e_local, h2d, d2h = e2e_run(p, e2e_steps)
    barrier(world)
    e2e_k_local, h2d_k, d2h_k = e2e_run(p, max(a.steps, 2))
    # every replica ran the same job: the slowest one sets the time
    cells = p.nx * p.ny * p.nz
    e2e_t = max_over_ranks(cells * e2e_steps / (e2e_local * 1e6), world)
    e2e_mlups = world * cells * e2e_steps / e2e_t / 1e6
    e2e_k_t = max_over_ranks(cells * max(a.steps, 2) / (e2e_k_local * 1e6), world)
    e2e_k_mlups = world * cells * max(a.steps, 2) / e2e_k_t / 1e6

    line = {
        "metric": "MLUPS", "value": round(value, 1), "unit": "MLUPS", "n_gpus": world,
        "steps": a.steps, "warmup": a.warmup, "ms_per_step": round(dt * 1e3 / a.steps, 4),
        "higher_is_better": True, "scaling": "weak",
        "vs_baseline": round(value / PUBLISHED_MLUPS[a.vs], 2),
        "vs_baseline_note": (f"the reference's published {PUBLISHED_MLUPS[a.vs]} MLUPS for D3Q{a.vs}+D3Q7 "
                             "(its README, RTX 3050, lattice size not stated)"),
        "dtype": "f32",
        "data": "synthetic: quiescent water + noisy oil inlet (the reference's initial state)",
        "config": {"workload": f"oil jet D3Q{a.vs}+D3Q7 {NX}x{NY}x{NZ}, {a.storage} storage, nozzle 16, "
                               "tau 0.52, w 0.05 + 1% noise, seed 1",
                   "cells": NX * NY * NZ, "velocity_set": f"D3Q{a.vs}", "storage": a.storage,
                   "parallelism": f"replicas x{world}",
                   "bulk_path": sim_path, "tile_z": sim_tz,
                   "autotuned": tuned is not None,
                   "l2": "inputs larger than L2 (populations 0.9 GB per buffer)"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 4),
                     "traffic": (int(NCU_BYTES_PER_CELL[(a.vs, a.storage)][0] * NX * NY * NZ)
                                 if (a.vs, a.storage) in NCU_BYTES_PER_CELL and not a.size else None),
                     "traffic_source": ("ncu capture of one launch on this lattice: {}, build {}".format(
                         *NCU_BYTES_PER_CELL[(a.vs, a.storage)][1:])
                         if (a.vs, a.storage) in NCU_BYTES_PER_CELL and not a.size else None),
                     "peak_kind": peak_kind, "kernel": f"ssmd::bulk_kernel<{a.vs},{a.storage}>",
                     "bytes_per_cell": b_alg(a.vs, s_f0, s_g0), "launch_ms": round(bulk_ms, 4)},
        "e2e": {"value": round(e2e_mlups, 1), "unit": "MLUPS", "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h), "steps": e2e_steps,
                "job": f"the jet's configured run: {e2e_steps} steps from the initial state uploaded "
                       "from pinned host memory to the download of phi and rho, through the C ABI",
                "k_steps": {"value": round(e2e_k_mlups, 1), "steps": max(a.steps, 2),
                            "h2d_bytes_per_step": int(h2d_k), "d2h_bytes_per_step": int(d2h_k)},
                "clocks": clk_e2e.summary()},
        "gpu_launches": a.steps * (1 + n_bc),
        "clocks": clocks,
        "variants": variants,
        "sweep": sweep,
        "precision": precision,
        "production": production,
        "stats": {"u_max": st["u_max"], "phi_sum": st["phi_sum_next"], "status": st["status"]},
    }
    if rank == 0 and world == 1 and not a.no_cpu:
        line["cpu_baseline"] = cpu_baseline(workload(_lib.STORAGE_F32, a.vs), steps=3)
    return line


def run_reference(a, world, rank):
    if rank != 0:
        return None
    sys.path.insert(0, ROOT)
    from oracle import build as obuild
    exe = obuild.ref_binary("q27_c2")
    if not os.path.exists(exe):
        return {"impl": "reference", "unavailable": f"reference harness not built ({exe})"}
    # the reference cannot express inlet noise, the centred nozzle, exact periodic
    # faces or M = 0.1; its closest run: same lattice, velocity sets, tau, sigma,
    # nozzle diameter and inlet speed, its own boundary set with y copy-periodic.
    def timed(case):
        out = subprocess.run([obuild.ref_binary(case), "--periodic-y", "--time", f"{a.warmup},{a.steps}"],
                             capture_output=True, text=True, timeout=1200, check=True).stdout
        return json.loads(out.strip().splitlines()[-1])

    r = timed("q27_c2")
    v = r["mlups"]
    # the reference's other builds of the same lattice: D3Q19 with FP32
    # populations, and D3Q27 with ENABLE_FP16=1 (its default build, compile.sh:69:
    # f - w as __half, g as float, src/cuda/utils.cuh:67-99)
    variants = {}
    for name, case, s_f, s_g in (("d3q19_f32", "q19_c2", 4, 4), ("d3q27_f16", "q27_c2_h", 2, 4)):
        if not os.path.exists(obuild.ref_binary(case)):
            variants[name] = {"unavailable": f"reference harness {case} not built"}
            continue
        rv = timed(case)
        variants[name] = {"mlups": round(rv["mlups"], 1), "ms_per_step": rv["ms_per_step"],
                          "build": f"D3Q{rv['Q']}, ENABLE_FP16={rv['fp16']}",
                          "population_bytes_per_cell": 2 * (rv["Q"] * s_f + 7 * s_g)}
    return {
        "metric": "MLUPS", "value": round(v, 1), "unit": "MLUPS", "n_gpus": 1, "steps": a.steps,
        "warmup": a.warmup, "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": round(v / PUBLISHED_MLUPS[27], 2), "dtype": "f32", "impl": "reference",
        "data": "synthetic: the reference's own initial state",
        "config": {"workload": f"oil jet D3Q27+D3Q7 {NX}x{NY}x{NZ}, FP32 storage, nozzle 16, tau 0.52 "
                               "(reference build: no noise, nozzle at (nx-1)/2, (ny-1)/4, M = 0.125)",
                   "cells": NX * NY * NZ, "velocity_set": "D3Q27", "storage": "f32",
                   "parallelism": "single GPU"},
        "cpu_baseline": {"value": round(v, 1), "unit": "MLUPS", "cores": 1, "kind": "reference",
                         "sample": "the reference's own CUDA kernels (its only implementation of the "
                                   "path), built for sm_100a from its sources, driven by one host "
                                   "thread with its per-step stream synchronisation"},
        "e2e": {"value": round(v, 1), "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_variants": variants,
    }


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=400)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--quick", action="store_true",
                    help="headline only: skip the variants, sweep, precision and production legs")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--size", default=None, help="nx,ny,nz of a smaller lattice (profiling runs)")
    ap.add_argument("--vs", type=int, default=Q, choices=[19, 27])
    ap.add_argument("--storage", default="f32", choices=sorted(STORAGE_NAMES))
    ap.add_argument("--no-tune", action="store_true", help="skip the autotuner (library defaults)")
    ap.add_argument("--no-production", action="store_true",
                    help="skip the production leg (384 x 384 x 1536 fine run, training, 192 x 192 x 768 coarse runs)")
    ap.add_argument("--c4", action="store_true",
                    help="run only the closure study's data generation and training (8 fine seeds, about 12 min)")
    ap.add_argument("--path", type=int, default=0, choices=[0, 1, 2, 3],
                    help="bulk kernel path: 0 auto, 1 gathers, 2 TMA phi boxes, 3 TMA population slabs")
    a = ap.parse_args()
    if a.size:
        global NX, NY, NZ
        NX, NY, NZ = (int(v) for v in a.size.split(","))
    a.warmup = max(a.warmup, 3)  # at least 3 untimed steps
    world, rank, local = dist_setup(a.gpus)
    if a.c4:
        line = {"metric": "closure study (C4)", **run_c4()} if rank == 0 else None
    elif a.impl == "reference":
        line = run_reference(a, world, rank)
    else:
        line = run_ours(a, world, rank, local)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0 and line is not None:
        print(json.dumps(line))
    return 0


if __name__ == "__main__":
    sys.exit(main())
