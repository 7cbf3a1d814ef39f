"""Learned closure: training data from fine runs, training, coarse runs with the closure.

The plain method on a 2x coarser lattice, corrected per cell by a small
network (ssmd_mlp_*: 12 features -> 64 -> 64 -> 2 on the tensor cores) that
predicts an eddy viscosity and a surface-tension factor.  Everything below
is host orchestration of the C ABI (include/ssmd.h); the arithmetic runs in
the library's kernels.

Lattice units follow acoustic scaling: the coarse lattice has twice the
spacing and twice the time step, so velocities are unchanged, viscosity and
mobility halve (nu dt / dx^2), surface tension halves (sigma dt^2 / dx^3),
the nozzle radius halves, and one coarse step spans two fine steps.  The
interface keeps its physical thickness, so its width in cells halves too (4
fine cells, 2 coarse), and the sharpening rate gamma = 4 M / (W c_s^2), with
both M and W halved, keeps its lattice value.  (Keeping 4 cells instead
doubles the physical thickness: on the 128 x 128 x 512 jet the plain coarse
run then loses 12.7 % of the fine run's phi volume instead of 6.8 %.)
"""
from __future__ import annotations

import ctypes
import math
import time
from dataclasses import dataclass, field

import numpy as np
import torch

from . import _lib
from ._lib import LBMFields, Params, check, lib

CS2_PHASE = 0.25


def init_net(seed: int = 0) -> np.ndarray:
    """Fan-in scaled normal weights, zero biases, identity normalisation."""
    rng = np.random.default_rng(seed)
    H, I, O = _lib.MLP_HIDDEN, _lib.MLP_IN, _lib.MLP_OUT
    net = np.zeros(_lib.MLP_NET_FLOATS, np.float32)
    w1 = np.zeros((H, 16), np.float32)
    w1[:, :I] = rng.normal(0, 1 / np.sqrt(I), (H, I))
    o = 0
    net[o:o + H * 16] = w1.reshape(-1)
    o += H * 16 + H
    net[o:o + H * H] = rng.normal(0, 1 / np.sqrt(H), H * H)
    o += H * H + H
    net[o:o + O * H] = rng.normal(0, 1 / np.sqrt(H), O * H)
    p = _lib.MLP_PARAMS
    net[p + I:p + 2 * I] = 1.0          # 1/std
    net[p + 2 * I:p + 2 * I + O] = 1.0  # output scale
    return net


def coarse_params(p: Params) -> Params:
    """The same jet on a lattice of half the size in every direction."""
    if (p.nx | p.ny | p.nz) & 1:
        raise ValueError("coarsening needs even lattice sizes")
    q = p.copy()
    q.nx, q.ny, q.nz = p.nx // 2, p.ny // 2, p.nz // 2
    f32 = np.float32
    for nu_name, omco_name in (("nu_water", "omco_water"), ("nu_oil", "omco_oil")):
        nu = f32(getattr(p, nu_name)) * f32(0.5)
        setattr(q, nu_name, nu)
        setattr(q, omco_name, f32(1) - f32(1.0 / (0.5 + 3.0 * float(nu))))
    q.omco_ref = q.omco_water
    q.sigma = f32(p.sigma) * f32(0.5)
    q.gamma = f32(p.gamma)  # mobility and width (in cells) both halve
    mob = (1.0 / float(p.omega_g) - 0.5) * CS2_PHASE * 0.5
    q.omega_g = f32(1.0 / (0.5 + mob / CS2_PHASE))
    q.oil_cx = f32((q.nx - 1) * 0.5) if abs(p.oil_cx - (p.nx - 1) * 0.5) < 1e-3 else f32(p.oil_cx * 0.5)
    q.oil_cy = f32((q.ny - 1) * 0.5) if abs(p.oil_cy - (p.ny - 1) * 0.5) < 1e-3 else f32(p.oil_cy * 0.5)
    q.oil_r2 = f32(p.oil_r2) * f32(0.25) if p.oil_r2 >= 0 else p.oil_r2
    q.water_cx, q.water_cz = f32(p.water_cx * 0.5), f32(p.water_cz * 0.5)
    q.water_r2 = f32(p.water_r2) * f32(0.25) if p.water_r2 >= 0 else p.water_r2
    q.f_alt = q.g_alt = q.workspace = None
    q.workspace_bytes = 0
    q.closure = None
    q.derived = None
    q.tile_z = 0
    return q


class Network:
    """A closure network on the device with its Adam state."""

    def __init__(self, seed: int = 0, device="cuda"):
        self.device = torch.device(device)
        self.net = torch.as_tensor(init_net(seed), device=self.device)
        self.m = torch.zeros(_lib.MLP_PARAMS, device=self.device)
        self.v = torch.zeros(_lib.MLP_PARAMS, device=self.device)
        self.grad = torch.zeros(_lib.MLP_PARAMS, device=self.device)
        self.loss = torch.zeros(1, dtype=torch.float64, device=self.device)
        # per-CTA gradient rows of ssmd_mlp_grad_ws: the same bits on every run
        self.ws = torch.empty(lib().ssmd_mlp_grad_workspace_bytes() // 4, device=self.device)
        self.t = 0

    def _grad(self, feats, targets, weights, n, stream) -> None:
        check(lib().ssmd_mlp_grad_ws(self.net.data_ptr(), feats.data_ptr(), targets.data_ptr(),
                                     weights.data_ptr() if weights is not None else None, n, self.grad.data_ptr(),
                                     self.loss.data_ptr(), self.ws.data_ptr(), self.ws.numel() * 4, stream))

    def normalise(self, feats: torch.Tensor, targets: torch.Tensor) -> None:
        """Feature standardisation and output scaling from training data."""
        p, I, O = _lib.MLP_PARAMS, _lib.MLP_IN, _lib.MLP_OUT
        mean = feats.mean(0)
        std = feats.std(0).clamp_min(1e-6)
        tm = targets.mean(0)
        ts = targets.std(0).clamp_min(1e-6)
        self.net[p:p + I] = mean
        self.net[p + I:p + 2 * I] = 1.0 / std
        self.net[p + 2 * I:p + 2 * I + O] = ts
        self.net[p + 2 * I + O:p + 2 * I + 2 * O] = tm

    def loss_on(self, feats, targets, weights=None) -> float:
        """Weighted mean squared error in normalised output units."""
        self._grad(feats, targets, weights, feats.shape[0], torch.cuda.current_stream(self.device).cuda_stream)
        return float(self.loss.item())

    def train(self, feats, targets, weights, steps: int, batch: int = 65536, lr: float = 1e-3, seed: int = 0,
              report_every: int = 0, average: float | None = None) -> list:
        """Adam on random mini-batches (rows drawn with replacement).  With
        `average` (a decay in (0, 1)) the network ends on the exponential
        moving average of its weights along the run (ssmd_mlp_average after
        every step) instead of the last step's weights."""
        L = lib()
        avg = self.net.clone() if average is not None else None
        st = torch.cuda.current_stream(self.device).cuda_stream
        gen = torch.Generator(device=self.device)
        gen.manual_seed(seed)
        n = feats.shape[0]
        b = min(batch, n)
        fb = torch.empty(b, feats.shape[1], device=self.device)
        tb = torch.empty(b, 2, device=self.device)
        wb = torch.empty(b, 2, device=self.device)
        losses = []
        for k in range(steps):
            idx = torch.randint(0, n, (b,), device=self.device, generator=gen)
            torch.index_select(feats, 0, idx, out=fb)
            torch.index_select(targets, 0, idx, out=tb)
            torch.index_select(weights, 0, idx, out=wb)
            self._grad(fb, tb, wb, b, st)
            self.t += 1
            check(L.ssmd_mlp_adam(self.net.data_ptr(), self.grad.data_ptr(), self.m.data_ptr(), self.v.data_ptr(),
                                  self.t, lr, 0.9, 0.999, 1e-8, st))
            if avg is not None:
                check(L.ssmd_mlp_average(avg.data_ptr(), self.net.data_ptr(), average, st))
            if report_every and (k % report_every == 0 or k == steps - 1):
                losses.append((k, float(self.loss.item())))
        if avg is not None:
            P = _lib.MLP_PARAMS
            self.net[:P] = avg[:P]
        return losses

    def predict(self, feats: torch.Tensor) -> torch.Tensor:
        out = torch.empty(feats.shape[0], 2, device=self.device)
        check(lib().ssmd_mlp_forward(self.net.data_ptr(), feats.data_ptr(), feats.shape[0], out.data_ptr(),
                                     torch.cuda.current_stream(self.device).cuda_stream))
        return out

    def status(self) -> int:
        s = ctypes.c_uint32()
        check(lib().ssmd_mlp_status(ctypes.byref(s)))
        return s.value


@dataclass
class Dataset:
    feats: list = field(default_factory=list)
    targets: list = field(default_factory=list)
    weights: list = field(default_factory=list)

    def cat(self):
        return torch.cat(self.feats), torch.cat(self.targets), torch.cat(self.weights)


# droplet-size histogram: detached component volume (sum of phi, fine-cell
# units) in powers-of-two bins
DROP_EDGES = np.concatenate([[0.0], 2.0 ** np.arange(0, 31)])


@dataclass
class JetStats:
    """Statistics of one run, on the coarse lattice's z planes.  The
    centreline profiles and the droplet counts are means over the sampled
    snapshots; the histogram counts every detached droplet of every snapshot."""
    centreline_uz: np.ndarray
    centreline_phi: np.ndarray
    droplets: int
    droplet_volume: float  # detached phi volume in fine-cell units (last snapshot)
    phi_volume: float      # total phi in fine-cell units
    device_s: float
    steps: int
    cells: int
    droplets_mean: float = 0.0       # detached droplets per snapshot
    droplet_hist: np.ndarray = None  # counts over DROP_EDGES, all snapshots


def _view(coarse: torch.Tensor, nc: int) -> LBMFields:
    """LBMFields whose rho, ux, uy, uz, phi are the five planes of a filtered array."""
    f = LBMFields()
    base = coarse.data_ptr()
    f.rho, f.ux, f.uy, f.uz, f.phi = (base + 4 * nc * k for k in range(5))
    return f


def _coarse_axis_cells(c: float) -> list:
    """Coarse cells whose mean is the centreline at coarse coordinate c."""
    return sorted({int(math.floor(c)), int(math.ceil(c))})


def _stats_snapshot(sim, acc: dict, cp: Params | None = None) -> None:
    """Accumulate the centreline profiles.  On the fine lattice (cp = the
    coarse lattice's parameters) the profile is the fine field filtered onto
    the coarse cells the coarse run samples: fine cells 2i and 2i + 1 under
    coarse cell i, so both runs average over the same region around the axis
    (the fine lattice's own nearest cells sit half as far from it)."""
    if cp is None:
        uz, phi = sim.centreline()
    else:
        uz = phi = 0.0
        cells = [(i, j) for i in _coarse_axis_cells(float(cp.oil_cx)) for j in _coarse_axis_cells(float(cp.oil_cy))]
        for i, j in cells:
            u, f = sim.centreline(2 * i + 0.5, 2 * j + 0.5)
            uz, phi = uz + u, phi + f
        uz, phi = uz / len(cells), phi / len(cells)
    acc["uz"] = acc.get("uz", 0) + uz
    acc["phi"] = acc.get("phi", 0) + phi
    acc["n"] = acc.get("n", 0) + 1
    d = sim.droplets(0.5)
    vol_unit = 1.0 if cp is not None else 8.0  # coarse cells hold 8 fine cells
    vols = d[d["touches_inlet"] == 0]["volume"].astype(np.float64) * vol_unit
    acc["hist"] = acc.get("hist", 0) + np.histogram(vols, bins=DROP_EDGES)[0]
    acc["ndrops"] = acc.get("ndrops", 0) + len(vols)


def _finish(sim, acc: dict, fine: bool, device_s: float, steps: int) -> JetStats:
    uz = acc["uz"] / acc["n"]
    phi = acc["phi"] / acc["n"]
    if fine:  # fine planes 2Z, 2Z + 1 -> coarse plane Z
        uz = 0.5 * (uz[0::2] + uz[1::2])
        phi = 0.5 * (phi[0::2] + phi[1::2])
    d = sim.droplets(0.5)
    vol_unit = 1.0 if fine else 8.0
    detached = d[d["touches_inlet"] == 0]
    total = float(sim.field("phi").astype(np.float64).sum()) * vol_unit
    return JetStats(uz, phi, int(len(detached)), float(detached["volume"].sum()) * vol_unit, total, device_s,
                    steps, sim.cells, droplets_mean=acc["ndrops"] / acc["n"],
                    droplet_hist=np.asarray(acc["hist"], np.int64))


def fine_run(p: Params, steps: int, sample_every: int, spinup: int, nut_max: float = 0.05,
             data: Dataset | None = None) -> JetStats:
    """Run the fine lattice; from step `spinup` on, every `sample_every` steps,
    accumulate centreline statistics and (if data is given) append filtered
    training samples."""
    from .lbm import Simulation
    L = lib()
    sim = Simulation(p)
    cp = coarse_params(sim.p)
    nc = int(cp.nx) * int(cp.ny) * int(cp.nz)
    coarse = torch.empty(5 * nc, device=sim.device)
    tau = torch.empty(6 * nc, device=sim.device)
    area = torch.empty(nc, device=sim.device)
    view = _view(coarse, nc)
    sim.init()
    acc: dict = {}
    t_dev = 0.0
    done = 0
    while done < steps:
        k = sample_every if done >= spinup else min(spinup - done, steps - done)
        k = min(k, steps - done)
        t_dev += _timed_steps(sim, k)
        done += k
        if done >= spinup:
            _stats_snapshot(sim, acc, cp)
            if data is not None:
                st = sim.stream
                check(L.ssmd_closure_filter(ctypes.byref(sim.p), ctypes.byref(sim.fields), coarse.data_ptr(),
                                            tau.data_ptr(), area.data_ptr(), st))
                feats = torch.empty(nc, _lib.MLP_IN, device=sim.device)
                tg = torch.empty(nc, 2, device=sim.device)
                wt = torch.empty(nc, 2, device=sim.device)
                check(L.ssmd_closure_targets(ctypes.byref(cp), coarse.data_ptr(), tau.data_ptr(), area.data_ptr(),
                                             nut_max, tg.data_ptr(), wt.data_ptr(), st))
                check(L.ssmd_closure_features(ctypes.byref(cp), ctypes.byref(view), feats.data_ptr(), st))
                sim.sync()
                data.feats.append(feats)
                data.targets.append(tg)
                data.weights.append(wt)
    stats = _finish(sim, acc, True, t_dev, steps)
    sim.close()
    return stats


def _timed_steps(sim, k: int) -> float:
    """k steps, the last storing the macroscopic fields; device seconds."""
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(sim.torch_stream)
    sim.step(k, store_macros=True)
    e1.record(sim.torch_stream)
    e1.synchronize()
    return e0.elapsed_time(e1) / 1e3


def coarse_run(cp: Params, steps: int, sample_every: int, spinup: int, net: Network | None = None,
               update_every: int = 1, nut_max: float = 0.05) -> JetStats:
    """The coarse lattice, plain (net None) or with the closure refreshed every
    `update_every` steps from the fields of the step before (features,
    network and bounds in one kernel, ssmd_closure_refresh)."""
    from .lbm import Simulation
    L = lib()
    sim = Simulation(cp)
    keep = None
    if net is not None:
        n = sim.cells
        nut = torch.zeros(n, device=sim.device)
        cs = torch.ones(n, device=sim.device)
        cl = _lib.Closure(nut.data_ptr(), cs.data_ptr())
        sim.p.closure = ctypes.addressof(cl)
        keep = (nut, cs, cl)
    sim.init()
    acc: dict = {}
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t_dev = 0.0
    done = 0
    st = sim.stream
    while done < steps:
        k = sample_every if done >= spinup else min(spinup - done, steps - done)
        k = min(k, steps - done)
        e0.record(sim.torch_stream)
        if net is None:
            sim.step(k, store_macros=True)
        else:
            nut, cs, _ = keep
            i = 0
            while i < k:
                j = min(update_every, k - i)
                # closure from the fields the previous step stored
                check(L.ssmd_closure_refresh(ctypes.byref(sim.p), ctypes.byref(sim.fields), net.net.data_ptr(),
                                             nut_max, nut.data_ptr(), cs.data_ptr(), st))
                sim.step(j, store_macros=True)
                i += j
        e1.record(sim.torch_stream)
        e1.synchronize()
        t_dev += e0.elapsed_time(e1) / 1e3
        done += k
        if done >= spinup:
            _stats_snapshot(sim, acc)
    stats = _finish(sim, acc, False, t_dev, steps)
    status = sim.check_status()
    sim.close()
    del keep
    if status:
        raise _lib.SSMDError(_lib.SSMD_ERR_UNSTABLE, f"coarse run status {status}")
    return stats


def stat_errors(s: JetStats, ref: JetStats) -> dict:
    """Relative errors of a coarse run's statistics against the fine run's."""
    z = slice(1, len(ref.centreline_uz) - 1)  # fluid planes
    def rel(a, b):
        return float(np.linalg.norm(a[z] - b[z]) / max(np.linalg.norm(b[z]), 1e-30))
    return {
        "centreline_uz": rel(s.centreline_uz, ref.centreline_uz),
        "centreline_phi": rel(s.centreline_phi, ref.centreline_phi),
        "droplets": (s.droplets, ref.droplets),
        "droplet_volume": (abs(s.droplet_volume - ref.droplet_volume) / ref.droplet_volume
                           if ref.droplet_volume > 0 else None),
        "droplets_per_snapshot": (s.droplets_mean, ref.droplets_mean),
        # droplet-size histogram: L1 distance over the fine run's droplet count
        "droplet_hist_l1": (float(np.abs(s.droplet_hist - ref.droplet_hist).sum()) / float(ref.droplet_hist.sum())
                            if ref.droplet_hist is not None and ref.droplet_hist.sum() > 0 else None),
        "phi_volume": abs(s.phi_volume - ref.phi_volume) / max(ref.phi_volume, 1e-30),
    }


def experiment(fine_p: Params, steps: int, sample_every: int, spinup: int, train_steps: int = 2000,
               batch: int = 65536, lr: float = 1e-3, seed: int = 0, update_every: int = 1,
               nut_max: float = 0.05, coarse_storage: int | None = None, average: float | None = None) -> dict:
    """Fine run (the judge and the data), training, then the coarse lattice
    plain and with the trained closure (population storage `coarse_storage`,
    default the fine run's); statistics, errors and device times."""
    data = Dataset()
    t0 = time.perf_counter()
    fine = fine_run(fine_p, steps, sample_every, spinup, nut_max, data)
    feats, tg, wt = data.cat()
    net = Network(seed)
    net.normalise(feats, tg)
    # held-out check: the last snapshot is not trained on
    nc = data.feats[-1].shape[0]
    f_tr, t_tr, w_tr = feats[:-nc], tg[:-nc], wt[:-nc]
    f_te, t_te, w_te = feats[-nc:], tg[-nc:], wt[-nc:]
    baseline = Network(seed)
    baseline.net.zero_()
    p = _lib.MLP_PARAMS
    I, O = _lib.MLP_IN, _lib.MLP_OUT
    baseline.net[p + I:p + 2 * I] = 1.0
    baseline.net[p:p + I] = 0.0
    baseline.net[p + 2 * I:p + 2 * I + O] = net.net[p + 2 * I:p + 2 * I + O]
    baseline.net[p + 2 * I + O:] = torch.tensor([0.0, 1.0], device=net.device)  # nu_t = 0, factor 1
    loss_plain = baseline.loss_on(f_te, t_te, w_te)
    loss_before = net.loss_on(f_te, t_te, w_te)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    curve = net.train(f_tr if f_tr.shape[0] else feats, t_tr if f_tr.shape[0] else tg,
                      w_tr if f_tr.shape[0] else wt, train_steps, batch, lr, seed,
                      report_every=max(1, train_steps // 10), average=average)
    e1.record()
    e1.synchronize()
    train_s = e0.elapsed_time(e1) / 1e3
    loss_after = net.loss_on(f_te, t_te, w_te)
    cp = coarse_params(fine_p)
    if coarse_storage is not None:
        cp.storage = coarse_storage
    csteps, cevery, cspin = steps // 2, max(1, sample_every // 2), spinup // 2
    plain = coarse_run(cp, csteps, cevery, cspin, None, nut_max=nut_max)
    closed = coarse_run(cp, csteps, cevery, cspin, net, update_every, nut_max)
    return {
        "fine": fine, "plain": plain, "closure": closed,
        "errors_plain": stat_errors(plain, fine), "errors_closure": stat_errors(closed, fine),
        "heldout_loss": {"no_closure": loss_plain, "untrained": loss_before, "trained": loss_after},
        "train_curve": curve, "train_device_s": train_s, "samples": int(feats.shape[0]),
        "wall_s": time.perf_counter() - t0, "mlp_status": net.status(), "net": net,
    }


def throughput(rows: int = 1 << 22, coarse=(96, 96, 192), reps: int = 3) -> dict:
    """Device throughput of the closure network: `reps` forward launches on
    `rows` random feature rows, then `reps` fused refreshes of a coarse D3Q27
    jet lattice of shape `coarse` (FP16 storage), CUDA events on the streams
    the launches use."""
    from .lbm import Simulation
    from . import configs
    L = lib()
    net = Network(0)
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    feats = torch.randn(rows, _lib.MLP_IN, device="cuda", generator=g)
    out = torch.empty(rows, 2, device="cuda")
    cur = torch.cuda.current_stream()

    def timed(fn, stream):
        fn()  # warm-up: module load and launch set-up stay out of the timing
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(reps):
            fn()
        e1.record(stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3 / reps

    t_fwd = timed(lambda: check(L.ssmd_mlp_forward(net.net.data_ptr(), feats.data_ptr(), rows, out.data_ptr(),
                                                   cur.cuda_stream)), cur)
    del feats, out
    nx, ny, nz = coarse
    cp = configs.oil_jet(nx, ny, nz, 27, tau=0.51, sigma=5e-4, width=2.0, mobility=0.05, diam=12, w_in=0.06,
                         noise=0.01, seed=3, storage=_lib.STORAGE_F16)
    sim = Simulation(cp)
    sim.init()
    sim.step(2, store_macros=True)
    nut = torch.empty(sim.cells, device=sim.device)
    cs = torch.empty(sim.cells, device=sim.device)
    t_ref = timed(lambda: check(L.ssmd_closure_refresh(ctypes.byref(sim.p), ctypes.byref(sim.fields),
                                                       net.net.data_ptr(), 0.05, nut.data_ptr(), cs.data_ptr(),
                                                       sim.stream)), sim.torch_stream)
    cells = sim.cells
    sim.close()
    flop_row = 2 * (12 * 64 + 64 * 64 + 64 * 2)
    return {"forward": {"rows": rows, "g_rows_per_s": rows / t_fwd / 1e9, "tflops": flop_row * rows / t_fwd / 1e12},
            "refresh": {"cells": cells, "g_cells_per_s": cells / t_ref / 1e9, "ms": t_ref * 1e3},
            "status": net.status()}


if __name__ == "__main__":
    import argparse
    import json
    ap = argparse.ArgumentParser(description="throughput of the closure network's kernels")
    ap.add_argument("--rows", type=int, default=1 << 22, help="feature rows of the forward launches")
    ap.add_argument("--coarse", default="96,96,192", help="nx,ny,nz of the refreshed coarse lattice")
    ap.add_argument("--reps", type=int, default=3)
    a = ap.parse_args()
    print(json.dumps(throughput(a.rows, tuple(int(v) for v in a.coarse.split(",")), a.reps)))
