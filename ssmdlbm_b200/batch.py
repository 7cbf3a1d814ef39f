"""Batched parameter sweeps: many jets advanced by one persistent launch per step.

``Sweep`` owns one ``lbm.Simulation`` per lattice (its own fields, buffers
and workspace) and the device table of the batched kernels; ``step`` /
``run_graph`` advance all lattices together through ssmd_batch_step.
``sweep_params`` draws the 48-lattice sweep of uneven N x N x 4N oil jets.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _lib, configs
from ._lib import LBMFields, Params, check, lib


def sweep_params(count: int = 48, seed: int = 2, velocity_set: int = 19, storage: int = _lib.STORAGE_F32):
    """Lattices N x N x 4N, N ~ U{32, 48, 64, 96}; inlet w ~ U[0.02, 0.08];
    nozzle diameter ~ U{6..12}; sigma log-uniform in [1e-4, 1e-2];
    tau ~ U[0.51, 0.6]; mobility ~ U[0.05, 0.2]; x, y exact periodic, oil inflow
    at z = 0, outflow at z = nz-1, 1 % inlet noise with per-lattice seeds."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        n = int(rng.choice([32, 48, 64, 96]))
        w = float(rng.uniform(0.02, 0.08))
        diam = int(rng.integers(6, 13))
        sigma = float(10 ** rng.uniform(-4, -2))
        tau = float(rng.uniform(0.51, 0.6))
        mob = float(rng.uniform(0.05, 0.2))
        out.append(configs.oil_jet(n, n, 4 * n, velocity_set, tau=tau, sigma=sigma, width=4.0, mobility=mob,
                                   diam=diam, w_in=w, noise=0.01, seed=1000 * seed + i, storage=storage))
    return out


class Sweep:
    def __init__(self, params: list[Params], device="cuda", tile_z: int = 0):
        from .lbm import Simulation
        self.sims = [Simulation(p, device) for p in params]
        self.count = len(self.sims)
        self.device = torch.device(device)
        self.params = (Params * self.count)(*[s.p for s in self.sims])
        self.fields = (LBMFields * self.count)(*[s.fields for s in self.sims])
        self.nbytes = int(lib().ssmd_batch_table_bytes(self.params, self.count))
        self.table = torch.zeros(self.nbytes, dtype=torch.uint8, device=self.device)
        torch.cuda.synchronize(self.device)
        self.torch_stream = torch.cuda.Stream(self.device)
        self.steps_done = 0
        self._graphs: dict = {}
        self.cells = sum(s.cells for s in self.sims)
        self.set_tile_z(tile_z)

    def set_tile_z(self, tile_z: int) -> None:
        """Rebuild the device table with z chunks of tile_z planes (0: 16)."""
        self.sync()
        for ex in self._graphs.values():
            check(lib().ssmd_graph_destroy(ex))
        self._graphs.clear()
        for i in range(self.count):
            self.params[i].tile_z = tile_z
        self.tile_z = tile_z
        self.table.zero_()
        torch.cuda.synchronize(self.device)
        check(lib().ssmd_batch_prepare(self.params, self.fields, self.count, self.table.data_ptr(), self.nbytes,
                                       self.stream))

    @property
    def stream(self) -> int:
        return self.torch_stream.cuda_stream

    def init(self) -> None:
        for s in self.sims:
            s.init()
            s.sync()
        self.steps_done = 0
        for s in self.sims:
            s.steps_done = 0

    def timed(self, steps: int, graph_steps: int = 2) -> float:
        """Device seconds of `steps` batched steps replayed as graphs (CUDA events on the stream)."""
        assert steps % graph_steps == 0
        self.run_graph(1, graph_steps)
        self.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(self.torch_stream)
        self.run_graph(steps // graph_steps, graph_steps)
        e1.record(self.torch_stream)
        e1.synchronize()
        return e0.elapsed_time(e1) / 1e3

    def timed_one_by_one(self, steps: int) -> float:
        """Device seconds of the same steps issued lattice by lattice (one
        ssmd_step per lattice and step, one stream): the launch pattern a
        sweep takes without the batched kernels, each lattice with the
        library's own z chunk (tile_z 0; the batched chunk does not carry
        over, since a lattice launched alone needs enough work items of its
        own)."""
        L = lib()
        singles = []
        for pr in self.params:
            q = pr.copy()
            q.tile_z = 0
            singles.append(q)
        args = [(ctypes.byref(s.fields), ctypes.byref(singles[i])) for i, s in enumerate(self.sims)]
        self.sync()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(self.torch_stream)
        for k in range(steps):
            for fl, pr in args:
                check(L.ssmd_step(fl, pr, self.steps_done + k, 0, self.stream))
        e1.record(self.torch_stream)
        e1.synchronize()
        self.steps_done += steps
        for s in self.sims:
            s.steps_done = self.steps_done
        return e0.elapsed_time(e1) / 1e3

    def step(self, n: int = 1, store_macros: bool = False) -> None:
        L = lib()
        for i in range(n):
            flags = _lib.STEP_STORE_MACROS if (store_macros and i == n - 1) else 0
            check(L.ssmd_batch_step(self.params, self.count, self.steps_done, flags, self.table.data_ptr(),
                                    self.stream))
            self.steps_done += 1
        for s in self.sims:
            s.steps_done = self.steps_done

    def run_graph(self, replays: int, steps: int = 2) -> None:
        key = (steps, self.steps_done & 1)
        if key not in self._graphs:
            ex = ctypes.c_void_p()
            check(lib().ssmd_batch_capture_graph(self.params, self.count, self.steps_done, steps, 0,
                                                 self.table.data_ptr(), self.stream, ctypes.byref(ex)))
            self._graphs[key] = ex.value
        L = lib()
        for _ in range(replays):
            check(L.ssmd_graph_launch(self._graphs[key], self.stream))
        self.steps_done += replays * steps
        for s in self.sims:
            s.steps_done = self.steps_done

    def sync(self) -> None:
        if hasattr(self, "torch_stream"):
            self.torch_stream.synchronize()

    def close(self) -> None:
        for ex in self._graphs.values():
            check(lib().ssmd_graph_destroy(ex))
        self._graphs.clear()
        for s in self.sims:
            s.close()
