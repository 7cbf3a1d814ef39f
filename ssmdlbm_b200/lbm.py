"""Host-side mirror of the reference's driver (src/main.cu:35-213).

``Simulation`` owns the device fields the way ``host::FieldAllocate`` does
(src/fieldAllocate/FieldAllocate.cuh:42-162): every LBMFields member the step
uses, zero-initialised, plus the second population buffers and the workspace
the C ABI asks for.  Memory comes from torch's CUDA allocator (plumbing
only); every computation goes through libssmd.so.
"""
from __future__ import annotations

import ctypes
import time
from dataclasses import dataclass

import numpy as np
import torch

from . import _lib
from ._lib import LBMFields, Params, Stats, check, lib

STORAGE_DTYPES = {_lib.STORAGE_F32: torch.float32, _lib.STORAGE_F16: torch.float16,
                  _lib.STORAGE_BF16: torch.bfloat16, _lib.STORAGE_F16_G32: torch.float16}
# element type of the phase populations g: BF16 runs keep g in half (phi in
# [0, 1] needs mantissa bits, not range); F16_G32 keeps it in float, as the
# reference's FP16 build does
PHASE_DTYPES = {_lib.STORAGE_F32: torch.float32, _lib.STORAGE_F16: torch.float16,
                _lib.STORAGE_BF16: torch.float16, _lib.STORAGE_F16_G32: torch.float32}
SCALARS = ("rho", "ux", "uy", "uz", "pxx", "pyy", "pzz", "pxy", "pxz", "pyz", "phi", "fsx", "fsy", "fsz")


@dataclass
class StepTiming:
    steps: int
    seconds: float
    cells: int

    @property
    def mlups(self) -> float:
        # reference convention: all nx*ny*nz cells per step (src/main.cu:199-203)
        return self.cells * self.steps / self.seconds / 1e6


class Simulation:
    """One lattice on one GPU: init, step, graph replay, reductions, I/O."""

    def __init__(self, params: Params, device: str | torch.device = "cuda"):
        self.p = params.copy()
        check(lib().ssmd_validate(ctypes.byref(self.p)))
        self.device = torch.device(device)
        n = int(self.p.nx) * int(self.p.ny) * int(self.p.nz)
        self.cells = n
        self.shape = (int(self.p.nz), int(self.p.ny), int(self.p.nx))  # [z][y][x]
        dt = STORAGE_DTYPES[self.p.storage]
        Q = int(self.p.velocity_set)
        self.t = {k: torch.zeros(n, dtype=torch.float32, device=self.device) for k in SCALARS}
        self.t["f"] = torch.zeros(Q * n, dtype=dt, device=self.device)
        dg = PHASE_DTYPES[self.p.storage]
        self.t["g"] = torch.zeros(7 * n, dtype=dg, device=self.device)
        self.t["f_alt"] = torch.zeros(Q * n, dtype=dt, device=self.device)
        self.t["g_alt"] = torch.zeros(7 * n, dtype=dg, device=self.device)
        wsb = int(lib().ssmd_workspace_bytes(ctypes.byref(self.p)))
        self.t["workspace"] = torch.zeros(wsb, dtype=torch.uint8, device=self.device)
        self.fields = LBMFields()
        for k in SCALARS:
            setattr(self.fields, k, self.t[k].data_ptr())
        self.fields.f = self.t["f"].data_ptr()
        self.fields.g = self.t["g"].data_ptr()
        self.p.f_alt = self.t["f_alt"].data_ptr()
        self.p.g_alt = self.t["g_alt"].data_ptr()
        self.p.workspace = self.t["workspace"].data_ptr()
        self.p.workspace_bytes = wsb
        self.steps_done = 0
        self._graphs: dict = {}
        # a non-default stream: graph capture is illegal on the legacy default stream
        torch.cuda.synchronize(self.device)
        self.torch_stream = torch.cuda.Stream(self.device)

    # ------------------------------------------------------------------ api
    @property
    def stream(self) -> int:
        return self.torch_stream.cuda_stream

    def sync(self) -> None:
        self.torch_stream.synchronize()

    def init(self) -> None:
        """Reference initial state (src/initialConditions.cu:33-140)."""
        check(lib().ssmd_init(ctypes.byref(self.p), ctypes.byref(self.fields), self.stream))
        self.steps_done = 0

    def init_from_macros(self, rho, ux, uy, uz, phi) -> None:
        """Populations at equilibrium of the given macroscopic fields ([z][y][x] arrays)."""
        with torch.cuda.stream(self.torch_stream):
            for k, v in zip(("rho", "ux", "uy", "uz", "phi"), (rho, ux, uy, uz, phi)):
                self.t[k].copy_(torch.as_tensor(np.ascontiguousarray(v, dtype=np.float32)).reshape(-1))
        check(lib().ssmd_init_from_macros(ctypes.byref(self.p), ctypes.byref(self.fields), self.stream))
        self.steps_done = 0

    def step(self, n: int = 1, store_macros: bool = False, average: bool = False) -> None:
        """n steps; store_macros: the last one writes the macroscopic fields;
        average: every step updates the running means (enable_derived first)."""
        L = lib()
        for i in range(n):
            last = i == n - 1
            flags = _lib.STEP_STORE_MACROS if (store_macros and last) else 0
            if average:
                flags |= _lib.STEP_AVERAGE
            check(L.ssmd_step(ctypes.byref(self.fields), ctypes.byref(self.p), self.steps_done, flags,
                              self.stream))
            self.steps_done += 1

    # ------------------------------------------------------- derived fields
    DERIVED = ("avg_phi", "avg_ux", "avg_uy", "avg_uz", "avg_uxux", "avg_uyuy", "avg_uzuz", "avg_uxuy",
               "avg_uxuz", "avg_uyuz", "vort_x", "vort_y", "vort_z", "vort_mag")

    def enable_derived(self, names=None) -> None:
        """Allocate (zeroed) derived-field arrays; names defaults to all of them."""
        names = self.DERIVED if names is None else tuple(names)
        self._derived = _lib.Derived()
        for k in names:
            if k not in self.DERIVED:
                raise KeyError(k)
            self.t[k] = torch.zeros(self.cells, dtype=torch.float32, device=self.device)
            setattr(self._derived, k, self.t[k].data_ptr())
        self.p.derived = ctypes.addressof(self._derived)
        for ex in self._graphs.values():
            check(lib().ssmd_graph_destroy(ex))
        self._graphs.clear()

    def derived_update(self, what: int = _lib.DERIVED_AVERAGES | _lib.DERIVED_VORTICITY) -> None:
        """The reference's per-step derived-field launch, from the stored macroscopic fields."""
        check(lib().ssmd_derived_update(ctypes.byref(self.p), ctypes.byref(self.fields), what, self.stream))

    def graph(self, steps: int = 2, flags: int = 0) -> int:
        """Instantiate (once) a CUDA graph of `steps` steps starting at the current parity."""
        key = (steps, flags, self.steps_done & 1)
        if key not in self._graphs:
            ex = ctypes.c_void_p()
            check(lib().ssmd_capture_graph(ctypes.byref(self.p), ctypes.byref(self.fields),
                                           self.steps_done, steps, flags, self.stream, ctypes.byref(ex)))
            self._graphs[key] = ex.value
        return self._graphs[key]

    def run_graph(self, replays: int, steps: int = 2) -> None:
        ex = self.graph(steps)
        L = lib()
        for _ in range(replays):
            check(L.ssmd_graph_launch(ex, self.stream))
        self.steps_done += replays * steps

    def reduce(self, raise_unstable: bool = True) -> dict:
        st = Stats()
        code = lib().ssmd_reduce(ctypes.byref(self.p), ctypes.byref(self.fields), self.steps_done,
                                 ctypes.byref(st), self.stream)
        if code != _lib.SSMD_OK and (raise_unstable or code != _lib.SSMD_ERR_UNSTABLE):
            check(code)
        d = st.as_dict()
        d["status"] = code
        return d

    def save(self, path: str) -> None:
        """Bit-exact checkpoint of the lattice (populations, macroscopic arrays, step)."""
        check(lib().ssmd_checkpoint_save(ctypes.byref(self.p), ctypes.byref(self.fields), self.steps_done,
                                         str(path).encode(), self.stream))

    def load(self, path: str) -> None:
        """Resume from a checkpoint written by save() for the same lattice."""
        n = ctypes.c_uint64()
        torch.cuda.synchronize(self.device)
        check(lib().ssmd_checkpoint_load(ctypes.byref(self.p), ctypes.byref(self.fields), str(path).encode(),
                                         ctypes.byref(n), self.stream))
        self.steps_done = int(n.value)

    def phase_flux(self) -> tuple:
        """(inflow, outflow) of phi in the last step, FP64."""
        a, b = ctypes.c_double(), ctypes.c_double()
        check(lib().ssmd_phase_flux(ctypes.byref(self.p), ctypes.byref(self.fields), self.steps_done,
                                    ctypes.byref(a), ctypes.byref(b), self.stream))
        return a.value, b.value

    def centreline(self, cx: float | None = None, cy: float | None = None):
        """Mean u_z and phi along the oil-nozzle axis, per z (FP64 numpy arrays):
        over the one, two or four cells nearest (cx, cy), by default the nozzle
        centre.  Needs the macroscopic fields of a step with store_macros."""
        p = self.p
        if cx is not None or cy is not None:
            p = self.p.copy()
            p.oil_cx = self.p.oil_cx if cx is None else cx
            p.oil_cy = self.p.oil_cy if cy is None else cy
        uz = torch.zeros(int(self.p.nz), dtype=torch.float64, device=self.device)
        phi = torch.zeros_like(uz)
        torch.cuda.synchronize(self.device)
        check(lib().ssmd_centreline(ctypes.byref(p), ctypes.byref(self.fields), uz.data_ptr(),
                                    phi.data_ptr(), self.stream))
        self.sync()
        return uz.cpu().numpy(), phi.cpu().numpy()

    def droplets(self, threshold: float = 0.5, max_droplets: int = 100000) -> np.ndarray:
        """Connected components of phi > threshold (structured array sorted by
        root: root, cells, volume, touches_inlet).  Needs store_macros fields."""
        L = lib()
        nbytes = int(L.ssmd_droplets_scratch_bytes(ctypes.byref(self.p), max_droplets))
        scratch = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        out = (_lib.Droplet * max_droplets)()
        n = ctypes.c_int32()
        torch.cuda.synchronize(self.device)
        check(L.ssmd_droplets(ctypes.byref(self.p), ctypes.byref(self.fields), threshold, scratch.data_ptr(),
                              nbytes, out, max_droplets, ctypes.byref(n), self.stream))
        k = min(n.value, max_droplets)
        arr = np.zeros(k, dtype=[("root", "u4"), ("cells", "u4"), ("volume", "f8"), ("touches_inlet", "u4")])
        for i in range(k):
            arr[i] = (out[i].root, out[i].cells, out[i].volume, out[i].touches_inlet)
        arr.sort(order="root")
        return arr

    def check_status(self) -> int:
        v = ctypes.c_uint32()
        check(lib().ssmd_check_status(ctypes.byref(self.p), ctypes.byref(v), self.stream))
        return v.value

    # --------------------------------------------------------------- access
    def field(self, name: str) -> np.ndarray:
        """A scalar field as a [z][y][x] float32 numpy array (synchronises)."""
        self.sync()
        return self.t[name].reshape(self.shape).cpu().numpy()

    def populations_push(self, which: int = 0) -> np.ndarray:
        """Current f (which=0) or g (which=1) in the reference's push layout, [q][z][y][x] float32."""
        Q = int(self.p.velocity_set) if which == 0 else 7
        dt = (STORAGE_DTYPES if which == 0 else PHASE_DTYPES)[self.p.storage]
        out = torch.empty(Q * self.cells, dtype=dt, device=self.device)
        torch.cuda.synchronize(self.device)
        check(lib().ssmd_populations_to_push(ctypes.byref(self.p), ctypes.byref(self.fields),
                                             self.steps_done, which, out.data_ptr(), self.stream))
        self.sync()
        return out.float().reshape((Q,) + self.shape).cpu().numpy()

    def timed(self, steps: int, use_graph: bool = True, graph_steps: int = 2) -> StepTiming:
        """Device-timed steps (CUDA events on the launching stream)."""
        s = self.torch_stream
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        if use_graph:
            assert steps % graph_steps == 0
            self.graph(graph_steps)
        torch.cuda.synchronize(self.device)
        e0.record(s)
        if use_graph:
            self.run_graph(steps // graph_steps, graph_steps)
        else:
            self.step(steps)
        e1.record(s)
        e1.synchronize()
        return StepTiming(steps, e0.elapsed_time(e1) / 1e3, self.cells)

    def close(self) -> None:
        for ex in self._graphs.values():
            check(lib().ssmd_graph_destroy(ex))
        self._graphs.clear()

