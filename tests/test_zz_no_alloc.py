"""ssmd_reduce_static: the reduction for callers that cannot allocate device memory.

Such callers (a plugin that only receives the simulation's fields, or code
where cudaMalloc is not allowed) get their scratch from a fixed array inside
the library instead of a caller workspace.  This test calls it through the C
ABI twice in a row and checks both results against ssmd_reduce, which uses
the caller's workspace: sums within 1e-12 relative (FP64, different block
count), maximum speed, cell and non-finite counts identical.  It runs last
(file name) so a failure here cannot hide the other tests, and it builds its
own lattice so it also passes alone in a fresh process.
"""
import ctypes

import numpy as np
import pytest

from ssmdlbm_b200 import _lib, configs
from ssmdlbm_b200._lib import Stats, lib
from oracle.oracle import seeded_macros

pytestmark = pytest.mark.gpu


def _stats(fn, sim):
    st = Stats()
    code = fn(ctypes.byref(sim.p), ctypes.byref(sim.fields), sim.steps_done, ctypes.byref(st), sim.stream)
    return code, st.as_dict()


def _close(a, b):
    for k in ("phi_sum", "phi_sum_next", "mass", "kinetic"):
        assert abs(a[k] - b[k]) <= 1e-12 * max(abs(b[k]), 1e-300), (k, a[k], b[k])
    for x, y in zip(a["momentum"], b["momentum"]):
        assert abs(x - y) <= 1e-12 * max(abs(y), 1e-12), ("momentum", x, y)
    for k in ("u_max", "nonfinite", "cells"):
        assert a[k] == b[k], (k, a[k], b[k])


@pytest.mark.parametrize("shape,vs,storage", [((18, 16, 20), 19, _lib.STORAGE_F32),
                                              ((64, 64, 256), 27, _lib.STORAGE_F16)])
def test_static_reduce_matches_workspace_reduce_twice(shape, vs, storage):
    from ssmdlbm_b200.lbm import Simulation
    nx, ny, nz = shape
    p = configs.periodic_box((nx, ny, nz), vs, storage=storage)
    sim = Simulation(p)
    sim.init_from_macros(*seeded_macros((nz, ny, nx), seed=7))
    sim.step(3, store_macros=True)
    L = lib()
    code_ref, ref = _stats(L.ssmd_reduce, sim)
    assert code_ref == _lib.SSMD_OK
    code1, first = _stats(L.ssmd_reduce_static, sim)
    code2, second = _stats(L.ssmd_reduce_static, sim)
    assert code1 == code2 == _lib.SSMD_OK
    _close(first, ref)
    _close(second, ref)
    assert first == second  # same kernels, same block count: bit-identical
    # the state moves on; the shared array must not leak the previous result
    sim.step(2, store_macros=True)
    _, ref2 = _stats(L.ssmd_reduce, sim)
    _, third = _stats(L.ssmd_reduce_static, sim)
    _close(third, ref2)
    sim.close()


def test_static_reduce_rejects_bad_input_without_touching_the_device():
    p = _lib.reference_params(4096, 4096, 4096, 19)  # > 2^32 - 1 cells
    f = _lib.LBMFields()
    st = Stats()
    code = lib().ssmd_reduce_static(ctypes.byref(p), ctypes.byref(f), 0, ctypes.byref(st), None)
    assert code == _lib.SSMD_ERR_INVALID_ARGUMENT
    assert "2^32" in lib().ssmd_last_error().decode()
