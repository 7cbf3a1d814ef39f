"""Derived fields: running means (timeAverage / reynoldsMoments) and
vorticity, standalone and fused into the step, against numpy."""
import numpy as np
import pytest

from ssmdlbm_b200 import _lib, configs

pytestmark = pytest.mark.gpu

MEANS = ("avg_phi", "avg_ux", "avg_uy", "avg_uz", "avg_uxux", "avg_uyuy", "avg_uzuz", "avg_uxuy", "avg_uxuz",
         "avg_uyuz")


def _params():
    return configs.reference_like(24, 40, 56, 19, diam_water=6, diam_oil=6, reynolds_water=10, reynolds_oil=8,
                                  weber=5)


def _np_update(acc, t, fields):
    f32 = np.float32
    ux, uy, uz, phi = fields["ux"], fields["uy"], fields["uz"], fields["phi"]
    vals = {"avg_phi": phi, "avg_ux": ux, "avg_uy": uy, "avg_uz": uz, "avg_uxux": ux * ux, "avg_uyuy": uy * uy,
            "avg_uzuz": uz * uz, "avg_uxuy": ux * uy, "avg_uxuz": ux * uz, "avg_uyuz": uy * uz}
    for k, v in vals.items():
        a = acc[k]
        acc[k] = (a + (v.astype(f32) - a) / f32(t)).astype(f32)


def _np_vorticity(f):
    f32 = np.float32
    ux, uy, uz = f["ux"], f["uy"], f["uz"]
    w = [np.zeros_like(ux) for _ in range(3)]
    s = (slice(1, -1),) * 3
    def d(a, axis):
        sl_p = [slice(1, -1)] * 3
        sl_m = [slice(1, -1)] * 3
        sl_p[axis] = slice(2, None)
        sl_m[axis] = slice(0, -2)
        return f32(0.5) * (a[tuple(sl_p)] - a[tuple(sl_m)])
    # arrays are [z][y][x]: axis 0 = z, 1 = y, 2 = x
    w[0][s] = d(uz, 1) - d(uy, 0)
    w[1][s] = d(ux, 0) - d(uz, 2)
    w[2][s] = d(uy, 2) - d(ux, 1)
    mag = np.sqrt((w[0] * w[0] + w[1] * w[1]) + w[2] * w[2]).astype(f32)
    return w[0], w[1], w[2], mag


def test_standalone_update_matches_numpy():
    from ssmdlbm_b200.lbm import Simulation
    s = Simulation(_params())
    s.enable_derived()
    s.init()
    acc = {k: np.zeros(s.shape, np.float32) for k in MEANS}
    for t in range(1, 6):
        s.step(1, store_macros=True)
        s.derived_update()
        f = {k: s.field(k) for k in ("ux", "uy", "uz", "phi")}
        _np_update(acc, t, f)
    for k in MEANS:
        assert np.array_equal(s.field(k), acc[k]), k
    wx, wy, wz, wm = _np_vorticity(f)
    for k, ref in zip(("vort_x", "vort_y", "vort_z", "vort_mag"), (wx, wy, wz, wm)):
        assert np.array_equal(s.field(k), ref), k
    assert s.check_status() == 0
    s.close()


def test_fused_averages_equal_standalone():
    from ssmdlbm_b200.lbm import Simulation
    a = Simulation(_params())
    a.enable_derived(MEANS)
    a.init()
    a.step(7, average=True)
    b = Simulation(_params())
    b.enable_derived(MEANS)
    b.init()
    for _ in range(7):
        b.step(1, store_macros=True)
        b.derived_update(_lib.DERIVED_AVERAGES)
    for k in MEANS:
        assert np.array_equal(a.field(k), b.field(k)), k
    a.close()
    b.close()


def test_fused_averages_in_a_graph():
    from ssmdlbm_b200.lbm import Simulation
    a = Simulation(_params())
    a.enable_derived(("avg_uz", "avg_uzuz"))
    a.init()
    a.step(6, average=True)
    b = Simulation(_params())
    b.enable_derived(("avg_uz", "avg_uzuz"))
    b.init()
    b.graph(2, _lib.STEP_AVERAGE)
    import ctypes
    L = _lib.lib()
    for _ in range(3):
        _lib.check(L.ssmd_graph_launch(b.graph(2, _lib.STEP_AVERAGE), b.stream))
        b.steps_done += 2
    for k in ("avg_uz", "avg_uzuz"):
        assert np.array_equal(a.field(k), b.field(k)), k
    a.close()
    b.close()


def test_average_flag_needs_arrays():
    from ssmdlbm_b200.lbm import Simulation
    s = Simulation(_params())
    s.init()
    with pytest.raises(_lib.SSMDError):
        s.step(1, average=True)
    s.close()
